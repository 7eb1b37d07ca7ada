"""Helpers that turn committed golden fixtures into oracle / engine inputs."""

from __future__ import annotations

import os

import numpy as np

from oracle import fdtd_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

H3 = O.CPML_3D_H_TERMS
E3 = O.CPML_3D_E_TERMS


def load(name: str):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def terms_from(data, prefix, comps, full_lens):
    """Rebuild oracle CpmlTerm records from fixture arrays ``{prefix}{i}_a/b/k/slab``."""
    terms = []
    for i, comp in enumerate(comps):
        axis, low, high, sign = (int(v) for v in data[f"{prefix}{i}_slab"])
        terms.append(O.CpmlTerm(comp, axis, float(sign), low, high,
                                data[f"{prefix}{i}_a"], data[f"{prefix}{i}_b"], data[f"{prefix}{i}_k"],
                                full_lens[i]))
    return terms


def terms3d(data, grid):
    shapes = O.component_shapes(tuple(int(v) for v in grid))
    h = terms_from(data, "h", [c for c, _ in H3], [shapes[c][ax] for c, ax in H3])
    e = terms_from(data, "e", [c for c, _ in E3], [shapes[c][ax] for c, ax in E3])
    return h, e, shapes
