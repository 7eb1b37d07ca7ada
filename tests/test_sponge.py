"""Sponge absorbers: the planner's graded conductivity against beamz's own
lowering (``tests/golden/sponge.npz`` from ``tests/golden/make_sponge.py``).
A sponge is a conductive material, so the step runs it through the per-site
lossy path (``tests/test_lossy*.py``); the GPU test checks that path on a
sponge scene and that the sponge absorbs."""

from __future__ import annotations

import numpy as np
import pytest

from beamz_b200 import plan as P
from tests.golden.make_sponge import CASES
from tests.golden_io import load


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_sponge_conductivity_matches_the_reference(case):
    name, grid, kind, edges, cells, sigma_max, order = case
    d = load("sponge")
    res = float(d["res"])
    got = P.sponge_conductivity(grid, res, base_sigma=d[f"{name}_base"],
                                edges=None if edges == "all" else edges,
                                thickness=None if cells is None else cells * res,
                                sigma_max=sigma_max, order=order)
    want = d[f"{name}_total"]
    assert got.dtype == np.float32 and got.shape == want.shape
    # float32 powers may differ by an ulp between numpy builds
    np.testing.assert_allclose(got, want, rtol=2e-6, atol=0.0)
    assert np.count_nonzero(want > d[f"{name}_base"]) > 0  # the sponge is there
