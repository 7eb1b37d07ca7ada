"""Golden vectors for sponge absorbers, from the reference's own code.

Run from the repository root, in a container that has the beamz source tree:

    python -m tests.golden.make_sponge [--reference /path/to/beamz]

For ``Absorber`` and ``PML(formulation="sponge")`` boundaries on 3D and 2D
uniform grids it runs ``_AbsorberCompiler.compile_absorber_regions``
(``beamz/devices/_boundary_compile.py:206-222``: the resolved sigma_max and
``_create_sponge_profiles``, 616-650) and ``_total_conductivity``
(``beamz/lattice.py:978-998``) on a seeded base conductivity, loaded by path
under the numpy stand-in for ``jax`` (``_refload.py``).  Writes
``tests/golden/sponge.npz``.
"""

from __future__ import annotations

import argparse
import os
import types
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# (name, grid, boundary kind, edges, thickness in cells or None, sigma_max or None, order)
CASES = (
    ("a3", (9, 11, 13), "absorber", "all", 3, None, 3),
    ("b3", (8, 10, 12), "absorber", ("left", "top", "back"), 2.5, None, 2),
    ("p3", (14, 15, 16), "pml", "all", None, None, 3),
    ("a2", (17, 19), "absorber", "all", 4, None, 3),
    ("b2", (16, 18), "absorber", ("right", "bottom"), 3, 5e5, 4),
)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("BEAMZ_REFERENCE_ROOT"),
                    help="root of the beamz source tree (or set BEAMZ_REFERENCE_ROOT)")
    ap.add_argument("--out", default=os.path.join(HERE, "sponge.npz"))
    args = ap.parse_args(argv)
    if not args.reference:
        ap.error("--reference (or BEAMZ_REFERENCE_ROOT) is required")
    os.environ["BEAMZ_REFERENCE_ROOT"] = args.reference
    from ._refload import load_reference

    ref = load_reference()
    rng = np.random.default_rng(99)
    res = 20e-9
    data = {"res": np.float64(res)}
    for name, grid, kind, edges, cells, sigma_max, order in CASES:
        thickness = None if cells is None else cells * res
        if kind == "absorber":
            spec = ref.boundaries.Absorber(edges=edges, thickness=thickness, sigma_max=sigma_max, m=order)
        else:
            spec = ref.boundaries.PML(edges=edges, formulation="sponge", m=order)
        eps = rng.choice(np.array([2.085, 12.11], np.float32), size=grid)
        base = np.where(rng.random(grid) < 0.2, np.float32(3e5), np.float32(0.0)).astype(np.float32)
        fields = types.SimpleNamespace(permittivity=eps)
        domain = tuple(n * res for n in reversed(grid)) + ((0.0,) if len(grid) == 2 else ())
        dt = 0.5 * res / 299792458.0
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            profiles = ref.boundary_compile.compile_absorber_regions(spec, fields, domain, res, dt)
        total = ref.lattice._total_conductivity(types.SimpleNamespace(
            conductivity=ref.jnp.asarray(base), has_pml=True, has_cpml=False, pml_data=profiles,
            permittivity=ref.jnp.asarray(eps), material_grid=None))
        data[f"{name}_base"] = base
        data[f"{name}_total"] = np.asarray(total)
        for axis in "xyz":
            data[f"{name}_sigma_{axis}"] = np.asarray(profiles[f"sigma_{axis}"])
        data[f"{name}_thickness"] = np.float64(-1.0 if thickness is None else thickness)
        data[f"{name}_sigma_max"] = np.float64(-1.0 if sigma_max is None else sigma_max)
    np.savez(args.out, **data)
    print(f"wrote {args.out}: {len(data)} arrays")


if __name__ == "__main__":
    main()
