"""Golden vectors for conductive 3D materials, from the reference's own code.

Run from the repository root, in a container that has the beamz source tree:

    python -m tests.golden.make_lossy [--reference /path/to/beamz]

It loads ``beamz/lattice.py`` and ``beamz/simulation/kernels.py`` by path under
the numpy stand-in for ``jax`` (``_refload.py``) and evaluates, on a seeded
cell-centred permittivity / conductivity grid, what beamz's CUDA path receives
for a conductive material (``beamz/simulation/compile.py:563-640``):

* ``sample_voxel_grid_at_e_component_3d_centered`` (lattice.py:732) of eps and
  sigma at the E sites;
* ``_magnetic_conductivity_terms_3d`` (lattice.py:1046-1068), the matched
  magnetic conductivity at the H sites;
* ``precompute_e_update_coefficients`` and ``precompute_h_update_coefficients``
  (kernels.py:704-728).

Writes ``tests/golden/lossy.npz``.
"""

from __future__ import annotations

import argparse
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("BEAMZ_REFERENCE_ROOT"),
                    help="root of the beamz source tree (or set BEAMZ_REFERENCE_ROOT)")
    ap.add_argument("--out", default=os.path.join(HERE, "lossy.npz"))
    args = ap.parse_args(argv)
    if not args.reference:
        ap.error("--reference (or BEAMZ_REFERENCE_ROOT) is required")
    os.environ["BEAMZ_REFERENCE_ROOT"] = args.reference
    from ._refload import load_reference

    ref = load_reference()
    jnp = ref.jnp
    rng = np.random.default_rng(77)
    grid = (5, 6, 7)
    eps = rng.choice(np.array([1.0, 2.085, 12.11], np.float32), size=grid)
    sigma = rng.choice(np.array([0.0, 2.5e3, 4.0e4], np.float32), size=grid)
    dt = float(0.99 * 20e-9 / (299792458.0 * 3.0**0.5))  # a Python float, weak-typed as in beamz
    out = {"eps": eps, "sigma": sigma, "dt": np.float64(dt)}
    shapes = {c: ref.lattice.component_shape_3d(c, grid) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    for c in ("Ex", "Ey", "Ez"):
        e = ref.lattice.sample_voxel_grid_at_e_component_3d_centered(jnp.asarray(eps), c)
        s = ref.lattice.sample_voxel_grid_at_e_component_3d_centered(jnp.asarray(sigma), c)
        dec, src = ref.kernels.precompute_e_update_coefficients(
            shape=shapes[c], conductivity=s, permittivity=e, dt=dt, region=(slice(None),) * 3)
        out[f"eps_{c}"], out[f"sig_{c}"] = np.asarray(e), np.asarray(s)
        out[f"decay_{c}"], out[f"source_{c}"] = np.asarray(dec), np.asarray(src)
    sig_m = ref.lattice._magnetic_conductivity_terms_3d(jnp.asarray(sigma), jnp.asarray(np.float32(1.0)),
                                                        shapes["Hx"], shapes["Hy"], shapes["Hz"])
    for c, sm in zip(("Hx", "Hy", "Hz"), sig_m):
        dec, src = ref.kernels.precompute_h_update_coefficients(sm, dt)
        out[f"sigm_{c}"] = np.asarray(sm)
        out[f"decay_{c}"], out[f"source_{c}"] = np.asarray(dec), np.asarray(src)
    # 2D (lattice.py:1091-1140): each active support samples eps, sigma and
    # the matched magnetic conductivity; then the same precompute functions.
    grid2 = (6, 7)
    eps2 = rng.choice(np.array([1.0, 2.085, 12.11], np.float32), size=grid2)
    sig2 = rng.choice(np.array([0.0, 2.5e3, 4.0e4], np.float32), size=grid2)
    dt2 = float(0.7 * 20e-9 / (299792458.0 * 2.0**0.5))
    out.update(eps2=eps2, sigma2=sig2, dt2=np.float64(dt2))
    base = jnp.asarray(sig2) * jnp.asarray(np.float32(1.0)) * 1.25663706212e-6 / 8.8541878128e-12
    for pol, e_comps, h_comps in (("tm", ("Ez",), ("Hx", "Hy")), ("te", ("Ex", "Ey"), ("Hz",))):
        for c in e_comps:
            e = ref.lattice.sample_voxel_grid_at_component_2d(jnp.asarray(eps2), c, "xy", pol)
            s = ref.lattice.sample_voxel_grid_at_component_2d(jnp.asarray(sig2), c, "xy", pol)
            dec, src = ref.kernels.precompute_e_update_coefficients(
                shape=np.shape(e), conductivity=s, permittivity=e, dt=dt2, region=(slice(None),) * 2)
            out[f"{pol}_eps_{c}"], out[f"{pol}_decay_{c}"], out[f"{pol}_source_{c}"] = map(np.asarray, (e, dec, src))
        for c in h_comps:
            sm = ref.lattice.sample_voxel_grid_at_component_2d(base, c, "xy", pol)
            dec, src = ref.kernels.precompute_h_update_coefficients(sm, dt2)
            out[f"{pol}_decay_{c}"], out[f"{pol}_source_{c}"] = np.asarray(dec), np.asarray(src)
    np.savez(args.out, **out)
    print(f"wrote {args.out}: {len(out)} arrays")


if __name__ == "__main__":
    main()
