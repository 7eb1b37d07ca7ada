"""Conductive 3D materials: per-site coefficients as beamz's CUDA path
receives them (beamz/simulation/compile.py:563-640), pinned to the reference's
own functions (``tests/golden/lossy.npz`` from ``tests/golden/make_lossy.py``),
and the step on them against the oracle.

beamz has two forms of the lossy update: its JAX path divides by (1 + beta)
after the CPML-corrected curl (kernels.py:554-626), its CUDA path applies
precomputed decay and source (cuda/src/update.cu:392-410, 585-597, 644-652).
This engine computes the CUDA form; the GPU tests check it bit for bit
against the oracle's restatement of that form and within the field tolerance
against the JAX form."""

from __future__ import annotations

import os

import numpy as np
import pytest

from beamz_b200 import plan as P
from oracle import fdtd_oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "lossy.npz"))


def test_lossy_coefficients_match_the_reference():
    e, h, eps = P.lossy_site_coefficients_3d(GOLD["eps"], GOLD["sigma"], float(GOLD["dt"]))
    for c in ("Ex", "Ey", "Ez"):
        np.testing.assert_array_equal(eps[c], GOLD[f"eps_{c}"], err_msg=c)
        np.testing.assert_array_equal(e[c][0], GOLD[f"decay_{c}"], err_msg=c)
        np.testing.assert_array_equal(e[c][1], GOLD[f"source_{c}"], err_msg=c)
    for c in ("Hx", "Hy", "Hz"):
        np.testing.assert_array_equal(h[c][0], GOLD[f"decay_{c}"], err_msg=c)
        np.testing.assert_array_equal(h[c][1], GOLD[f"source_{c}"], err_msg=c)
    # A NumPy float64 dt must not switch the arithmetic to float64.
    e64, _, _ = P.lossy_site_coefficients_3d(GOLD["eps"], GOLD["sigma"], np.float64(GOLD["dt"]))
    np.testing.assert_array_equal(e64["Ex"][0], GOLD["decay_Ex"])


def lossy_scene(grid=(10, 12, 20), seed=0, pml_cells=3, nsteps=12, sigma_of=None, metallic=()):
    """A conductive 3D scene (boxes of eps and of sigma, CPML on every face,
    a pre-E dipole, an H source and a DFT plane) as a ProgramSpec, and the
    oracle program with both lossy forms available.  ``sigma_of(sigma)``
    replaces the conductivity grid (e.g. adds a sponge); ``pml_cells`` 0
    leaves out the CPML."""
    rng = np.random.default_rng(seed)
    res = 20e-9
    dt = float(0.99 * res / (P.LIGHT_SPEED * 3.0**0.5))
    eps = np.full(grid, 2.085, np.float32)
    sigma = np.zeros(grid, np.float32)
    for _ in range(3):
        lo = [int(rng.integers(1, n - 2)) for n in grid]
        hi = [min(n - 1, a + int(rng.integers(2, max(3, n // 2)))) for a, n in zip(lo, grid)]
        box = tuple(slice(a, b) for a, b in zip(lo, hi))
        eps[box] = rng.choice([12.11, 4.0])
        sigma[box] = rng.choice([5e3, 4e4])
    if sigma_of is not None:
        sigma = sigma_of(sigma)
    e_site, h_site, e_eps = P.lossy_site_coefficients_3d(eps, sigma, dt)
    h_terms, e_terms = P.plan_cpml(grid, dt, res, pml_cells=pml_cells) if pml_cells else ([], [])
    f0 = P.LIGHT_SPEED / 1.55e-6
    wave = P.gaussian_pulse((np.arange(nsteps) + 0.5) * dt, f0, 0.5 * f0, offset=0.3)
    c = tuple(n // 2 for n in grid)
    srcs = [P.SourcePlan("Ey", "pre_e", c, np.array([[[-dt / (P.EPS_0 * 2.085)]]], np.float32), wave),
            P.SourcePlan("Hz", "h", (1, 2, 1), rng.standard_normal((2, 2, 3)).astype(np.float32),
                         (rng.standard_normal(nsteps) * 1e-3).astype(np.float32))]
    mon = P.plane_monitor(grid, res, "x", 0.6 * grid[2] * res, (np.arange(pml_cells, grid[0] - pml_cells) + 0.5) * res,
                          (np.arange(pml_cells, grid[1] - pml_cells) + 0.5) * res, np.array([0.9, 1.1]) * f0)
    spec = P.ProgramSpec(tuple(grid), dt, res, e_site=e_site, h_site=h_site, e_site_eps=e_eps, h_terms=h_terms,
                         e_terms=e_terms, sources=srcs, monitors=[mon], total_steps=nsteps,
                         metallic_edges=frozenset(metallic))
    shapes = O.component_shapes(grid)
    terms = lambda ts: [O.CpmlTerm(t.component, t.axis, t.sign, t.low, t.high, t.a, t.b, t.inv_kappa,  # noqa: E731
                                   shapes[t.component][t.axis]) for t in ts]
    sig_m = tuple(P.h_site_sample_3d(sigma * np.float32(1.0) * P.MU_0 / P.EPS_0, c) for c in ("Hx", "Hy", "Hz"))
    material = O.Material3D(tuple(e_eps[c] for c in ("Ex", "Ey", "Ez")),
                            tuple(P.e_site_average_3d(sigma, c) for c in ("Ex", "Ey", "Ez")), sig_m)
    sources = [O.SlabSource(s.component, s.timing, tuple(s.start), np.asarray(s.coeff, np.float32),
                            np.asarray(s.waveform, np.float32)) for s in srcs]
    monitors = [O.DftMonitor(m.freqs, m.indices, m.weights, m.component_mask, m.t_start, m.t_end, m.interval,
                             m.window_code, m.normalization_code, m.length_unit) for m in spec.monitors]
    monitors[0].value_offset, monitors[0].weight_offset = 0, 0
    oprog = O.OracleProgram(tuple(grid), dt, res, terms(h_terms), terms(e_terms), material=material,
                            sources=sources, monitors=monitors, metallic_edges=frozenset(metallic))
    return spec, oprog, e_site, h_site, (eps, sigma)


def test_oracle_lossy_forms_agree():
    """The CUDA form (precomputed decay/source) and the JAX form (division by
    1 + beta after the curl) of the reference agree within the field tolerance."""
    spec, oprog, e_site, h_site, _ = lossy_scene(nsteps=16)
    jax_form = O.run(O.new_state(oprog), oprog, 16)
    oprog.e_coeffs, oprog.h_coeffs_3d = e_site, h_site
    cuda_form = O.run(O.new_state(oprog), oprog, 16)
    assert_family_close(cuda_form.fields, jax_form.fields, 1e-5)
    assert np.abs(cuda_form.fields["Ey"]).max() > 0


def assert_family_close(got: dict, ref: dict, tol: float) -> None:
    """|got_c - ref_c| <= tol * |ref of c's family (E or H)|: a component that
    the scene leaves near zero (Ez beside a centred Ey dipole) is measured
    against its family's norm, not its own rounding-level one."""
    for fam in ("E", "H"):
        comps = [c for c in O.COMPONENTS if c[0] == fam]
        scale = float(np.sqrt(sum(np.linalg.norm(np.asarray(ref[c], np.float64)) ** 2 for c in comps)))
        for c in comps:
            err = float(np.linalg.norm(np.asarray(got[c], np.float64) - np.asarray(ref[c], np.float64)))
            assert err <= tol * scale, f"{c}: {err:.3e} > {tol} * {scale:.3e}"


def test_lossy_2d_coefficients_match_the_reference():
    for pol in ("tm", "te"):
        e, h, eps = P.lossy_site_coefficients_2d(GOLD["eps2"], GOLD["sigma2"], float(GOLD["dt2"]), pol)
        for c, (dec, src) in {**e, **h}.items():
            np.testing.assert_array_equal(dec, GOLD[f"{pol}_decay_{c}"], err_msg=f"{pol} {c}")
            np.testing.assert_array_equal(src, GOLD[f"{pol}_source_{c}"], err_msg=f"{pol} {c}")
        for c in e:
            np.testing.assert_array_equal(eps[c], GOLD[f"{pol}_eps_{c}"], err_msg=f"{pol} {c}")


def lossy_scene_2d(grid=(21, 26), polarization="tm", seed=0, pml_cells=4, nsteps=12):
    """A conductive 2D scene (eps and sigma boxes, CPML, a pre-E point source,
    a line monitor) and the matching oracle program (per-component E and H
    coefficient arrays: beamz's 2D path applies decay/source in both backends)."""
    rng = np.random.default_rng(seed)
    res = 20e-9
    dt = float(0.7 * res / (P.LIGHT_SPEED * 2.0**0.5))
    eps = np.full(grid, 2.085, np.float32)
    sigma = np.zeros(grid, np.float32)
    for _ in range(2):
        y0, x0 = int(rng.integers(1, grid[0] - 5)), int(rng.integers(1, grid[1] - 5))
        eps[y0:y0 + 5, x0:x0 + 6] = 12.11
        sigma[y0:y0 + 5, x0:x0 + 6] = rng.choice([5e3, 4e4])
    e_site, h_site, e_eps = P.lossy_site_coefficients_2d(eps, sigma, dt, polarization)
    h_terms, e_terms = P.plan_cpml(grid, dt, res, pml_cells=pml_cells, polarization=polarization)
    f0 = P.LIGHT_SPEED / 1.55e-6
    wave = P.gaussian_pulse((np.arange(nsteps) + 0.5) * dt, f0, 0.5 * f0, offset=0.3)
    comp = "Ez" if polarization == "tm" else "Ey"
    srcs = [P.SourcePlan(comp, "pre_e", (grid[0] // 2, grid[1] // 3), np.array([[-dt / (P.EPS_0 * 2.085)]], np.float32),
                         wave)]
    idx, w = [], []
    rows = np.arange(2, grid[0] - 2)
    for c in P.COMPONENTS:
        sy, sx = P.component_shape(c, grid, polarization)
        idx.append((np.minimum(rows, sy - 1) * sx + min(2 * grid[1] // 3, sx - 1)).astype(np.int32)[:, None])
        w.append(np.ones((rows.size, 1), np.float32))
    mask = np.array([1.0 if c in P.active_components(2, polarization) else 0.0 for c in P.COMPONENTS], np.float32)
    mon = P.DftMonitorPlan(np.array([0.95 * f0, 1.05 * f0], np.float32), idx, w, mask)
    spec = P.ProgramSpec(tuple(grid), dt, res, polarization=polarization, e_site=e_site, h_site=h_site,
                         e_site_eps=e_eps, h_terms=h_terms, e_terms=e_terms, sources=srcs, monitors=[mon],
                         total_steps=nsteps)
    shapes = O.component_shapes(grid, polarization)
    terms = lambda ts: [O.CpmlTerm(t.component, t.axis, t.sign, t.low, t.high, t.a, t.b, t.inv_kappa,  # noqa: E731
                                   shapes[t.component][t.axis]) for t in ts]
    sources = [O.SlabSource(s.component, s.timing, tuple(s.start), np.asarray(s.coeff, np.float32),
                            np.asarray(s.waveform, np.float32)) for s in srcs]
    monitors = [O.DftMonitor(mon.freqs, mon.indices, mon.weights, mon.component_mask)]
    oprog = O.OracleProgram(tuple(grid), dt, res, terms(h_terms), terms(e_terms), sources=sources,
                            monitors=monitors, polarization=polarization)
    oprog.h_coeffs = h_site
    oprog.e_coeffs = e_site
    return spec, oprog
