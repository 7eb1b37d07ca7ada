"""Automatic termination on the device: the diagnostics and monitor-change
reductions (fdtd_field_diagnostics, fdtd_dft_change) against the oracle, and
bounded runs end to end (beamz/simulation/execute.py:1312-1484; the pulse test
follows tests/validation/invariants/test_automatic_termination.py:64-140 of
the reference)."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from beamz_b200 import plan as P  # noqa: E402
from beamz_b200 import runtime as R  # noqa: E402
from beamz_b200 import termination as T  # noqa: E402
from oracle import fdtd_oracle as O  # noqa: E402
from tests.scenarios import random_initial_fields, scenario_2d, scenario_3d  # noqa: E402

pytestmark = pytest.mark.gpu


def _site_eps(spec):
    if spec.ndim == 3:
        return {c: P.site_eps_3d(spec.voxel_ids, spec.eps_table, c) for c in ("Ex", "Ey", "Ez")}
    return dict(spec.e_site_eps)


CASES = {
    "3d_pitched": (lambda: scenario_3d(grid=(9, 12, 40), seed=3, nsteps=4), "fused"),
    "3d_dense": (lambda: scenario_3d(grid=(9, 12, 40), seed=3, nsteps=4), "phases"),
    "2d_tm": (lambda: scenario_2d(grid=(17, 23), polarization="tm"), "fused"),
    "2d_te": (lambda: scenario_2d(grid=(17, 23), polarization="te"), "phases"),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_device_diagnostics_match_the_oracle(case):
    build, schedule = CASES[case]
    spec = build()
    fields = random_initial_fields(spec, seed=11, scale=3.0)
    prog = R.compile_program(spec, schedule=schedule)
    assert (prog.layout == "pitched") == (case == "3d_pitched")
    st = R.initial_state(prog, fields=fields)
    got = R.field_diagnostics(st, prog)
    energy, max_field, finite = O.field_diagnostics(fields, _site_eps(spec), spec.grid_shape, spec.resolution)
    assert got.finite and finite and got.nonfinite == 0
    # float products, double sums across rows (the reference sums in float32)
    assert got.energy == pytest.approx(energy, rel=1e-6)
    assert np.float32(got.max_field) == np.float32(max_field)
    again = R.field_diagnostics(st, prog)
    assert again.energy == got.energy  # fixed partition and order: identical


def test_nonfinite_values_are_counted_and_left_out():
    spec = scenario_3d(grid=(9, 12, 40), seed=4, nsteps=4)
    fields = random_initial_fields(spec, seed=12)
    planted = {k: v.copy() for k, v in fields.items()}
    planted["Ey"].reshape(-1)[5] = np.nan
    planted["Hz"].reshape(-1)[17] = np.inf
    planted["Hz"].reshape(-1)[18] = -np.inf
    prog = R.compile_program(spec)
    got = R.field_diagnostics(R.initial_state(prog, fields=planted), prog)
    assert not got.finite and got.nonfinite == 3
    clean = {k: np.where(np.isfinite(v), v, 0.0).astype(np.float32) for k, v in planted.items()}
    energy, max_field, _ = O.field_diagnostics(clean, _site_eps(spec), spec.grid_shape, spec.resolution)
    assert got.energy == pytest.approx(energy, rel=1e-6)
    assert np.float32(got.max_field) == np.float32(max_field)


@pytest.mark.parametrize("dims", [3, 2])
def test_monitor_change_matches_the_oracle(dims):
    spec = (scenario_3d(grid=(9, 12, 40), seed=5, nsteps=40) if dims == 3
            else scenario_2d(grid=(17, 23), polarization="tm", nsteps=40))
    prog = R.compile_program(spec)
    st = R.initial_state(prog, fields=random_initial_fields(spec, seed=13))
    R.run_steps(st, prog, 9)
    first, finite = R.dft_change(st, prog)
    assert first is None and finite
    before = st.numpy()
    R.run_steps(st, prog, 11)
    change, finite = R.dft_change(st, prog)
    after = st.numpy()
    cur, prev = {}, {}
    for m, mon in enumerate(spec.monitors):
        voff, nf, npts, _ = prog.arena.layout[m]
        for c in range(6):
            if mon.component_mask[c] <= 0:
                continue
            for f in range(nf):
                sl = slice(voff + (c * nf + f) * npts, voff + (c * nf + f + 1) * npts)
                cur[(m, c, f)] = after["dft_re"][sl].astype(np.float64) + 1j * after["dft_im"][sl]
                prev[(m, c, f)] = before["dft_re"][sl].astype(np.float64) + 1j * before["dft_im"][sl]
    assert finite
    assert change == pytest.approx(O.relative_monitor_change(cur, prev), rel=1e-9)


def _pulse_scene(total=420):
    """An 8 um vacuum square at 10 points per 1 um wavelength with a 1 um CPML,
    a soft Ez pulse that ends at step 65, and an Ez line monitor across the
    far side (the reference's pulse-convergence scene)."""
    wavelength = 1e-6
    res = wavelength / 10
    n = 80
    dt = 0.7 * res / (P.LIGHT_SPEED * np.sqrt(2.0))
    f0 = P.LIGHT_SPEED / wavelength
    step = np.arange(total)
    signal = (np.exp(-0.5 * ((step - 24) / 7.0) ** 2) * np.cos(2.0 * np.pi * f0 * step * dt)).astype(np.float32)
    signal[65:] = 0.0
    h_terms, e_terms = P.plan_cpml((n, n), dt, res, pml_cells=10, polarization="tm")
    eps = np.ones((n, n), np.float32)
    site = P.site_values_2d(eps, "Ez", "tm")
    e_site = {"Ez": (np.float32(1.0), P.e_source_2d(site, dt))}
    src = P.SourcePlan("Ez", "pre_e", (40, 20), np.array([[-dt / P.EPS_0]], np.float32), signal)
    rows = np.arange(20, 61)
    idx, w = [], []
    for c in P.COMPONENTS:
        sy, sx = P.component_shape(c, (n, n), "tm")
        idx.append((np.minimum(rows, sy - 1) * sx + min(60, sx - 1)).astype(np.int32)[:, None])
        w.append(np.ones((rows.size, 1), np.float32))
    mask = np.array([0, 0, 1, 0, 0, 0], np.float32)
    mon = P.DftMonitorPlan(np.array([f0], np.float32), idx, w, mask)
    return P.ProgramSpec((n, n), dt, res, polarization="tm", e_site=e_site, e_site_eps={"Ez": site},
                         h_terms=h_terms, e_terms=e_terms, sources=[src], monitors=[mon], total_steps=total)


def test_pulse_convergence_keeps_the_frequency_domain_result():
    spec = _pulse_scene()
    policy = T.AutoTermination(field_decay=1e-5, monitor_change=1e-3, source_decay=1e-6, chunk_steps=30,
                               consecutive_checks=3)
    prog = R.compile_program(spec)
    bounded = R.initial_state(prog)
    report = T.run_until_terminated(bounded, prog, policy)
    full = R.initial_state(prog)
    R.run_steps(full, prog, spec.total_steps)
    assert report.reason == "converged" and report.converged
    assert report.steps < spec.total_steps and report.steps == bounded.step
    assert report.source_decay == 0.0
    assert report.field_decay <= policy.field_decay
    assert report.monitor_change is not None and report.monitor_change <= policy.monitor_change
    a, b = bounded.numpy(), full.numpy()
    za = a["dft_re"].astype(np.float64) + 1j * a["dft_im"]
    zb = b["dft_re"].astype(np.float64) + 1j * b["dft_im"]
    assert np.linalg.norm(za - zb) / max(np.linalg.norm(za), np.linalg.norm(zb)) < 5e-3
    np.testing.assert_allclose(a["dft_w"], b["dft_w"])


def test_nonfinite_fields_stop_the_run_at_the_first_check():
    spec = _pulse_scene(total=200)
    prog = R.compile_program(spec)
    fields = {c: np.zeros(P.component_shape(c, spec.grid_shape, "tm"), np.float32) for c in ("Ez", "Hx", "Hy")}
    fields["Hx"][3, 3] = np.nan
    st = R.initial_state(prog, fields=fields)
    report = T.run_until_terminated(st, prog, T.AutoTermination(chunk_steps=25))
    assert report.reason == "nonfinite" and report.steps == 25 and not report.converged
