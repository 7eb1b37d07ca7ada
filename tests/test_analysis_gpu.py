"""Monitor analysis on the device (fdtd_monitor_reduce): the DFT flux and
modal overlaps of a run's monitors against the oracle's restatement of beamz
(pinned in tests/test_analysis.py) applied to a host copy of the same arena.
The sums run in another order than numpy's, so the bound is relative to the
sum of the terms' magnitudes (1e-12, double accumulation)."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from beamz_b200 import runtime as R  # noqa: E402
from oracle import fdtd_oracle as O  # noqa: E402
from tests.scenarios import random_initial_fields, scenario_2d, scenario_3d  # noqa: E402

pytestmark = pytest.mark.gpu


def _run(spec, steps, schedule="fused"):
    prog = R.compile_program(spec, schedule=schedule)
    st = R.run_steps(R.initial_state(prog, fields=random_initial_fields(spec, seed=2)), prog, steps)
    return prog, st


def _normalised(state, prog, m, base_dt):
    values = R.monitor_values(state, prog, m)
    _voff, nf, _npts, woff = prog.arena.layout[m]
    wsum = state.dft_w[woff:woff + nf].cpu().numpy()
    freqs = np.asarray(prog.spec.monitors[m].freqs, dtype=float)
    return {c: O.flux_component(v, wsum, c, freqs, base_dt) for c, v in values.items()}


@pytest.mark.parametrize("base_dt", [0.0, 3.7e-17])
@pytest.mark.parametrize("layout", ["pitched", "dense"])
def test_device_flux_matches_the_oracle(layout, base_dt):
    spec = scenario_3d(grid=(10, 14, 30), seed=4, nsteps=24)
    prog, st = _run(spec, 24, "fused" if layout == "pitched" else "phases")
    assert prog.layout == layout
    rng = np.random.default_rng(1)
    for m, axis in ((0, "x"), (1, "z")):
        npts = prog.arena.layout[m][2]
        iw = rng.uniform(0.5, 1.5, npts) * 4e-16
        got = R.monitor_dft_flux(st, prog, m, axis, sign=-1.0, integration_weights=iw, base_dt=base_dt)
        fields = _normalised(st, prog, m, base_dt)
        want = O.monitor_dft_flux(fields, axis, -1.0, iw)
        e1, e2, h1, h2 = O.TANGENTIAL_COMPONENTS[axis]
        terms = np.abs(fields[e1] * fields[h1]) + np.abs(fields[e2] * fields[h2])  # [F, P]
        scale = 0.5 * np.sum(terms * iw, axis=1)
        assert np.all(np.abs(got - want) <= 1e-12 * scale), (got, want)
        assert np.any(np.abs(want) > 1e-6 * scale)
        # a constant measure instead of per-point weights
        got_m = R.monitor_dft_flux(st, prog, m, axis, measure=2.5e-16, base_dt=base_dt)
        want_m = O.monitor_dft_flux(fields, axis, 1.0, None, measure=2.5e-16)
        assert np.all(np.abs(got_m - want_m) <= 1e-12 * 0.5 * np.sum(terms, axis=1) * 2.5e-16)


@pytest.mark.parametrize("kind", ["mapping", "array", "scalar"])
def test_device_modal_overlap_matches_the_oracle(kind):
    spec = scenario_3d(grid=(10, 14, 30), seed=5, nsteps=24)
    prog, st = _run(spec, 24)
    m, axis = 0, "x"
    _voff, nf, npts, _woff = prog.arena.layout[m]
    names = O.TANGENTIAL_COMPONENTS[axis]
    rng = np.random.default_rng(7)
    cplx = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)  # noqa: E731
    modes = [{c: cplx(nf, npts) * 1e-3 for c in names}, {c: cplx(npts) for c in names}]
    measure = ({c: rng.uniform(0.5, 1.5, npts) for c in names[:2]} if kind == "mapping"
               else rng.uniform(0.5, 1.5, npts) if kind == "array" else 0.8)
    got = R.modal_overlap(st, prog, m, modes, axis, measure, direction_sign=-1.0, base_dt=2.9e-17)
    assert got.shape == (2, nf)
    fields = _normalised(st, prog, m, 2.9e-17)
    for r, mode in enumerate(modes):
        for f in range(nf):
            mf = {c: np.broadcast_to(np.asarray(mode[c]).reshape(-1, npts), (nf, npts))[f] for c in names}
            ff = {c: fields[c][f] for c in names}
            want = O.modal_overlap(ff, mf, axis, measure, -1.0)
            scale = 0.0
            for q in range(2):
                e, h = names[q], names[2 + q]
                w = measure[e] if isinstance(measure, dict) else np.broadcast_to(measure, (npts,))
                scale += 0.25 * np.sum(w * (np.abs(ff[e] * mf[h]) + np.abs(mf[e] * ff[h])))
            assert abs(got[r, f] - want) <= 1e-12 * scale, (got[r, f], want)
            assert abs(want) > 1e-6 * scale


def test_device_flux_of_a_2d_line_monitor():
    spec = scenario_2d(grid=(23, 29), polarization="tm", nsteps=30)
    prog, st = _run(spec, 30)
    got = R.monitor_dft_flux(st, prog, 0, "x", measure=20e-9)
    want = O.monitor_dft_flux(_normalised(st, prog, 0, None), "x", 1.0, None, measure=20e-9)
    np.testing.assert_allclose(got, want, rtol=1e-10)


def test_s_parameters_from_device_dft_values():
    """The S-parameter path on a device run: two x-normal lines of a 2D TM
    scene, their DFT values (Ez, Hy phase-aligned) projected on a mode that is
    the input line's own field, then assembled.  Projecting a field on itself
    gives a pure forward wave (a_plus = its power normalisation, a_minus = 0),
    so the input port reflects nothing."""
    from beamz_b200 import sparameters as S
    from beamz_b200 import workloads as W

    spec = W.scene_2d(total_steps=240, seed=2, shape=(96, 96), pml_cells=10, n_monitors=2)
    prog = R.compile_program(spec)
    st = R.initial_state(prog)
    R.run_steps(st, prog, 240)
    freqs = np.asarray(spec.monitors[0].freqs, dtype=float)
    dl = float(spec.resolution)
    fields = []
    for m in range(2):
        v = R.monitor_values(st, prog, m)
        fields.append((v["Ez"], v["Hy"] * S.monitor_projection_phase("Hy", freqs, spec.dt)[:, None]))
    waves = {"in": {"a_plus": [], "a_minus": []}, "out": {"a_plus": [], "a_minus": []}}
    e_in, h_in = fields[0]
    for f in range(len(freqs)):
        proj = S.port_projection(e_in[f], h_in[f], dl, -1.0)
        power = 0.5 * np.real(np.sum(dl * -1.0 * e_in[f] * np.conjugate(h_in[f])))
        for name, (e, h) in zip(("in", "out"), fields):
            ap, am = S.project_waves(proj, e[f], h[f])
            waves[name]["a_plus"].append(ap)
            waves[name]["a_minus"].append(am)
        assert abs(waves["in"]["a_plus"][-1] - np.sqrt(abs(power))) <= 1e-9 * np.sqrt(abs(power))
        assert abs(waves["in"]["a_minus"][-1]) <= 1e-9 * np.sqrt(abs(power))
    flux = {p: R.monitor_dft_flux(st, prog, m, "x", measure=dl) for m, p in enumerate(("in", "out"))}
    ports = [S.PortSpec("in", "x", "+"), S.PortSpec("out", "x", "+")]
    res = S.s_parameters(waves, ports, "in", frequencies=freqs, is_3d=False, monitor_flux=flux)
    assert res.diagnostics["valid_mask"].all()
    assert np.abs(res.s_matrix[("in", "in")]).max() <= 1e-9
    s21 = res.s_matrix[("out", "in")]
    assert np.isfinite(s21).all() and np.abs(s21).max() > 0
    np.testing.assert_allclose(res.diagnostics["P_in"], np.abs(np.asarray(waves["in"]["a_plus"])) ** 2)
    assert np.isfinite(res.diagnostics["monitor_flux_checks"]["out"]["monitor_flux"]).all()
