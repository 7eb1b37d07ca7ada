"""Automatic termination on the CPU: the oracle's diagnostics and the host
policy against outputs of the reference's own functions
(``tests/golden/termination.npz``, made by ``tests/golden/make_termination.py``),
a known-answer energy, and the check loop's decisions on synthetic sequences
(beamz/simulation/execute.py:1312-1484)."""

from __future__ import annotations

import types

import numpy as np
import pytest

from beamz_b200 import termination as T
from oracle import fdtd_oracle as O

GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "termination.npz"))
RES = 20e-9


@pytest.mark.parametrize("n,off", [(1, 0.0), (1, 0.5), (5, 0.0), (5, 0.5), (8, 0.0)])
def test_axis_weights_equal_the_reference(n, off):
    got = O.axis_integration_weights(np.arange(n + 1) * RES, off, n + 1 if off == 0.0 else n)
    np.testing.assert_array_equal(got, GOLD[f"axisw_{n}_{off}"])


@pytest.mark.parametrize("case", ["3d", "tm", "te", "3d_nan"])
def test_oracle_diagnostics_match_the_reference(case):
    grid = tuple(int(v) for v in GOLD[f"diag_{case}_grid"])
    comps = [k.split("_field_")[1] for k in GOLD.files if k.startswith(f"diag_{case}_field_")]
    fields = {c: GOLD[f"diag_{case}_field_{c}"] for c in comps}
    eps = {c: GOLD[f"diag_{case}_eps_{c}"] for c in comps if c[0] == "E"}
    energy, max_field, finite = O.field_diagnostics(fields, eps, grid, RES)
    ref = GOLD[f"diag_{case}_result"]
    assert finite == bool(ref[2])
    if finite:
        # The reference sums in float32; the oracle in float64.
        assert energy == pytest.approx(ref[0], rel=1e-6)
        assert np.float32(max_field) == np.float32(ref[1])


def test_unit_fields_integrate_to_the_domain_volume():
    """Every component's control volumes tile the domain, so unit fields hold
    0.5 eps0 eps_r V per E component and 0.5 mu0 V per H component."""
    grid = (3, 4, 5)
    fields = {c: np.ones(O.component_shapes(grid)[c], np.float32) for c in O.COMPONENTS}
    eps = {c: np.full(O.component_shapes(grid)[c], 2.5, np.float32) for c in ("Ex", "Ey", "Ez")}
    energy, max_field, finite = O.field_diagnostics(fields, eps, grid, RES)
    volume = np.prod(grid) * RES**3
    assert energy == pytest.approx(3 * 0.5 * O.EPS_0 * 2.5 * volume + 3 * 0.5 * O.MU_0 * volume, rel=1e-12)
    assert max_field == 1.0 and finite


def test_monitor_change_matches_the_reference():
    keys = [("m", "Ez", 0), ("m", "Ez", 1), ("m", "Ez", 2), ("m", "Hx", 0)]
    cur = {k: GOLD[f"mon_cur_{i}"] for i, k in enumerate(keys)}
    prev = {k: GOLD[f"mon_prev_{i}"] for i, k in enumerate(keys)}
    assert O.relative_monitor_change(cur, prev) == pytest.approx(float(GOLD["mon_change"][0]), rel=1e-12)
    assert O.relative_monitor_change(cur, None) is None


def test_source_activity_matches_the_reference():
    waves = [GOLD[f"src_wave_{i}"] for i in range(4)]
    activity = T.remaining_source_activity(waves, 60)
    np.testing.assert_array_equal(activity, GOLD["src_activity"])
    got = [T.source_residual(activity, s) for s in (0, 10, 30, 59, 60, 75)]
    np.testing.assert_array_equal(got, GOLD["src_residual"])
    with pytest.raises(ValueError):
        T.source_residual(activity, -1)


def test_configured_weight_sums_match_the_reference():
    for (interval, t0, t1, code), want in zip(GOLD["weight_cases"], GOLD["weight_sums"]):
        mon = types.SimpleNamespace(interval=int(interval), t_start=t0, t_end=t1, window_code=int(code))
        assert T.configured_dft_weight_sum(mon, 1e-15, 3e-17, 200) == pytest.approx(float(want), rel=1e-12)


def test_policy_validation():
    with pytest.raises(ValueError):
        T.AutoTermination(field_decay=-1.0)
    with pytest.raises(ValueError):
        T.AutoTermination(monitor_change=float("nan"))
    with pytest.raises(ValueError):
        T.AutoTermination(chunk_steps=0)
    with pytest.raises(ValueError):
        T.AutoTermination(growth_factor=1.0)
    assert T.AutoTermination(monitor_change=None).monitor_change is None


class _Script:
    """A fake run: each check returns the next (energy, max, finite, change, monitors_finite)."""

    def __init__(self, values):
        self.values = list(values)
        self.step = 0

    def advance(self, n):
        self.step += n
        return self.step

    def diagnose(self):
        return self.values.pop(0)


def _run(policy, total, activity, values, use_monitor):
    s = _Script(values)
    return T.decide(policy, total, activity, s.advance, s.diagnose, use_monitor), s


def test_policy_converges_after_consecutive_checks():
    policy = T.AutoTermination(field_decay=1e-3, monitor_change=1e-2, chunk_steps=10, consecutive_checks=3)
    activity = np.r_[np.ones(25), np.zeros(175)]  # sources off from step 25
    energies = [1.0, 2.0, 1.0, 1e-4, 1e-4, 1e-5, 1e-6, 1e-6]
    changes = [None, 0.5, 0.2, 1e-3, 1e-3, 1e-3, 1e-3, 1e-3]
    values = [(e, 1.0, True, c, True) for e, c in zip(energies, changes)]
    report, s = _run(policy, 200, activity, values, use_monitor=True)
    # Checks at steps 10..60: eligible from 30; decayed from 40 -> 40, 50, 60.
    assert report.reason == "converged" and report.converged
    assert report.steps == 60 and report.consecutive_checks == 3
    assert report.peak_energy == 2.0 and report.field_decay == pytest.approx(1e-5 / 2.0)
    assert report.source_decay == 0.0 and report.monitor_change == 1e-3


def test_policy_first_check_has_no_monitor_change():
    policy = T.AutoTermination(field_decay=1.0, monitor_change=1.0, chunk_steps=10, consecutive_checks=1)
    report, _ = _run(policy, 100, np.zeros(100), [(1.0, 1.0, True, None, True), (1.0, 1.0, True, 0.0, True)], True)
    assert report.reason == "converged" and report.steps == 20


def test_policy_diverges_on_growth_after_the_sources():
    policy = T.AutoTermination(chunk_steps=5, growth_checks=3)
    values = [(1.1**n, 1.0, True, None, True) for n in range(10)]
    report, _ = _run(policy, 100, np.zeros(100), values, use_monitor=False)
    # Growth events at checks 2, 3, 4 (each 1.1x the previous check).
    assert report.reason == "diverged" and report.steps == 20


def test_policy_stops_on_nonfinite_values():
    policy = T.AutoTermination(chunk_steps=7)
    values = [(1.0, 1.0, True, None, True), (1.0, 1.0, True, None, False)]
    report, _ = _run(policy, 100, np.zeros(100), values, use_monitor=False)
    assert report.reason == "nonfinite" and report.steps == 14
    values = [(float("nan"), 1.0, True, None, True)]
    report, _ = _run(policy, 100, np.zeros(100), values, use_monitor=False)
    assert report.reason == "nonfinite" and report.steps == 7


def test_policy_time_limit_with_a_partial_last_chunk():
    policy = T.AutoTermination(chunk_steps=30)
    values = [(1.0, 1.0, True, None, True)] * 4
    report, s = _run(policy, 100, np.ones(100), values, use_monitor=False)
    assert report.reason == "time_limit" and report.steps == 100 and not report.converged


def test_run_needs_a_criterion():
    spec = types.SimpleNamespace(monitors=[], sources=[], total_steps=10)
    with pytest.raises(ValueError, match="no applicable"):
        T.run_until_terminated(types.SimpleNamespace(step=0), types.SimpleNamespace(spec=spec),
                               T.AutoTermination(field_decay=0.0))
