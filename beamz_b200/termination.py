"""Automatic termination: chunked runs stopped on convergence, divergence or
non-finite fields (beamz/simulation/execute.py:1312-1484, run_until_terminated;
policy beamz/simulation/model.py:336-396, AutoTermination; report
beamz/simulation/results.py:97-125, RunTermination).

The engine advances whole chunks on the device; between chunks two device
reductions (:func:`beamz_b200.runtime.field_diagnostics` and
:func:`beamz_b200.runtime.dft_change`) supply the energy, the largest
|field|, finiteness and the monitors' relative change, and the host applies the
reference's rules:

* a check is *eligible* once every source's remaining drive is at most
  ``source_decay`` of its peak and the step is at least ``min_steps``;
* it *succeeds* when the energy is at most ``field_decay`` of its running peak
  and (if monitors are watched) the monitor change is at most
  ``monitor_change``; ``consecutive_checks`` successes in a row converge;
* after the sources are off, an energy above ``growth_factor`` times the
  previous check's is a growth event; ``growth_checks`` in a row diverge;
* a non-finite field, energy or monitor value stops the run at once;
* the configured step count is a hard limit ("time_limit").

On convergence each monitor's DFT weight sum is completed to its value at the
time limit (beamz/simulation/execute.py:319-352), as though the negligible tail
had been sampled.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class AutoTermination:
    """Chunked convergence checks (beamz/simulation/model.py:336-396).

    ``monitors`` selects DFT monitors by index (beamz selects them by name);
    empty selects every monitor with a frequency, a point and an unmasked
    component.
    """

    field_decay: float = 1e-5
    monitor_change: float | None = 1e-3
    source_decay: float = 1e-6
    chunk_steps: int = 256
    min_steps: int = 0
    consecutive_checks: int = 3
    monitors: tuple = ()
    growth_factor: float = 1.05
    growth_checks: int = 3

    def __post_init__(self) -> None:
        for name in ("field_decay", "source_decay"):
            value = float(getattr(self, name))
            if not np.isfinite(value) or value < 0.0:
                raise ValueError(f"AutoTermination.{name} must be finite and non-negative.")
            object.__setattr__(self, name, value)
        if self.monitor_change is not None:
            value = float(self.monitor_change)
            if not np.isfinite(value) or value < 0.0:
                raise ValueError("AutoTermination.monitor_change must be finite, non-negative, or None.")
            object.__setattr__(self, "monitor_change", value)
        for name in ("chunk_steps", "consecutive_checks", "growth_checks"):
            if int(getattr(self, name)) < 1:
                raise ValueError(f"AutoTermination.{name} must be a positive integer.")
            object.__setattr__(self, name, int(getattr(self, name)))
        if int(self.min_steps) < 0:
            raise ValueError("AutoTermination.min_steps must be non-negative.")
        growth = float(self.growth_factor)
        if not np.isfinite(growth) or growth <= 1.0:
            raise ValueError("AutoTermination.growth_factor must be finite and greater than one.")
        object.__setattr__(self, "growth_factor", growth)
        object.__setattr__(self, "monitors", tuple(int(m) for m in self.monitors))


@dataclass(frozen=True)
class RunTermination:
    """Why a bounded run stopped and its final residuals
    (beamz/simulation/results.py:97-125)."""

    reason: str  # "converged" | "time_limit" | "nonfinite" | "diverged"
    steps: int
    time: float
    converged: bool
    field_decay: float | None = None
    monitor_change: float | None = None
    source_decay: float | None = None
    energy: float | None = None
    peak_energy: float | None = None
    max_field: float | None = None
    consecutive_checks: int = 0


def remaining_source_activity(waveforms, total_steps: int) -> np.ndarray:
    """Largest future drive of any source relative to its own peak, per step
    (beamz/simulation/execute.py:225-244): waveforms shorter than the run hold
    their last sample."""
    total_steps = int(total_steps)
    activity = np.zeros(total_steps, dtype=np.float64)
    for wave in waveforms:
        w = np.abs(np.asarray(wave, dtype=np.float64).reshape(-1))
        if w.size == 0:
            continue
        peak = float(np.max(w, initial=0.0))
        if peak > 0.0:
            sampled = np.empty(total_steps, dtype=np.float64)
            n = min(total_steps, w.size)
            sampled[:n] = w[:n]
            if n < total_steps:
                sampled[n:] = w[-1]
            activity = np.maximum(activity, sampled / peak)
    return np.maximum.accumulate(activity[::-1])[::-1] if activity.size else activity


def source_residual(activity: np.ndarray, step: int) -> float:
    """Normalised source drive at or after ``step`` (execute.py:247-252)."""
    if int(step) < 0:
        raise ValueError("current_step must be non-negative.")
    return float(activity[int(step)]) if int(step) < activity.size else 0.0


def configured_dft_weight_sum(monitor, t0: float, dt: float, total_steps: int) -> float:
    """A monitor's DFT window weight over the configured run
    (beamz/simulation/execute.py:319-337)."""
    steps = np.arange(int(total_steps), dtype=np.int64)
    times = float(t0) + (steps.astype(np.float64) + 1.0) * float(dt)
    selected = ((steps % max(1, int(monitor.interval)) == 0) & (times >= float(monitor.t_start))
                & (times <= float(monitor.t_end)))
    if not np.any(selected):
        return 0.0
    if int(monitor.window_code) != 1 or not np.isfinite(monitor.t_end):
        return float(np.count_nonzero(selected))
    span = max(float(monitor.t_end) - float(monitor.t_start), 1e-30)
    tau = np.clip((times[selected] - float(monitor.t_start)) / span, 0.0, 1.0)
    return float(np.sum(0.5 * (1.0 - np.cos(2.0 * np.pi * tau))))


def applicable_monitors(monitors) -> tuple:
    """Indices of monitors with a frequency, a point and an unmasked component
    (execute.py:255-275)."""
    return tuple(i for i, m in enumerate(monitors)
                 if len(m.freqs) > 0 and m.points > 0 and np.any(np.asarray(m.component_mask) > 0.0))


def decide(policy: AutoTermination, total_steps: int, activity: np.ndarray, advance, diagnose, use_monitor: bool):
    """The reference's check loop (execute.py:1350-1455) over injected device
    work: ``advance(steps)`` runs a chunk and returns the step reached;
    ``diagnose()`` returns (energy, max_field, fields_finite, monitor_change,
    monitors_finite) for the state after it.  Returns a RunTermination without
    its time (the caller knows the clock)."""
    tiny = np.finfo(float).tiny
    chunk = min(int(policy.chunk_steps), int(total_steps))
    step = 0
    previous_energy = None
    energy = peak_energy = max_field = 0.0
    field_decay = monitor_change = None
    source_decay = source_residual(activity, 0)
    successes = growth = 0
    reason = "time_limit"
    while step < int(total_steps):
        step = advance(min(chunk, int(total_steps) - step))
        energy, max_field, fields_finite, monitor_change, monitors_finite = diagnose()
        if not fields_finite or not np.isfinite(energy) or not monitors_finite:
            reason = "nonfinite"
            break
        peak_energy = max(peak_energy, energy)
        field_decay = energy / peak_energy if peak_energy > tiny else 0.0
        source_decay = source_residual(activity, step)
        source_off = source_decay <= policy.source_decay
        if source_off and previous_energy is not None and previous_energy > tiny and \
                energy > policy.growth_factor * previous_energy:
            growth += 1
        else:
            growth = 0
        if growth >= policy.growth_checks:
            reason = "diverged"
            break
        eligible = source_off and step >= policy.min_steps
        energy_ok = policy.field_decay == 0.0 or field_decay <= policy.field_decay
        monitor_ok = not use_monitor or (monitor_change is not None and policy.monitor_change is not None
                                         and monitor_change <= policy.monitor_change)
        successes = successes + 1 if eligible and energy_ok and monitor_ok else 0
        if successes >= policy.consecutive_checks:
            reason = "converged"
            break
        previous_energy = energy
    return RunTermination(reason=reason, steps=step, time=0.0, converged=reason == "converged",
                          field_decay=field_decay, monitor_change=monitor_change if use_monitor else None,
                          source_decay=source_decay, energy=energy, peak_energy=peak_energy, max_field=max_field,
                          consecutive_checks=successes)


def run_until_terminated(state, program, policy: AutoTermination, total_steps: int | None = None):
    """Advance ``state`` in chunks of ``policy.chunk_steps`` until the policy
    stops it or ``total_steps`` (default: the spec's) have run; returns the
    RunTermination (beamz/simulation/execute.py:1312-1484)."""
    from . import runtime

    spec = program.spec
    total = int(spec.total_steps if total_steps is None else total_steps)
    watched = policy.monitors or applicable_monitors(spec.monitors)
    for m in watched:
        if m not in applicable_monitors(spec.monitors):
            raise ValueError(f"Automatic termination monitors must be applicable frequency-domain monitors: {m}.")
    use_monitor = policy.monitor_change is not None and bool(watched)
    if policy.field_decay == 0.0 and not use_monitor:
        raise ValueError("Automatic termination has no applicable field or monitor criterion.")
    activity = remaining_source_activity([s.waveform for s in spec.sources], total)
    start = state.step

    def advance(n: int) -> int:
        runtime.run_steps(state, program, n)
        state.check()
        return state.step - start

    def diagnose():
        d = runtime.field_diagnostics(state, program)
        change, monitors_finite = runtime.dft_change(state, program, watched) if watched else (None, True)
        return d.energy, d.max_field, d.finite, change, monitors_finite

    state._dft_prev = None  # the first check records the vectors later checks compare with
    report = decide(policy, total, activity, advance, diagnose, use_monitor)
    report = RunTermination(**{**report.__dict__, "time": float(state.t)})
    if report.converged and program.arena is not None:
        complete_dft_weights(state, program, total)
    return report


def complete_dft_weights(state, program, total_steps: int) -> None:
    """Set every monitor's DFT weight sums to their value at the time limit
    (beamz/simulation/execute.py:340-352, _complete_converged_dft_weights)."""
    import torch

    spec = program.spec
    host = state.dft_w.cpu().numpy()
    for m, mon in enumerate(spec.monitors):
        _voff, nf, _p, woff = program.arena.layout[m]
        host[woff:woff + nf] = configured_dft_weight_sum(mon, spec.t0, spec.dt, total_steps)
    state.dft_w.copy_(torch.as_tensor(host, device=state.dft_w.device))
