"""Broadband modal S-parameters from port wave amplitudes.

The last step of beamz's S-parameter extraction
(beamz/analysis/sparameters.py:424-566 ``s_parameters`` and 581-644
``_modal_dft_flux_diagnostics``): given, per port and frequency, the complex
amplitudes of the forward ("plus") and backward ("minus") mode at the port's
monitor, pick each port's incident and scattered wave by its axis and inward
direction, divide every output port's scattered amplitude by the source port's
incident one where that exceeds a floor, and report the power balance and the
monitor-flux cross-checks.

The amplitudes come from projecting a monitor's DFT fields on mode profiles.
``modal_overlap`` in :mod:`beamz_b200.runtime` forms the overlap sums on the
device arena; the mode profiles come from a mode solver, which is outside
this engine. ``monitor_flux`` takes the device flux
(``runtime.monitor_dft_flux``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class PortSpec:
    """A modal port: a name, the monitor that samples it (a name or index,
    as the caller keys ``monitor_flux``), the plane-normal axis ("x", "y" or
    "z") and the inward propagation direction ("+" or "-")
    (beamz/devices/ports.py ``Port``: name, monitor_name, axis, direction)."""

    name: str
    axis: str
    direction: str = "+"
    monitor: object = None

    def __post_init__(self):
        if self.axis not in ("x", "y", "z"):
            raise ValueError(f"port axis must be 'x', 'y' or 'z', got {self.axis!r}")
        if self.direction not in ("+", "-"):
            raise ValueError(f"port direction must be '+' or '-', got {self.direction!r}")

    @property
    def monitor_name(self):
        return self.name if self.monitor is None else self.monitor


@dataclass(frozen=True)
class SParameters:
    """``s_matrix[(output_port, source_port)]``: complex vector over
    ``frequencies``; ``diagnostics``: the power balance and flux checks."""

    s_matrix: dict
    frequencies: np.ndarray
    diagnostics: dict = field(default_factory=dict)


def wave_selectors(port: PortSpec, is_3d: bool) -> tuple[str, str]:
    """(incident, scattered) branch of a port (sparameters.py:99-108): in 3D
    the positive-axis wave of an x- or y-normal port is the "minus" branch."""
    positive_axis_wave = "minus" if is_3d and port.axis in {"x", "y"} else "plus"
    if port.direction == "+":
        incident = positive_axis_wave
    else:
        incident = "minus" if positive_axis_wave == "plus" else "plus"
    return incident, "minus" if incident == "plus" else "plus"


def _safe_ratio(num, den, eps=1e-18):
    out = np.zeros_like(num, dtype=np.complex128)
    valid = np.abs(den) > eps
    out[valid] = num[valid] / den[valid]
    return out


def _ports(ports) -> dict:
    values = tuple(ports.values()) if isinstance(ports, dict) else tuple(ports)
    if not values:
        raise ValueError("ports must contain at least one PortSpec")
    if any(not isinstance(p, PortSpec) for p in values):
        raise TypeError("ports must be PortSpec objects")
    if len({p.name for p in values}) != len(values):
        raise ValueError("port names must be unique")
    return {p.name: p for p in values}


def monitor_projection_phase(component: str, frequencies, dt: float) -> np.ndarray:
    """Phase that aligns a monitor's DFT phasors to the E sample time
    (beamz/analysis/modal_projection/geometry.py:41-60): exp(-i pi f dt) for
    H components (stored half a step earlier), 1 for E."""
    f = np.atleast_1d(np.asarray(frequencies, dtype=float))
    if str(component).startswith("H"):
        return np.exp(-1j * np.pi * f * float(dt))
    return np.ones_like(f, dtype=np.complex128)


def port_projection(e_profile, h_profile, measure, signed_flux_sign: float) -> dict:
    """Least-squares projection of a port's (E, H) DFT fields onto its
    forward and backward mode (beamz/analysis/mode_projection.py:485-535, the
    2D port projection after the mode solve): the solved tangential profiles
    normalised to unit power 0.5 Re sum w s E conj(H), the mode matrix of the
    forward [E; H] and backward [E; -H] fields, and its pseudo-inverse,
    weighted by sqrt(w) when ``measure`` is per point.  The profiles come from
    a mode solver, which is outside this engine."""
    e = np.asarray(e_profile, dtype=np.complex128)
    h = np.asarray(h_profile, dtype=np.complex128)
    measure = np.asarray(measure, dtype=float)
    weights = measure if measure.ndim == 0 else measure.reshape(-1)[: e.size]
    power = 0.5 * np.real(np.sum(weights * signed_flux_sign * e * np.conjugate(h)))
    norm = np.sqrt(max(abs(power), 1e-30))
    e_fwd, h_fwd = e / norm, h / norm
    mode_matrix = np.column_stack([np.concatenate([e_fwd, h_fwd]), np.concatenate([e_fwd, -h_fwd])])
    out = {"mode_matrix": mode_matrix, "condition_number": float(np.linalg.cond(mode_matrix))}
    if np.ndim(weights) == 0:  # uniform measure: the unweighted solve, as beamz keeps it
        out["pinv"] = np.linalg.pinv(mode_matrix)
    else:
        pw = np.concatenate([np.broadcast_to(np.sqrt(weights), e_fwd.shape),
                             np.broadcast_to(np.sqrt(weights), h_fwd.shape)])
        out["pinv"] = np.linalg.pinv(pw[:, None] * mode_matrix)
        out["projection_weights"] = pw
    return out


def project_waves(projection: dict, e_values, h_values) -> tuple[complex, complex]:
    """(a_plus, a_minus) of one frequency: the projection's pseudo-inverse
    applied to the weighted field vector [E; H] (beamz/analysis/sparameters.py
    377-393).  ``e_values`` / ``h_values`` are the monitor's DFT values of the
    port's components (``runtime.monitor_values``) with beamz's phase
    alignment applied (:func:`monitor_projection_phase`, and in 2D the
    modal-plane delay)."""
    field_vec = np.concatenate([np.asarray(e_values, dtype=np.complex128), np.asarray(h_values, dtype=np.complex128)])
    weights = np.asarray(projection.get("projection_weights", np.ones(field_vec.size)), dtype=float)
    coeff = projection["pinv"] @ (weights * field_vec)
    return coeff[0], coeff[1]


def modal_flux_diagnostics(ports, waves: dict, frequencies, is_3d: bool = True, monitor_flux=None) -> dict:
    """Per port: the modal powers of both branches, the selected (scattered)
    and rejected ones, and their differences from the monitor's DFT flux
    (sparameters.py:581-644; NaN where a flux or a power is missing)."""
    freqs = np.atleast_1d(np.asarray(frequencies, dtype=float))
    flux_by_monitor = {} if monitor_flux is None else monitor_flux
    out = {}
    for name, spec in _ports(ports).items():
        wave = waves.get(name, {})

        def power(pkey, akey, wave=wave):
            if pkey in wave:
                p = np.asarray(wave[pkey], dtype=float)
            elif akey in wave:
                p = np.abs(np.asarray(wave[akey], dtype=np.complex128)) ** 2
            else:
                p = np.asarray([], dtype=float)
            return p if p.size == freqs.size else np.full(freqs.shape, np.nan, dtype=float)

        p_plus, p_minus = power("P_plus", "a_plus"), power("P_minus", "a_minus")
        incident, scattered = wave_selectors(spec, is_3d)
        selected, rejected = (p_plus, p_minus) if scattered == "plus" else (p_minus, p_plus)
        flux = flux_by_monitor.get(spec.monitor_name)
        flux = (np.full(freqs.shape, np.nan, dtype=float) if flux is None
                else np.asarray(flux, dtype=float).reshape(freqs.shape))
        modal_net = p_plus - p_minus
        out[name] = {
            "monitor": spec.monitor_name,
            "monitor_flux": flux,
            "incident_wave": incident,
            "scattered_wave": scattered,
            "P_plus": p_plus,
            "P_minus": p_minus,
            "P_modal_sum": p_plus + p_minus,
            "P_modal_net": modal_net,
            "P_selected": selected,
            "P_rejected": rejected,
            "P_selected_modal_net": selected - rejected,
            "flux_minus_modal_net": flux - modal_net,
            "flux_minus_selected_modal_net": flux - (selected - rejected),
            "abs_flux_minus_modal_sum": np.abs(flux) - (p_plus + p_minus),
        }
    return out


def s_parameters(waves: dict, ports, source_port: str, output_ports=None, frequencies=None,
                 min_incident_db: float = -40.0, is_3d: bool = True, monitor_flux=None) -> SParameters:
    """S[(out, source)] = scattered amplitude at ``out`` / incident amplitude
    at ``source_port`` (sparameters.py:424-566), zero where the incident
    amplitude is below ``min_incident_db`` relative to its peak.

    ``waves[port]`` holds ``a_plus`` and ``a_minus`` (complex, one per
    frequency; ``P_plus`` / ``P_minus`` optional), ``frequencies`` the grid
    they are on (the source monitor's DFT frequencies), ``monitor_flux`` an
    optional mapping monitor -> DFT flux per frequency for the cross-checks."""
    port_map = _ports(ports)
    if source_port not in port_map:
        raise ValueError(f"source_port '{source_port}' not found in ports")
    names = list(port_map) if output_ports is None else list(output_ports)
    missing = [n for n in names if n not in port_map]
    if missing:
        raise ValueError(f"output_ports contains unknown ports: {missing}")
    if frequencies is None:
        raise ValueError("frequencies (the grid of the wave amplitudes) is required")
    frequencies = np.atleast_1d(np.asarray(frequencies, dtype=float))

    incident_branch, _ = wave_selectors(port_map[source_port], is_3d)
    a_incident = np.asarray(waves[source_port][f"a_{incident_branch}"], dtype=np.complex128)
    max_incident = float(np.max(np.abs(a_incident))) if a_incident.size else 0.0
    abs_floor = max(1e-18, max_incident * (10.0 ** (float(min_incident_db) / 20.0)))
    valid = np.abs(a_incident) >= abs_floor

    scattered_waves, s_matrix = {}, {}
    for out_port in names:
        _, branch = wave_selectors(port_map[out_port], is_3d)
        b_out = np.asarray(waves[out_port][f"a_{branch}"], dtype=np.complex128)
        scattered_waves[out_port] = b_out
        s_matrix[(out_port, source_port)] = np.where(valid, _safe_ratio(b_out, a_incident), 0.0 + 0.0j)

    p_in = np.abs(a_incident) ** 2
    p_out = np.zeros_like(p_in, dtype=float)
    for out_port in names:
        p_out += np.abs(scattered_waves[out_port]) ** 2
    power_sum = p_out / np.maximum(p_in, 1e-18)
    loss = 1.0 - power_sum
    diagnostics = {
        "frequencies": frequencies,
        "source_port": source_port,
        "output_ports": names,
        "P_in": p_in,
        "P_guided_out": p_out,
        "power_sum": np.where(valid, power_sum, np.nan),
        "loss_est": np.where(valid, loss, np.nan),
        "valid_mask": valid,
        "monitor_flux_checks": modal_flux_diagnostics(port_map, waves, frequencies, is_3d, monitor_flux),
        "scattered_waves": scattered_waves,
    }
    return SParameters(s_matrix, frequencies, diagnostics)
