"""Golden vectors for the S-parameter assembly, from the reference's own code.

Run from the repository root, in a container that has the beamz source tree:

    python -m tests.golden.make_sparams [--reference /path/to/beamz]

It loads ``beamz/analysis/sparameters.py`` by path under the numpy stand-in
for ``jax`` (``_refload.py``), with small stand-ins for the modules it imports
for mode projection and monitor data (unused by the assembly), and replaces
its ``_extract_port_waves_dft`` and ``analysis_inputs`` by functions that
return seeded port waves and monitor records.  ``s_parameters``
(sparameters.py:424-566) then runs its own wave selection, incident floor,
ratios, power balance and ``_modal_dft_flux_diagnostics`` (581-644) on them.

It also loads ``beamz/analysis/mode_projection.py`` (its solver and geometry
imports stood in for) and runs ``_build_port_projection_2d`` (485-535: power
normalisation, mode matrix, pseudo-inverse) with the mode solver replaced by
seeded profiles, then the coefficient step of sparameters.py:377-393 on
seeded field vectors.

Writes ``tests/golden/sparams.npz``.
"""

from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# (tag, is_3d, ports [(name, axis, direction)], source, outputs or None, min_incident_db)
CASES = (
    ("c3x", True, (("in", "x", "+"), ("out", "x", "-"), ("drop", "y", "+")), "in", None, -40.0),
    ("c3z", True, (("a", "z", "-"), ("b", "z", "+")), "a", ("b",), -20.0),
    ("c2", False, (("p1", "x", "+"), ("p2", "y", "-")), "p2", None, -30.0),
)
# (tag, points, measure: "scalar" or "array", signed flux sign)
PROJ_CASES = (("pu", 23, "scalar", -1.0), ("pw", 31, "array", 1.0))
DIAG_KEYS = ("P_in", "P_guided_out", "power_sum", "loss_est", "valid_mask")
FLUX_KEYS = ("monitor_flux", "P_plus", "P_minus", "P_modal_sum", "P_modal_net", "P_selected", "P_rejected",
             "P_selected_modal_net", "flux_minus_modal_net", "flux_minus_selected_modal_net",
             "abs_flux_minus_modal_sum")


def _stub(name, **attrs):
    mod = types.ModuleType(name)
    mod.__path__ = []
    for k, v in attrs.items():
        setattr(mod, k, v)
    sys.modules[name] = mod
    return mod


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("BEAMZ_REFERENCE_ROOT"),
                    help="root of the beamz source tree (or set BEAMZ_REFERENCE_ROOT)")
    ap.add_argument("--out", default=os.path.join(HERE, "sparams.npz"))
    args = ap.parse_args(argv)
    if not args.reference:
        ap.error("--reference (or BEAMZ_REFERENCE_ROOT) is required")
    os.environ["BEAMZ_REFERENCE_ROOT"] = args.reference
    from ._refload import _load, load_reference

    load_reference()
    _load("beamz.devices._immutable", "beamz/devices/_immutable.py")

    class Port:  # the attributes sparameters.py reads (beamz/devices/ports.py)
        def __init__(self, name, axis, direction):
            self.name, self.axis, self.direction, self.monitor_name = name, axis, direction, name

    _stub("beamz.analysis")
    _stub("beamz.analysis.mode_projection")
    _stub("beamz.analysis.data", analysis_inputs=None)
    _stub("beamz.analysis.modal_projection")
    _stub("beamz.analysis.modal_projection.colocation", _colocate_field_components_to_projection_3d=None)
    _stub("beamz.analysis.modal_projection.diagnostics", _modal_projection_reconstruction_residual=None)
    _stub("beamz.analysis.modal_projection.geometry", _apply_modal_projection_spatial_phase=None,
          _monitor_projection_phase=None)
    _stub("beamz.devices.ports", Port=Port)
    sp = _load("beamz.analysis.sparameters", "beamz/analysis/sparameters.py")

    rng = np.random.default_rng(57)
    F = 7
    data = {"F": np.int32(F)}
    for tag, is_3d, ports, source, outputs, floor in CASES:
        freqs = np.linspace(1.8e14, 2.1e14, F)
        waves, inputs = {}, {}
        for n, (name, _axis, _d) in enumerate(ports):
            for br in ("plus", "minus"):
                amp = (rng.standard_normal(F) + 1j * rng.standard_normal(F)) * rng.uniform(0.1, 2.0)
                if name == source and n == 0:
                    amp[1] *= 1e-3  # below a -40 dB floor: masked
                waves.setdefault(name, {})[f"a_{br}"] = amp
                data[f"{tag}_{name}_a_{br}"] = amp
            w = waves[name]
            w["P_plus"], w["P_minus"] = np.abs(w["a_plus"]) ** 2, np.abs(w["a_minus"]) ** 2
            flux = rng.standard_normal(F)
            data[f"{tag}_{name}_flux"] = flux
            inputs[name] = types.SimpleNamespace(is_3d=is_3d, frequencies=freqs, fields={"flux": flux})
        data[f"{tag}_freqs"] = freqs
        sp.analysis_inputs = lambda _x, inputs=inputs: inputs
        sp._extract_port_waves_dft = lambda *_a, waves=waves, **_k: waves
        res = sp.s_parameters(None, source, [Port(*p) for p in ports], output_ports=outputs, frequencies=freqs,
                              min_incident_db=floor)
        for (o, s), v in res.s_matrix.items():
            data[f"{tag}_S_{o}_{s}"] = np.asarray(v)
        for key in DIAG_KEYS:
            data[f"{tag}_{key}"] = np.asarray(res.diagnostics[key])
        for name, entry in res.diagnostics["monitor_flux_checks"].items():
            for key in FLUX_KEYS:
                data[f"{tag}_{name}_{key}"] = np.asarray(entry[key])
            data[f"{tag}_{name}_incident"] = np.asarray(entry["incident_wave"])
    _stub("beamz.analysis.modal_projection.colocation", _discrete_mode_projection_grids_3d=None)
    _stub("beamz.analysis.modal_projection.diagnostics",
          _modal_projection_reconstruction_diagnostics_from_matrix=None)
    _stub("beamz.analysis.modal_projection.geometry", _analysis_plane_sample_area=None,
          _modal_projection_plane_delay_s=None, _mode_components_for_port=None, _monitor_analysis_plane_3d=None)
    _stub("beamz.analysis.data", AnalysisData=object)
    _stub("beamz.devices._placement", line_region_points=None, snap_axis_aligned_line_region_grid=None,
          snap_plane_region_grid=None)
    _stub("beamz.devices.modes")
    _stub("beamz.devices.modes.discrete", DISCRETE_MODE_CONTRACT=None, solve_beamz_mode=None)
    _stub("beamz.devices.modes.fields", _modal_overlap=None, _normalize_profiles=None)
    _stub("beamz.devices.modes.plane", solve_mode_plane_3d=None, solve_modes=None)
    _stub("beamz.devices.monitors")
    _stub("beamz.devices.monitors.monitors", ModeMonitor=object)
    mp = _load("beamz.analysis.mode_projection", "beamz/analysis/mode_projection.py")
    for tag, n, kind, sign in PROJ_CASES:
        e = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * 3.0
        h = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * 0.01
        dl = np.float64(2e-8) if kind == "scalar" else rng.uniform(1e-8, 3e-8, n)
        mp._monitor_profile_slice = lambda *_a, n=n, dl=dl: (np.ones(n), np.arange(n), dl)
        mp.solve_modes = lambda *_a, e=e, h=h, **_k: ([1.7], [[e]], [[h]], None)
        mp._modal_projection_plane_delay_s = lambda *_a: 0.0
        spec = types.SimpleNamespace(mode_index=0, projection_direction="+", polarization=None, name=tag)
        parts = {"axis": "x", "e_mode_index": 0, "h_mode_index": 0, "signed_flux_sign": sign,
                 "e_component": "Ez", "h_component": "Hy"}
        proj = mp._build_port_projection_2d(types.SimpleNamespace(resolution=2e-8), spec=spec, monitor=None,
                                            frequency=1.9e14, parts=parts, mode_pad_cells=0)
        field_vec = rng.standard_normal(2 * n) + 1j * rng.standard_normal(2 * n)
        pw = np.asarray(proj.get("projection_weights", np.ones(field_vec.size)), dtype=float)
        coeff = proj["pinv"] @ (pw * field_vec)
        data.update({f"{tag}_e": e, f"{tag}_h": h, f"{tag}_dl": np.asarray(dl), f"{tag}_field": field_vec,
                     f"{tag}_mode_matrix": proj["mode_matrix"], f"{tag}_pinv": proj["pinv"],
                     f"{tag}_cond": np.float64(proj["condition_number"]), f"{tag}_coeff": coeff})
    np.savez(args.out, **data)
    print(f"wrote {args.out} ({len(data)} arrays)")


if __name__ == "__main__":
    main()
