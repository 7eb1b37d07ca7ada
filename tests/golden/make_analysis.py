"""Golden vectors for monitor analysis (DFT flux, modal overlap), from the
reference's own code.

Run from the repository root, in a container that has the beamz source tree:

    python -m tests.golden.make_analysis [--reference /path/to/beamz]

It runs, on seeded float32 DFT values (as an arena holds them):

* ``monitor_dft_flux`` (``beamz/simulation/observe.py:198-234``, with
  ``monitor_dft_component`` 166-179 and ``_flux_component`` 182-187) on a
  monitor record carrying ``dft_fields``, ``dft_weight_sum``,
  ``dft_frequencies``, ``dft_base_dt`` and integration weights or a power
  scale, loaded by path under the numpy stand-in for ``jax`` (``_refload.py``);
* ``_modal_overlap`` (``beamz/devices/modes/fields.py:76-129``), loaded by path.

Writes ``tests/golden/analysis.npz``.
"""

from __future__ import annotations

import argparse
import os
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")

# (tag, normal axis, sign, base dt or 0, integration weights?)
FLUX_CASES = (("fx", "x", 1.0, 3.1e-17, True), ("fy", "y", -1.0, 0.0, True), ("fz", "z", 1.0, 2.7e-17, False))
# (tag, axis, direction sign, measure kind)
OVERLAP_CASES = (("ox", "x", 1.0, "mapping"), ("oy", "y", -1.0, "array"), ("oz", "z", 1.0, "scalar"))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("BEAMZ_REFERENCE_ROOT"),
                    help="root of the beamz source tree (or set BEAMZ_REFERENCE_ROOT)")
    ap.add_argument("--out", default=os.path.join(HERE, "analysis.npz"))
    args = ap.parse_args(argv)
    if not args.reference:
        ap.error("--reference (or BEAMZ_REFERENCE_ROOT) is required")
    os.environ["BEAMZ_REFERENCE_ROOT"] = args.reference
    from ._refload import _load, load_reference

    ref = load_reference()
    modes = _load("beamz.devices.modes.fields", "beamz/devices/modes/fields.py")
    rng = np.random.default_rng(31)
    F, P = 3, 57
    data = {"F": np.int32(F), "P": np.int32(P)}
    for tag, axis, sign, base_dt, with_iw in FLUX_CASES:
        re = rng.standard_normal((6, F, P)).astype(np.float32)
        im = rng.standard_normal((6, F, P)).astype(np.float32)
        wsum = rng.uniform(5.0, 50.0, F).astype(np.float32)
        freqs = (rng.uniform(1.5e14, 2.5e14, F)).astype(np.float32)
        iw = rng.uniform(0.5, 1.5, P) * 4e-16 if with_iw else np.zeros(0)
        monitor = types.SimpleNamespace(
            name=tag, dft_fields={c: (re[i] + 1j * im[i]).reshape(-1) for i, c in enumerate(COMPONENTS)},
            dft_weight_sum=wsum, dft_frequencies=freqs, dft_base_dt=base_dt,
            resolution=20e-9, normal_axis="xyz".index(axis), normal_sign=sign, integration_weights=iw,
            power_scale=0.0 if with_iw else 3.3e-16,
            monitor=types.SimpleNamespace(freqs=freqs, is_3d=True, start=None, end=None, plane_normal=axis))
        flux = ref.observe.monitor_dft_flux(monitor)
        data.update({f"{tag}_re": re, f"{tag}_im": im, f"{tag}_wsum": wsum, f"{tag}_freqs": freqs,
                     f"{tag}_iw": iw, f"{tag}_base_dt": np.float64(base_dt),
                     f"{tag}_power_scale": np.float64(monitor.power_scale), f"{tag}_flux": np.asarray(flux)})
    for tag, axis, direction, kind in OVERLAP_CASES:
        names = modes._TANGENTIAL_COMPONENTS[axis]
        fields = {c: rng.standard_normal(P) + 1j * rng.standard_normal(P) for c in names}
        mode = {c: rng.standard_normal(P) + 1j * rng.standard_normal(P) for c in names}
        if kind == "mapping":
            measure = {c: rng.uniform(0.5, 1.5, P) for c in names[:2]}
        elif kind == "array":
            measure = rng.uniform(0.5, 1.5, P)
        else:
            measure = 0.75
        value = modes._modal_overlap(fields, mode, axis, measure, direction_sign=direction)
        for c in names:
            data[f"{tag}_field_{c}"] = fields[c]
            data[f"{tag}_mode_{c}"] = mode[c]
        if kind == "mapping":
            for c in names[:2]:
                data[f"{tag}_measure_{c}"] = measure[c]
        else:
            data[f"{tag}_measure"] = np.asarray(measure, dtype=float)
        data[f"{tag}_overlap"] = np.asarray(value)
    np.savez(args.out, **data)
    print(f"wrote {args.out}: {len(data)} arrays")


if __name__ == "__main__":
    main()
