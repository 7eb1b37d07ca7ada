"""Oracle programs from the engine's ``ProgramSpec`` -- TEST INFRASTRUCTURE.

The same planner outputs (CPML terms, sources, monitors, materials, metrics,
recorders) that the CUDA path receives, as an :class:`OracleProgram`, so the
checker and the engine see identical inputs.  Used by the tests and by
bench.py's CPU-baseline leg (its accuracy report).
"""

from __future__ import annotations

import numpy as np

from . import fdtd_oracle as O


def oracle_program(spec, dtype=np.float32) -> O.OracleProgram:
    """The oracle's program for ``spec`` in ``dtype`` (float32: the reference's
    arithmetic; float64: the FP64 oracle).  3D voxel programs sample the
    voxel permittivities at the E sites; 2D programs take the per-site
    coefficients (the H pair of the first active H component)."""
    shapes = O.component_shapes(spec.grid_shape, spec.polarization)

    def terms(ts):
        return [O.CpmlTerm(t.component, t.axis, t.sign, t.low, t.high, t.a, t.b, t.inv_kappa,
                           shapes[t.component][t.axis]) for t in ts]

    sources = [O.SlabSource(s.component, s.timing, tuple(s.start), np.asarray(s.coeff, np.float32),
                            np.asarray(s.waveform, np.float32)) for s in spec.sources]
    monitors = [O.DftMonitor(m.freqs, m.indices, m.weights, m.component_mask, m.t_start, m.t_end, m.interval,
                             m.window_code, m.normalization_code, m.length_unit) for m in spec.monitors]
    # Arena offsets follow declaration order (beamz/simulation/observe.py:403-410).
    voff = woff = 0
    for m in monitors:
        m.value_offset, m.weight_offset = voff, woff
        voff += 6 * len(m.freqs) * m.point_count
        woff += len(m.freqs)
    prog = O.OracleProgram(tuple(spec.grid_shape), float(spec.dt), float(spec.resolution), terms(spec.h_terms),
                           terms(spec.e_terms), metallic_edges=frozenset(spec.metallic_edges), sources=sources,
                           monitors=monitors, polarization=spec.polarization,
                           metrics=spec.metrics.as_dict() if spec.metrics is not None else None,
                           recorders=[O.FieldRecorder(r.components, r.interval, r.capacity, r.indices, r.weights,
                                                      r.signs) for r in spec.recorders])
    if spec.ndim == 3 and spec.voxel_ids is None:
        # Per-site coefficients (beamz's CUDA-path form, cuda/src/update.cu:392-410):
        # E <- decay E + source curl, H <- decay H - source curl.
        prog.e_coeffs = {c: (np.asarray(d, dtype), np.asarray(s, dtype)) for c, (d, s) in spec.e_site.items()}
        prog.h_coeffs_3d = {c: (np.asarray(d, dtype), np.asarray(s, dtype)) for c, (d, s) in spec.h_coefficients().items()}
    elif spec.ndim == 3:
        eps = np.asarray(spec.eps_table, np.float32)[spec.voxel_ids]
        prog.material = O.material_from_voxels(eps, dtype=dtype)
    else:
        hc = spec.h_coefficients()
        prog.h_coeffs = hc["Hx" if spec.polarization == "tm" else "Hz"]
        prog.e_coeffs = {c: (np.asarray(d, dtype), np.asarray(s, dtype)) for c, (d, s) in spec.e_site.items()}
    return prog
