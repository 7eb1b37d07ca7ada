"""beamz's native program entry points, on this engine.

beamz's ``execute.build_scan`` hands its native branch a compiled program in
four pieces (beamz/simulation/execute.py:555-681) and calls
``beamz.simulation.cuda.run_program_steps`` / ``run_source_group_steps`` /
``run_steps`` (beamz/simulation/cuda/runtime.py:496-700) on 256-step chunks:

* ``state`` -- ``SimulationState`` (beamz/simulation/model.py:127-259): ``hx``,
  ``hy``, ``hz``, ``ex``, ``ey``, ``ez`` (complete Yee supports, (z, y, x)),
  ``cpml_psi_h_terms`` / ``cpml_psi_e_terms`` (packed slabs), ``dft_vec_re``,
  ``dft_vec_im``, ``dft_weight_sum``, ``t``, ``current_step``;
* ``ctx`` -- the step context: ``dt``, ``resolution``, ``boundary.cpml``
  (``enabled``, ``metallic_edges``, ``h_terms`` / ``e_terms`` of ``CpmlTerm``,
  model.py:306-324), ``config.metric_kind`` and ``metrics``
  (``DerivativeMetricPlan``, model.py:290-303);
* ``coeffs`` -- ``UpdateCoefficients`` (model.py:262-287) as beamz compiles
  them for its CUDA backend (compile.py:563-660): uniform H decay/source
  scalars, and per E component either decay/source arrays or, for a lossless
  low-cardinality material, the coefficient table in ``e_decay_*`` and four
  uint8 table ids per int32 word in ``e_source_*`` (compile.py:146-187);
* ``groups`` -- nine ``BatchedSlabGroup`` or None (sources/compiler.py:52-113)
  in the order of ``SOURCE_PHASE_COMPONENTS`` (execute.py:48-52);
* ``packed_monitors`` -- the seven arrays of ``pack_dft_monitors``
  (cuda/runtime.py:530-618).

:func:`program_spec` maps them onto this engine's :class:`ProgramSpec`
(lossless 3D coefficient tables become the pitched class step's codebook),
and the ``run_*`` functions below are drop-ins for beamz's: they advance the
state ``nsteps`` steps on the device and return it with every array replaced
(numpy arrays; a JAX caller wraps them).  Compiled programs are cached per
(ctx, coeffs, groups, monitors) identity, the way beamz's graph cache keys
on its launch.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from . import plan as P
from . import runtime as R

#: beamz/simulation/execute.py:48-52: the nine source groups, in order.
SOURCE_PHASE_COMPONENTS = (("pre_e", ("Ex", "Ey", "Ez")), ("h", ("Hx", "Hy", "Hz")), ("e", ("Ex", "Ey", "Ez")))
GROUP_ORDER = tuple((timing, c) for timing, comps in SOURCE_PHASE_COMPONENTS for c in comps)

_STATE_FIELDS = (("Ex", "ex"), ("Ey", "ey"), ("Ez", "ez"), ("Hx", "hx"), ("Hy", "hy"), ("Hz", "hz"))


def _np(value, dtype=None):
    a = np.asarray(value)
    return a.astype(dtype) if dtype is not None and a.dtype != dtype else a


def grid_shape(state) -> tuple:
    """Cells (nz, ny, nx) from the state's Ex support (Z+1, Y+1, X)."""
    ex = np.shape(state.ex)
    return int(ex[0]) - 1, int(ex[1]) - 1, int(ex[2])


def unpack_coefficient_ids(table, packed, shape) -> np.ndarray:
    """Per-site coefficients from beamz's lossless CUDA packing: four uint8
    ids per int32 word over the C-order site index (compile.py:146-171)."""
    words = _np(packed).astype(np.int32).view(np.uint32)
    ids = np.stack([(words >> np.uint32(8 * b)) & np.uint32(0xFF) for b in range(4)], axis=1).reshape(-1)
    n = int(np.prod(shape))
    return _np(table, np.float32)[ids[:n].astype(np.int64)].reshape(shape)


def e_site_coefficients(coeffs, shapes) -> dict:
    """Component -> (decay, source) of beamz's compiled E coefficients."""
    out = {}
    for c, tag in (("Ex", "x"), ("Ey", "y"), ("Ez", "z")):
        dec, src = _np(getattr(coeffs, f"e_decay_{tag}")), _np(getattr(coeffs, f"e_source_{tag}"))
        if src.dtype == np.int32 and src.ndim == 1:  # table + packed ids
            out[c] = (np.float32(1.0), unpack_coefficient_ids(dec, src, shapes[c]))
        else:
            out[c] = (dec.astype(np.float32), src.astype(np.float32))
    return out


def h_site_coefficients(coeffs) -> dict:
    return {c: (_np(getattr(coeffs, f"h_decay_{t}"), np.float32), _np(getattr(coeffs, f"h_source_{t}"), np.float32))
            for c, t in (("Hx", "x"), ("Hy", "y"), ("Hz", "z"))}


def cpml_terms(terms) -> list:
    """beamz CpmlTerm records -> planner terms (same order, axis, sign and
    packed coefficient slabs)."""
    return [P.CpmlTermPlan(t.component, int(t.axis), float(t.sign), int(t.slab.low), int(t.slab.high),
                           _np(t.a, np.float32).reshape(-1), _np(t.b, np.float32).reshape(-1),
                           _np(t.inv_kappa, np.float32).reshape(-1)) for t in terms]


def slab_sources(groups) -> list:
    """The batched slab groups -> one source per slab, group by group."""
    out = []
    if not groups:
        return out
    for (timing, component), g in zip(GROUP_ORDER, groups):
        if g is None:
            continue
        coeffs, waves, starts = _np(g.coeffs, np.float32), _np(g.waveforms, np.float32), _np(g.starts)
        for n in range(int(coeffs.shape[0])):
            out.append(P.SourcePlan(component, timing, tuple(int(v) for v in starts[n]), coeffs[n], waves[n]))
    return out


def dft_monitors(packed) -> list:
    """pack_dft_monitors' arrays -> one monitor plan per monitor, in order."""
    if not packed:
        return []
    indices, weights, freqs, masks, counts, codes, windows = (_np(v) for v in packed)
    out = []
    voff = woff = 0
    for m in range(int(indices.shape[0])):
        nf, npt, interval, value_offset, weight_offset = (int(v) for v in counts[m])
        if (value_offset, weight_offset) != (voff, woff):
            raise ValueError("DFT arena offsets must follow monitor order")
        voff += 6 * nf * npt
        woff += nf
        out.append(P.DftMonitorPlan(
            freqs[m, :nf].astype(np.float32), [indices[m, c, :npt].astype(np.int32) for c in range(6)],
            [weights[m, c, :npt].astype(np.float32) for c in range(6)], masks[m].astype(np.float32),
            t_start=float(windows[m, 0]), t_end=float(windows[m, 1]), interval=interval,
            window_code=int(codes[m, 0]), normalization_code=int(codes[m, 1]), length_unit=float(windows[m, 2])))
    return out


def derivative_metrics(ctx):
    kind = getattr(getattr(ctx, "config", None), "metric_kind", "isotropic_uniform")
    if kind == "isotropic_uniform":
        return None
    m = ctx.metrics
    return P.DerivativeMetrics(**{name: _np(getattr(m, name), np.float32) for name in P.METRIC_NAMES})


def program_spec(state, ctx, coeffs, groups=None, packed_monitors=None, total_steps: int = 1) -> P.ProgramSpec:
    """This engine's program for a beamz compiled program (see the module doc)."""
    grid = grid_shape(state)
    shapes = {c: P.component_shape(c, grid) for c in P.COMPONENTS}
    cpml = ctx.boundary.cpml
    enabled = bool(getattr(cpml, "enabled", True))
    return P.ProgramSpec(
        grid, float(ctx.dt), float(ctx.resolution),
        e_site=e_site_coefficients(coeffs, shapes), h_site=h_site_coefficients(coeffs),
        h_terms=cpml_terms(cpml.h_terms) if enabled else [], e_terms=cpml_terms(cpml.e_terms) if enabled else [],
        metallic_edges=frozenset(cpml.metallic_edges), sources=slab_sources(groups),
        monitors=dft_monitors(packed_monitors), total_steps=max(int(total_steps), 1), t0=0.0,
        metrics=derivative_metrics(ctx))


_CACHE: dict = {}


def compile_program(state, ctx, coeffs, groups=None, packed_monitors=None, *, device="cuda", total_steps=1,
                    **kwargs) -> R.DeviceProgram:
    """Compile (or fetch from the cache) the device program of beamz's pieces."""
    key = (id(ctx), id(coeffs), id(groups), id(packed_monitors), grid_shape(state), str(device),
           tuple(sorted(kwargs.items())))
    hit = _CACHE.get(key)
    if hit is not None and hit[0] is ctx and hit[1] is coeffs:
        prog = hit[2]
        prog._times_for(max(int(total_steps), 1))
        return prog
    spec = program_spec(state, ctx, coeffs, groups, packed_monitors, total_steps)
    prog = R.compile_program(spec, device=device, **kwargs)
    if len(_CACHE) >= 32:  # bounded like beamz's graph cache: evicted wholesale
        _CACHE.clear()
    _CACHE[key] = (ctx, coeffs, prog)
    return prog


def device_state(program: R.DeviceProgram, state) -> R.DeviceState:
    """The beamz state's fields, CPML memories and DFT arena on the device, at
    its step counter (the clock is the program's float32 accumulation from
    t = 0, beamz's own for runs that start at step 0)."""
    torch = R._torch()
    fields = {c: _np(getattr(state, name), np.float32) for c, name in _STATE_FIELDS}
    psi_h = [_np(v, np.float32) for v in (getattr(state, "cpml_psi_h_terms", None) or ())] or None
    psi_e = [_np(v, np.float32) for v in (getattr(state, "cpml_psi_e_terms", None) or ())] or None
    st = R.initial_state(program, fields=fields, psi_h=psi_h if program.h_terms else None,
                         psi_e=psi_e if program.e_terms else None, step=int(np.asarray(state.current_step)))
    if program.arena is not None:
        for name, dst in (("dft_vec_re", st.dft_re), ("dft_vec_im", st.dft_im), ("dft_weight_sum", st.dft_w)):
            src = getattr(state, name, None)
            if src is not None and np.size(src) == dst.numel():
                dst.copy_(torch.as_tensor(_np(src, np.float32).reshape(-1), device=dst.device))
    return st


def simulation_state(device: R.DeviceState, state):
    """``state`` with every array replaced by the device state's values."""
    out = device.numpy()
    values = {name: out[c] for c, name in _STATE_FIELDS}
    values["cpml_psi_h_terms"] = tuple(out["psi_h"])
    values["cpml_psi_e_terms"] = tuple(out["psi_e"])
    if device.program.arena is not None:
        values.update(dft_vec_re=out["dft_re"], dft_vec_im=out["dft_im"], dft_weight_sum=out["dft_w"])
    values["t"] = np.float32(out["t"])
    values["current_step"] = np.int32(out["step"])
    if hasattr(state, "_replace"):
        keep = {k: v for k, v in values.items() if k in state._fields}
        return state._replace(**keep)
    merged = dict(vars(state))
    merged.update(values)
    return SimpleNamespace(**merged)


def run_program_steps(state, ctx, coeffs, groups, packed_monitors, nsteps: int, *, device="cuda", **kwargs):
    """Drop-in for beamz.simulation.cuda.run_program_steps: slab sources and
    packed vector DFTs advanced ``nsteps`` steps on the device."""
    if nsteps < 1:
        raise ValueError("CUDA step count must be positive")
    total = int(np.asarray(state.current_step)) + int(nsteps)
    prog = compile_program(state, ctx, coeffs, groups, packed_monitors, device=device, total_steps=total, **kwargs)
    st = device_state(prog, state)
    R.run_steps(st, prog, int(nsteps))
    return simulation_state(st, state)


def run_source_group_steps(state, ctx, coeffs, groups, nsteps: int, **kwargs):
    """Drop-in for beamz.simulation.cuda.run_source_group_steps (no monitors)."""
    return run_program_steps(state, ctx, coeffs, groups, None, nsteps, **kwargs)


def run_steps(state, ctx, coeffs, nsteps: int, **kwargs):
    """Drop-in for beamz.simulation.cuda.run_steps (no sources, no monitors)."""
    return run_program_steps(state, ctx, coeffs, None, None, nsteps, **kwargs)
