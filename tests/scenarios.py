"""Seeded scenarios shared by the CPU and GPU tests.

Each builder returns a product-side :class:`beamz_b200.plan.ProgramSpec` and a
matching oracle program (same planner outputs), so the CUDA path and the CPU
oracle see identical inputs.
"""

from __future__ import annotations

import numpy as np

from beamz_b200 import plan as P
from oracle import fdtd_oracle as O


def to_oracle(spec: P.ProgramSpec, dtype=np.float32) -> O.OracleProgram:
    from oracle.from_spec import oracle_program

    return oracle_program(spec, dtype)


def _dt3(res, courant=0.99):
    return courant * res / (P.LIGHT_SPEED * np.sqrt(3.0))


def scenario_3d(grid=(9, 10, 11), seed=0, pml_cells=3, cpml_edges="all", metallic=(), sources=True,
                monitors=True, nsteps=12):
    """Random box geometry, CPML on ``cpml_edges``, PEC on ``metallic``."""
    rng = np.random.default_rng(seed)
    res = 20e-9
    dt = _dt3(res)
    eps = np.full(grid, 2.085, np.float32)
    for _ in range(3):
        lo = [int(rng.integers(0, n - 1)) for n in grid]
        hi = [min(n, lo_ + int(rng.integers(1, max(2, n // 2)))) for lo_, n in zip(lo, grid)]
        eps[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = rng.choice([12.11, 4.0])
    edges = None if cpml_edges == "all" else cpml_edges
    h_terms, e_terms = P.plan_cpml(grid, dt, res, pml_cells=pml_cells, edges=edges) if cpml_edges else ([], [])
    if cpml_edges:
        eps = P.extend_into_absorber(eps, P.absorber_edge_counts(grid, pml_cells, edges))
    ids, table = P.voxel_codebook(eps)
    srcs = []
    if sources:
        f0 = P.LIGHT_SPEED / 1.55e-6
        times = (np.arange(nsteps) + 0.5) * dt
        wave = P.gaussian_pulse(times, f0, 0.5 * f0, offset=0.3)
        c = grid[0] // 2, grid[1] // 2, grid[2] // 2
        srcs.append(P.SourcePlan("Ey", "pre_e", c, np.array([[[-dt / (P.EPS_0 * 2.085)]]], np.float32), wave))
        srcs.append(P.SourcePlan("Hz", "h", (1, 2, 1), rng.standard_normal((2, 2, min(3, grid[2] - 1))).astype(np.float32),
                                 (rng.standard_normal(nsteps) * 1e-3).astype(np.float32)))
        srcs.append(P.SourcePlan("Ex", "e", (0, 1, 1), rng.standard_normal((grid[0] + 1, 1, 2)).astype(np.float32),
                                 (rng.standard_normal(nsteps) * 1e-2).astype(np.float32)))
        srcs.append(P.SourcePlan("Ez", "pre_e", (2, 0, 0), rng.standard_normal((1, grid[1] + 1, grid[2] + 1)).astype(np.float32),
                                 (rng.standard_normal(nsteps + 3) * 1e-2).astype(np.float32)))
    mons = []
    if monitors:
        f0 = P.LIGHT_SPEED / 1.55e-6
        a = (np.arange(grid[0] - 2) + 1.5) * res
        b = (np.arange(grid[1] - 2) + 1.25) * res
        mons.append(P.plane_monitor(grid, res, "x", (grid[2] * 0.6) * res, a, b, [0.9 * f0, f0, 1.1 * f0]))
        c = (np.arange(grid[1] - 3) + 1.0) * res
        d = (np.arange(grid[2] - 3) + 1.5) * res
        mons.append(P.plane_monitor(grid, res, "z", (grid[0] * 0.4) * res, c, d, [f0, 1.2 * f0],
                                    components=("Ex", "Ey", "Hx", "Hy"), window_code=1, normalization_code=1,
                                    t_start=2 * dt, t_end=(nsteps - 1) * dt))
    spec = P.ProgramSpec(tuple(grid), dt, res, voxel_ids=ids, eps_table=table, h_terms=h_terms, e_terms=e_terms,
                         metallic_edges=frozenset(metallic), sources=srcs, monitors=mons, total_steps=nsteps)
    return spec


def scenario_2d(grid=(13, 15), polarization="tm", seed=0, pml_cells=3, metallic=(), nsteps=20, cpml=True):
    rng = np.random.default_rng(seed)
    res = 20e-9
    dt = 0.7 * res / (P.LIGHT_SPEED * np.sqrt(2.0))
    eps = np.full(grid, 2.085, np.float32)
    eps[grid[0] // 3: 2 * grid[0] // 3, :] = 12.11
    h_terms, e_terms = P.plan_cpml(grid, dt, res, pml_cells=pml_cells, polarization=polarization) if cpml else ([], [])
    e_comps = ("Ez",) if polarization == "tm" else ("Ex", "Ey")
    site_eps = {c: P.site_values_2d(eps, c, polarization) for c in e_comps}
    e_site = {c: (np.float32(1.0), P.e_source_2d(site_eps[c], dt)) for c in e_comps}
    f0 = P.LIGHT_SPEED / 1.55e-6
    wave = P.gaussian_pulse((np.arange(nsteps) + 0.5) * dt, f0, 0.5 * f0, offset=0.3)
    comp = "Ez" if polarization == "tm" else "Ey"
    srcs = [P.SourcePlan(comp, "pre_e", (grid[0] // 2, grid[1] // 3), np.array([[-dt / (P.EPS_0 * 12.11)]], np.float32), wave)]
    hcomp = "Hx" if polarization == "tm" else "Hz"
    srcs.append(P.SourcePlan(hcomp, "h", (1, 1), rng.standard_normal((2, 3)).astype(np.float32),
                             (rng.standard_normal(nsteps) * 1e-4).astype(np.float32)))
    # A line monitor: gather one column of the active components.
    shapes = {c: P.component_shape(c, grid, polarization) for c in P.COMPONENTS}
    idx, w = [], []
    P_ = grid[0] - 2
    for c in P.COMPONENTS:
        sy, sx = shapes[c]
        rows = np.minimum(np.arange(1, 1 + P_), sy - 1)
        col = min(2 * grid[1] // 3, sx - 1)
        idx.append((rows * sx + col).astype(np.int32)[:, None])
        w.append(np.ones((P_, 1), np.float32))
    mask = np.array([1.0 if c in P.active_components(2, polarization) else 0.0 for c in P.COMPONENTS], np.float32)
    mons = [P.DftMonitorPlan(np.array([0.95 * f0, f0, 1.05 * f0], np.float32), idx, w, mask)]
    return P.ProgramSpec(tuple(grid), dt, res, polarization=polarization, e_site=e_site, e_site_eps=site_eps,
                         h_terms=h_terms, e_terms=e_terms, metallic_edges=frozenset(metallic), sources=srcs,
                         monitors=mons, total_steps=nsteps)


def random_initial_fields(spec: P.ProgramSpec, seed=1, scale=1.0):
    rng = np.random.default_rng(seed)
    active = P.active_components(spec.ndim, spec.polarization)
    out = {}
    for c in P.COMPONENTS:
        if c in active:
            shape = P.component_shape(c, spec.grid_shape, spec.polarization)
            s = scale if c.startswith("E") else scale / 376.73
            out[c] = (rng.standard_normal(shape) * s).astype(np.float32)
    return out


def oracle_state(prog: O.OracleProgram, fields=None, dtype=np.float32):
    st = O.new_state(prog, dtype)
    if fields:
        for c, v in fields.items():
            st.fields[c] = np.asarray(v, dtype).copy()
    return st


def pack_dft_monitors_host(monitors, shapes, strides):
    """Host restatement of the device gather packing (the engine's earlier host
    path), for equivalence tests: per monitor and component, the (P, K) plan
    remapped to the device layout's offsets and reordered nonzero weights
    first (stable), laid out neighbour-major [M, 6, K, Pmax], K the most
    nonzero weights any point has."""
    M = len(monitors)
    P = max(m.points for m in monitors)
    K = max(max(np.asarray(a).reshape(m.points, -1).shape[1] for a in m.indices) for m in monitors)
    indices = np.zeros((M, 6, K, P), np.int32)
    weights = np.zeros((M, 6, K, P), np.float32)
    for m, mon in enumerate(monitors):
        p = mon.points
        for c in range(6):
            ic = np.asarray(mon.indices[c]).reshape(p, -1).astype(np.int64)
            wc = np.asarray(mon.weights[c], np.float32).reshape(p, -1)
            dims = (1,) * (3 - len(shapes[c])) + tuple(shapes[c])
            k, j, i = np.unravel_index(ic, dims)
            row, plane = strides(c)
            ic = (k * plane + j * row + i).astype(np.int32)
            order = np.argsort(wc == 0.0, axis=1, kind="stable")
            ic, wc = np.take_along_axis(ic, order, axis=1), np.take_along_axis(wc, order, axis=1)
            indices[m, c, : ic.shape[1], :p] = ic.T
            weights[m, c, : wc.shape[1], :p] = wc.T
    # as the runtime: K shrinks to the most nonzero weights of any point
    k_eff = max(1, int((weights != 0).sum(axis=2).max()))
    return indices[:, :, :k_eff], weights[:, :, :k_eff]


def with_metrics(spec: P.ProgramSpec, kind="rectilinear", seed=0, spread=(1.0, 1.6)) -> P.ProgramSpec:
    """``spec`` on an axis-uniform or rectilinear grid: seeded cell widths in
    ``spread`` x the cell size on every axis (never below it, so the spec's
    time step stays stable)."""
    import dataclasses

    rng = np.random.default_rng(seed)
    axes = ("z", "y", "x") if spec.ndim == 3 else ("y", "x")
    widths = {}
    for a, n in zip(axes, spec.grid_shape):
        if kind == "axis_uniform":
            widths[a] = np.full(int(n), spec.resolution * rng.uniform(*spread))
        else:
            widths[a] = spec.resolution * rng.uniform(*spread, int(n))
    return dataclasses.replace(spec, metrics=P.derivative_metrics(widths, kind))
