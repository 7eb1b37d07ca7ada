"""Seeded synthetic scenes for the benchmark workloads.

No public dataset is involved: permittivity voxels are written directly from
seeded random geometry, the way beamz's own performance workloads do
(tests/performance/h100_workloads.py:74-88 in beamz).

* ``scene_3d_512``: 512 x 512 x 256 cells at 20 nm, 12-cell CPML on all faces,
  oxide background (eps 2.085) with 8-16 Si boxes (eps 12.11, 220 nm tall,
  200-2000 nm lateral) on one layer, an Ey Gaussian-pulse dipole at 1.55 um and
  four x-normal DFT planes at five frequencies.
* ``scene_capacity``: 1536 x 1024 x 1024 cells, 12-cell CPML, Si slab
  waveguides with Gaussian sidewall roughness (sigma 2 cells).
* ``scene_2d_400``: 400 x 400 TM cells, 20-cell CPML, a 500 nm Si strip along x,
  a soft Ez source and one DFT line monitor at three frequencies.
"""

from __future__ import annotations

import numpy as np

from . import plan as P

SI = 12.11
OXIDE = 2.085
RES = 20e-9
F0 = P.LIGHT_SPEED / 1.55e-6


def _dt(ndim, courant):
    return courant * RES / (P.LIGHT_SPEED * np.sqrt(float(ndim)))


def _dipole(component, site, eps_site, dt, total_steps, fwidth, offset, ndim=3):
    """Point source with coeff -dt / (eps0 eps_r) at pre-E timing, sampled at
    t0 + (i + 1/2) dt (beamz/devices/sources/compiler.py:419-461)."""
    times = (np.arange(max(total_steps, 1), dtype=np.float64) + 0.5) * dt
    wave = P.gaussian_pulse(times, F0, fwidth, offset=offset)
    shape = (1,) * ndim
    coeff = np.full(shape, -dt / (P.EPS_0 * eps_site), np.float32)
    return P.SourcePlan(component, "pre_e", tuple(int(v) for v in site), coeff, wave)


def scene_3d_512(total_steps=1000, seed=0, shape=(256, 512, 512), pml_cells=12, monitors=True, sources=True,
                 n_monitors=4, n_freqs=5, cpml_edges=None):
    """``cpml_edges``: the faces with an absorber (default all six; an empty
    tuple gives a closed box), for measuring the absorber's cost per axis."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    dt = _dt(3, 0.99)
    # Voxel ids: 0 = oxide, 1 = Si (the sorted codebook of the two permittivities).
    ids = np.zeros(shape, np.uint8)
    z0 = nz // 2 - 5
    for _ in range(int(rng.integers(8, 17))):
        sy, sx = (int(v) for v in rng.integers(10, 101, size=2))
        y0 = int(rng.integers(0, max(1, ny - sy)))
        x0 = int(rng.integers(0, max(1, nx - sx)))
        ids[z0:z0 + 11, y0:y0 + sy, x0:x0 + sx] = 1
    if cpml_edges is not None and len(cpml_edges) == 0:
        h_terms, e_terms = [], []
    else:
        h_terms, e_terms = P.plan_cpml(shape, dt, RES, pml_cells=pml_cells, edges=cpml_edges)
    ids = P.extend_into_absorber(ids, P.absorber_edge_counts(shape, pml_cells, resolution=RES))
    table = np.ones(256, np.float32)
    table[0], table[1] = OXIDE, SI
    srcs = []
    if sources:
        site = (nz // 2, ny // 2, nx // 2)
        # Ey site permittivity: mean of the voxels sharing the edge.
        k, j, i = site
        eps = table[ids[k - 1:k + 1, j, i - 1:i + 1]]
        e_site = 0.25 * (eps[0, 0] + eps[1, 0] + eps[0, 1] + eps[1, 1])
        srcs.append(_dipole("Ey", site, float(e_site), dt, total_steps, 0.2 * F0, 0.5))
    mons = []
    if monitors:
        zc = (np.arange(pml_cells, nz - pml_cells) + 0.5) * RES
        yc = (np.arange(pml_cells, ny - pml_cells) + 0.5) * RES
        freqs = np.linspace(0.9, 1.1, n_freqs) * F0
        for frac in (0.2, 0.4, 0.6, 0.8)[:n_monitors]:
            mons.append(P.plane_monitor(shape, RES, "x", frac * nx * RES, zc, yc, freqs,
                                        components=("Ey", "Ez", "Hy", "Hz")))
    return P.ProgramSpec(shape, dt, RES, voxel_ids=ids, eps_table=table, h_terms=h_terms, e_terms=e_terms,
                         sources=srcs, monitors=mons, total_steps=total_steps)


def conductive(spec: P.ProgramSpec, sigma_by_id=(0.0, 4e4)) -> P.ProgramSpec:
    """The same scene with conductive material: voxel id v gets conductivity
    ``sigma_by_id[v]`` (S/m; default lossy Si, lossless oxide), lowered to
    beamz's per-site E and H (decay, source) coefficients
    (:func:`plan.lossy_site_coefficients_3d`, compile.py:563-640)."""
    import dataclasses

    ids = np.asarray(spec.voxel_ids)
    table = np.ones(256, np.float32)
    table[: len(spec.eps_table)] = spec.eps_table
    sig = np.zeros(256, np.float32)
    sig[: len(sigma_by_id)] = sigma_by_id
    e_site, h_site, e_eps = P.lossy_site_coefficients_3d(table[ids], sig[ids], spec.dt)
    return dataclasses.replace(spec, voxel_ids=None, eps_table=None, e_site=e_site, h_site=h_site, e_site_eps=e_eps)


def graded(spec: P.ProgramSpec, kind: str = "rectilinear", seed: int = 0, spread=(1.0, 1.25)) -> P.ProgramSpec:
    """The same scene on an axis-uniform or rectilinear grid: seeded cell
    widths within ``spread`` x the cell size on every axis (never below it, so
    the scene's time step stays stable), lowered to beamz's per-axis inverse
    distances (:func:`plan.derivative_metrics`, kernels.py:164-176)."""
    import dataclasses

    rng = np.random.default_rng(seed)
    widths = {}
    for a, n in zip(("z", "y", "x"), spec.grid_shape):
        if kind == "axis_uniform":
            widths[a] = np.full(int(n), spec.resolution * rng.uniform(*spread))
        else:
            widths[a] = spec.resolution * rng.uniform(*spread, int(n))
    return dataclasses.replace(spec, metrics=P.derivative_metrics(widths, kind))


def scene_capacity(total_steps=500, seed=0, shape=(1024, 1024, 1536), pml_cells=12, monitors=False):
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    dt = _dt(3, 0.99)
    ids = np.zeros(shape, np.uint8)  # id 0 = oxide, id 1 = Si
    # Layered slab waveguides along x: 220 nm (11-cell) Si cores every 96 cells in
    # z, sidewalls wandering with a smoothed Gaussian random walk (sigma 2 cells).
    kernel = np.exp(-0.5 * (np.arange(-12, 13) / 4.0) ** 2)
    kernel /= kernel.sum()
    for zc in range(48, nz - 48, 96):
        for yc in range(64, ny - 64, 128):
            walk = np.convolve(rng.normal(0.0, 2.0, nx + 24), kernel, mode="same")[12:12 + nx]
            lo = np.clip(np.round(yc - 12 + walk).astype(int), 0, ny)
            hi = np.clip(np.round(yc + 12 + walk).astype(int), 0, ny)
            for x in range(nx):
                ids[zc - 5:zc + 6, lo[x]:hi[x], x] = 1
    table = np.ones(256, np.float32)
    table[0], table[1] = OXIDE, SI
    counts = P.absorber_edge_counts(shape, pml_cells)
    ids = P.extend_into_absorber(ids, counts)
    h_terms, e_terms = P.plan_cpml(shape, dt, RES, pml_cells=pml_cells)
    site = (nz // 2, ny // 2 + 64, nx // 4)
    srcs = [_dipole("Ey", site, float(table[ids[site]]), dt, total_steps, 0.2 * F0, 0.5)]
    return P.ProgramSpec(shape, dt, RES, voxel_ids=ids, eps_table=table, h_terms=h_terms, e_terms=e_terms,
                         sources=srcs, monitors=[], total_steps=total_steps)


def scene_2d_400(total_steps=2000, shape=(400, 400), pml_cells=20):
    """2D TM (Ez, Hx, Hy): beamz's "TE with an Ez source" maps to its TM lattice
    (beamz/lattice.py:789-813)."""
    ny, nx = shape
    dt = _dt(2, 0.7)
    eps = np.full(shape, OXIDE, np.float32)
    yc = ny // 2
    eps[yc - 12:yc + 13, :] = SI  # 25 cells = 500 nm
    h_terms, e_terms = P.plan_cpml(shape, dt, RES, pml_cells=pml_cells, polarization="tm")
    eps = P.extend_into_absorber(eps, P.absorber_edge_counts(shape, pml_cells, resolution=RES, explicit_thickness=True))
    e_site = {"Ez": (np.float32(1.0), P.e_source_2d(P.site_values_2d(eps, "Ez", "tm"), dt))}
    site = (yc, nx // 4)
    src = _dipole("Ez", site, float(eps[site]), dt, total_steps, 0.1 * F0, 0.5, ndim=2)
    # Line monitor across the strip at x = 0.75 L: points along y at Ez nodes.
    x_col = int(0.75 * nx)
    ys = np.arange(yc - 40, yc + 41)
    idx, w = [], []
    for c in P.COMPONENTS:
        sh = P.component_shape(c, shape, "tm")
        rows = np.minimum(ys, sh[0] - 1)
        col = min(x_col, sh[1] - 1)
        idx.append((rows * sh[1] + col).astype(np.int32)[:, None])
        w.append(np.ones((ys.size, 1), np.float32))
    mask = np.array([0, 0, 1, 1, 1, 0], np.float32)
    mon = P.DftMonitorPlan(np.array([0.95, 1.0, 1.05], np.float32) * np.float32(F0), idx, w, mask)
    return P.ProgramSpec(shape, dt, RES, polarization="tm", e_site=e_site, h_terms=h_terms, e_terms=e_terms,
                         sources=[src], monitors=[mon], total_steps=total_steps)


def _line_monitor(shape, x_col, ys, freqs):
    """DFT line monitor along y at column x_col of a 2D TM grid (Ez, Hx, Hy)."""
    idx, w = [], []
    for c in P.COMPONENTS:
        sh = P.component_shape(c, shape, "tm")
        rows = np.minimum(ys, sh[0] - 1)
        col = min(x_col, sh[1] - 1)
        idx.append((rows * sh[1] + col).astype(np.int32)[:, None])
        w.append(np.ones((ys.size, 1), np.float32))
    mask = np.array([0, 0, 1, 1, 1, 0], np.float32)
    return P.DftMonitorPlan(np.asarray(freqs, np.float32), idx, w, mask)


def scene_2d(total_steps=2000, seed=0, shape=(512, 512), pml_cells=12, n_monitors=1, n_boxes=(2, 7)):
    """2D TM request: oxide with seeded random Si boxes, a soft Ez point source
    (Gaussian pulse at 1.55 um) and 1-4 x-normal DFT lines at 3 frequencies."""
    ny, nx = shape
    rng = np.random.default_rng(seed)
    dt = _dt(2, 0.7)
    eps = np.full(shape, OXIDE, np.float32)
    for _ in range(int(rng.integers(*n_boxes))):
        sy, sx = (int(v) for v in rng.integers(10, max(11, min(ny, nx) // 3), size=2))
        y0 = int(rng.integers(0, max(1, ny - sy)))
        x0 = int(rng.integers(0, max(1, nx - sx)))
        eps[y0:y0 + sy, x0:x0 + sx] = SI
    h_terms, e_terms = P.plan_cpml(shape, dt, RES, pml_cells=pml_cells, polarization="tm")
    eps = P.extend_into_absorber(eps, P.absorber_edge_counts(shape, pml_cells, resolution=RES, explicit_thickness=True))
    e_site = {"Ez": (np.float32(1.0), P.e_source_2d(P.site_values_2d(eps, "Ez", "tm"), dt))}
    site = (ny // 2, nx // 4)
    src = _dipole("Ez", site, float(eps[site]), dt, total_steps, 0.1 * F0, 0.5, ndim=2)
    freqs = np.array([0.95, 1.0, 1.05], np.float32) * np.float32(F0)
    ys = np.arange(pml_cells, ny - pml_cells)
    mons = [_line_monitor(shape, int(frac * nx), ys, freqs) for frac in (0.6, 0.7, 0.8, 0.9)[:n_monitors]]
    return P.ProgramSpec(shape, dt, RES, polarization="tm", e_site=e_site, h_terms=h_terms, e_terms=e_terms,
                         sources=[src], monitors=mons, total_steps=total_steps)


SERVING_3D_SHAPES = ((128, 128, 128), (192, 192, 192), (128, 256, 256))


def serving_requests(n=256, rate=50.0, seed=0, steps=(500, 4000), sizes_2d=(256, 1024), shapes_3d=SERVING_3D_SHAPES,
                     frac_3d=0.5):
    """Seeded request stream: Poisson arrivals at `rate` per second, half 2D TM
    grids (square, 256^2-1024^2 in steps of 32) and half 3D grids (128^3,
    192^3, 256x256x128 in x, y, z), uniform step counts, 1-4 DFT monitors and
    seeded random Si/oxide boxes.  Returns ``[(arrival_s, spec), ...]``."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for r in range(n):
        t += float(rng.exponential(1.0 / rate)) if rate > 0 else 0.0
        nsteps = int(rng.integers(steps[0], steps[1] + 1))
        nmon = int(rng.integers(1, 5))
        sub = int(rng.integers(0, 2**31 - 1))
        if rng.random() < frac_3d:
            shape = tuple(shapes_3d[int(rng.integers(0, len(shapes_3d)))])
            spec = scene_3d_512(total_steps=nsteps, seed=sub, shape=shape, n_monitors=nmon, n_freqs=3)
        else:
            side = int(rng.integers(sizes_2d[0] // 32, sizes_2d[1] // 32 + 1)) * 32
            spec = scene_2d(total_steps=nsteps, seed=sub, shape=(side, side), n_monitors=nmon)
        out.append((t, spec))
    return out


SCENES = {"3d_512": scene_3d_512, "capacity": scene_capacity, "2d_400": scene_2d_400}


def algorithmic_bytes(spec: P.ProgramSpec) -> int:
    """DRAM bytes one step must move at minimum: every field element read and
    written once (4 B each way), one material byte per cell (a voxel id, or an
    E class and, with per-site H, an H class), every CPML psi element read and
    written once.  DFT and coefficient traffic is excluded."""
    active = P.active_components(spec.ndim, spec.polarization)
    shapes = {c: P.component_shape(c, spec.grid_shape, spec.polarization) for c in active}
    field = sum(int(np.prod(s)) for s in shapes.values())
    psi = sum(int(np.prod(t.psi_shape(shapes[t.component]))) for t in list(spec.h_terms) + list(spec.e_terms))
    cells = int(np.prod(spec.grid_shape))
    if spec.voxel_ids is not None:
        material = cells  # one voxel id per cell
    elif spec.e_site is not None and spec.ndim == 3:
        # Per-site material: one E class per cell, and one H class where H is per site too.
        h_site = any(np.ndim(d) or np.ndim(s) for d, s in spec.h_coefficients().values())
        material = cells * (2 if h_site else 1)
    else:
        material = 0
    return 8 * field + material + 8 * psi
