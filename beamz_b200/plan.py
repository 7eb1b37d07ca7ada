"""Host-side planning: everything the step kernels consume, built on the CPU.

This is setup, not the hot path.  It produces, in beamz's conventions, the
inputs that beamz's compiler hands its native step (beamz/simulation/compile.py
:241-305 and 540-733): packed CPML recurrence slabs, material encodings,
slab sources with sampled waveforms, DFT gather plans and the float32 clock.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# beamz/const.py:1-5
LIGHT_SPEED = 299792458.0
EPS_0 = 8.8541878128e-12
MU_0 = 1.25663706212e-6

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
COMPONENT_INDEX = {c: i for i, c in enumerate(COMPONENTS)}
ACTIVE = {3: COMPONENTS, "tm": ("Ez", "Hx", "Hy"), "te": ("Ex", "Ey", "Hz")}

# Which axes (z, y, x) carry a +1 sample on each Yee support (beamz/lattice.py:14-45).
_FACE_AXES_3D = {
    "Ex": (1, 1, 0), "Ey": (1, 0, 1), "Ez": (0, 1, 1),
    "Hx": (0, 0, 1), "Hy": (0, 1, 0), "Hz": (1, 0, 0),
}
_SHAPE_2D = {
    "tm": {"Ez": (1, 1), "Hx": (0, 1), "Hy": (1, 0)},
    "te": {"Ex": (1, 0), "Ey": (0, 1), "Hz": (0, 0)},
}


def component_shape(component: str, grid_shape, polarization: str = "tm") -> tuple:
    """Complete stored Yee support of one component (beamz/lattice.py:32-45, 789-813)."""
    if len(grid_shape) == 3:
        return tuple(int(n) + e for n, e in zip(grid_shape, _FACE_AXES_3D[component]))
    extra = _SHAPE_2D[polarization].get(component)
    if extra is None:
        return (1, 1)
    return tuple(int(n) + e for n, e in zip(grid_shape, extra))


def active_components(ndim: int, polarization: str = "tm") -> tuple:
    return ACTIVE[3] if ndim == 3 else ACTIVE[polarization]


# ---------------------------------------------------------------------------
# CPML
# ---------------------------------------------------------------------------


@dataclass
class CpmlTermPlan:
    """A packed recurrence: a, b, 1/kappa over the low and high slabs of
    ``axis`` (beamz/simulation/model.py:306-324)."""

    component: str
    axis: int  # storage axis of the component's array (3D: 0=z 1=y 2=x; 2D: 0=y 1=x)
    sign: float
    low: int
    high: int
    a: np.ndarray
    b: np.ndarray
    inv_kappa: np.ndarray

    @property
    def width(self) -> int:
        return self.low + self.high

    def psi_shape(self, target_shape) -> tuple:
        shape = list(target_shape)
        shape[self.axis] = self.width
        return tuple(shape)


# (component, axis, sign) per 3D derivative term, beamz/devices/_boundary_compile.py:44-60
# and beamz/simulation/compile.py:271-283.
TERMS_3D_H = (("Hx", 1, 1.0), ("Hx", 0, -1.0), ("Hy", 0, 1.0), ("Hy", 2, -1.0), ("Hz", 2, 1.0), ("Hz", 1, -1.0))
TERMS_3D_E = (("Ex", 1, 1.0), ("Ex", 0, -1.0), ("Ey", 0, 1.0), ("Ey", 2, -1.0), ("Ez", 2, 1.0), ("Ez", 1, -1.0))
# 2D terms, beamz/simulation/compile.py:285-304.
TERMS_2D = {
    "tm": ((("Hx", 0, 1.0), ("Hy", 1, -1.0)), (("Ez", 1, 1.0), ("Ez", 0, -1.0))),
    "te": ((("Hz", 1, 1.0), ("Hz", 0, -1.0)), (("Ex", 0, 1.0), ("Ey", 1, -1.0))),
}
_WALLS_3D = (("front", "back"), ("bottom", "top"), ("left", "right"))
_WALLS_2D = (("bottom", "top"), ("left", "right"))
ALL_EDGES_3D = ("left", "right", "top", "bottom", "front", "back")
ALL_EDGES_2D = ("left", "right", "top", "bottom")


def _graded_profile(samples, pml_cells, on_low, on_high, electric, sigma_max, alpha_max, kappa_max, order):
    """Staggered sigma/kappa/alpha along one axis in float32
    (beamz/devices/_boundary_compile.py:479-614, uniform grid)."""
    f32 = np.float32
    pml = max(int(pml_cells), 1)
    n_cells = samples - 1 if electric else samples
    pos = np.arange(samples, dtype=f32) + (f32(0.0) if electric else f32(0.5))
    sigma = np.zeros(samples, f32)
    kappa = np.ones(samples, f32)
    alpha = np.zeros(samples, f32)
    distances = []
    if on_low:
        distances.append(np.clip(f32(pml) - pos, f32(0.0), f32(pml)))
    if on_high:
        distances.append(np.clip(pos - f32(n_cells - pml), f32(0.0), f32(pml)))
    for dist in distances:
        inside = dist > 0
        u = np.clip(dist / f32(pml), f32(0.0), f32(1.0))
        graded = np.power(u, f32(order))
        sigma = np.where(inside, np.maximum(sigma, f32(sigma_max) * graded), sigma)
        kappa = np.where(inside, np.maximum(kappa, f32(1.0) + (f32(kappa_max) - f32(1.0)) * graded), kappa)
        alpha = np.where(inside, np.maximum(alpha, f32(alpha_max) * np.power(f32(1.0) - u, f32(1.0))), alpha)
    return sigma, kappa, alpha


def recurrence_coefficients(sigma, kappa, alpha, dt):
    """a, b, 1/kappa of one CPML recurrence in float32 (beamz/simulation/kernels.py:130-144)."""
    f32 = np.float32
    kappa = np.maximum(kappa.astype(f32), f32(1.0))
    rate = (sigma / kappa + alpha) * (f32(dt) / f32(EPS_0))
    b = np.exp(-rate).astype(f32)
    den = np.maximum((sigma + kappa * alpha) * kappa, f32(1e-30))
    a = np.nan_to_num(((b - f32(1.0)) * sigma) / den).astype(f32)
    return a, b, (f32(1.0) / kappa).astype(f32)


def _slab_extent(a, inv_kappa):
    """Active run lengths from each end (beamz/simulation/kernels.py:225-235)."""
    on = (np.abs(a) > 1e-30) | (np.abs(inv_kappa - 1.0) > 1e-7)
    low = int(np.argmin(on)) if not on.all() else on.size
    rest = on[low:][::-1]
    high = int(np.argmin(rest)) if not rest.all() else rest.size
    return low, high


def plan_cpml(grid_shape, dt, resolution, pml_cells=12, edges=None, polarization="tm",
              kappa_max=2.0, order=3, reflection=1e-6):
    """Every CPML term of a uniform grid, H terms then E terms.

    sigma_max = -(m+1) ln R / (2 eta d), alpha_max = 2 eps0 a_n / dt with a_n =
    0.05 (3D) or 0.1 (2D) (beamz/devices/_boundary_compile.py:244-261,
    beamz/devices/boundaries.py:133-141).
    """
    ndim = len(grid_shape)
    edges = set(ALL_EDGES_3D if ndim == 3 else ALL_EDGES_2D) if edges is None else set(edges)
    eta = np.sqrt(MU_0 / EPS_0)
    thickness = max(pml_cells * float(resolution), float(resolution))
    sigma_max = -(order + 1) * np.log(max(reflection, 1e-16)) / (2.0 * eta * thickness)
    alpha_max = 2.0 * EPS_0 * (0.05 if ndim == 3 else 0.1) / max(float(dt), 1e-30)
    if ndim == 3:
        specs_h, specs_e, walls = TERMS_3D_H, TERMS_3D_E, _WALLS_3D
    else:
        (specs_h, specs_e), walls = TERMS_2D[polarization], _WALLS_2D

    def one(component, axis, sign):
        shape = component_shape(component, grid_shape, polarization)
        n = shape[axis]
        electric = component.startswith("E") if ndim == 2 else _FACE_AXES_3D[component][axis] == 1
        lo_wall, hi_wall = walls[axis]
        s, k, al = _graded_profile(n, pml_cells, lo_wall in edges, hi_wall in edges, electric,
                                   sigma_max, alpha_max, kappa_max, order)
        a, b, ik = recurrence_coefficients(s, k, al, dt)
        low, high = _slab_extent(a, ik)
        keep = np.concatenate([np.arange(low), np.arange(n - high, n)]).astype(np.int64)
        return CpmlTermPlan(component, axis, sign, low, high, a[keep], b[keep], ik[keep])

    return [one(*s) for s in specs_h], [one(*s) for s in specs_e]


def absorber_edge_counts(grid_shape, pml_cells, edges=None, resolution=None, explicit_thickness=False):
    """Cells of each active wall that the absorber covers, in beamz's wall order
    (beamz/devices/_boundary_compile.py:278-319, 404-440)."""
    ndim = len(grid_shape)
    order = ALL_EDGES_3D if ndim == 3 else ALL_EDGES_2D
    chosen = order if edges is None else tuple(edges)
    axis_of = {"left": ndim - 1, "right": ndim - 1, "bottom": ndim - 2, "top": ndim - 2, "front": 0, "back": 0}
    out = []
    for edge in chosen:
        if ndim == 2 and edge in ("front", "back"):
            continue
        axis = axis_of[edge]
        n = int(grid_shape[axis])
        if explicit_thickness:
            centers = np.linspace(0, float(n * float(resolution)), n).astype(np.float32)
            span, depth = np.float32(n * float(resolution)), np.float32(pml_cells * float(resolution))
        else:
            centers = np.arange(n, dtype=np.float32) + np.float32(0.5)
            span, depth = np.float32(n), np.float32(pml_cells)
        if edge in ("left", "bottom", "front"):
            covered = (depth - centers) > 0
            side = "low"
        else:
            covered = (centers - (span - depth)) > 0
            covered = covered[::-1]
            side = "high"
        count = int(np.argmin(covered)) if not covered.all() else 0
        out.append((edge, axis, side, count))
    return out


def extend_into_absorber(grid: np.ndarray, counts) -> np.ndarray:
    """Copy the first interior layer outward through every absorber slab
    (beamz/devices/_boundary_compile.py:334-363)."""
    out = np.array(grid, copy=True)
    for _edge, axis, side, count in counts:
        n = out.shape[axis]
        if count <= 0 or count >= n:
            continue
        src = count if side == "low" else n - count - 1
        dst = slice(0, count) if side == "low" else slice(n - count, n)
        index = [slice(None)] * out.ndim
        index[axis] = dst
        ref = [slice(None)] * out.ndim
        ref[axis] = slice(src, src + 1)
        out[tuple(index)] = out[tuple(ref)]
    return out


# ---------------------------------------------------------------------------
# Materials
# ---------------------------------------------------------------------------


def voxel_codebook(eps_grid: np.ndarray):
    """uint8 voxel ids and a 256-entry float32 permittivity table."""
    table, ids = np.unique(np.asarray(eps_grid, dtype=np.float32), return_inverse=True)
    if table.size > 256:
        raise ValueError(f"voxel material needs <= 256 distinct permittivities, got {table.size}")
    padded = np.ones(256, np.float32)
    padded[: table.size] = table
    return ids.reshape(np.shape(eps_grid)).astype(np.uint8), padded


# E-site coefficient codebook (pitched 3D layout).  The E update coefficient at
# a site is fl(fl(dt)/fl(eps0) * fl(1/eps_site)), with eps_site the centered
# average 0.5*(0.5*(t0+t1) + 0.5*(t2+t3)) of four voxel samples
# (beamz/lattice.py:732-786: z, then y, then x, each with clipped indices).
# On the edge-replicated voxel grid vp (Z+2, Y+2, X+2), vp[k+dk, j+dj, i+di]
# is voxel (clip(k-1+dk), clip(j-1+dj), clip(i-1+di)); these are the (dk, dj,
# di) of t0..t3 per component, in averaging order.
CODEBOOK_TAPS = {
    "Ex": ((0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1)),  # average z, then y
    "Ey": ((0, 1, 0), (1, 1, 0), (0, 1, 1), (1, 1, 1)),  # average z, then x
    "Ez": ((1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1)),  # average y, then x
}
#: The 4-tuple key space m**4 must stay addressable by int32 keys.
CODEBOOK_MAX_MATERIALS = 46


class CodebookOverflow(ValueError):
    """The program has more distinct E-site coefficients than a codebook holds."""


def codebook_keys(vp, m: int, component: str, k0: int, k1: int):
    """Tuple keys ((t0*m + t1)*m + t2)*m + t3 of one component's sites on
    lattice planes [k0, k1) x (Y+1) x (X+1).

    ``vp`` is the edge-replicated grid of compact material indices (0..m-1),
    as a numpy array or a torch tensor of an integer type wide enough for m**4.
    """
    ny, nx = vp.shape[1] - 1, vp.shape[2] - 1
    t = [vp[k0 + dk:k1 + dk, dj:dj + ny, di:di + nx] for dk, dj, di in CODEBOOK_TAPS[component]]
    return ((t[0] * m + t[1]) * m + t[2]) * m + t[3]


def edge_replicated(compact: np.ndarray) -> np.ndarray:
    """(Z, Y, X) -> (Z+2, Y+2, X+2) with each face copied outward once."""
    return np.pad(compact, 1, mode="edge")


def codebook_tables(eps_used: np.ndarray, dt_over_eps, present: dict, with_eps: bool = False):
    """Per-component lookup tables from tuple key to codebook id, and the
    coefficient tables.

    ``eps_used`` holds the m permittivities in compact-index order and
    ``present[c]`` flags which of the m**4 keys occur.  Returns ``(luts, coef)``:
    ``luts[c]`` is a uint8 array of m**4 ids (0 where a key is absent) and
    ``coef`` the float32 (3, 256) tables.  Raises :class:`CodebookOverflow` when
    a component has more than 256 distinct coefficients.  With ``with_eps``
    also returns the float32 (3, 256) site permittivities of the ids (an id's
    sites share one coefficient; the table keeps one of their permittivities).
    """
    f32 = np.float32
    e = np.asarray(eps_used, f32)
    half = f32(0.5)
    a = half * (e[:, None, None, None] + e[None, :, None, None])
    b = half * (e[None, None, :, None] + e[None, None, None, :])
    eps_site = (half * (a + b)).reshape(-1)
    coef_all = f32(dt_over_eps) * (f32(1.0) / eps_site)
    luts, coef, eps = {}, np.zeros((3, 256), f32), np.ones((3, 256), f32)
    for n, c in enumerate(("Ex", "Ey", "Ez")):
        mask = np.asarray(present[c], bool)
        values, inverse = np.unique(coef_all[mask], return_inverse=True)
        if values.size > 256:
            raise CodebookOverflow(f"{c}: {values.size} distinct E-site coefficients (> 256)")
        lut = np.zeros(coef_all.size, np.uint8)
        lut[mask] = inverse.astype(np.uint8)
        luts[c] = lut
        coef[n, : values.size] = values
        eps[n, inverse] = eps_site[mask]
    return (luts, coef, eps) if with_eps else (luts, coef)


def compact_materials(voxel_ids: np.ndarray, eps_table: np.ndarray, counts=None):
    """Compact voxel ids to 0..m-1 over the ids that occur.

    Returns ``(remap, eps_used)``: ``remap`` is a 256-entry int32 table from
    voxel id to compact index and ``eps_used`` the m permittivities.
    ``counts`` (the 256-bin voxel-id histogram, e.g. from the device) saves
    counting the ids here.
    """
    if counts is None:
        counts = np.bincount(np.asarray(voxel_ids, np.uint8).reshape(-1), minlength=256)
    used = np.flatnonzero(np.asarray(counts))
    if used.size > CODEBOOK_MAX_MATERIALS:
        raise CodebookOverflow(f"{used.size} materials (> {CODEBOOK_MAX_MATERIALS}) for the site codebook")
    remap = np.zeros(256, np.int32)
    remap[used] = np.arange(used.size, dtype=np.int32)
    table = np.ones(256, np.float32)
    table[: len(eps_table)] = np.asarray(eps_table, np.float32)
    return remap, table[used]


def site_codebook(voxel_ids: np.ndarray, eps_table: np.ndarray, dt_over_eps):
    """Host build of the site-id words and coefficient tables.

    Returns ``(words, coef)``: ``words`` is an int32 (Z+1, Y+1, X+1) array whose
    bytes 0, 1, 2 are the Ex, Ey, Ez codebook ids at each lattice point, and
    ``coef`` the float32 (3, 256) coefficient tables.
    """
    remap, eps_used = compact_materials(voxel_ids, eps_table)
    m = eps_used.size
    vp = edge_replicated(remap[np.asarray(voxel_ids, np.uint8)])
    nz = vp.shape[0] - 2
    keys = {c: codebook_keys(vp, m, c, 0, nz + 1) for c in ("Ex", "Ey", "Ez")}
    present = {c: np.bincount(keys[c].reshape(-1), minlength=m**4) > 0 for c in keys}
    luts, coef = codebook_tables(eps_used, dt_over_eps, present)
    words = np.zeros(keys["Ex"].shape, np.int32)
    for shift, c in ((0, "Ex"), (8, "Ey"), (16, "Ez")):
        words |= luts[c][keys[c]].astype(np.int32) << shift
    return words, coef


def e_site_average_3d(grid: np.ndarray, component: str) -> np.ndarray:
    """float32 E-site sample of a cell-centred float grid over the component's
    stored shape: the four-voxel average 0.5*(0.5*(t0+t1) + 0.5*(t2+t3)) with
    clipped indices (beamz/lattice.py:732-786), as the codebook uses."""
    f32 = np.float32
    g = np.asarray(grid, f32)
    vp = edge_replicated(g)
    nz, ny, nx = g.shape
    t = [vp[dk:dk + nz + 1, dj:dj + ny + 1, di:di + nx + 1] for dk, dj, di in CODEBOOK_TAPS[component]]
    half = f32(0.5)
    site = half * (half * (t[0] + t[1]) + half * (t[2] + t[3]))
    dz, dy, dx = component_shape(component, (nz, ny, nx))
    return np.ascontiguousarray(site[:dz, :dy, :dx], dtype=f32)


def site_eps_3d(voxel_ids: np.ndarray, eps_table: np.ndarray, component: str) -> np.ndarray:
    """float32 E-site permittivity of one component over its stored shape
    (voxel ids and a permittivity table)."""
    table = np.ones(256, np.float32)
    table[: len(eps_table)] = np.asarray(eps_table, np.float32)
    return e_site_average_3d(table[np.asarray(voxel_ids, np.uint8)], component)


# Yee offsets (z, y, x) in cells, beamz/lattice.py:14-21.
_OFFSETS_3D = {"Ex": (0.0, 0.0, 0.5), "Ey": (0.0, 0.5, 0.0), "Ez": (0.5, 0.0, 0.0),
               "Hx": (0.5, 0.5, 0.0), "Hy": (0.5, 0.0, 0.5), "Hz": (0.0, 0.5, 0.5)}


def h_site_sample_3d(grid: np.ndarray, component: str) -> np.ndarray:
    """Sample of a cell-centred grid at an H component's sites: the owning
    voxel floor(index + offset), clipped (beamz/lattice.py:670-729)."""
    g = np.asarray(grid)
    shape = component_shape(component, g.shape)
    idx = [np.clip(np.floor(np.arange(n, dtype=np.float64) + off).astype(np.int64), 0, m - 1)
           for n, off, m in zip(shape, _OFFSETS_3D[component], g.shape)]
    return np.ascontiguousarray(g[np.ix_(*idx)])


def sponge_conductivity(grid_shape, resolution, base_sigma=0.0, edges=None, thickness=None, sigma_max=None,
                        order: int = 3, reflection: float = 1e-6) -> np.ndarray:
    """Cell-centred float32 conductivity of a graded sponge absorber on a
    uniform grid, combined with the material's own: beamz's ``Absorber`` /
    ``PML(formulation="sponge")`` lowering (beamz/devices/_boundary_compile.py:
    206-262, 406-423, 616-650) and ``_total_conductivity`` (lattice.py:978-998).

    Per axis (3D z, y, x; 2D y, x) the cell coordinates are ``linspace(0, L,
    n)`` (L = n * resolution, float64 rounded to float32) and the profile
    sigma_max * (d / thickness)**order grows with the depth d into each chosen
    face; the three axis profiles are summed (x, y, z order) and the larger of
    that sum and ``base_sigma`` is kept per cell.  ``thickness`` defaults to 12
    cells (beamz's ``PML``; its ``Absorber`` takes metres), and ``sigma_max`` to
    -(order + 1) ln(reflection) / (2 eta max(thickness, resolution)).  The
    result feeds :func:`lossy_site_coefficients_3d` / ``_2d``."""
    f32 = np.float32
    shape = tuple(int(n) for n in grid_shape)
    ndim = len(shape)
    res = float(resolution)
    edges = set(ALL_EDGES_3D if ndim == 3 else ALL_EDGES_2D) if edges is None else set(edges)
    thk = 12 * res if thickness is None else float(thickness)
    if sigma_max is None:
        eta = np.sqrt(MU_0 / (EPS_0 * 1.0))
        sigma_max = -(order + 1) * np.log(max(reflection, 1e-16)) / (2.0 * eta * max(thk, res))
    walls = dict(zip(("z", "y", "x"), _WALLS_3D)) if ndim == 3 else dict(zip(("y", "x"), _WALLS_2D))
    names = ("z", "y", "x") if ndim == 3 else ("y", "x")
    profiles = {}
    for axis, name in enumerate(names):
        n = shape[axis]
        length = n * res
        coords = np.linspace(0.0, length, n).astype(f32)
        sigma = np.zeros(n, f32)
        low, high = walls[name]
        if low in edges:
            dist = np.clip(f32(thk) - coords, f32(0.0), None)
            sigma = sigma + f32(sigma_max) * (dist / f32(thk)) ** order
        if high in edges:
            dist = np.clip(coords - f32(length - thk), f32(0.0), None)
            sigma = sigma + f32(sigma_max) * (dist / f32(thk)) ** order
        bshape = [1] * ndim
        bshape[axis] = n
        profiles[name] = np.broadcast_to(sigma.reshape(bshape), shape)
    total = np.zeros(shape, f32) + np.asarray(base_sigma, f32)
    pml = np.zeros_like(np.asarray(base_sigma, f32))
    for name in ("x", "y", "z"):
        if name in profiles:
            pml = pml + profiles[name]
    return np.maximum(total, pml).astype(f32)


def lossy_site_coefficients_3d(eps_grid: np.ndarray, sigma_grid: np.ndarray, dt: float):
    """Per-site update coefficients of a conductive, non-magnetic 3D material,
    as beamz's CUDA path receives them (beamz/simulation/compile.py:563-640):
    sigma sampled at E sites like eps (lattice.py:1031-1044), the matched
    magnetic conductivity sigma * MU_0 / EPS_0 at the H sites' owning voxels
    (lattice.py:1046-1068), then decay and source by
    precompute_e/h_update_coefficients (kernels.py:704-728), float32 throughout.
    Returns ``(e_site, h_site, e_site_eps)`` for a :class:`ProgramSpec`."""
    f32 = np.float32
    dt = float(dt)  # a Python float: float32 arithmetic, as in beamz (JAX weak typing)
    eps = np.asarray(eps_grid, f32)
    sig = np.asarray(sigma_grid, f32)
    e_site, h_site, e_eps = {}, {}, {}
    for c in ("Ex", "Ey", "Ez"):
        ep = e_site_average_3d(eps, c)
        sg = e_site_average_3d(sig, c)
        denom = 1.0 + sg * dt / (2.0 * EPS_0 * ep)
        decay = ((1.0 - sg * dt / (2.0 * EPS_0 * ep)) / denom).astype(f32)
        source = ((dt / (EPS_0 * ep)) / denom).astype(f32)
        e_site[c], e_eps[c] = (decay, source), ep
    base = sig * f32(1.0) * MU_0 / EPS_0
    for c in ("Hx", "Hy", "Hz"):
        sm = h_site_sample_3d(base, c)
        denom = 1.0 + sm * dt / (2.0 * MU_0)
        decay = ((1.0 - sm * dt / (2.0 * MU_0)) / denom).astype(f32)
        source = ((dt / MU_0) / denom).astype(f32)
        h_site[c] = (decay, source)
    return e_site, h_site, e_eps


def lossy_site_coefficients_2d(eps_grid: np.ndarray, sigma_grid: np.ndarray, dt: float, polarization: str = "tm"):
    """2D analogue of :func:`lossy_site_coefficients_3d`: eps and sigma sampled
    on each active component's support (lattice.py:919-972, the H supports of
    the matched magnetic conductivity sigma * MU_0 / EPS_0 included,
    lattice.py:1117-1129), then precompute_e/h_update_coefficients
    (kernels.py:704-728).  Returns ``(e_site, h_site, e_site_eps)``."""
    f32 = np.float32
    dt = float(dt)
    eps = np.asarray(eps_grid, f32)
    sig = np.asarray(sigma_grid, f32)
    e_comps = ("Ez",) if polarization == "tm" else ("Ex", "Ey")
    h_comps = ("Hx", "Hy") if polarization == "tm" else ("Hz",)
    e_site, h_site, e_eps = {}, {}, {}
    for c in e_comps:
        ep = np.asarray(site_values_2d(eps, c, polarization), f32)
        sg = np.asarray(site_values_2d(sig, c, polarization), f32)
        denom = 1.0 + sg * dt / (2.0 * EPS_0 * ep)
        decay = ((1.0 - sg * dt / (2.0 * EPS_0 * ep)) / denom).astype(f32)
        source = ((dt / (EPS_0 * ep)) / denom).astype(f32)
        e_site[c], e_eps[c] = (decay, source), ep
    base = sig * f32(1.0) * MU_0 / EPS_0
    for c in h_comps:
        sm = np.asarray(site_values_2d(base, c, polarization), f32)
        denom = 1.0 + sm * dt / (2.0 * MU_0)
        decay = ((1.0 - sm * dt / (2.0 * MU_0)) / denom).astype(f32)
        source = ((dt / MU_0) / denom).astype(f32)
        h_site[c] = (decay, source)
    return e_site, h_site, e_eps


def site_values_2d(eps_grid: np.ndarray, component: str, polarization: str = "tm") -> np.ndarray:
    """2D supports take the owning voxel (beamz/lattice.py:935-972)."""
    ny, nx = eps_grid.shape
    sy, sx = component_shape(component, (ny, nx), polarization)
    half = {"Ez": (0, 0), "Hx": (1, 0), "Hy": (0, 1), "Ex": (0, 1), "Ey": (1, 0), "Hz": (1, 1)}[component]
    rows = np.minimum((2 * np.arange(sy) + half[0]) // 2, ny - 1)
    cols = np.minimum((2 * np.arange(sx) + half[1]) // 2, nx - 1)
    return np.asarray(eps_grid)[rows][:, cols]


def e_source_2d(eps_site: np.ndarray, dt: float) -> np.ndarray:
    """dt / (EPS_0 * eps) in float32 (beamz/simulation/kernels.py:711-728)."""
    f32 = np.float32
    return (f32(dt) / (f32(EPS_0) * np.asarray(eps_site, f32))).astype(f32)


# ---------------------------------------------------------------------------
# Sources and monitors
# ---------------------------------------------------------------------------


@dataclass
class SourcePlan:
    """field[start + idx] += coeff[idx] * waveform[clamp(step)] at one timing."""

    component: str
    timing: str  # "pre_e" | "h" | "e"
    start: tuple
    coeff: np.ndarray
    waveform: np.ndarray


def gaussian_pulse(times, freq0, fwidth, amplitude=1.0, offset=4.0, remove_dc=True) -> np.ndarray:
    """Gaussian-modulated carrier sampled at ``times`` (beamz/devices/sources/time.py:459-487)."""
    t = np.asarray(times, dtype=np.float64)
    sigma_t = 1.0 / (2.0 * np.pi * max(float(fwidth), 1e-30))
    t_peak = float(offset) / max(float(fwidth), 1e-30)
    wave = float(amplitude) * np.exp(-0.5 * ((t - t_peak) / sigma_t) ** 2) * np.cos(2.0 * np.pi * float(freq0) * t)
    if remove_dc and wave.size:
        wave = wave - wave.mean()
    return wave.astype(np.float32)


@dataclass
class DftMonitorPlan:
    """A vector-DFT monitor (beamz/devices/monitors/compiler.py:62-102)."""

    freqs: np.ndarray
    indices: list  # 6 x (P, K) int32 flat offsets
    weights: list  # 6 x (P, K) float32
    component_mask: np.ndarray  # (6,) float32
    t_start: float = 0.0
    t_end: float = float("inf")
    interval: int = 1
    window_code: int = 0
    normalization_code: int = 0
    length_unit: float = 1e-6

    @property
    def points(self) -> int:
        return int(self.indices[0].shape[0])


def _axis_samples(n, offset, resolution):
    return (np.arange(n, dtype=np.float64) + offset) * float(resolution)


def _bracket(src, dst):
    """Linear interpolation brackets and weights (beamz/lattice.py:241-271)."""
    src = np.asarray(src, np.float64)
    dst = np.asarray(dst, np.float64)
    if src.size == 1:
        z = np.zeros(dst.size, np.int32)
        return z, z, np.ones(dst.size, np.float32), np.zeros(dst.size, np.float32)
    hi = np.clip(np.searchsorted(src, dst, side="right"), 1, src.size - 1)
    lo = hi - 1
    below, above = dst <= src[0], dst >= src[-1]
    lo[below] = hi[below] = 0
    lo[above] = hi[above] = src.size - 1
    span = src[hi] - src[lo]
    frac = np.zeros_like(dst)
    ok = (hi != lo) & (np.abs(span) > 0)
    frac[ok] = (dst[ok] - src[lo[ok]]) / span[ok]
    w_hi = frac.astype(np.float32)
    w_lo = (1.0 - frac).astype(np.float32)
    same = hi == lo
    w_lo[same], w_hi[same] = 1.0, 0.0
    return lo.astype(np.int32), hi.astype(np.int32), w_lo, w_hi


def plane_gather(component, normal_axis, position, coords_a, coords_b, resolution, grid_shape):
    """Trilinear gather plan of one component onto a plane's sample points
    (beamz/lattice.py:274-355).  Axes are named "z", "y", "x"; ``coords_a``
    and ``coords_b`` lie on the two in-plane axes in storage order."""
    names = ("z", "y", "x")
    shape = component_shape(component, grid_shape)
    offs = {n: 0.0 if e else 0.5 for n, e in zip(names, _FACE_AXES_3D[component])}
    in_plane = [n for n in names if n != normal_axis]
    ga, gb = np.meshgrid(np.asarray(coords_a, float), np.asarray(coords_b, float), indexing="ij")
    targets = {in_plane[0]: ga.ravel(), in_plane[1]: gb.ravel(), normal_axis: np.full(ga.size, float(position))}
    axes = {}
    for ax, n in zip(names, shape):
        axes[ax] = _bracket(_axis_samples(n, offs[ax], resolution), targets[ax])
    corner = np.array([[a, b, c] for a in (0, 1) for b in (0, 1) for c in (0, 1)])
    order = (in_plane[0], in_plane[1], normal_axis)
    pick = {}
    weight = np.ones((ga.size, 8), np.float32)
    for d, ax in enumerate(order):
        lo, hi, wl, wh = axes[ax]
        use_hi = corner[:, d][None, :] == 1
        pick[ax] = np.where(use_hi, hi[:, None], lo[:, None])
        weight = weight * np.where(use_hi, wh[:, None], wl[:, None])
    flat = (pick["z"].astype(np.int64) * shape[1] + pick["y"]) * shape[2] + pick["x"]
    keep = np.abs(weight) > 4.0 * np.finfo(np.float32).eps
    weight = np.where(keep, weight, np.float32(0.0))
    total = weight.sum(axis=1, keepdims=True)
    weight = np.where(np.abs(total) > 0, weight / np.where(total == 0, 1, total), 0).astype(np.float32)
    width = int(keep.sum(axis=1).max(initial=0))
    if 0 < width < 8:
        idx = np.argsort(~keep, axis=1, kind="stable")[:, :width]
        flat = np.take_along_axis(flat, idx, axis=1)
        weight = np.take_along_axis(weight, idx, axis=1)
    return flat.astype(np.int32), weight.astype(np.float32)


def plane_monitor(grid_shape, resolution, normal_axis, position, coords_a, coords_b, freqs,
                  components=("Ey", "Ez", "Hy", "Hz"), **kwargs) -> DftMonitorPlan:
    """A plane DFT monitor over the named components (others masked off)."""
    idx, w = [], []
    for c in COMPONENTS:
        i, ww = plane_gather(c, normal_axis, position, coords_a, coords_b, resolution, grid_shape)
        idx.append(i)
        w.append(ww)
    k = max(a.shape[1] for a in idx)
    idx = [np.pad(a, ((0, 0), (0, k - a.shape[1]))) for a in idx]
    w = [np.pad(a, ((0, 0), (0, k - a.shape[1]))) for a in w]
    mask = np.array([1.0 if c in components else 0.0 for c in COMPONENTS], np.float32)
    return DftMonitorPlan(np.asarray(freqs, np.float32), idx, w, mask, **kwargs)


@dataclass
class RecorderPlan:
    """A time-domain field recorder (beamz's ``FieldRecorder``:
    devices/monitors/compiler.py:286-412, recorded by
    simulation/observe.py:588-646): after each step s with (s + 1) % interval
    == 0, while fewer than ``capacity`` records exist, one record of every
    listed component, times its sign.  ``indices``/``weights`` (per component,
    (V, K) dense flat offsets and interpolation weights, summed over K) sample
    a plane or line; None records the whole component in its own order."""

    components: tuple
    interval: int = 1
    capacity: int = 1
    indices: list | None = None
    weights: list | None = None
    shapes: tuple | None = None  # per component, the shape of one record
    signs: tuple | None = None

    def sign(self, q: int) -> float:
        return 1.0 if self.signs is None else float(self.signs[q])


def records_for(num_steps: int, interval: int) -> int:
    """Record slots of a run: ceil(num_steps / interval) (compiler.py:282-284)."""
    return int(np.ceil(int(num_steps) / max(1, int(interval))))


def domain_recorder(grid_shape, components, interval: int, num_steps: int, polarization: str = "tm") -> RecorderPlan:
    """Whole-component snapshots every ``interval`` steps (``region="domain"``)."""
    shapes = tuple(component_shape(c, grid_shape, polarization) for c in components)
    return RecorderPlan(tuple(components), max(1, int(interval)), records_for(num_steps, interval), shapes=shapes)


def plane_recorder(grid_shape, resolution, normal_axis, position, coords_a, coords_b, components, interval: int,
                   num_steps: int) -> RecorderPlan:
    """Interpolated samples of a 3D plane every ``interval`` steps, on the
    (coords_a, coords_b) points (the DFT plane gather of :func:`plane_gather`)."""
    idx, w = [], []
    for c in components:
        i, ww = plane_gather(c, normal_axis, position, coords_a, coords_b, resolution, grid_shape)
        idx.append(i)
        w.append(ww)
    shape = (len(coords_a), len(coords_b))
    return RecorderPlan(tuple(components), max(1, int(interval)), records_for(num_steps, interval), idx, w,
                        shapes=(shape,) * len(components))


def sources_clear_of_monitors(spec) -> bool:
    """True when no pre-E source cell is read by a DFT monitor's gather (same
    component, nonzero weight, component not masked off).

    A pre-E source writes the bank that the previous step's DFT sample reads,
    so only then may that sample run beside the next step."""
    boxes: dict = {}
    for src in spec.sources:
        if src.timing != "pre_e":
            continue
        ext = (1,) * (len(spec.grid_shape) - np.ndim(src.coeff)) + tuple(np.shape(src.coeff))
        boxes.setdefault(src.component, []).append((tuple(int(v) for v in src.start), ext))
    if not boxes:
        return True
    for mon in spec.monitors:
        for ci, c in enumerate(COMPONENTS):
            if c not in boxes or float(mon.component_mask[ci]) == 0.0:
                continue
            idx = np.asarray(mon.indices[ci])
            flat = idx[np.asarray(mon.weights[ci]) != 0]
            if flat.size == 0:
                continue
            shape = component_shape(c, spec.grid_shape, spec.polarization)
            flat = flat.astype(np.int64)
            for start, ext in boxes[c]:
                # only offsets between the box's first and last cell can be in it
                first = tuple(max(lo, 0) for lo in start)
                last = tuple(min(lo + n, d) - 1 for lo, n, d in zip(start, ext, shape))
                if any(a > b for a, b in zip(first, last)):
                    continue
                lo_flat, hi_flat = np.ravel_multi_index(first, shape), np.ravel_multi_index(last, shape)
                near = flat[(flat >= lo_flat) & (flat <= hi_flat)]
                if near.size == 0:
                    continue
                coords = np.unravel_index(near, shape)
                inside = np.ones(near.shape, bool)
                for a, (lo, n) in enumerate(zip(start, ext)):
                    inside &= (coords[a] >= lo) & (coords[a] < lo + n)
                if inside.any():
                    return False
    return True


def step_times(t0: float, dt: float, nsteps: int) -> np.ndarray:
    """t + dt after each step, accumulated in float32 like beamz's clock
    (beamz/simulation/execute.py:524-541)."""
    out = np.empty(max(int(nsteps), 1), np.float32)
    t = np.float32(t0)
    d = np.float32(dt)
    for s in range(out.size):
        t = np.float32(t + d)
        out[s] = t
    return out


# ---------------------------------------------------------------------------
# Program description
# ---------------------------------------------------------------------------


METRIC_NAMES = ("e_to_h_x", "e_to_h_y", "e_to_h_z", "h_to_e_x", "h_to_e_y", "h_to_e_z")


@dataclass(frozen=True)
class DerivativeMetrics:
    """Separable inverse distances of the staggered derivatives of an
    axis-uniform or rectilinear grid (beamz/simulation/model.py:290-303).

    ``e_to_h_a`` multiplies the forward differences along axis ``a`` that
    feed H (one value per cell, or one scalar on an axis-uniform grid);
    ``h_to_e_a`` the backward differences that feed E (cells + 1 values, or
    one scalar).  An axis the grid lacks (z in 2D) holds an empty array."""

    e_to_h_x: np.ndarray
    e_to_h_y: np.ndarray
    e_to_h_z: np.ndarray
    h_to_e_x: np.ndarray
    h_to_e_y: np.ndarray
    h_to_e_z: np.ndarray

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n in METRIC_NAMES}

    def along(self, name: str, n: int) -> np.ndarray:
        """``name``'s inverse distances as ``n`` float32 values (a scalar is
        repeated), the form the device takes."""
        v = np.asarray(getattr(self, name), np.float32)
        if v.ndim == 0:
            return np.full(n, v, np.float32)
        if v.shape != (n,):
            raise ValueError(f"{name}: {v.shape[0]} inverse distances for {n} positions")
        return np.ascontiguousarray(v)


def derivative_metrics(widths: dict, kind: str = "rectilinear") -> DerivativeMetrics | None:
    """Inverse distances from per-axis cell widths (``{"x": w, "y": w[, "z": w]}``
    in metres, float64), as beamz compiles them (compile.py:209-239):

    * ``"isotropic_uniform"``: None (every difference over the cell size);
    * ``"axis_uniform"``: one float32 scalar 1/w[0] per axis, both staggers;
    * ``"rectilinear"``: forward 1/w per cell; backward 1/w[0], then
      2/(w[i-1] + w[i]) between cells, then 1/w[-1]; each computed in float64
      and rounded once to float32.
    """
    if kind == "isotropic_uniform":
        return None
    if kind not in ("axis_uniform", "rectilinear"):
        raise ValueError(f"unknown metric kind {kind!r}")
    empty = np.zeros((0,), np.float32)
    forward, backward = {}, {}
    for axis in ("x", "y", "z"):
        if axis not in widths:
            continue
        w = np.asarray(widths[axis], np.float64).reshape(-1)
        if w.size == 0 or not np.all(w > 0):
            raise ValueError(f"axis {axis}: cell widths must be positive")
        if kind == "axis_uniform":
            forward[axis] = backward[axis] = np.float32(1.0 / float(w[0]))
            continue
        back = np.empty(w.size + 1, np.float64)
        back[0], back[-1] = 1.0 / w[0], 1.0 / w[-1]
        if w.size > 1:
            back[1:-1] = 2.0 / (w[:-1] + w[1:])
        forward[axis] = (1.0 / w).astype(np.float32)
        backward[axis] = back.astype(np.float32)
    return DerivativeMetrics(*(forward.get(a, empty) for a in ("x", "y", "z")),
                             *(backward.get(a, empty) for a in ("x", "y", "z")))


@dataclass
class ProgramSpec:
    """Host description of one simulation's step program."""

    grid_shape: tuple
    dt: float
    resolution: float
    polarization: str = "tm"
    # Voxel material (3D): uint8 ids [nz, ny, nx] and a 256-entry eps table.
    voxel_ids: np.ndarray | None = None
    eps_table: np.ndarray | None = None
    # Per-site material: component -> (decay, source), scalars or full arrays.
    e_site: dict | None = None
    h_site: dict | None = None
    # Relative permittivity per E site (component -> array over its stored
    # shape), for energy diagnostics of per-site programs; optional.
    e_site_eps: dict | None = None
    h_terms: list = field(default_factory=list)
    e_terms: list = field(default_factory=list)
    metallic_edges: frozenset = frozenset()
    sources: list = field(default_factory=list)
    monitors: list = field(default_factory=list)
    total_steps: int = 1
    t0: float = 0.0
    # Derivative metrics of an axis-uniform or rectilinear grid; None on the
    # isotropic grid (differences over `resolution`).
    metrics: DerivativeMetrics | None = None
    # Time-domain field recorders (at most four).
    recorders: list = field(default_factory=list)

    @property
    def ndim(self) -> int:
        return len(self.grid_shape)

    @property
    def cells(self) -> int:
        return int(np.prod(self.grid_shape))

    def h_coefficients(self):
        """Uniform H decay/source: fl32(dt)/fl32(mu0) in 3D (kernels.py:495-500),
        fl32(dt/mu0) in 2D (kernels.py:704-708)."""
        if self.h_site is not None:
            return self.h_site
        if self.ndim == 3:
            src = np.float32(np.float32(self.dt) / np.float32(MU_0))
        else:
            src = np.float32(float(self.dt) / MU_0)
        return {c: (np.float32(1.0), src) for c in ("Hx", "Hy", "Hz")}
