"""CPU oracle for the beamz FDTD leapfrog step -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it.
It restates, in numpy, the reference (QuentinWach/beamz v0.5.0) JAX CPU path
for the hot path -- the 3D / 2D Yee E/H updates, packed CPML psi recurrences,
slab source injection, PEC masking and running DFT monitors -- operation for
operation, so that float32 rounding follows the reference's order of
operations.  Passing ``dtype=np.float64`` gives the FP64 oracle.

Parity pin: ``tests/golden/make_golden.py`` runs the reference's own source
files (under a numpy stand-in for ``jax``) and commits their outputs as
fixtures; ``tests/test_oracle_golden.py`` checks this restatement against them.

All citations are ``path:line`` inside the beamz source tree.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

# beamz/const.py:1-5
LIGHT_SPEED = 299792458.0
EPS_0 = 8.8541878128e-12
MU_0 = 1.25663706212e-6

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")

# beamz/lattice.py:14-21 -- Yee offsets (z, y, x) in cell units.
_OFFSETS_3D = {
    "Ex": (0.0, 0.0, 0.5),
    "Ey": (0.0, 0.5, 0.0),
    "Ez": (0.5, 0.0, 0.0),
    "Hx": (0.5, 0.5, 0.0),
    "Hy": (0.5, 0.0, 0.5),
    "Hz": (0.0, 0.5, 0.5),
}

# beamz/devices/boundaries.py:13-14 -- wall order used by every boundary pass.
PLANAR_EDGES = ("left", "right", "top", "bottom")
VOLUME_EDGES = (*PLANAR_EDGES, "front", "back")

# Metallic-edge bitmask order (front, back, bottom, top, left, right),
# beamz/simulation/cuda/runtime.py:38-40.
EDGE_BITS = {"front": 0, "back": 1, "bottom": 2, "top": 3, "left": 4, "right": 5}


def component_shape_3d(component: str, grid_shape) -> tuple[int, int, int]:
    """beamz/lattice.py:32-45: +1 on every axis where the Yee offset is 0."""
    off = _OFFSETS_3D[component]
    return tuple(int(n) + int(o == 0.0) for n, o in zip(grid_shape, off))


def component_shape_2d(component: str, grid_shape, polarization: str = "tm"):
    """beamz/lattice.py:789-813 (canonical xy plane)."""
    ny, nx = (int(v) for v in grid_shape)
    table = {
        "tm": {"Ez": (ny + 1, nx + 1), "Hx": (ny, nx + 1), "Hy": (ny + 1, nx)},
        "te": {"Ex": (ny + 1, nx), "Ey": (ny, nx + 1), "Hz": (ny, nx)},
    }[polarization]
    return table.get(component, (1, 1))


def component_shapes(grid_shape, polarization: str = "tm") -> dict:
    """beamz/lattice.py:816-828."""
    if len(grid_shape) == 3:
        return {c: component_shape_3d(c, grid_shape) for c in COMPONENTS}
    return {c: component_shape_2d(c, grid_shape, polarization) for c in COMPONENTS}


# ---------------------------------------------------------------------------
# Materials
# ---------------------------------------------------------------------------


def sample_e_site_3d(voxels: np.ndarray, component: str) -> np.ndarray:
    """Centered E-site sampling, beamz/lattice.py:732-786.

    Axes are walked in storage order (z, y, x); on an axis where the E site sits
    on a cell face (offset 0) the two bracketing voxel centers are averaged as
    ``0.5 * (lo + hi)`` with clipped indices, otherwise the owning voxel is taken.
    Arithmetic is in the voxel array's dtype.
    """
    grid_shape = voxels.shape
    shape = component_shape_3d(component, grid_shape)
    off = _OFFSETS_3D[component]
    out = np.asarray(voxels)
    for axis in range(3):
        coord = np.arange(shape[axis], dtype=np.float64) + off[axis]
        if off[axis] == 0.0:
            hi = np.floor(coord).astype(np.int64)
            lo = np.clip(hi - 1, 0, grid_shape[axis] - 1)
            hi = np.clip(hi, 0, grid_shape[axis] - 1)
            half = out.dtype.type(0.5)
            out = half * (np.take(out, lo, axis=axis) + np.take(out, hi, axis=axis))
        else:
            idx = np.clip(np.floor(coord).astype(np.int64), 0, grid_shape[axis] - 1)
            out = np.take(out, idx, axis=axis)
    return out


def sample_site_2d(voxels: np.ndarray, component: str, polarization: str = "tm"):
    """beamz/lattice.py:935-972: 2D supports take the owning voxel (no averaging)."""
    ny, nx = voxels.shape
    shape = component_shape_2d(component, voxels.shape, polarization)
    y_off, x_off = {
        "Ez": (0.0, 0.0),
        "Hx": (0.5, 0.0),
        "Hy": (0.0, 0.5),
        "Ex": (0.0, 0.5),
        "Ey": (0.5, 0.0),
        "Hz": (0.5, 0.5),
    }[component]
    yi = np.clip(np.floor(np.arange(shape[0]) + y_off).astype(np.int64), 0, ny - 1)
    xi = np.clip(np.floor(np.arange(shape[1]) + x_off).astype(np.int64), 0, nx - 1)
    return np.asarray(voxels)[np.ix_(yi, xi)]


def extend_materials_into_absorber(
    voxels: np.ndarray, counts: Sequence[tuple[str, int, str, int]]
) -> np.ndarray:
    """beamz/devices/_boundary_compile.py:334-363 -- copy the first interior
    material layer outward through each active CPML slab, wall by wall."""
    out = np.array(voxels, copy=True)
    for _edge, axis, side, count in counts:
        if count <= 0 or count >= out.shape[axis]:
            continue
        dst = [slice(None)] * out.ndim
        ref = [slice(None)] * out.ndim
        if side == "low":
            dst[axis] = slice(0, count)
            ref[axis] = count
        else:
            dst[axis] = slice(out.shape[axis] - count, None)
            ref[axis] = out.shape[axis] - count - 1
        out[tuple(dst)] = np.expand_dims(out[tuple(ref)], axis=axis)
    return out


# ---------------------------------------------------------------------------
# CPML planning
# ---------------------------------------------------------------------------


def cpml_sigma_max(pml_cells: int, resolution: float, m: int = 3, reflection=1e-6):
    """beamz/devices/_boundary_compile.py:244-253 (float64)."""
    eta = np.sqrt(MU_0 / (EPS_0 * 1.0))
    thickness = max(pml_cells * float(resolution), float(resolution))
    return float(-(m + 1) * np.log(max(reflection, 1e-16)) / (2.0 * eta * thickness))


def cpml_alpha_max(dt: float, is_3d: bool) -> float:
    """beamz/devices/_boundary_compile.py:254-261, boundaries.py:133-134."""
    alpha_normalized = 0.05 if is_3d else 0.1
    return float(2.0 * EPS_0 * alpha_normalized / max(float(dt), 1e-30))


def staggered_profile_1d(
    total_samples: int,
    pml_cells: int,
    low_active: bool,
    high_active: bool,
    sample_kind: str,
    sigma_max: float,
    alpha_max: float,
    kappa_max: float = 2.0,
    m: float = 3.0,
    dtype=np.float32,
):
    """beamz/devices/_boundary_compile.py:479-614 (uniform grid branch).

    E samples sit at i (i = 0..N), H samples at i + 0.5 (i = 0..N-1); the graded
    coordinate u = dist / pml_cells with dist clipped to [0, pml_cells].
    """
    f = np.dtype(dtype).type
    n = int(total_samples)
    sigma = np.zeros(n, dtype)
    kappa = np.ones(n, dtype)
    alpha = np.zeros(n, dtype)
    pml = max(int(pml_cells), 1)
    if sample_kind == "E":
        offset, domain_cells = 0.0, n - 1
    else:
        offset, domain_cells = 0.5, n
    coords = np.arange(n, dtype=dtype) + f(offset)
    scale = f(max(float(pml), 1e-30))

    def apply_u(u):
        u = np.clip(np.asarray(u, dtype=dtype), f(0.0), f(1.0))
        s = f(sigma_max) * np.power(u, f(m))
        k = f(1.0) + (f(kappa_max) - f(1.0)) * np.power(u, f(m))
        a = f(alpha_max) * np.power(f(1.0) - u, f(1.0))
        return s, k, a

    sides = []
    if low_active:
        sides.append(np.clip(f(pml) - coords, f(0.0), f(pml)))
    if high_active:
        sides.append(np.clip(coords - f(domain_cells - pml), f(0.0), f(pml)))
    for dist in sides:
        mask = dist > f(0.0)
        s, k, a = apply_u(dist / scale)
        sigma = np.where(mask, np.maximum(sigma, s), sigma)
        kappa = np.where(mask, np.maximum(kappa, k), kappa)
        alpha = np.where(mask, np.maximum(alpha, a), alpha)
    return sigma.astype(dtype), kappa.astype(dtype), alpha.astype(dtype)


def cpml_coefficients(sigma, kappa, alpha, dt, dtype=np.float32):
    """beamz/simulation/kernels.py:130-144: b = exp(-(s/k + a) dt/eps0),
    a = (b - 1) s / ((s + k a) k), and 1/k, in ``dtype``."""
    f = np.dtype(dtype).type
    sigma = np.asarray(sigma, dtype)
    kappa = np.maximum(np.asarray(kappa, dtype), f(1.0))
    alpha = np.asarray(alpha, dtype)
    one = f(1.0)
    decay = (sigma / kappa + alpha) * (f(dt) / f(EPS_0))
    b = np.exp(-decay)
    a = np.nan_to_num(((b - one) * sigma) / np.maximum((sigma + kappa * alpha) * kappa, f(1e-30)))
    return a.astype(dtype), b.astype(dtype), (one / kappa).astype(dtype)


def active_slab_counts(a: np.ndarray, inv_kappa: np.ndarray) -> tuple[int, int]:
    """beamz/simulation/kernels.py:225-235 for a 1-D profile."""
    active = (np.abs(np.asarray(a)) > 1e-30) | (np.abs(np.asarray(inv_kappa) - 1.0) > 1e-7)
    low = next((i for i, v in enumerate(active) if not v), active.size)
    tail = active[low:][::-1]
    high = next((i for i, v in enumerate(tail) if not v), tail.size)
    return int(low), int(high)


@dataclass
class CpmlTerm:
    """One packed CPML recurrence (beamz/simulation/model.py:306-324).

    ``a``, ``b``, ``inv_kappa`` are 1-D, of length ``low + high``, along ``axis``
    of the target component; psi has the target shape with that axis replaced
    by ``low + high``.
    """

    component: str
    axis: int
    sign: float
    low: int
    high: int
    a: np.ndarray
    b: np.ndarray
    inv_kappa: np.ndarray
    full_len: int

    def psi_shape(self, target_shape):
        shape = list(target_shape)
        shape[self.axis] = self.low + self.high
        return tuple(shape)


def compile_cpml_term(component, axis, sign, sigma, kappa, alpha, dt, full_len, dtype=np.float32):
    """beamz/simulation/kernels.py:238-254."""
    a, b, k = cpml_coefficients(sigma, kappa, alpha, dt, dtype)
    low, high = active_slab_counts(a, k)
    sel = np.r_[0:low, full_len - high : full_len].astype(np.int64)
    return CpmlTerm(component, int(axis), float(sign), low, high, a[sel], b[sel], k[sel], int(full_len))


# Derivative order and signs: beamz/devices/_boundary_compile.py:44-60 and
# beamz/simulation/compile.py:271-283 (index % 2 == 0 -> +1).  Axis: 0=z 1=y 2=x.
CPML_3D_H_TERMS = (("Hx", 1), ("Hx", 0), ("Hy", 0), ("Hy", 2), ("Hz", 2), ("Hz", 1))
CPML_3D_E_TERMS = (("Ex", 1), ("Ex", 0), ("Ey", 0), ("Ey", 2), ("Ez", 2), ("Ez", 1))
# 2D (beamz/simulation/compile.py:285-304): (component, axis, sign).
CPML_2D_TERMS = {
    "tm": ((("Hx", 0, 1.0), ("Hy", 1, -1.0)), (("Ez", 1, 1.0), ("Ez", 0, -1.0))),
    "te": ((("Hz", 1, 1.0), ("Hz", 0, -1.0)), (("Ex", 0, 1.0), ("Ey", 1, -1.0))),
}
_AXIS_FACES = {0: ("front", "back"), 1: ("bottom", "top"), 2: ("left", "right")}
_AXIS_FACES_2D = {0: ("bottom", "top"), 1: ("left", "right")}


def plan_cpml(
    grid_shape,
    dt: float,
    resolution: float,
    pml_cells: int = 12,
    edges=None,
    polarization: str = "tm",
    dtype=np.float32,
    kappa_max: float = 2.0,
    m: int = 3,
    reflection: float = 1e-6,
):
    """Plan every CPML term for a uniform grid (compile.py:241-305 with the
    profiles of _boundary_compile.py:735-820 / 660-733).

    Returns ``(h_terms, e_terms)``.
    """
    is_3d = len(grid_shape) == 3
    edges = set(VOLUME_EDGES if is_3d else PLANAR_EDGES) if edges is None else set(edges)
    sigma_max = cpml_sigma_max(pml_cells, resolution, m, reflection)
    alpha_max = cpml_alpha_max(dt, is_3d)
    shapes = component_shapes(grid_shape, polarization)
    if is_3d:
        specs = [(c, ax, 1.0 if i % 2 == 0 else -1.0) for i, (c, ax) in enumerate(CPML_3D_H_TERMS)]
        specs_e = [(c, ax, 1.0 if i % 2 == 0 else -1.0) for i, (c, ax) in enumerate(CPML_3D_E_TERMS)]
        faces = _AXIS_FACES
    else:
        specs, specs_e = CPML_2D_TERMS[polarization]
        faces = _AXIS_FACES_2D

    def build(spec_list):
        terms = []
        for comp, axis, sign in spec_list:
            target = shapes[comp]
            cells = int(grid_shape[axis])
            if is_3d:
                kind = "E" if _OFFSETS_3D[comp][axis] == 0.0 else "H"
            else:
                kind = "E" if comp.startswith("E") else "H"
            samples = target[axis]
            low_face, high_face = faces[axis]
            s, k, a = staggered_profile_1d(
                samples, pml_cells, low_face in edges, high_face in edges, kind,
                sigma_max, alpha_max, kappa_max, m, dtype,
            )
            terms.append(compile_cpml_term(comp, axis, sign, s, k, a, dt, samples, dtype))
        return terms

    return build(specs), build(specs_e)


def cpml_material_edge_counts(grid_shape, pml_cells, edges=None, resolution=None, explicit_thickness=False):
    """(edge, axis, side, count) per active wall, in the wall order of
    beamz/devices/boundaries.py:13-14 (_boundary_compile.py:278-319), where
    ``count`` is the run of cell-centred CPML sigma > 0 from that wall.

    The default cell-count PML grades logical centres ``i + 0.5`` against a
    thickness of ``pml_cells``; an explicit physical thickness grades
    ``linspace(0, L, n)`` against ``pml_cells * resolution``
    (_boundary_compile.py:424-440, 404-421).
    """
    is_3d = len(grid_shape) == 3
    edges = tuple(VOLUME_EDGES if is_3d else PLANAR_EDGES) if edges is None else tuple(edges)
    axis_map = {"z": 0, "y": 1, "x": 2} if is_3d else {"y": 0, "x": 1}
    edge_axes = {
        "left": ("x", "low"), "right": ("x", "high"), "bottom": ("y", "low"),
        "top": ("y", "high"), "front": ("z", "low"), "back": ("z", "high"),
    }
    out = []
    for edge in edges:
        axis_name, side = edge_axes[edge]
        if axis_name not in axis_map:
            continue
        axis = axis_map[axis_name]
        n = int(grid_shape[axis])
        if explicit_thickness:
            length = np.float32(n * float(resolution))
            thickness = np.float32(pml_cells * float(resolution))
            coords = np.linspace(0, float(n * float(resolution)), n).astype(np.float32)
        else:
            length = np.float32(n)
            thickness = np.float32(pml_cells)
            coords = np.arange(n, dtype=np.float32) + np.float32(0.5)
        if side == "low":
            active = np.clip(thickness - coords, 0.0, None) > 0
            count = int(np.argmax(~active)) if np.any(~active) else 0
        else:
            active = np.clip(coords - (length - thickness), 0.0, None) > 0
            rev = active[::-1]
            count = int(np.argmax(~rev)) if np.any(~rev) else 0
        out.append((edge, axis, side, count))
    return out


# ---------------------------------------------------------------------------
# PEC
# ---------------------------------------------------------------------------

# beamz/devices/_boundary_compile.py:129-153
_WALLS_3D = {
    "front": (0, 0, ("Ex", "Ey", "Hz")), "back": (0, -1, ("Ex", "Ey", "Hz")),
    "bottom": (1, 0, ("Ex", "Ez", "Hy")), "top": (1, -1, ("Ex", "Ez", "Hy")),
    "left": (2, 0, ("Ey", "Ez", "Hx")), "right": (2, -1, ("Ey", "Ez", "Hx")),
}
_WALLS_2D = {
    "tm": {
        "bottom": (0, 0, ("Ez", "Hy")), "top": (0, -1, ("Ez", "Hy")),
        "left": (1, 0, ("Ez", "Hx")), "right": (1, -1, ("Ez", "Hx")),
    },
    "te": {
        "bottom": (0, 0, ("Ex",)), "top": (0, -1, ("Ex",)),
        "left": (1, 0, ("Ey",)), "right": (1, -1, ("Ey",)),
    },
}


def pec_masks(shapes: dict, ndim: int, metallic_edges, polarization="tm") -> dict:
    """beamz/devices/_boundary_compile.py:118-160 -- boolean masks per component."""
    masks = {c: np.zeros(shapes[c], dtype=bool) for c in COMPONENTS}
    walls = _WALLS_3D if ndim == 3 else _WALLS_2D[polarization]
    for edge in metallic_edges:
        axis, index, comps = walls[edge]
        for comp in comps:
            sel = [slice(None)] * ndim
            sel[axis] = index
            masks[comp][tuple(sel)] = True
    return masks


# ---------------------------------------------------------------------------
# Packed CPML slab algebra (beamz/simulation/kernels.py:184-264)
# ---------------------------------------------------------------------------


def _region(ndim, axis, start, stop):
    r = [slice(None)] * ndim
    r[axis] = slice(start, stop)
    return tuple(r)


def _bshape(ndim, axis, n):
    s = [1] * ndim
    s[axis] = n
    return tuple(s)


def _pack(arr, term: CpmlTerm):
    parts = []
    stop = arr.shape[term.axis]
    if term.low:
        parts.append(arr[_region(arr.ndim, term.axis, 0, term.low)])
    if term.high:
        parts.append(arr[_region(arr.ndim, term.axis, stop - term.high, stop)])
    return parts[0] if len(parts) == 1 else np.concatenate(parts, axis=term.axis)


def _unpack(base, packed, term: CpmlTerm):
    out = np.array(base, copy=True)
    stop = base.shape[term.axis]
    if term.low:
        out[_region(base.ndim, term.axis, 0, term.low)] = packed[_region(base.ndim, term.axis, 0, term.low)]
    if term.high:
        out[_region(base.ndim, term.axis, stop - term.high, stop)] = packed[
            _region(base.ndim, term.axis, term.low, term.low + term.high)
        ]
    return out


def correct_cpml_term(derivative, psi, term: CpmlTerm):
    """beamz/simulation/kernels.py:257-264: psi <- b psi + a d; d' = d / kappa + psi;
    returns (sign * d', psi) with d' spliced into the slabs only."""
    dtype = derivative.dtype
    sign = dtype.type(term.sign)
    if not term.low and not term.high:
        return sign * derivative, psi
    nd = derivative.ndim
    ds = _pack(derivative, term)
    b = term.b.astype(dtype).reshape(_bshape(nd, term.axis, term.b.size))
    a = term.a.astype(dtype).reshape(_bshape(nd, term.axis, term.a.size))
    k = term.inv_kappa.astype(dtype).reshape(_bshape(nd, term.axis, term.inv_kappa.size))
    psi = b * psi + a * ds
    corrected = ds * k + psi
    return sign * _unpack(derivative, corrected, term), psi


# ---------------------------------------------------------------------------
# 3D updates
# ---------------------------------------------------------------------------


def _ghost_pad(arr, axis, metallic_edges):
    """beamz/lattice.py:523-551: one ghost plane per side; zero on a metallic
    face, else a copy of the edge plane (so the edge derivative vanishes)."""
    low_edge, high_edge = (("front", "back"), ("bottom", "top"), ("left", "right"))[axis]
    shape = list(arr.shape)
    shape[axis] = 1
    zero = np.zeros(shape, dtype=arr.dtype)
    low = zero if low_edge in metallic_edges else np.take(arr, [0], axis=axis)
    high = zero if high_edge in metallic_edges else np.take(arr, [arr.shape[axis] - 1], axis=axis)
    return np.concatenate((low, arr, high), axis=axis)


def _ghost_pad_2d(arr, axis, metallic_edges):
    """beamz/simulation/kernels.py:741-756 / 812-826 (axis 0 = y, 1 = x)."""
    low_edge, high_edge = (("bottom", "top"), ("left", "right"))[axis]
    shape = list(arr.shape)
    shape[axis] = 1
    zero = np.zeros(shape, dtype=arr.dtype)
    low = zero if low_edge in metallic_edges else np.take(arr, [0], axis=axis)
    high = zero if high_edge in metallic_edges else np.take(arr, [arr.shape[axis] - 1], axis=axis)
    return np.concatenate((low, arr, high), axis=axis)


def _metric_diff(arr, axis, res, inverse_distance=None):
    """Difference along ``axis`` over the cell size: ``np.diff / res`` on an
    isotropic grid (kernels.py:477-488), ``np.diff * inverse_distance`` (a
    scalar or one value per difference along the axis) with a derivative
    metric (kernels.py:164-176)."""
    d = np.diff(arr, axis=axis)
    if inverse_distance is None:
        return d / res
    m = np.asarray(inverse_distance, d.dtype)
    if m.ndim == 0:
        return d * m
    shape = [1] * d.ndim
    shape[axis] = m.shape[0]
    return d * m.reshape(shape)


def _metric(metrics, name):
    return None if metrics is None else metrics[name]


@dataclass
class Material3D:
    """E-site permittivity (and optional conductivity) plus H-site magnetic
    conductivity, as used by beamz/simulation/kernels.py:1074-1170."""

    eps: tuple  # (eps_x, eps_y, eps_z) on Ex/Ey/Ez supports
    sigma: tuple = (0.0, 0.0, 0.0)  # electric conductivity on E supports (or scalars)
    sigma_m: tuple = (0.0, 0.0, 0.0)  # magnetic conductivity on H supports (or scalars)


def material_from_voxels(voxel_eps: np.ndarray, voxel_sigma=None, dtype=np.float32) -> Material3D:
    """E-site sampling of a voxel permittivity grid (lattice.py:1003-1012)."""
    v = np.asarray(voxel_eps, dtype=dtype)
    eps = tuple(sample_e_site_3d(v, c) for c in ("Ex", "Ey", "Ez"))
    if voxel_sigma is None or not np.any(np.asarray(voxel_sigma)):
        return Material3D(eps)
    s = np.asarray(voxel_sigma, dtype=dtype)
    return Material3D(eps, tuple(sample_e_site_3d(s, c) for c in ("Ex", "Ey", "Ez")))


def update_h_3d(fields, psi_h, h_terms, dt, resolution, sigma_m=(0.0, 0.0, 0.0), coeffs=None, metrics=None):
    """beamz/simulation/kernels.py:458-503 (``h_terms`` empty => kernels.py:267-290
    without CPML).  Returns (hx, hy, hz, psi_h).

    ``metrics`` (a mapping with beamz's ``DerivativeMetricPlan`` names,
    model.py:290-303) scales each difference by its inverse distance instead
    of dividing by the cell size (kernels.py:293-323, 506-551).

    ``coeffs`` (component -> (decay, source) arrays) selects the form of
    beamz's CUDA path instead, which receives precomputed coefficients:
    H <- decay * H - source * curl with the same (CPML-corrected) curl
    (cuda/src/update.cu:392-410 and 585-597)."""
    ex, ey, ez, hx, hy, hz = (fields[c] for c in COMPONENTS)
    dtype = hx.dtype
    f = dtype.type
    res = f(resolution)
    derivs = (
        _metric_diff(ez, 1, res, _metric(metrics, "e_to_h_y")),
        _metric_diff(ey, 0, res, _metric(metrics, "e_to_h_z")),
        _metric_diff(ex, 0, res, _metric(metrics, "e_to_h_z")),
        _metric_diff(ez, 2, res, _metric(metrics, "e_to_h_x")),
        _metric_diff(ey, 2, res, _metric(metrics, "e_to_h_x")),
        _metric_diff(ex, 1, res, _metric(metrics, "e_to_h_y")),
    )
    one = f(1.0)
    dt_over_mu = f(dt) / f(MU_0)
    new_psi = list(psi_h) if psi_h else []
    if h_terms:
        corrected = []
        for i, (d, term) in enumerate(zip(derivs, h_terms)):
            c, p = correct_cpml_term(d, psi_h[i], term)
            corrected.append(c)
            new_psi[i] = p
        curls = tuple(corrected[i] + corrected[i + 1] for i in (0, 2, 4))
        out = []
        if coeffs is not None:
            for c, fld, curl in zip(("Hx", "Hy", "Hz"), (hx, hy, hz), curls):
                decay, source = (np.asarray(v, dtype) for v in coeffs[c])
                out.append(decay * fld - source * curl)
            return out[0].astype(dtype), out[1].astype(dtype), out[2].astype(dtype), new_psi
        for fld, curl, sm in zip((hx, hy, hz), curls, sigma_m):
            alpha = np.asarray(sm, dtype) * (f(0.5) * dt_over_mu)
            out.append(((one - alpha) * fld - dt_over_mu * curl) / (one + alpha))
    else:
        curls = (derivs[0] - derivs[1], derivs[2] - derivs[3], derivs[4] - derivs[5])
        out = []
        if coeffs is not None:
            for c, fld, curl in zip(("Hx", "Hy", "Hz"), (hx, hy, hz), curls):
                decay, source = (np.asarray(v, dtype) for v in coeffs[c])
                out.append(decay * fld - source * curl)
            return out[0].astype(dtype), out[1].astype(dtype), out[2].astype(dtype), new_psi
        for fld, curl, sm in zip((hx, hy, hz), curls, sigma_m):
            alpha = np.asarray(sm, dtype) * (f(0.5) * dt_over_mu)
            denom = one + alpha
            out.append((one - alpha) / denom * fld - (dt_over_mu / denom) * curl)
    return out[0].astype(dtype), out[1].astype(dtype), out[2].astype(dtype), new_psi


def update_e_3d(fields, psi_e, e_terms, dt, resolution, material: Material3D, metallic_edges=(), coeffs=None,
                metrics=None):
    """beamz/simulation/kernels.py:554-626 (``e_terms`` empty =>
    kernels.py:326-388).  Returns (ex, ey, ez, psi_e).  ``metrics`` as in
    :func:`update_h_3d` (kernels.py:391-455, 629-701)."""
    ex, ey, ez, hx, hy, hz = (fields[c] for c in COMPONENTS)
    dtype = ex.dtype
    f = dtype.type
    res = f(resolution)
    views = {
        "hz_y": _ghost_pad(hz, 1, metallic_edges),
        "hy_z": _ghost_pad(hy, 0, metallic_edges),
        "hx_z": _ghost_pad(hx, 0, metallic_edges),
        "hz_x": _ghost_pad(hz, 2, metallic_edges),
        "hy_x": _ghost_pad(hy, 2, metallic_edges),
        "hx_y": _ghost_pad(hx, 1, metallic_edges),
    }
    derivs = (
        _metric_diff(views["hz_y"], 1, res, _metric(metrics, "h_to_e_y")),
        _metric_diff(views["hy_z"], 0, res, _metric(metrics, "h_to_e_z")),
        _metric_diff(views["hx_z"], 0, res, _metric(metrics, "h_to_e_z")),
        _metric_diff(views["hz_x"], 2, res, _metric(metrics, "h_to_e_x")),
        _metric_diff(views["hy_x"], 2, res, _metric(metrics, "h_to_e_x")),
        _metric_diff(views["hx_y"], 1, res, _metric(metrics, "h_to_e_y")),
    )
    one = f(1.0)
    dt_over_eps = f(dt) / f(EPS_0)
    # (per-site coefficient programs carry no material: only ``coeffs`` is read)
    inv = tuple(one / np.asarray(e, dtype) for e in material.eps) if material is not None else (None,) * 3
    new_psi = list(psi_e) if psi_e else []
    if e_terms:
        corrected = []
        for i, (d, term) in enumerate(zip(derivs, e_terms)):
            c, p = correct_cpml_term(d, psi_e[i], term)
            corrected.append(c)
            new_psi[i] = p
        curls = tuple(corrected[i] + corrected[i + 1] for i in (0, 2, 4))
        out = []
        if coeffs is not None:  # beamz's CUDA path: cuda/src/update.cu:644-652
            for c, fld, curl in zip(("Ex", "Ey", "Ez"), (ex, ey, ez), curls):
                decay, source = (np.asarray(v, dtype) for v in coeffs[c])
                out.append(decay * fld + source * curl)
            return out[0].astype(dtype), out[1].astype(dtype), out[2].astype(dtype), new_psi
        for fld, curl, cond, iv in zip((ex, ey, ez), curls, material.sigma, inv):
            beta = np.asarray(cond, dtype) * (f(0.5) * dt_over_eps) * iv
            out.append(((one - beta) * fld + dt_over_eps * iv * curl) / (one + beta))
    else:
        curls = (derivs[0] - derivs[1], derivs[2] - derivs[3], derivs[4] - derivs[5])
        out = []
        if coeffs is not None:  # cuda/src/update.cu:392-410
            for c, fld, curl in zip(("Ex", "Ey", "Ez"), (ex, ey, ez), curls):
                decay, source = (np.asarray(v, dtype) for v in coeffs[c])
                out.append(decay * fld + source * curl)
            return out[0].astype(dtype), out[1].astype(dtype), out[2].astype(dtype), new_psi
        for fld, curl, cond, iv in zip((ex, ey, ez), curls, material.sigma, inv):
            beta = np.asarray(cond, dtype) * (f(0.5) * dt_over_eps) * iv
            denom = one + beta
            out.append((one - beta) / denom * fld + (dt_over_eps * iv / denom) * curl)
    return out[0].astype(dtype), out[1].astype(dtype), out[2].astype(dtype), new_psi


# ---------------------------------------------------------------------------
# 2D updates (canonical xy plane)
# ---------------------------------------------------------------------------


def h_coefficients_2d(dt, dtype=np.float32):
    """beamz/simulation/kernels.py:704-708 with zero magnetic conductivity:
    decay = 1, source = fl(dt / MU_0)."""
    f = np.dtype(dtype).type
    return f(1.0), f(float(dt) / MU_0)


def e_coefficients_2d(eps_site, dt, dtype=np.float32):
    """beamz/simulation/kernels.py:711-728 with zero conductivity:
    decay = 1, source = dt / (EPS_0 * eps) evaluated in ``dtype``."""
    f = np.dtype(dtype).type
    eps = np.asarray(eps_site, dtype)
    return np.ones_like(eps), (f(dt) / (f(EPS_0) * eps)).astype(dtype)


def update_h_2d(fields, psi_h, h_terms, resolution, h_coeffs, polarization="tm", metrics=None):
    """TM: beamz/simulation/kernels.py:731-738, 771-788, 1217-1243;
    TE: kernels.py:791-797, 838-850, 1286-1300.  ``h_coeffs`` is one
    (decay, source) pair for every H component, or a dict component ->
    (decay, source) (per-site arrays of a magnetically lossy material).
    ``metrics``: inverse distances as in :func:`update_h_3d` (kernels.py:880-1012)."""
    dtype = fields["Ez" if polarization == "tm" else "Hz"].dtype
    res = dtype.type(resolution)
    per = h_coeffs if isinstance(h_coeffs, dict) else None
    decay, source = h_coeffs["Hx" if polarization == "tm" else "Hz"] if per else h_coeffs
    new_psi = list(psi_h) if psi_h else []
    if polarization == "tm":
        ez, hx, hy = fields["Ez"], fields["Hx"], fields["Hy"]
        d0 = _metric_diff(ez, 0, res, _metric(metrics, "e_to_h_y"))
        d1 = _metric_diff(ez, 1, res, _metric(metrics, "e_to_h_x"))
        if h_terms:
            c0, new_psi[0] = correct_cpml_term(d0, psi_h[0], h_terms[0])
            c1, new_psi[1] = correct_cpml_term(d1, psi_h[1], h_terms[1])
        else:
            c0, c1 = d0, -d1
        hx_n = decay * hx - source * c0
        if per:
            decay, source = per["Hy"]
        hy_n = decay * hy - source * c1
        return {"Hx": hx_n.astype(dtype), "Hy": hy_n.astype(dtype)}, new_psi
    ex, ey, hz = fields["Ex"], fields["Ey"], fields["Hz"]
    d0 = _metric_diff(ey, 1, res, _metric(metrics, "e_to_h_x"))
    d1 = _metric_diff(ex, 0, res, _metric(metrics, "e_to_h_y"))
    if h_terms:
        c0, new_psi[0] = correct_cpml_term(d0, psi_h[0], h_terms[0])
        c1, new_psi[1] = correct_cpml_term(d1, psi_h[1], h_terms[1])
        curl = c0 + c1
    else:
        curl = d0 - d1
    return {"Hz": (decay * hz - source * curl).astype(dtype)}, new_psi


def update_e_2d(fields, psi_e, e_terms, resolution, e_coeffs, metallic_edges=(), polarization="tm", metrics=None):
    """TM: kernels.py:741-769, 800-823, 1258-1283; TE: kernels.py:800-836,
    852-860, 1303-1342.  ``e_coeffs`` maps component -> (decay, source)."""
    new_psi = list(psi_e) if psi_e else []
    if polarization == "tm":
        hx, hy, ez = fields["Hx"], fields["Hy"], fields["Ez"]
        dtype = ez.dtype
        res = dtype.type(resolution)
        phy = _ghost_pad_2d(hy, 1, metallic_edges)
        phx = _ghost_pad_2d(hx, 0, metallic_edges)
        d_hy_dx = _metric_diff(phy, 1, res, _metric(metrics, "h_to_e_x"))
        d_hx_dy = _metric_diff(phx, 0, res, _metric(metrics, "h_to_e_y"))
        if e_terms:
            c0, new_psi[0] = correct_cpml_term(d_hy_dx, psi_e[0], e_terms[0])
            c1, new_psi[1] = correct_cpml_term(d_hx_dy, psi_e[1], e_terms[1])
            curl = (c0 + c1).astype(dtype)
        else:
            curl = d_hy_dx - d_hx_dy
        decay, source = e_coeffs["Ez"]
        return {"Ez": (decay * ez + source * curl).astype(dtype)}, new_psi
    hz, ex, ey = fields["Hz"], fields["Ex"], fields["Ey"]
    dtype = ex.dtype
    res = dtype.type(resolution)
    py = _ghost_pad_2d(hz, 0, metallic_edges)
    px = _ghost_pad_2d(hz, 1, metallic_edges)
    d_hz_dy = _metric_diff(py, 0, res, _metric(metrics, "h_to_e_y"))
    d_hz_dx = _metric_diff(px, 1, res, _metric(metrics, "h_to_e_x"))
    if e_terms:
        c0, new_psi[0] = correct_cpml_term(d_hz_dy, psi_e[0], e_terms[0])
        c1, new_psi[1] = correct_cpml_term(d_hz_dx, psi_e[1], e_terms[1])
        curls = (c0, c1)
    else:
        curls = (d_hz_dy, -d_hz_dx)
    dx_, sx_ = e_coeffs["Ex"]
    dy_, sy_ = e_coeffs["Ey"]
    return {
        "Ex": (dx_ * ex + sx_ * curls[0]).astype(dtype),
        "Ey": (dy_ * ey + sy_ * curls[1]).astype(dtype),
    }, new_psi


# ---------------------------------------------------------------------------
# Sources
# ---------------------------------------------------------------------------


@dataclass
class SlabSource:
    """One slab injection ``field[start:start+shape] += coeff * waveform[step]``
    (beamz/devices/sources/compiler.py:116-129, execute.py:374-433)."""

    component: str
    timing: str  # "pre_e" | "h" | "e"
    start: tuple
    coeff: np.ndarray
    waveform: np.ndarray


def gaussian_pulse_sample(times, freq0, fwidth, amplitude=1.0, offset=4.0, remove_dc=True):
    """beamz/devices/sources/time.py:459-487 (in-phase float32 samples)."""
    t = np.asarray(times, dtype=float)
    width = 1.0 / (2.0 * np.pi * max(float(fwidth), 1e-30))
    peak = float(offset) / max(float(fwidth), 1e-30)
    envelope = float(amplitude) * np.exp(-((t - peak) ** 2) / (2.0 * width**2))
    signal = envelope * np.cos(2.0 * np.pi * float(freq0) * t)
    if remove_dc and signal.size:
        signal = signal - np.mean(signal)
    return signal.astype(np.float32)


def apply_sources(fields, sources: Sequence[SlabSource], timing: str, step: int):
    """beamz/simulation/execute.py:436-461: in declaration order, each slab adds
    ``(coeff * waveform[clip(step)]).astype(field dtype)``."""
    for src in sources:
        if src.timing != timing:
            continue
        arr = fields[src.component]
        wf = np.asarray(src.waveform)
        amp = wf[min(max(int(step), 0), wf.shape[0] - 1)]
        coeff = np.asarray(src.coeff)
        patch = (coeff.astype(np.float32) * np.float32(amp)).astype(arr.dtype) if arr.dtype == np.float32 else (
            coeff.astype(arr.dtype) * arr.dtype.type(amp)
        )
        sl = tuple(slice(int(s), int(s) + int(n)) for s, n in zip(src.start, coeff.shape))
        arr[sl] = arr[sl] + patch


# ---------------------------------------------------------------------------
# DFT monitors
# ---------------------------------------------------------------------------


def linear_interpolation_plan(source, target):
    """beamz/lattice.py:241-271."""
    source = np.asarray(source, dtype=np.float64).reshape(-1)
    target = np.asarray(target, dtype=np.float64).reshape(-1)
    if source.size == 1:
        idx = np.zeros(target.size, dtype=np.int32)
        return idx, idx, np.ones(target.size, np.float32), np.zeros(target.size, np.float32)
    high = np.clip(np.searchsorted(source, target, side="right"), 1, source.size - 1)
    low = high - 1
    low[target <= source[0]] = 0
    high[target <= source[0]] = 0
    low[target >= source[-1]] = source.size - 1
    high[target >= source[-1]] = source.size - 1
    den = source[high] - source[low]
    alpha = np.divide(target - source[low], den, out=np.zeros_like(target),
                      where=(high != low) & (np.abs(den) > 0.0))
    wh = alpha.astype(np.float32)
    wl = (1.0 - alpha).astype(np.float32)
    wl[high == low] = 1.0
    wh[high == low] = 0.0
    return low.astype(np.int32), high.astype(np.int32), wl, wh


def plane_gather_plan_3d(component, normal_axis, plane_position, coords0, coords1, resolution, grid_shape):
    """beamz/lattice.py:274-355 for a uniform grid.

    ``normal_axis`` in {"x","y","z"}; ``coords0``/``coords1`` are the in-plane
    target coordinates (metres) on the two remaining axes in (z, y, x) order.
    Returns (flat_indices (P, K) int32, weights (P, K) float32).
    """
    axes = [a for a in ("z", "y", "x") if a != normal_axis]
    axis0, axis1 = axes
    shape = component_shape_3d(component, grid_shape)
    off = dict(zip(("z", "y", "x"), _OFFSETS_3D[component]))
    lengths = dict(zip(("z", "y", "x"), shape))
    um = 1e-6
    dx_um = float(resolution / um)
    coords = {a: (np.arange(lengths[a], dtype=np.float64) + off[a]) * dx_um * um for a in ("z", "y", "x")}
    g0, g1 = np.meshgrid(coords0, coords1, indexing="ij")
    t0, t1 = g0.reshape(-1), g1.reshape(-1)
    tn = np.full_like(t0, float(plane_position))
    plans = (
        linear_interpolation_plan(coords[axis0], t0),
        linear_interpolation_plan(coords[axis1], t1),
        linear_interpolation_plan(coords[normal_axis], tn),
    )
    bits = np.asarray([(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)], dtype=np.int32)
    indices, weights = [], []
    for d, (lo, hi, wl, wh) in enumerate(plans):
        bit = bits[:, d][None, :]
        indices.append(np.where(bit == 0, lo[:, None], hi[:, None]))
        weights.append(np.where(bit == 0, wl[:, None], wh[:, None]))
    imap = {axis0: indices[0], axis1: indices[1], normal_axis: indices[2]}
    flat = np.asarray(np.ravel_multi_index((imap["z"], imap["y"], imap["x"]), dims=shape), dtype=np.int32)
    w = np.prod(np.stack(weights), axis=0).astype(np.float32)
    nz = np.abs(w) > 4.0 * np.finfo(np.float32).eps
    w = np.where(nz, w, 0.0)
    rs = np.sum(w, axis=1, keepdims=True)
    w = np.divide(w, rs, out=np.zeros_like(w), where=np.abs(rs) > 0.0)
    width = int(np.max(np.sum(nz, axis=1), initial=0))
    if 0 < width < w.shape[1]:
        order = np.argsort(~nz, axis=1, kind="stable")[:, :width]
        flat = np.take_along_axis(flat, order, axis=1)
        w = np.take_along_axis(w, order, axis=1)
    return flat, w.astype(np.float32)


@dataclass
class DftMonitor:
    """Compiled vector-DFT plan (beamz/devices/monitors/compiler.py:62-102).

    ``indices[c]``/``weights[c]`` (P, K) gather component ``c`` (order Ex..Hz);
    ``component_mask[c]`` enables it.  Accumulators are laid out as
    ``value_offset + (c * F + f) * P + p`` (beamz/simulation/observe.py:569-577).
    """

    freqs: np.ndarray
    indices: list
    weights: list
    component_mask: np.ndarray
    t_start: float = 0.0
    t_end: float = float("inf")
    interval: int = 1
    window_code: int = 0  # 1 = Hann
    normalization_code: int = 0  # 1 = physical units
    length_unit: float = 1e-6
    value_offset: int = 0
    weight_offset: int = 0

    @property
    def point_count(self):
        return int(self.indices[0].shape[0])


def dft_arena_sizes(monitors: Sequence[DftMonitor]):
    """beamz/simulation/observe.py:403-410."""
    values = sum(6 * len(m.freqs) * m.point_count for m in monitors)
    weights = sum(len(m.freqs) for m in monitors)
    return values, weights


def dft_window_weight(t, t0, t1, use_hann, dtype=np.float32):
    """beamz/simulation/observe.py:337-343."""
    f = np.dtype(dtype).type
    t, t0, t1 = f(t), f(t0), f(t1)
    span = np.maximum(t1 - t0, f(1e-30))
    tau = np.clip((t - t0) / span, f(0.0), f(1.0))
    hann = f(0.5) * (f(1.0) - np.cos(f(2.0 * np.pi) * tau))
    return hann if (use_hann and np.isfinite(t1) and t1 > t0) else f(1.0)


def dft_sample_scale(weight, code, base_dt, interval, length_unit, dtype=np.float32):
    """beamz/simulation/observe.py:346-357."""
    f = np.dtype(dtype).type
    native = np.maximum(f(weight), f(0.0))
    if code != 1:
        return native
    # base_dt is the float32 clock scalar, so each product rounds in dtype.
    phys = ((f(base_dt) * f(interval)) * f(LIGHT_SPEED)) / f(length_unit)
    return native * (phys / np.sqrt(f(2.0 * np.pi)))


def accumulate_dft(mon: DftMonitor, arena, fields, t_phys, step, dt):
    """beamz/simulation/observe.py:327-334 (gate) and 529-585 (accumulate)."""
    re, im, w = arena
    dtype = re.dtype
    f = dtype.type
    t = np.float32(t_phys) if dtype == np.float32 else f(t_phys)
    if not (t >= f(mon.t_start) and t <= f(mon.t_end) and step % max(1, mon.interval) == 0):
        return
    theta = f(2.0 * np.pi) * np.asarray(mon.freqs, dtype) * f(t)
    cre, cim = np.cos(theta), np.sin(theta)
    window = dft_window_weight(t, mon.t_start, mon.t_end, mon.window_code == 1, dtype)
    scale = f(dft_sample_scale(window, mon.normalization_code, dt, mon.interval, mon.length_unit, dtype))
    nf, npt = len(mon.freqs), mon.point_count
    arrays = [fields[c] for c in COMPONENTS]
    for c in range(6):
        vec = np.sum(arrays[c].reshape(-1)[mon.indices[c]].astype(dtype) * mon.weights[c].astype(dtype), axis=-1)
        m = f(mon.component_mask[c])
        base = mon.value_offset + c * nf * npt
        for fi in range(nf):
            sl = slice(base + fi * npt, base + (fi + 1) * npt)
            re[sl] += (scale * m) * (cre[fi] * vec)
            im[sl] += (scale * m) * (cim[fi] * vec)
    w[mon.weight_offset : mon.weight_offset + nf] += f(window)


# ---------------------------------------------------------------------------
# The step (beamz/simulation/execute.py:467-541)
# ---------------------------------------------------------------------------


@dataclass
class OracleState:
    """Mutable stand-in for beamz's SimulationState (model.py:127-259)."""

    fields: dict
    psi_h: list = field(default_factory=list)
    psi_e: list = field(default_factory=list)
    dft_re: np.ndarray | None = None
    dft_im: np.ndarray | None = None
    dft_w: np.ndarray | None = None
    t: float = 0.0
    step: int = 0
    records: list = field(default_factory=list)  # per field recorder (see record_fields)


@dataclass
class FieldRecorder:
    """A compiled time-domain field recorder (beamz/devices/monitors/
    compiler.py:286-412): ``indices``/``weights`` per component are (V, K)
    dense flat offsets and interpolation weights, or None for the whole
    component."""

    components: tuple
    interval: int = 1
    capacity: int = 1
    indices: list | None = None
    weights: list | None = None
    signs: tuple | None = None


def new_records(recorders, shapes: dict, dtype=np.float32) -> list:
    out = []
    for rec in recorders:
        sizes = [int(np.prod(shapes[c])) if rec.indices is None else int(np.shape(rec.indices[q])[0])
                 for q, c in enumerate(rec.components)]
        out.append({"values": [np.zeros((rec.capacity, v), dtype) for v in sizes],
                    "steps": np.zeros(rec.capacity, np.int32), "times": np.zeros(rec.capacity, dtype), "count": 0})
    return out


def record_fields(recorders, records, fields, step: int, t_phys) -> None:
    """beamz/simulation/observe.py:588-646 (_record_fields): after step ``step``
    with (step + 1) % interval == 0 (monitor_records_on_step, 322-324), while
    fewer than ``capacity`` records exist, record each component (the whole
    array, or sum_k field[idx[:, k]] * w[:, k] in slot order) times its sign,
    the step + 1 and the time t + dt.  beamz sums the K slots with jnp.sum;
    the slot order here is the engine's, as for the DFT gather."""
    for rec, store in zip(recorders, records):
        n = store["count"]
        if (int(step) + 1) % max(1, int(rec.interval)) != 0 or n >= rec.capacity:
            continue
        for q, c in enumerate(rec.components):
            f = np.asarray(fields[c]).reshape(-1)
            if rec.indices is None:
                value = f
            else:
                idx = np.asarray(rec.indices[q]).reshape(len(rec.indices[q]), -1)
                w = np.asarray(rec.weights[q], f.dtype).reshape(idx.shape)
                value = f[idx[:, 0]] * w[:, 0]
                for k in range(1, idx.shape[1]):
                    value = value + f[idx[:, k]] * w[:, k]
            sign = f.dtype.type(1.0 if rec.signs is None else rec.signs[q])
            store["values"][q][n] = value * sign
        store["steps"][n] = int(step) + 1
        store["times"][n] = t_phys
        store["count"] = n + 1


@dataclass
class OracleProgram:
    """Static plan for the oracle step."""

    grid_shape: tuple
    dt: float
    resolution: float
    h_terms: list = field(default_factory=list)
    e_terms: list = field(default_factory=list)
    material: Material3D | None = None  # 3D
    h_coeffs: tuple | None = None  # 2D (decay, source)
    e_coeffs: dict | None = None  # 2D component -> (decay, source); 3D with h_coeffs_3d: coefficient form
    h_coeffs_3d: dict | None = None  # 3D component -> (decay, source) (beamz's CUDA path)
    metallic_edges: frozenset = frozenset()
    sources: list = field(default_factory=list)
    monitors: list = field(default_factory=list)
    polarization: str = "tm"
    metrics: dict | None = None  # DerivativeMetricPlan names -> inverse distances (None: isotropic)
    recorders: list = field(default_factory=list)  # FieldRecorder

    @property
    def ndim(self):
        return len(self.grid_shape)


def new_state(program: OracleProgram, dtype=np.float32, t0: float = 0.0) -> OracleState:
    shapes = component_shapes(program.grid_shape, program.polarization)
    fields = {c: np.zeros(shapes[c], dtype=dtype) for c in COMPONENTS}
    psi_h = [np.zeros(t.psi_shape(shapes[t.component]), dtype) for t in program.h_terms]
    psi_e = [np.zeros(t.psi_shape(shapes[t.component]), dtype) for t in program.e_terms]
    nv, nw = dft_arena_sizes(program.monitors)
    return OracleState(fields, psi_h, psi_e, np.zeros(nv, dtype), np.zeros(nv, dtype), np.zeros(nw, dtype), t0, 0,
                       new_records(program.recorders, shapes, dtype))


def forward_step(state: OracleState, program: OracleProgram) -> OracleState:
    """One leapfrog step in the order of beamz/simulation/execute.py:467-541."""
    fields = state.fields
    step = state.step
    masks = pec_masks({c: fields[c].shape for c in COMPONENTS}, program.ndim,
                      program.metallic_edges, program.polarization)
    dtype = next(iter(fields.values())).dtype
    # 1. pre-E sources, then H.
    apply_sources(fields, program.sources, "pre_e", step)
    if program.ndim == 3:
        sm = program.material.sigma_m if program.material is not None else (0.0, 0.0, 0.0)
        hx, hy, hz, state.psi_h = update_h_3d(fields, state.psi_h, program.h_terms, program.dt,
                                              program.resolution, sm, program.h_coeffs_3d, program.metrics)
        fields["Hx"], fields["Hy"], fields["Hz"] = hx, hy, hz
    else:
        new, state.psi_h = update_h_2d(fields, state.psi_h, program.h_terms, program.resolution,
                                       program.h_coeffs, program.polarization, program.metrics)
        fields.update(new)
    # 2. H sources and H masks.
    apply_sources(fields, program.sources, "h", step)
    for c in ("Hx", "Hy", "Hz"):
        fields[c] = np.where(masks[c], dtype.type(0.0), fields[c])
    # 3. E, E sources, E masks.
    if program.ndim == 3:
        ex, ey, ez, state.psi_e = update_e_3d(fields, state.psi_e, program.e_terms, program.dt,
                                              program.resolution, program.material, program.metallic_edges,
                                              program.e_coeffs if program.h_coeffs_3d is not None else None,
                                              program.metrics)
        fields["Ex"], fields["Ey"], fields["Ez"] = ex, ey, ez
    else:
        new, state.psi_e = update_e_2d(fields, state.psi_e, program.e_terms, program.resolution,
                                       program.e_coeffs, program.metallic_edges, program.polarization,
                                       program.metrics)
        fields.update(new)
    apply_sources(fields, program.sources, "e", step)
    for c in ("Ex", "Ey", "Ez"):
        fields[c] = np.where(masks[c], dtype.type(0.0), fields[c])
    # 4. Monitors at t + dt, then the clocks (FP32 accumulation in FP32 mode).
    if dtype == np.float32:
        t_phys = np.float32(np.float32(state.t) + np.float32(program.dt))
    else:
        t_phys = float(state.t) + float(program.dt)
    for mon in program.monitors:
        accumulate_dft(mon, (state.dft_re, state.dft_im, state.dft_w), fields, t_phys, step, program.dt)
    record_fields(program.recorders, state.records, fields, step, t_phys)
    state.t = t_phys
    state.step = step + 1
    return state


def run(state: OracleState, program: OracleProgram, nsteps: int) -> OracleState:
    for _ in range(int(nsteps)):
        state = forward_step(state, program)
    return state


def relative_l2(actual, expected) -> float:
    a = np.asarray(actual, dtype=np.float64)
    e = np.asarray(expected, dtype=np.float64)
    den = float(np.linalg.norm(e))
    num = float(np.linalg.norm(a - e))
    return 0.0 if den == 0.0 and num == 0.0 else num / max(den, 1e-300)


# ---------------------------------------------------------------------------
# Field diagnostics for automatic termination
# ---------------------------------------------------------------------------

# beamz/lattice.py:14-21: Yee offsets (z, y, x) in cells; 2D (y, x) from
# beamz/simulation/execute.py:66-73.
COMPONENT_OFFSETS_3D = {
    "Ex": (0.0, 0.0, 0.5), "Ey": (0.0, 0.5, 0.0), "Ez": (0.5, 0.0, 0.0),
    "Hx": (0.5, 0.5, 0.0), "Hy": (0.5, 0.0, 0.5), "Hz": (0.0, 0.5, 0.5),
}
COMPONENT_OFFSETS_2D = {
    "Ex": (0.0, 0.5), "Ey": (0.5, 0.0), "Ez": (0.0, 0.0),
    "Hx": (0.5, 0.0), "Hy": (0.0, 0.5), "Hz": (0.5, 0.5),
}


def axis_integration_weights(edges, offset: float, count: int) -> np.ndarray:
    """Control-volume widths along one axis (beamz/simulation/execute.py:77-93):
    cell widths for a centre-aligned support; half cells at the two ends and
    averages of neighbouring cells inside for an edge-aligned one."""
    edges = np.asarray(edges, dtype=np.float64)
    widths = np.diff(edges)
    if offset == 0.5:
        return widths
    out = np.empty(int(count), dtype=np.float64)
    out[0] = 0.5 * widths[0]
    out[-1] = 0.5 * widths[-1]
    if count > 2:
        out[1:-1] = 0.5 * (widths[:-1] + widths[1:])
    return out


def component_integration_weights(component: str, grid_shape, resolution: float) -> np.ndarray:
    """Physical integration weights of one component on a uniform grid
    (beamz/simulation/execute.py:95-111)."""
    offsets = COMPONENT_OFFSETS_3D[component] if len(grid_shape) == 3 else COMPONENT_OFFSETS_2D[component]
    axes = []
    for n, off in zip(grid_shape, offsets):
        edges = np.arange(int(n) + 1, dtype=np.float64) * float(resolution)
        axes.append(axis_integration_weights(edges, off, int(n) + (1 if off == 0.0 else 0)))
    w = axes[0]
    for a in axes[1:]:
        w = np.multiply.outer(w, a)
    return w


def field_diagnostics(fields: dict, eps_sites: dict, grid_shape, resolution: float):
    """(energy, max |field|, all finite) of scalar-material fields
    (beamz/simulation/execute.py:127-222, _energy_terms / _field_diagnostics
    without the full-tensor cross terms), in float64: energy =
    sum_c 0.5 * const_c * sum(material * v^2 * weights), const = eps0 for E,
    mu0 for H; H material is mu_r = 1."""
    energy, max_field, finite = 0.0, 0.0, True
    for c, v in fields.items():
        v = np.asarray(v, dtype=np.float64)
        finite = finite and bool(np.all(np.isfinite(v)))
        max_field = max(max_field, float(np.max(np.abs(v), initial=0.0)))
        mat = np.asarray(eps_sites.get(c, 1.0), dtype=np.float64) if c[0] == "E" else 1.0
        const = EPS_0 if c[0] == "E" else MU_0
        w = component_integration_weights(c, grid_shape, resolution)
        energy += 0.5 * const * float(np.sum(mat * v * v * w))
    return energy, max_field, finite


def relative_monitor_change(current: dict, previous: dict | None):
    """Largest |cur - prev| / max(|cur|, |prev|) over the monitor vectors, 0 for
    a pair of vanishing vectors, None without a previous check
    (beamz/simulation/execute.py:292-316)."""
    if previous is None:
        return None
    tiny = np.finfo(float).tiny
    changes = []
    for key, cur in current.items():
        prev = previous[key]
        num = float(np.linalg.norm(cur - prev))
        den = max(float(np.linalg.norm(cur)), float(np.linalg.norm(prev)))
        changes.append(0.0 if den <= tiny and num <= tiny else num / den)
    return max(changes, default=0.0)


# ---------------------------------------------------------------------------
# Monitor analysis: DFT flux and modal overlaps (float64 / complex128)
# ---------------------------------------------------------------------------

# beamz/devices/modes/fields.py:15-19 -- (E1, E2, H1, H2) tangential to a plane
# normal; E1 pairs with H1 (+), E2 with H2 (-).
TANGENTIAL_COMPONENTS = {
    "x": ("Ey", "Ez", "Hz", "Hy"),
    "y": ("Ez", "Ex", "Hx", "Hz"),
    "z": ("Ex", "Ey", "Hy", "Hx"),
}


def monitor_dft_component(values, weight_sum):
    """beamz/simulation/observe.py:166-179: the stored DFT values of one
    component, [F, P] complex, over half the accumulated window weight."""
    values = np.asarray(values, np.complex128)
    weights = np.maximum(np.asarray(weight_sum, dtype=float), 1e-18).reshape(-1, 1)
    return (2.0 / weights) * values


def flux_component(values, weight_sum, component: str, freqs, base_dt):
    """beamz/simulation/observe.py:182-187: H values also carry the half-step
    phase exp(-i pi f dt) when the monitor has a base time step."""
    v = monitor_dft_component(values, weight_sum)
    if component.startswith("H") and base_dt:
        phase = np.exp(-1j * np.pi * np.asarray(freqs, dtype=float) * base_dt)
        v = v * phase[:, None]
    return v


def monitor_dft_flux(fields: dict, axis: str, sign: float = 1.0, integration_weights=None, measure=None):
    """beamz/simulation/observe.py:198-234 on flux-normalised fields
    (component -> [F, P]): 0.5 Re sum sign (E1 conj(H1) - E2 conj(H2)) w, with
    per-point integration weights when given (size P), else times ``measure``."""
    e1, e2, h1, h2 = TANGENTIAL_COMPONENTS[axis]
    component = fields[e1] * np.conjugate(fields[h1]) - fields[e2] * np.conjugate(fields[h2])
    iw = np.asarray(() if integration_weights is None else integration_weights, dtype=float).reshape(-1)
    if iw.size == component.shape[1]:
        return 0.5 * np.real(np.sum(sign * component * iw[None, :], axis=1))
    return 0.5 * np.real(np.sum(sign * component, axis=1)) * float(measure)


def modal_overlap(fields: dict, mode: dict, axis: str, measure, direction_sign: float = 1.0):
    """beamz/devices/modes/fields.py:76-129 for equal-size profiles:
    0.25 dir [sum w1 (E1 conj(Hm1) + conj(Em1) H1) - sum w2 (E2 conj(Hm2) + conj(Em2) H2)],
    ``measure`` a scalar, a per-point array or a mapping E name -> weights."""
    names = TANGENTIAL_COMPONENTS[axis]

    def paired(e_name, h_name, sign):
        ef = np.asarray(fields[e_name], np.complex128).reshape(-1)
        hf = np.asarray(fields[h_name], np.complex128).reshape(-1)
        em = np.asarray(mode[e_name], np.complex128).reshape(-1)
        hm = np.asarray(mode[h_name], np.complex128).reshape(-1)
        if isinstance(measure, dict):
            w = np.asarray(measure[e_name], dtype=float).reshape(-1)
        else:
            raw = np.asarray(measure, dtype=float)
            w = raw if raw.ndim == 0 else raw.reshape(-1)
        return np.complex128(np.sum(w * sign * (ef * np.conjugate(hm) + np.conjugate(em) * hf)))

    overlap = paired(names[0], names[2], 1.0) + paired(names[1], names[3], -1.0)
    return np.complex128(0.25 * float(direction_sign) * overlap)
