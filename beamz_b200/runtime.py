"""Python side of the C ABI: device programs, device state and step entry points.

Mirrors beamz's native runtime surface (beamz/simulation/cuda/runtime.py):
``update_h`` / ``update_e`` advance one half step in place (184, 234),
``run_steps`` / ``run_program_steps`` advance whole leapfrog steps with
sources and monitors (621, 685) and ``pack_dft_monitors`` builds the monitor
arena (530).  PyTorch tensors own every device buffer; the library only sees
raw pointers.  There is no CPU fallback: without the library or a CUDA device
these functions raise :class:`~beamz_b200.abi.CudaBackendUnavailable`.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import abi
from .plan import (
    COMPONENT_INDEX,
    COMPONENTS,
    EPS_0,
    MU_0,
    CodebookOverflow,
    ProgramSpec,
    active_components,
    codebook_keys,
    codebook_tables,
    compact_materials,
    component_shape,
    site_eps_3d,
    sources_clear_of_monitors,
    step_times,
)

#: Steps per native call; beamz replays 256-step CUDA-graph chunks
#: (beamz/simulation/execute.py:64).
GRAPH_CHUNK_STEPS = 256


def _torch():
    import torch

    return torch


def _require_cuda(device):
    torch = _torch()
    dev = torch.device(device)
    if dev.type != "cuda" or not torch.cuda.is_available():
        raise abi.CudaBackendUnavailable("beamz_b200 runs on a CUDA device only (no CPU fallback)")
    return dev


def _f32(x, device):
    torch = _torch()
    return torch.as_tensor(np.ascontiguousarray(np.asarray(x, dtype=np.float32)), device=device)


def _pad_last(arrays, k):
    return [np.pad(a, ((0, 0), (0, k - a.shape[1]))) for a in arrays]


def _replicated_slab(torch, ids, remap, k0: int, k1: int):
    """Edge-replicated compact material planes for lattice planes [k0, k1):
    voxel planes clip(k0-1) .. clip(k1), one replicated row/column per side."""
    nz = ids.shape[0]
    zi = torch.arange(k0 - 1, k1 + 1, device=ids.device).clamp_(0, nz - 1)
    slab = remap[ids.index_select(0, zi).long()]
    slab = torch.cat([slab[:, :1], slab, slab[:, -1:]], dim=1)
    return torch.cat([slab[:, :, :1], slab, slab[:, :, -1:]], dim=2)


def device_site_codebook(voxel_ids, eps_table, dt_over_eps, pitch: int, device, z_block: int = 32,
                         with_eps: bool = False, ids=None, counts=None):
    """Site-id words (Z+1, Y+1, pitch) int32 and coefficient tables (3, 256) on
    the device; equal bit for bit to :func:`beamz_b200.plan.site_codebook` (the
    device part is integer gathers only; coefficients come from the host).
    With ``with_eps`` also the (3, 256) site permittivities of the ids.
    ``ids`` (the voxel ids already on the device) and ``counts`` (their
    histogram) save an upload and a host count."""
    torch = _torch()
    remap_np, eps_used = compact_materials(voxel_ids, eps_table, counts)
    m = int(eps_used.size)
    if ids is None:
        ids = torch.as_tensor(np.ascontiguousarray(voxel_ids, np.uint8), device=device)
    remap = torch.as_tensor(remap_np, device=device)
    nz, ny, nx = (int(v) for v in ids.shape)
    blocks = [(k, min(k + z_block, nz + 1)) for k in range(0, nz + 1, z_block)]
    comps = ("Ex", "Ey", "Ez")
    present = {c: torch.zeros(m**4, dtype=torch.bool, device=device) for c in comps}
    for k0, k1 in blocks:
        vp = _replicated_slab(torch, ids, remap, k0, k1)
        for c in comps:
            keys = codebook_keys(vp, m, c, 0, k1 - k0).reshape(-1).long()
            present[c] |= torch.bincount(keys, minlength=m**4) > 0
    luts, coef, eps = codebook_tables(eps_used, dt_over_eps, {c: present[c].cpu().numpy() for c in comps},
                                      with_eps=True)
    lut = {c: torch.as_tensor(luts[c].astype(np.int32), device=device) for c in comps}
    words = torch.zeros((nz + 1, ny + 1, pitch), dtype=torch.int32, device=device)
    for k0, k1 in blocks:
        vp = _replicated_slab(torch, ids, remap, k0, k1)
        w = words[k0:k1, :, : nx + 1]
        for shift, c in ((0, "Ex"), (8, "Ey"), (16, "Ez")):
            w |= lut[c][codebook_keys(vp, m, c, 0, k1 - k0).long()] << shift
    if with_eps:
        return words, torch.as_tensor(coef, device=device), torch.as_tensor(eps, device=device)
    return words, torch.as_tensor(coef, device=device)


def lossless_site_sources(spec: ProgramSpec):
    """The per-site E sources of a 3D program whose E decay is exactly 1
    everywhere (beamz's lossless material: E <- E + source * curl), else None."""
    if spec.ndim != 3 or spec.e_site is None or spec.voxel_ids is not None:
        return None
    out = {}
    for c in ("Ex", "Ey", "Ez"):
        if c not in spec.e_site:
            return None
        dec, src = spec.e_site[c]
        if np.any(np.asarray(dec, np.float32) != np.float32(1.0)):
            return None
        out[c] = src
    return out


def device_codebook_from_sites(sources: dict, shapes: dict, pitch: int, dt: float, device):
    """Codebook words (Z+1, Y+1, pitch) int32 and (3, 256) tables from per-site
    lossless E sources: per component the distinct source values (at most 256,
    in increasing order) and each site's index among them -- beamz packs its
    lossless CUDA coefficients the same way (compile.py:146-187) -- plus the
    relative permittivity dt / (eps0 source) of each table entry (energy
    diagnostics).  Raises :class:`CodebookOverflow` above 256 values."""
    torch = _torch()
    ez = shapes["Ex"]  # (Z+1, Y+1, X): the lattice's z and y extents
    words = torch.zeros((int(ez[0]), int(ez[1]), pitch), dtype=torch.int32, device=device)
    coef = np.zeros((3, 256), np.float32)
    eps = np.ones((3, 256), np.float32)
    for n, c in enumerate(("Ex", "Ey", "Ez")):
        src = torch.as_tensor(np.ascontiguousarray(np.broadcast_to(np.asarray(sources[c], np.float32), shapes[c])),
                              device=device)
        table, ids = torch.unique(src, return_inverse=True)
        if table.numel() > 256:
            raise CodebookOverflow(f"{c}: {table.numel()} distinct E-site coefficients (> 256)")
        dz, dy, dx = (int(v) for v in shapes[c])
        words[:dz, :dy, :dx] |= ids.to(torch.int32) << (8 * n)
        t = table.cpu().numpy()
        coef[n, : t.size] = t
        with np.errstate(divide="ignore"):
            eps[n, : t.size] = np.where(t != 0, np.float64(dt) / (EPS_0 * t.astype(np.float64)), 1.0)
    return words, torch.as_tensor(coef, device=device), torch.as_tensor(eps, device=device)


class ClassOverflow(ValueError):
    """More than 256 distinct (Ex, Ey, Ez) coefficient triples: no uint8 class ids."""


def _word_classes(words, nx: int, limit: int, what: str, z_block: int = 64):
    """uint8 classes of codebook words: each distinct word (a triple of
    per-component ids) one class, numbered in increasing word order, on rows of
    a 16-byte multiple; returns the classes and the words of the classes."""
    torch = _torch()
    dev = words.device
    nz1, ny1, _ = (int(v) for v in words.shape)
    pitch8 = -(-(nx + 1) // 16) * 16
    present = torch.zeros(1 << 24, dtype=torch.int32, device=dev)
    for k0 in range(0, nz1, z_block):
        w = words[k0:k0 + z_block, :, : nx + 1].reshape(-1).long()
        present += torch.bincount(w, minlength=1 << 24).to(torch.int32)[: 1 << 24].clamp_(max=1)
        present.clamp_(max=1)
    keys = torch.nonzero(present, as_tuple=False).reshape(-1)
    if keys.numel() > limit:
        raise ClassOverflow(f"{keys.numel()} distinct {what} coefficient triples (> {limit})")
    lut = torch.zeros(1 << 24, dtype=torch.uint8, device=dev)
    lut[keys] = torch.arange(keys.numel(), device=dev, dtype=torch.int32).to(torch.uint8)
    classes = torch.zeros((nz1, ny1, pitch8), dtype=torch.uint8, device=dev)
    for k0 in range(0, nz1, z_block):
        w = words[k0:k0 + z_block, :, : nx + 1].long()
        classes[k0:k0 + z_block, :, : nx + 1] = lut[w]
    return classes, keys.cpu().numpy().astype(np.int64)


def device_site_classes(words, coef, res: float, nx: int, z_block: int = 64, over_dx: bool = False):
    """uint8 material classes of the codebook words (each distinct (Ex, Ey, Ez)
    id triple one class, numbered in increasing word order) on rows of a
    16-byte multiple, and the (256, 4) float32 table of each class's Ex, Ey,
    Ez coefficients: the codebook's own values, or with ``over_dx`` divided by
    the cell size (rounded once from float64) for the tolerance arithmetic.
    Raises :class:`ClassOverflow` above 256 classes."""
    torch = _torch()
    dev = words.device
    classes, k = _word_classes(words, nx, 256, "E", z_block)
    c64 = np.asarray(coef.cpu().numpy() if hasattr(coef, "cpu") else coef, np.float64)
    table = np.zeros((256, 4), np.float32)
    for n in range(3):
        v = c64[n, (k >> (8 * n)) & 0xFF]
        table[: k.size, n] = (v / np.float64(np.float32(res)) if over_dx else v).astype(np.float32)
    return classes, torch.as_tensor(table, device=dev)


def _pair_words(pairs: dict, comps, shapes: dict, lattice, device):
    """Codebook words of per-site (decay, source) pairs: per component the
    distinct pairs (at most 256, numbered in increasing bit order) and each
    site's index, in bytes 0-2 of an int32 word per lattice point (0 where the
    component has no site); returns the words and the (3, 256) decay and source
    tables.  Raises :class:`ClassOverflow` above 256 pairs."""
    torch = _torch()
    words = torch.zeros(lattice, dtype=torch.int32, device=device)
    dec_t = np.zeros((3, 256), np.float32)
    src_t = np.zeros((3, 256), np.float32)
    for n, c in enumerate(comps):
        dec, src = pairs[c]
        d = torch.as_tensor(np.ascontiguousarray(np.broadcast_to(np.asarray(dec, np.float32), shapes[c])), device=device)
        v = torch.as_tensor(np.ascontiguousarray(np.broadcast_to(np.asarray(src, np.float32), shapes[c])), device=device)
        key = (d.view(torch.int32).long() << 32) | (v.view(torch.int32).long() & 0xFFFFFFFF)
        del d, v
        table, ids = torch.unique(key, return_inverse=True)
        del key
        if table.numel() > 256:
            raise ClassOverflow(f"{c}: {table.numel()} distinct (decay, source) pairs (> 256)")
        dz, dy, dx = (int(x) for x in shapes[c])
        words[:dz, :dy, :dx] |= ids.to(torch.int32) << (8 * n)
        t = table.cpu().numpy()
        dec_t[n, : t.size] = (t >> 32).astype(np.int32).view(np.float32)
        src_t[n, : t.size] = (t & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
    return words, dec_t, src_t


def device_lossy_classes(e_pairs: dict, h_pairs: dict, shapes: dict, lattice, nx: int, device):
    """Conductive material on the class step (FDTD_FLAG_LOSSY): uint8 E and H
    classes per lattice point -- each distinct (Ex, Ey, Ez), resp. (Hx, Hy,
    Hz), triple of (decay, source) pairs one class -- and their [classes, 4, 2]
    float32 tables, at most 128 E and 64 H classes (shared-memory tables of the
    step).  The pairs are beamz's per-site coefficients as they are (E <-
    decay E + source curl, H <- decay H - source curl).  Raises
    :class:`ClassOverflow` above those counts."""
    torch = _torch()
    out = []
    for pairs, comps, limit, what in ((e_pairs, ("Ex", "Ey", "Ez"), 128, "E"), (h_pairs, ("Hx", "Hy", "Hz"), 64, "H")):
        words, dec_t, src_t = _pair_words(pairs, comps, shapes, lattice, device)
        classes, k = _word_classes(words, nx, limit, what)
        del words
        table = np.zeros((limit, 4, 2), np.float32)
        for n in range(3):
            ids = (k >> (8 * n)) & 0xFF
            table[: k.size, n, 0] = dec_t[n, ids]
            table[: k.size, n, 1] = src_t[n, ids]
        out += [classes, torch.as_tensor(table, device=device)]
    return tuple(out)


@dataclass
class DftArena:
    """Device buffers of the packed monitor plan (beamz/simulation/cuda/runtime.py:530-618)."""

    indices: object
    weights: object
    freqs: object
    masks: object
    counts: object
    codes: object
    windows: object
    value_count: int
    weight_count: int
    layout: list  # per monitor: (value_offset, freq_count, point_count, weight_offset)
    affine: object = None  # [M, 6, 24] int32: affine forms of the plans (FdtdDft.affine)


def voxel_histogram(ids, device):
    """Counts of every voxel id of a device uint8 tensor (fdtd_voxel_histogram)."""
    torch = _torch()
    counts = torch.empty(256, dtype=torch.int32, device=device)
    lib = abi.load_library()
    stream = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    b_ids, b_counts = abi.buffer_of(ids), abi.buffer_of(counts)
    abi.check(lib.fdtd_voxel_histogram(stream, ctypes.byref(b_ids), ctypes.byref(b_counts)), "fdtd_voxel_histogram")
    return counts.cpu().numpy()


def pack_dft_monitors(monitors, device, shapes, strides) -> DftArena | None:
    """Pad every monitor to a common (P, K, F), lay out the ragged arena, and
    pack each (monitor, component) gather plan on the device
    (fdtd_pack_gather): per point the nonzero-weight neighbours first, in
    order, so a gather may stop at the first zero weight, and every offset in
    the device layout.  ``shapes[c]`` is component ``c``'s stored shape and
    ``strides(c)`` the (row, plane) element strides of its device array."""
    if not monitors:
        return None
    M = len(monitors)
    P = max(m.points for m in monitors)
    F = max(len(m.freqs) for m in monitors)
    if F > 64:
        raise ValueError("at most 64 frequencies per monitor")
    torch = _torch()
    lib = abi.load_library()
    cur = torch.cuda.current_stream(device)
    stream = ctypes.c_void_p(cur.cuda_stream)
    # Every (monitor, component) plan goes up in one pinned staging copy.
    plans = [(m, c, np.asarray(mon.indices[c]).reshape(mon.points, -1), np.asarray(mon.weights[c]))
             for m, mon in enumerate(monitors) for c in range(6)]
    total = sum(a.size for _m, _c, a, _w in plans)
    host_i = torch.empty(total, dtype=torch.int32, pin_memory=True)
    host_w = torch.empty(total, dtype=torch.float32, pin_memory=True)
    hi, hw = host_i.numpy(), host_w.numpy()
    o = 0
    for _m, _c, a, w in plans:
        hi[o : o + a.size] = a.reshape(-1)
        hw[o : o + a.size] = w.reshape(-1)
        o += a.size
    dev_i = host_i.to(device, non_blocking=True)
    dev_w = host_w.to(device, non_blocking=True)
    # K = the most nonzero weights any point has: the packed plans keep them
    # first, so the zero-weight slots past them are dropped.
    nonzero, o = [], 0
    for _m, _c, a, _w in plans:
        if a.size:
            nonzero.append(torch.count_nonzero(dev_w[o : o + a.size].view(a.shape), dim=1).max())
        o += a.size
    K = max(1, int(torch.stack(nonzero).max().item())) if nonzero else 1
    indices = torch.zeros((M, 6, K, P), dtype=torch.int32, device=device)  # neighbour-major (see FdtdDft)
    weights = torch.zeros((M, 6, K, P), dtype=torch.float32, device=device)
    o = 0
    for m, c, a, _w in plans:
        g = abi.FdtdGatherPack()
        g.indices_in = abi.buffer_of(dev_i[o : o + a.size].view(a.shape))
        g.weights_in = abi.buffer_of(dev_w[o : o + a.size].view(a.shape))
        g.indices_out, g.weights_out = abi.buffer_of(indices[m, c]), abi.buffer_of(weights[m, c])
        dims = (1,) * (3 - len(shapes[c])) + tuple(shapes[c])  # 2D: z extent 1
        for ax, n in enumerate(dims):
            g.dims[ax] = int(n)
        g.row, g.plane = strides(c)
        abi.check(lib.fdtd_pack_gather(stream, ctypes.byref(g)), "fdtd_pack_gather")
        o += a.size
    freqs = np.zeros((M, F), np.float32)
    masks = np.zeros((M, 6), np.float32)
    counts = np.zeros((M, 5), np.int32)
    codes = np.zeros((M, 2), np.int32)
    windows = np.zeros((M, 3), np.float32)
    voff = woff = 0
    layout = []
    for m, mon in enumerate(monitors):
        p, nf = mon.points, len(mon.freqs)
        freqs[m, :nf] = mon.freqs
        masks[m] = mon.component_mask
        counts[m] = (nf, p, max(1, int(mon.interval)), voff, woff)
        codes[m] = (int(mon.window_code), int(mon.normalization_code))
        windows[m] = (mon.t_start, mon.t_end, mon.length_unit)
        layout.append((voff, nf, p, woff))
        voff += 6 * nf * p
        woff += nf
    t = lambda a: torch.as_tensor(a, device=device)  # noqa: E731
    affine = np.zeros((M, 6, 24), np.int32)
    for m, mon in enumerate(monitors):
        for c in range(6):
            if mon.component_mask[c] != 0 and mon.points > 0:
                words = _affine_plan(indices[m, c, :, : mon.points], weights[m, c, :, : mon.points])
                if words is not None:
                    affine[m, c] = words
    arena = DftArena(indices, weights, t(freqs), t(masks), t(counts), t(codes), t(windows), voff, woff, layout,
                     t(affine))
    cur.synchronize()  # the plan is complete before any stream of the program reads it
    return arena


def _affine_plan(idx, w):
    """The 24-word affine form (FdtdDft.affine) of one packed [K, n] gather
    plan on the device, or None when the plan does not have it exactly: the
    nonzero-weight slots (at most 4, first) carry the same weight and the same
    offset from slot 0 at every point, and slot 0's index is
    base + (p // nb) * sa + (p % nb) * sb.  Plane monitors on uniform
    coordinates have this form; sampling them then reads no plan."""
    torch = _torch()
    K, n = idx.shape
    nonzero = (w != 0).sum(dim=1)
    full, empty = nonzero == n, nonzero == 0
    if not bool((full | empty).all()):
        return None
    k = int(full.sum())
    if not 1 <= k <= 4 or not bool(full[:k].all()):
        return None
    wk, ik = w[:k], idx[:k].long()
    if not bool((wk == wk[:, :1]).all()):
        return None
    delta = ik - ik[:1]
    if not bool((delta == delta[:, :1]).all()):
        return None
    b0 = ik[0]
    na, nb, sa, sb = 1, n, 0, 0
    if n > 1:
        sb = int(b0[1] - b0[0])
        breaks = ((b0[1:] - b0[:-1]) != sb).nonzero()
        nb = int(breaks[0, 0]) + 1 if breaks.numel() else n
        if n % nb:
            return None
        na = n // nb
        sa = int(b0[nb] - b0[0]) if na > 1 else 0
        p = torch.arange(n, device=idx.device)
        if not bool((b0 == b0[0] + (p // nb) * sa + (p % nb) * sb).all()):
            return None
    if max(abs(sa), abs(sb), abs(int(b0[0]))) >= 2**31:
        return None
    bits = wk[:, 0].contiguous().view(torch.int32).tolist()
    return ([1, na, nb, int(b0[0]), sa, sb, k, 0] + [int(v) for v in delta[:, 0].tolist()] + [0] * (8 - k)
            + [int(v) for v in bits] + [0] * (8 - k))


def _pack_plan(lib, stream, indices, weights, dims, strides, device):
    """One (V, K) gather plan as device [K, V] arrays in the device layout,
    nonzero weights first per value (fdtd_pack_gather)."""
    torch = _torch()
    ic = torch.as_tensor(np.ascontiguousarray(np.asarray(indices).reshape(len(indices), -1), np.int32), device=device)
    wc = torch.as_tensor(np.ascontiguousarray(np.asarray(weights, np.float32).reshape(ic.shape)), device=device)
    V, K = (int(v) for v in ic.shape)
    out_i = torch.zeros((K, V), dtype=torch.int32, device=device)
    out_w = torch.zeros((K, V), dtype=torch.float32, device=device)
    g = abi.FdtdGatherPack()
    g.indices_in, g.weights_in = abi.buffer_of(ic), abi.buffer_of(wc)
    g.indices_out, g.weights_out = abi.buffer_of(out_i), abi.buffer_of(out_w)
    for a, n in enumerate((1,) * (3 - len(dims)) + tuple(dims)):
        g.dims[a] = int(n)
    g.row, g.plane = strides
    abi.check(lib.fdtd_pack_gather(stream, ctypes.byref(g)), "fdtd_pack_gather")
    torch.cuda.current_stream(device).synchronize()
    return out_i, out_w


class DeviceProgram:
    """A compiled program: every static input of the step, resident on the device."""

    def __init__(self, spec: ProgramSpec, device="cuda", schedule="fused", tile=(32, 8), z_chunk=16,
                 graphs=True, layout="auto", dft_batch: int = 16, dft_overlap: bool = True,
                 arithmetic: str = "exact", step_kernel: str = "classes", wait_limit_ns: int = 0,
                 test_stall: bool = False):
        self.lib = abi.load_library()
        self.device = _require_cuda(device)
        torch = _torch()
        self.spec = spec
        self.ndim = spec.ndim
        self.polarization = spec.polarization
        self.active = active_components(spec.ndim, spec.polarization)
        self.schedule = {"fused": abi.FDTD_SCHEDULE_FUSED, "phases": abi.FDTD_SCHEDULE_PHASES}[schedule]
        self.shapes = {c: component_shape(c, spec.grid_shape, spec.polarization) for c in COMPONENTS}
        dev = self.device
        h_uniform = all(np.ndim(d) == 0 and np.ndim(s_) == 0 for d, s_ in spec.h_coefficients().values())
        site_sources = lossless_site_sources(spec)
        # Derivative metrics (axis-uniform / rectilinear grids) ride on the
        # class step in exact arithmetic; the codebook step has none.
        layout_arg = layout
        metric_ok = spec.metrics is None or (step_kernel == "classes" and arithmetic == "exact")
        pitched_ok = (spec.ndim == 3 and (spec.voxel_ids is not None or site_sources is not None)
                      and schedule == "fused" and h_uniform and metric_ok)
        lossy_ok = (spec.ndim == 3 and spec.voxel_ids is None and site_sources is None and spec.e_site is not None
                    and all(c in spec.e_site for c in ("Ex", "Ey", "Ez")) and schedule == "fused"
                    and spec.metrics is None and step_kernel == "classes" and arithmetic == "exact")
        if layout == "pitched" and not (pitched_ok or lossy_ok):
            raise ValueError("the pitched layout needs a 3D voxel or per-site program and the fused schedule; "
                             "conductive material or a non-isotropic grid also need the class step in exact "
                             "arithmetic")
        f32 = np.float32
        dt_over_eps = f32(spec.dt) / f32(EPS_0)
        self.site_ids = self.site_coef = self.site_eps_table = None
        self._diag_eps = None
        if layout in ("auto", "pitched") and pitched_ok:
            nz, ny, nx = (int(v) for v in spec.grid_shape)
            self.pitch = -(-(nx + 1) // 4) * 4
            self.bank_shape = (nz + 1, ny + 1, self.pitch)
            try:
                if spec.voxel_ids is not None:
                    ids = torch.as_tensor(np.ascontiguousarray(spec.voxel_ids, np.uint8), device=dev)
                    self.site_ids, self.site_coef, self.site_eps_table = device_site_codebook(
                        spec.voxel_ids, spec.eps_table, dt_over_eps, self.pitch, dev, with_eps=True, ids=ids,
                        counts=voxel_histogram(ids, dev))
                else:
                    self.site_ids, self.site_coef, self.site_eps_table = device_codebook_from_sites(
                        site_sources, self.shapes, self.pitch, float(spec.dt), dev)
                layout = "pitched"
            except CodebookOverflow:
                if layout == "pitched":
                    raise
                layout = "dense"
        elif layout == "auto" and not lossy_ok:
            layout = "dense"
        # Conductive (per-site decay) 3D programs: the class step with E and H
        # classes of (decay, source) pairs (FDTD_FLAG_LOSSY), when at most 128
        # E and 64 H classes occur; else the dense per-site step.
        self.lossy = False
        self.h_class = self.h_class_coef = None
        if lossy_ok and layout in ("auto", "pitched"):
            nz, ny, nx = (int(v) for v in spec.grid_shape)
            self.pitch = -(-(nx + 1) // 4) * 4
            self.bank_shape = (nz + 1, ny + 1, self.pitch)
            try:
                e_pairs = {c: spec.e_site[c] for c in ("Ex", "Ey", "Ez")}
                self.site_class, self.class_coef, self.h_class, self.h_class_coef = device_lossy_classes(
                    e_pairs, spec.h_coefficients(), self.shapes, self.bank_shape, nx, dev)
                # Energy diagnostics read the E-site permittivity through codebook words.
                if spec.e_site_eps is not None and all(c in spec.e_site_eps for c in ("Ex", "Ey", "Ez")):
                    eps = {c: (spec.e_site_eps[c], spec.e_site_eps[c]) for c in ("Ex", "Ey", "Ez")}
                    self.site_ids, eps_t, _ = _pair_words(eps, ("Ex", "Ey", "Ez"), self.shapes, self.bank_shape, dev)
                    self.site_eps_table = torch.as_tensor(eps_t, device=dev)
                else:
                    self.site_ids = torch.zeros(self.bank_shape, dtype=torch.int32, device=dev)
                self.site_coef = torch.zeros((3, 256), dtype=torch.float32, device=dev)
                self.lossy = True
                layout = "pitched"
            except ClassOverflow:
                if layout == "pitched":
                    raise
                self.site_class = self.class_coef = self.h_class = self.h_class_coef = None
                layout = "dense"
        self.layout = layout
        # The pitched 3D step: the class step (uint8 material classes, 128-wide
        # tiles) unless the scene has more than 256 distinct E coefficient
        # triples or the codebook step is asked for.  Its arithmetic is
        # beamz's float32 order; "fast" opts into the tolerance form.
        if arithmetic not in ("fast", "exact"):
            raise ValueError("arithmetic is 'fast' or 'exact'")
        if step_kernel not in ("classes", "codebook"):
            raise ValueError("step_kernel is 'classes' or 'codebook'")
        if not self.lossy:
            self.site_class = self.class_coef = None
        if layout == "pitched" and step_kernel == "classes" and not self.lossy:
            try:
                self.site_class, self.class_coef = device_site_classes(
                    self.site_ids, self.site_coef, float(spec.resolution), int(spec.grid_shape[2]),
                    over_dx=arithmetic == "fast")
            except ClassOverflow:
                if spec.metrics is not None:  # the codebook step carries no metrics: the dense step
                    if layout_arg == "pitched":
                        raise
                    layout = self.layout = "dense"
                    self.site_ids = self.site_coef = self.site_eps_table = None
                else:
                    step_kernel = "codebook"
        if layout != "pitched":
            step_kernel = "dense"
        if step_kernel != "classes":
            arithmetic = "exact"
        self.step_kernel = step_kernel
        self.arithmetic = arithmetic
        s = abi.FdtdProgram()
        s.abi_version = abi.FDTD_ABI_VERSION
        s.flags = abi.FDTD_FLAG_GRAPH_CACHE if graphs else 0
        if step_kernel == "classes":
            s.flags |= abi.FDTD_FLAG_CLASSES
            if arithmetic == "fast":
                s.flags |= abi.FDTD_FLAG_FAST_MATH
            if self.lossy:
                s.flags |= abi.FDTD_FLAG_LOSSY
        s.wait_limit_ns = int(wait_limit_ns)
        if test_stall:  # test only: the pitched step's first wait runs out (nothing in flight)
            s.flags |= abi.FDTD_FLAG_TEST_STALL
        s.ndim = spec.ndim
        s.polarization = 0 if spec.polarization == "tm" else 1
        s.schedule = self.schedule
        mask = 0
        for edge in spec.metallic_edges:
            mask |= 1 << abi.EDGE_BITS[edge]
        s.metallic_edges = mask
        if spec.ndim == 3:
            s.cells[:] = [int(v) for v in spec.grid_shape]
        else:
            s.cells[:] = [1, int(spec.grid_shape[0]), int(spec.grid_shape[1])]
        s.dt = f32(spec.dt)
        s.resolution = f32(spec.resolution)
        s.inv_resolution = f32(1.0) / f32(spec.resolution)
        s.dt_over_eps = dt_over_eps
        s.dt_over_mu = f32(spec.dt) / f32(MU_0)
        s.h_source = f32(float(spec.dt) / MU_0)
        s.tile_x, s.tile_y = int(tile[0]), int(tile[1])
        s.z_chunk = int(z_chunk)
        if layout == "pitched":
            s.layout = abi.FDTD_LAYOUT_PITCHED
            s.pitch = self.pitch
        self._keep = []  # tensors referenced by the struct
        # DFT samples are buffered and added to the arena every `dft_batch` steps
        # (bit-identical to per-step accumulation; 1 disables the buffer).
        self.dft_batch = max(1, min(16, int(dft_batch)))
        # ... and the sample of step n runs on a side stream beside step n+1
        # when no pre-E source writes a gathered cell (bit-identical either way).
        self.dft_overlap = bool(dft_overlap) and schedule == "fused" and sources_clear_of_monitors(spec)
        self.e_source = {}  # per-site E source coefficients (site material), by component

        def buf(t):
            self._keep.append(t)
            return abi.buffer_of(t)

        # Material.
        if layout == "pitched":
            s.material_kind = abi.FDTD_MATERIAL_CODEBOOK
            s.site_ids = buf(self.site_ids)
            s.site_coef = buf(self.site_coef)
            if self.site_class is not None:
                s.site_class = buf(self.site_class)
                s.class_coef = buf(self.class_coef)
            if self.lossy:
                s.h_class = buf(self.h_class)
                s.h_class_coef = buf(self.h_class_coef)
        elif spec.voxel_ids is not None:
            s.material_kind = abi.FDTD_MATERIAL_VOXEL
            ids = np.ascontiguousarray(spec.voxel_ids, dtype=np.uint8)
            self.voxels = torch.as_tensor(ids, device=dev)
            table = np.ones(256, np.float32)
            table[: len(spec.eps_table)] = spec.eps_table
            self.eps_table = _f32(table, dev)
            s.voxels = buf(self.voxels)
            s.eps_table = buf(self.eps_table)
        else:
            s.material_kind = abi.FDTD_MATERIAL_SITE
            for c in ("Ex", "Ey", "Ez"):
                if c not in self.active:
                    continue
                dec, src = spec.e_site[c]
                i = COMPONENT_INDEX[c]
                s.e_decay[i] = buf(_f32(dec, dev))
                self.e_source[c] = _f32(src, dev)
                s.e_source[i] = buf(self.e_source[c])
        for c, (dec, src) in spec.h_coefficients().items():
            if c not in self.active:
                continue
            i = COMPONENT_INDEX[c] - 3
            if self.lossy:  # the H classes carry them; the pitched layout takes scalars here
                dec, src = np.float32(1.0), np.float32(0.0)
            s.h_decay[i] = buf(_f32(dec, dev))
            s.h_source_site[i] = buf(_f32(src, dev))
        # CPML coefficient slabs.
        s.cpml = 1 if (spec.h_terms or spec.e_terms) else 0
        self.h_terms, self.e_terms = list(spec.h_terms), list(spec.e_terms)
        for dst, terms in ((s.h_terms, self.h_terms), (s.e_terms, self.e_terms)):
            for t, term in enumerate(terms):
                dst[t].axis, dst[t].low, dst[t].high = term.axis, term.low, term.high
                if term.width:
                    dst[t].a = buf(_f32(term.a, dev))
                    dst[t].b = buf(_f32(term.b, dev))
                    dst[t].inv_kappa = buf(_f32(term.inv_kappa, dev))
        # Sources.
        if len(spec.sources) > abi.FDTD_MAX_SOURCES:
            raise ValueError(f"at most {abi.FDTD_MAX_SOURCES} sources")
        s.source_count = len(spec.sources)
        for n, src in enumerate(spec.sources):
            d = s.sources[n]
            d.component = COMPONENT_INDEX[src.component]
            d.timing = abi.TIMINGS[src.timing]
            start = tuple(int(v) for v in src.start)
            d.start[:] = list(start) if spec.ndim == 3 else [0, *start]
            coeff = np.asarray(src.coeff, np.float32)
            if spec.ndim == 2:
                coeff = coeff.reshape((1, *coeff.shape))
            d.coeff = buf(_f32(coeff, dev))
            d.waveform = buf(_f32(np.asarray(src.waveform, np.float32).reshape(-1), dev))
        # Derivative metrics (axis-uniform / rectilinear grids).
        if spec.metrics is not None:
            cells = tuple(int(v) for v in spec.grid_shape)
            axes = (("z", cells[0]), ("y", cells[1]), ("x", cells[2])) if spec.ndim == 3 else (
                (None, 0), ("y", cells[0]), ("x", cells[1]))
            for a, (name, n) in enumerate(axes):
                if name is None:
                    continue
                s.metric_h[a] = buf(_f32(spec.metrics.along(f"e_to_h_{name}", n), dev))
                s.metric_e[a] = buf(_f32(spec.metrics.along(f"h_to_e_{name}", n + 1), dev))
        # Monitors.
        self.arena = pack_dft_monitors(spec.monitors, dev, [self.shapes[c] for c in COMPONENTS], self._strides)
        if self.arena is not None:
            a = self.arena
            s.dft.monitor_count = len(spec.monitors)
            for name in ("indices", "weights", "freqs", "masks", "counts", "codes", "windows", "affine"):
                setattr(s.dft, name, buf(getattr(a, name)))
        # Time-domain field recorders.
        if len(spec.recorders) > abi.FDTD_MAX_RECORDERS:
            raise ValueError(f"at most {abi.FDTD_MAX_RECORDERS} field recorders")
        self.recorders = []  # per recorder: values per record of each component
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        s.recorder_count = len(spec.recorders)
        for r, rec in enumerate(spec.recorders):
            d = s.recorders[r]
            d.interval, d.capacity = max(1, int(rec.interval)), max(0, int(rec.capacity))
            if not 1 <= len(rec.components) <= 6:
                raise ValueError("a field recorder records 1 to 6 components")
            d.component_count = len(rec.components)
            counts = []
            for q, c in enumerate(rec.components):
                if c not in self.active:
                    raise ValueError(f"field recorder component {c} is inactive in this program")
                ci = COMPONENT_INDEX[c]
                d.components[q] = ci
                d.signs[q] = rec.sign(q)
                if rec.indices is None:
                    counts.append(int(np.prod(self.shapes[c])))
                    continue
                pi, pw = _pack_plan(self.lib, stream, rec.indices[q], rec.weights[q], self.shapes[c],
                                    self._strides(ci), dev)
                d.indices[q], d.weights[q] = buf(pi), buf(pw)
                counts.append(int(pi.shape[1]))
            self.recorders.append(counts)
        self._times_for(max(int(spec.total_steps), 1))
        self.struct = s

    def _strides(self, c: int):
        """(row, plane) element strides of component ``c``'s device array."""
        if self.layout == "pitched":
            return self.pitch, self.bank_shape[1] * self.pitch
        shape = tuple(self.shapes[COMPONENTS[c]])
        _dz, dy, dx = (1,) * (3 - len(shape)) + shape  # 2D: z extent 1
        return dx, dy * dx

    def diag_site_eps(self, component: str):
        """Device relative permittivity of one E component over its stored
        shape, for energy diagnostics of dense programs: the spec's
        ``e_site_eps``, else the voxel sampling of the update (3D voxel
        material), else dt / (eps0 * source) of lossless per-site material."""
        if self._diag_eps is None:
            self._diag_eps = {}
        if component in self._diag_eps:
            return self._diag_eps[component]
        spec = self.spec
        if spec.e_site_eps is not None and component in spec.e_site_eps:
            eps = np.asarray(spec.e_site_eps[component], np.float32)
        elif spec.ndim == 3 and spec.voxel_ids is not None:
            eps = site_eps_3d(spec.voxel_ids, spec.eps_table, component)
        elif spec.e_site is not None and component in spec.e_site:
            decay, src = (np.asarray(v, np.float64) for v in spec.e_site[component])
            if np.any(decay != 1.0):
                raise ValueError(f"{component}: lossy per-site material needs e_site_eps for energy diagnostics")
            eps = (float(spec.dt) / (EPS_0 * src)).astype(np.float32)
        else:
            eps = np.ones(1, np.float32)
        eps = np.broadcast_to(eps, self.shapes[component]).astype(np.float32)
        self._diag_eps[component] = _f32(eps, self.device)
        return self._diag_eps[component]

    def view(self, bank_tensor, component: str):
        """The component's own extent inside a device field tensor."""
        if self.layout != "pitched":
            return bank_tensor
        dz, dy, dx = self.shapes[component]
        return bank_tensor[:dz, :dy, :dx]

    def _times_for(self, nsteps: int):
        have = getattr(self, "_step_time_len", 0)
        if nsteps <= have:
            return
        n = max(nsteps, 2 * have)
        self.step_time_host = step_times(self.spec.t0, self.spec.dt, n)
        self.step_time = _f32(self.step_time_host, self.device)
        self._step_time_len = n

    def clock_after(self, step: int) -> float:
        """Float32 clock after ``step`` completed steps."""
        if step <= 0:
            return float(np.float32(self.spec.t0))
        self._times_for(step)
        return float(self.step_time_host[step - 1])

    # -- struct assembly ---------------------------------------------------
    def fill(self, state: "DeviceState", nsteps: int) -> abi.FdtdProgram:
        s = abi.FdtdProgram.from_buffer_copy(self.struct)
        s.nsteps = int(nsteps)
        for c in range(6):
            s.fields[c] = abi.buffer_of(state.fields[c])
            if state.alt is not None:
                s.fields_alt[c] = abi.buffer_of(state.alt[c])
        for t, term in enumerate(self.h_terms):
            if term.width:
                s.h_terms[t].psi = abi.buffer_of(state.psi_h[t])
                if state.psi_h_alt is not None:
                    s.h_terms[t].psi_alt = abi.buffer_of(state.psi_h_alt[t])
        for t, term in enumerate(self.e_terms):
            if term.width:
                s.e_terms[t].psi = abi.buffer_of(state.psi_e[t])
        if self.arena is not None:
            s.dft.re = abi.buffer_of(state.dft_re)
            s.dft.im = abi.buffer_of(state.dft_im)
            s.dft.weight_sum = abi.buffer_of(state.dft_w)
            if state.dft_samples is not None:
                s.dft.batch = self.dft_batch
                s.dft.samples = abi.buffer_of(state.dft_samples)
                if self.dft_overlap:
                    s.flags |= abi.FDTD_FLAG_DFT_OVERLAP
        for r, bufs in enumerate(state.records):
            d = s.recorders[r]
            for q, v in enumerate(bufs["values"]):
                d.values[q] = abi.buffer_of(v)
            d.steps, d.times, d.count = (abi.buffer_of(bufs[k]) for k in ("steps", "times", "count"))
        s.step_counter = abi.buffer_of(state.counter)
        s.step_time = abi.buffer_of(self.step_time)
        s.status = abi.buffer_of(state.status)
        return s


class DeviceState:
    """Evolving fields, CPML memories, DFT arena and clocks (beamz/simulation/model.py:127-259)."""

    def __init__(self, program: DeviceProgram, fields=None, psi_h=None, psi_e=None, step: int = 0):
        torch = _torch()
        dev = program.device
        self.program = program
        sh = program.shapes
        empty = torch.zeros(0, dtype=torch.float32, device=dev)

        def zeros(c):
            if c not in program.active:
                return empty
            shape = program.bank_shape if program.layout == "pitched" else sh[c]
            return torch.zeros(shape, dtype=torch.float32, device=dev)

        self.fields = [zeros(c) for c in COMPONENTS]
        if fields is not None:
            self.set_fields(fields)
        fused = program.schedule == abi.FDTD_SCHEDULE_FUSED
        self.alt = [torch.empty_like(f) for f in self.fields] if fused else None

        def psi_list(terms, given):
            out = []
            for i, t in enumerate(terms):
                shape = t.psi_shape(sh[t.component])
                if given is not None:
                    out.append(_f32(given[i], dev).reshape(shape).contiguous())
                else:
                    out.append(torch.zeros(shape, dtype=torch.float32, device=dev))
            return out

        self.psi_h = psi_list(program.h_terms, psi_h)
        self.psi_e = psi_list(program.e_terms, psi_e)
        self.psi_h_alt = [torch.empty_like(p) for p in self.psi_h] if fused else None
        a = program.arena
        nv = a.value_count if a else 0
        nw = a.weight_count if a else 0
        self.dft_re = torch.zeros(nv, dtype=torch.float32, device=dev)
        self.dft_im = torch.zeros(nv, dtype=torch.float32, device=dev)
        self.dft_w = torch.zeros(nw, dtype=torch.float32, device=dev)
        self.dft_samples = None
        if a is not None and program.dft_batch > 1:
            M, P = len(a.layout), int(a.indices.shape[3])
            self.dft_samples = torch.empty((program.dft_batch, M, 6, P), dtype=torch.float32, device=dev)
        self.records = []
        for rec, counts in zip(program.spec.recorders, program.recorders):
            cap = max(0, int(rec.capacity))
            self.records.append({
                "values": [torch.zeros((cap, v), dtype=torch.float32, device=dev) for v in counts],
                "steps": torch.zeros(cap, dtype=torch.int32, device=dev),
                "times": torch.zeros(cap, dtype=torch.float32, device=dev),
                "count": torch.zeros(2, dtype=torch.int32, device=dev),
            })
        self.counter = torch.full((1,), int(step), dtype=torch.int32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.step = int(step)
        self.t = program.clock_after(self.step)

    def swap_banks(self):
        self.fields, self.alt = self.alt, self.fields
        if self.psi_h_alt is not None:
            self.psi_h, self.psi_h_alt = self.psi_h_alt, self.psi_h

    def set_fields(self, fields: dict) -> None:
        """Load host or device arrays (beamz component shapes) into the current bank."""
        for i, c in enumerate(COMPONENTS):
            if c in fields and c in self.program.active:
                src = fields[c]
                if not isinstance(src, _torch().Tensor):
                    src = _f32(src, self.program.device)
                self.program.view(self.fields[i], c).copy_(src.reshape(self.program.shapes[c]))

    def field(self, component: str):
        """Device view of one component in beamz's shape (may be strided)."""
        return self.program.view(self.fields[COMPONENT_INDEX[component]], component)

    def check(self) -> None:
        """Raise if a bounded device wait expired in an earlier launch."""
        if int(self.status.item()) != 0:
            raise abi.FdtdError(int(self.status.item()), "device wait expired", "step kernel")

    def numpy(self) -> dict:
        """Host copies of every field, memory and accumulator."""
        self.check()
        out = {c: self.field(c).cpu().numpy() for c in COMPONENTS if c in self.program.active}
        out["psi_h"] = [p.cpu().numpy() for p in self.psi_h]
        out["psi_e"] = [p.cpu().numpy() for p in self.psi_e]
        out["dft_re"] = self.dft_re.cpu().numpy()
        out["dft_im"] = self.dft_im.cpu().numpy()
        out["dft_w"] = self.dft_w.cpu().numpy()
        out["t"] = np.float32(self.t)
        out["step"] = self.step
        return out


def compile_program(spec: ProgramSpec, device="cuda", tile=(32, 8), z_chunk=16, tune: bool = False,
                    **kwargs) -> DeviceProgram:
    """Upload a program's static inputs (beamz/simulation/compile.py:796-895 analogue).

    ``tile="auto"`` / ``z_chunk="auto"`` take the 3D launch shape from the
    per-shape autotuner (measuring it now when ``tune``)."""
    if tile == "auto" or z_chunk == "auto":
        from . import autotune

        ty, zc = autotune.choose(spec, device=device, tune=tune)
        tile = (32, ty) if tile == "auto" else tile
        z_chunk = zc if z_chunk == "auto" else z_chunk
    return DeviceProgram(spec, device=device, tile=tile, z_chunk=z_chunk, **kwargs)


def initial_state(program: DeviceProgram, **kwargs) -> DeviceState:
    return DeviceState(program, **kwargs)


def _stream(program: DeviceProgram):
    return ctypes.c_void_p(_torch().cuda.current_stream(program.device).cuda_stream)


def update_h(state: DeviceState, program: DeviceProgram) -> DeviceState:
    """H half step in place, with CPML and PEC (beamz/simulation/cuda/runtime.py:184)."""
    s = program.fill(state, 0)
    abi.check(program.lib.fdtd_launch_phase(_stream(program), ctypes.byref(s), 0), "fdtd_launch_phase(H)")
    return state


def update_e(state: DeviceState, program: DeviceProgram) -> DeviceState:
    """E half step in place, with CPML and PEC (beamz/simulation/cuda/runtime.py:234)."""
    s = program.fill(state, 0)
    abi.check(program.lib.fdtd_launch_phase(_stream(program), ctypes.byref(s), 1), "fdtd_launch_phase(E)")
    return state


def apply_sources(state: DeviceState, program: DeviceProgram, timing: str) -> DeviceState:
    """Inject every source of one timing at the state's current step."""
    s = program.fill(state, 0)
    abi.check(program.lib.fdtd_apply_sources(_stream(program), ctypes.byref(s), abi.TIMINGS[timing], 0),
              "fdtd_apply_sources")
    return state


def accumulate_monitors(state: DeviceState, program: DeviceProgram) -> DeviceState:
    """The end-of-step monitor updates: DFT accumulation, then the field
    recorders (beamz/simulation/observe.py:649-795)."""
    s = program.fill(state, 0)
    abi.check(program.lib.fdtd_accumulate_dft(_stream(program), ctypes.byref(s), 0), "fdtd_accumulate_dft")
    if s.recorder_count:
        abi.check(program.lib.fdtd_record_fields(_stream(program), ctypes.byref(s), 0), "fdtd_record_fields")
    return state


def step_by_phases(state: DeviceState, program: DeviceProgram) -> DeviceState:
    """One step composed from the phase-level entries in beamz's order
    (beamz/simulation/execute.py:467-541)."""
    apply_sources(state, program, "pre_e")
    update_h(state, program)
    apply_sources(state, program, "h")
    update_e(state, program)
    apply_sources(state, program, "e")
    accumulate_monitors(state, program)
    state.counter += 1
    state.step += 1
    state.t = program.clock_after(state.step)
    return state


def run_steps(state: DeviceState, program: DeviceProgram, nsteps: int, chunk: int = GRAPH_CHUNK_STEPS) -> DeviceState:
    """Advance ``nsteps`` complete steps (beamz/simulation/cuda/runtime.py:621/685)."""
    if nsteps < 0:
        raise ValueError("step count must be non-negative")
    program._times_for(state.step + nsteps)
    done = 0
    stream = _stream(program)
    while done < nsteps:
        n = min(chunk, nsteps - done)
        s = program.fill(state, n)
        abi.check(program.lib.fdtd_launch_program(stream, ctypes.byref(s)), "fdtd_launch_program")
        if program.schedule == abi.FDTD_SCHEDULE_FUSED and n % 2 == 1:
            state.swap_banks()
        done += n
    state.step += nsteps
    state.t = program.clock_after(state.step)
    return state


run_program_steps = run_steps


@dataclass
class FieldDiagnostics:
    """Integrated electromagnetic energy (J; per metre of depth in 2D), largest
    |field| and finiteness of a state's fields."""

    energy: float
    max_field: float
    finite: bool
    nonfinite: int


def field_diagnostics(state: DeviceState, program: DeviceProgram) -> FieldDiagnostics:
    """beamz/simulation/execute.py:184-222 (_field_diagnostics) as one device
    reduction (fdtd_field_diagnostics): sum over components of
    0.5 * const * sum(eps_r * v^2 * control volume), const = eps0 for E and mu0
    for H.  Non-finite values are counted, and left out of the sum and max."""
    torch = _torch()
    dev = program.device
    if getattr(state, "_diag_scratch", None) is None:
        state._diag_scratch = (torch.empty(6 * abi.FDTD_DIAG_BLOCKS * 3, dtype=torch.float64, device=dev),
                               torch.empty(18, dtype=torch.float64, device=dev))
    partials, out = state._diag_scratch
    d = abi.FdtdDiagnostics()
    if program.layout == "pitched":
        if program.site_eps_table is None:
            raise ValueError("energy diagnostics of a conductive program need the spec's e_site_eps")
        d.site_eps_table = abi.buffer_of(program.site_eps_table)
    else:
        for i, c in enumerate(("Ex", "Ey", "Ez")):
            if c in program.active:
                d.site_eps[i] = abi.buffer_of(program.diag_site_eps(c))
    d.partials = abi.buffer_of(partials)
    d.out = abi.buffer_of(out)
    s = program.fill(state, 0)
    abi.check(program.lib.fdtd_field_diagnostics(_stream(program), ctypes.byref(s), ctypes.byref(d)),
              "fdtd_field_diagnostics")
    r = out.cpu().numpy().reshape(6, 3)
    volume = float(program.spec.resolution) ** program.ndim
    energy = sum(0.5 * (EPS_0 if i < 3 else MU_0) * float(r[i, 0]) * volume
                 for i, c in enumerate(COMPONENTS) if c in program.active)
    nonfinite = int(r[:, 2].sum())
    return FieldDiagnostics(float(energy), float(r[:, 1].max()), nonfinite == 0 and np.isfinite(energy), nonfinite)


def dft_change(state: DeviceState, program: DeviceProgram, monitors=None):
    """Largest relative change of any (monitor, component, frequency) DFT vector
    since the previous call, and whether every monitor value is finite
    (beamz/simulation/execute.py:294-316, _relative_monitor_change): per vector
    |cur - prev| / max(|cur|, |prev|), 0 when both norms vanish.  The first
    call only records the arena and returns (None, finite).  ``monitors``
    selects monitor indices (default: every monitor)."""
    torch = _torch()
    if program.arena is None:
        return None, True
    first = getattr(state, "_dft_prev", None) is None
    if first:
        F = int(program.arena.freqs.shape[1])
        state._dft_prev = (torch.zeros_like(state.dft_re), torch.zeros_like(state.dft_im),
                           torch.empty(len(program.arena.layout) * 6 * F * 3, dtype=torch.float64,
                                       device=program.device))
    prev_re, prev_im, out = state._dft_prev
    c = abi.FdtdDftChange(abi.buffer_of(prev_re), abi.buffer_of(prev_im), abi.buffer_of(out))
    s = program.fill(state, 0)
    abi.check(program.lib.fdtd_dft_change(_stream(program), ctypes.byref(s), ctypes.byref(c)), "fdtd_dft_change")
    M = len(program.arena.layout)
    r = out.cpu().numpy().reshape(M, 6, -1, 3)
    chosen = range(M) if monitors is None else monitors
    keys = [(m, ci, f) for m in chosen for ci in range(6) if program.spec.monitors[m].component_mask[ci] > 0
            for f in range(program.arena.layout[m][1])]
    finite = all(np.isfinite(r[k][1]) for k in keys)
    if first:
        return None, finite
    tiny = np.finfo(float).tiny
    changes = []
    for k in keys:
        num = float(np.sqrt(r[k][0]))
        den = max(float(np.sqrt(r[k][1])), float(np.sqrt(r[k][2])))
        changes.append(0.0 if den <= tiny and num <= tiny else num / den)
    return max(changes, default=0.0), finite


def monitor_values(state: DeviceState, program: DeviceProgram, monitor: int) -> dict:
    """Host copy of one monitor's stored DFT values: component -> complex128
    [F, P] (the arena slice beamz records as ``dft_fields``)."""
    voff, nf, npts, _woff = program.arena.layout[monitor]
    n = 6 * nf * npts
    re = state.dft_re[voff:voff + n].cpu().numpy().astype(np.float64).reshape(6, nf, npts)
    im = state.dft_im[voff:voff + n].cpu().numpy().astype(np.float64).reshape(6, nf, npts)
    return {c: re[i] + 1j * im[i] for i, c in enumerate(COMPONENTS)}


def _tangential_pairs(axis: str):
    """(E1, E2, H1, H2) tangential to a plane normal (beamz/devices/modes/
    fields.py:15-19) as component indices: pair 0 = (E1, H1), pair 1 = (E2, H2)."""
    names = {"x": ("Ey", "Ez", "Hz", "Hy"), "y": ("Ez", "Ex", "Hx", "Hz"), "z": ("Ex", "Ey", "Hy", "Hx")}[axis]
    return names, [COMPONENT_INDEX[names[0]], COMPONENT_INDEX[names[1]]], \
        [COMPONENT_INDEX[names[2]], COMPONENT_INDEX[names[3]]]


def _flux_scales(state: DeviceState, program: DeviceProgram, monitor: int, base_dt):
    """Per frequency (alpha, phase re, phase im): stored values times alpha =
    2 / max(window weight sum, 1e-18) (beamz/simulation/observe.py:166-179),
    H values also times exp(-i pi f dt) with a base time step (observe.py:182-187)."""
    _voff, nf, _npts, woff = program.arena.layout[monitor]
    wsum = state.dft_w[woff:woff + nf].cpu().numpy().astype(np.float64)
    alpha = 2.0 / np.maximum(wsum, 1e-18)
    freqs = np.asarray(program.spec.monitors[monitor].freqs, dtype=float)[:nf]
    phase = np.exp(-1j * np.pi * freqs * base_dt) if base_dt else np.ones(nf, np.complex128)
    return np.stack([alpha, phase.real, phase.imag], axis=1)


def _monitor_reduce(state, program, monitor, e, h, scale, weights, profiles=None):
    torch = _torch()
    voff, nf, npts, _woff = program.arena.layout[monitor]
    rows = 0 if profiles is None else int(profiles.shape[0])
    dev = program.device
    f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)  # noqa: E731
    keep = [f64(scale), f64(weights)]
    out = torch.empty((max(rows, 1), nf, 2, 2), dtype=torch.float64, device=dev)
    r = abi.FdtdMonitorReduce()
    r.abi_version = abi.FDTD_ABI_VERSION
    r.freq_count, r.value_offset, r.point_count = nf, voff, npts
    r.e[:], r.h[:] = e, h
    r.rows = rows
    r.scale, r.weights, r.out = abi.buffer_of(keep[0]), abi.buffer_of(keep[1]), abi.buffer_of(out)
    if rows:
        keep += [f64(profiles.real), f64(profiles.imag)]
        r.profile_re, r.profile_im = abi.buffer_of(keep[2]), abi.buffer_of(keep[3])
    s = program.fill(state, 0)
    abi.check(program.lib.fdtd_monitor_reduce(_stream(program), ctypes.byref(s), ctypes.byref(r)),
              "fdtd_monitor_reduce")
    o = out.cpu().numpy()
    return o[..., 0] + 1j * o[..., 1]  # [rows or 1, F, pair]


def monitor_dft_flux(state: DeviceState, program: DeviceProgram, monitor: int, axis: str, sign: float = 1.0,
                     integration_weights=None, measure=None, base_dt=None) -> np.ndarray:
    """Power through a plane monitor per frequency, on the device arena
    (beamz/simulation/observe.py:198-234 monitor_dft_flux):
    0.5 Re sum_p sign (E1 conj(H1) - E2 conj(H2)) w_p over the flux-normalised
    fields, ``axis`` the plane normal ("x", "y", "z"), w the per-point
    ``integration_weights`` (size P) or else a constant ``measure``."""
    _voff, nf, npts, _woff = program.arena.layout[monitor]
    _names, e, h = _tangential_pairs(axis)
    iw = np.asarray(() if integration_weights is None else integration_weights, dtype=float).reshape(-1)
    per_point = iw.size == npts
    if not per_point and measure is None:
        raise ValueError("monitor_dft_flux needs integration weights of one per point or a measure")
    w = iw if per_point else np.ones(npts)
    sums = _monitor_reduce(state, program, monitor, e, h, _flux_scales(state, program, monitor, base_dt),
                           np.stack([w, w]))[0]
    flux = 0.5 * np.real(sign * (sums[:, 0] - sums[:, 1]))
    return flux if per_point else flux * float(measure)


def modal_overlap(state: DeviceState, program: DeviceProgram, monitor: int, modes, axis: str, measure=1.0,
                  direction_sign: float = 1.0, base_dt=None) -> np.ndarray:
    """Overlap of a plane monitor's flux-normalised DFT fields with each mode,
    per frequency, on the device arena (beamz/devices/modes/fields.py:76-129
    _modal_overlap): 0.25 dir [sum w1 (E1 conj(Hm1) + conj(Em1) H1) -
    sum w2 (E2 conj(Hm2) + conj(Em2) H2)].  ``modes`` is a list of mappings
    component name -> complex profile [F, P] (or [P] for every frequency) of
    the four tangential components; ``measure`` a scalar, a per-point array
    or a mapping E name -> per-point weights.  Returns [len(modes), F]."""
    _voff, nf, npts, _woff = program.arena.layout[monitor]
    names, e, h = _tangential_pairs(axis)
    weights = np.empty((2, npts))
    for q in range(2):
        m = measure[names[q]] if isinstance(measure, dict) else measure
        weights[q] = np.broadcast_to(np.asarray(m, dtype=float).reshape(-1) if np.ndim(m) else float(m), (npts,))
    prof = np.empty((len(modes), nf, 4, npts), np.complex128)
    for r, mode in enumerate(modes):
        for k, name in enumerate(names):
            prof[r, :, k] = np.broadcast_to(np.asarray(mode[name], np.complex128).reshape(-1, npts), (nf, npts))
    sums = _monitor_reduce(state, program, monitor, e, h, _flux_scales(state, program, monitor, base_dt),
                           weights, prof)
    return 0.25 * float(direction_sign) * (sums[:, :, 0] - sums[:, :, 1])


def recorded(state: DeviceState, program: DeviceProgram, recorder: int) -> dict:
    """What field recorder ``recorder`` holds so far, as beamz returns it
    (observe.py:588-646): ``steps`` (absolute step + 1 of each record),
    ``times`` (t + dt), and per component its records [n, *shape]."""
    rec = program.spec.recorders[recorder]
    bufs = state.records[recorder]
    n = int(bufs["count"][state.step & 1].item())
    out = {"steps": bufs["steps"][:n].cpu().numpy(), "times": bufs["times"][:n].cpu().numpy()}
    for q, c in enumerate(rec.components):
        shape = rec.shapes[q] if rec.shapes is not None else program.shapes[c]
        out[c] = bufs["values"][q][:n].cpu().numpy().reshape((n, *shape))
    return out
