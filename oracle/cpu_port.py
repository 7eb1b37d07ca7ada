"""ctypes driver for the C restatement (oracle/fdtd_cpu.c) -- TEST INFRASTRUCTURE.

Used only by tests and by bench.py's CPU-baseline / reference arm.  It fills
the same FdtdProgram struct as the CUDA library, but with host (numpy)
buffers, and runs the OpenMP loops of ``fdtd_cpu_run`` on all host threads.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from beamz_b200 import abi
from beamz_b200.plan import COMPONENT_INDEX, COMPONENTS, EPS_0, MU_0, ProgramSpec, active_components, component_shape
from beamz_b200.plan import step_times

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libfdtd_cpu.so")


def build() -> str:
    """Compile oracle/fdtd_cpu.c with the committed Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        build()  # make is incremental; rebuilds when fdtd_cpu.c or the ABI header changed
        lib = ctypes.CDLL(LIB)
        lib.fdtd_cpu_run.argtypes = [ctypes.POINTER(abi.FdtdProgram), ctypes.c_int]
        lib.fdtd_cpu_run.restype = ctypes.c_int
        lib.fdtd_cpu_max_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def _buf(arr: np.ndarray) -> abi.FdtdBuffer:
    b = abi.FdtdBuffer()
    b.data = arr.ctypes.data if arr.size else None
    b.rank = arr.ndim
    b.element_type = {np.dtype(np.float32): abi.FDTD_F32, np.dtype(np.int32): abi.FDTD_S32,
                      np.dtype(np.uint8): abi.FDTD_U8}[arr.dtype]
    for a, n in enumerate(arr.shape):
        b.dims[a] = n
    return b


class HostRun:
    """Host state + program for the C restatement."""

    def __init__(self, spec: ProgramSpec, fields=None):
        self.spec = spec
        self.active = active_components(spec.ndim, spec.polarization)
        keep = self.keep = []

        def k(a):
            a = np.ascontiguousarray(a)
            keep.append(a)
            return a

        s = self.struct = abi.FdtdProgram()
        s.abi_version = abi.FDTD_ABI_VERSION
        s.ndim = spec.ndim
        s.polarization = 0 if spec.polarization == "tm" else 1
        s.schedule = abi.FDTD_SCHEDULE_PHASES
        m = 0
        for e in spec.metallic_edges:
            m |= 1 << abi.EDGE_BITS[e]
        s.metallic_edges = m
        s.cells[:] = list(spec.grid_shape) if spec.ndim == 3 else [1, *spec.grid_shape]
        f32 = np.float32
        s.dt = f32(spec.dt)
        s.resolution = f32(spec.resolution)
        s.inv_resolution = f32(1.0) / f32(spec.resolution)
        s.dt_over_eps = f32(spec.dt) / f32(EPS_0)
        s.dt_over_mu = f32(spec.dt) / f32(MU_0)
        self.fields = {}
        for c in COMPONENTS:
            if c in self.active:
                shape = component_shape(c, spec.grid_shape, spec.polarization)
                v = np.zeros(shape, f32) if fields is None or c not in fields else np.array(fields[c], f32)
                self.fields[c] = k(v)
                s.fields[COMPONENT_INDEX[c]] = _buf(self.fields[c])
        if spec.voxel_ids is not None:
            s.material_kind = abi.FDTD_MATERIAL_VOXEL
            s.voxels = _buf(k(spec.voxel_ids.astype(np.uint8)))
            table = np.ones(256, f32)
            table[: len(spec.eps_table)] = spec.eps_table
            s.eps_table = _buf(k(table))
        else:
            s.material_kind = abi.FDTD_MATERIAL_SITE
            for c, (dec, src) in spec.e_site.items():
                i = COMPONENT_INDEX[c]
                s.e_decay[i] = _buf(k(np.asarray(dec, f32)))
                s.e_source[i] = _buf(k(np.asarray(src, f32)))
        for c, (dec, src) in spec.h_coefficients().items():
            if c in self.active:
                i = COMPONENT_INDEX[c] - 3
                s.h_decay[i] = _buf(k(np.asarray(dec, f32)))
                s.h_source_site[i] = _buf(k(np.asarray(src, f32)))
        s.cpml = 1 if (spec.h_terms or spec.e_terms) else 0
        self.psi_h, self.psi_e = [], []
        for dst, terms, store in ((s.h_terms, spec.h_terms, self.psi_h), (s.e_terms, spec.e_terms, self.psi_e)):
            for t, term in enumerate(terms):
                dst[t].axis, dst[t].low, dst[t].high = term.axis, term.low, term.high
                psi = k(np.zeros(term.psi_shape(component_shape(term.component, spec.grid_shape, spec.polarization)), f32))
                store.append(psi)
                if term.width:
                    dst[t].a = _buf(k(np.asarray(term.a, f32)))
                    dst[t].b = _buf(k(np.asarray(term.b, f32)))
                    dst[t].inv_kappa = _buf(k(np.asarray(term.inv_kappa, f32)))
                    dst[t].psi = _buf(psi)
        s.source_count = len(spec.sources)
        for n, src in enumerate(spec.sources):
            d = s.sources[n]
            d.component = COMPONENT_INDEX[src.component]
            d.timing = abi.TIMINGS[src.timing]
            d.start[:] = list(src.start) if spec.ndim == 3 else [0, *src.start]
            coeff = np.asarray(src.coeff, f32)
            if spec.ndim == 2:
                coeff = coeff.reshape((1, *coeff.shape))
            d.coeff = _buf(k(coeff))
            d.waveform = _buf(k(np.asarray(src.waveform, f32).reshape(-1)))
        self.dft_re = self.dft_im = self.dft_w = np.zeros(0, f32)
        if spec.monitors:
            mons = spec.monitors
            M, P = len(mons), max(m.points for m in mons)
            K = max(max(a.shape[1] for a in m.indices) for m in mons)
            F = max(len(m.freqs) for m in mons)
            idx = np.zeros((M, 6, K, P), np.int32)  # neighbour-major, as the ABI lays it out
            w = np.zeros((M, 6, K, P), f32)
            fr = np.zeros((M, F), f32)
            masks = np.zeros((M, 6), f32)
            counts = np.zeros((M, 5), np.int32)
            codes = np.zeros((M, 2), np.int32)
            win = np.zeros((M, 3), f32)
            vo = wo = 0
            for mi, mon in enumerate(mons):
                p, nf = mon.points, len(mon.freqs)
                for c in range(6):
                    idx[mi, c, : mon.indices[c].shape[1], :p] = np.asarray(mon.indices[c]).T
                    w[mi, c, : mon.weights[c].shape[1], :p] = np.asarray(mon.weights[c]).T
                fr[mi, :nf] = mon.freqs
                masks[mi] = mon.component_mask
                counts[mi] = (nf, p, max(1, mon.interval), vo, wo)
                codes[mi] = (mon.window_code, mon.normalization_code)
                win[mi] = (mon.t_start, mon.t_end, mon.length_unit)
                vo += 6 * nf * p
                wo += nf
            self.dft_re, self.dft_im, self.dft_w = k(np.zeros(vo, f32)), k(np.zeros(vo, f32)), k(np.zeros(wo, f32))
            d = s.dft
            d.monitor_count = M
            for name, arr in (("indices", idx), ("weights", w), ("freqs", fr), ("masks", masks), ("counts", counts),
                              ("codes", codes), ("windows", win), ("re", self.dft_re), ("im", self.dft_im),
                              ("weight_sum", self.dft_w)):
                setattr(d, name, _buf(k(arr)))
        self.counter = k(np.zeros(1, np.int32))
        s.step_counter = _buf(self.counter)
        self.step_time = k(step_times(spec.t0, spec.dt, max(spec.total_steps, 1)))
        s.step_time = _buf(self.step_time)

    def run(self, nsteps: int, threads: int = 0) -> "HostRun":
        lib = load()
        need = int(self.counter[0]) + int(nsteps)
        if need > self.step_time.size:
            self.step_time = np.ascontiguousarray(step_times(self.spec.t0, self.spec.dt, need))
            self.keep.append(self.step_time)
            self.struct.step_time = _buf(self.step_time)
        self.struct.nsteps = int(nsteps)
        lib.fdtd_cpu_run(ctypes.byref(self.struct), int(threads))
        return self


def max_threads() -> int:
    return int(load().fdtd_cpu_max_threads())
