"""Continuous-batching serving loop for FDTD simulation requests.

Requests (a planned :class:`~beamz_b200.plan.ProgramSpec` plus a step count)
arrive over time.  The engine admits them FIFO as soon as the HBM budget, the
slot limit and the resident-cell bound allow -- also while others are running
-- compiles each onto the device once, and keeps its fields, CPML memories and
DFT arena resident until it finishes.  Every admitted simulation gets its own
CUDA stream and its own executable graphs of up to ``chunk`` steps
(``fdtd_graph_create``); the host loop keeps up to ``queue_depth`` chunks
queued per stream, so the simulations' step kernels overlap on the device and
small grids fill the GPU together.  Results (the
DFT arena and, optionally, the fields) are copied back when a simulation's
last chunk completes, and its memory and graphs are released, which admits
the next request.

beamz runs one simulation per call (beamz/simulation/execute.py:603-681); the
sequential baseline here is that plain path, one request at a time
(:func:`run_sequential`).  Each result is identical, bit for bit, alone and in
the mix: a simulation's kernels touch only its own buffers, in the same order.
"""

from __future__ import annotations

import ctypes
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .plan import COMPONENTS, ProgramSpec, active_components, component_shape


@dataclass
class Request:
    rid: int
    spec: ProgramSpec
    nsteps: int
    arrival: float = 0.0  # seconds after the stream starts


@dataclass
class Result:
    rid: int
    nsteps: int
    dft_re: np.ndarray
    dft_im: np.ndarray
    dft_w: np.ndarray
    fields: dict | None
    arrival: float
    admitted: float
    finished: float
    records: list | None = None  # per field recorder: runtime.recorded(...)
    gpu_s: float | None = None  # device time of the request's steps (sequential path: CUDA events)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def estimate_bytes(spec: ProgramSpec, schedule: str = "fused") -> int:
    """Device bytes one simulation holds: two field banks (one for the phase
    schedule), CPML memories (H double-banked), material, DFT arena, field
    recorders, clock."""
    active = active_components(spec.ndim, spec.polarization)
    shapes = {c: component_shape(c, spec.grid_shape, spec.polarization) for c in COMPONENTS}
    banks = 2 if schedule == "fused" else 1
    if spec.ndim == 3:
        nz, ny, nx = spec.grid_shape
        pitch = -(-(nx + 1) // 4) * 4
        field_bytes = 6 * (nz + 1) * (ny + 1) * pitch * 4
        material = (nz + 1) * (ny + 1) * pitch * 4
    else:
        field_bytes = sum(int(np.prod(shapes[c])) * 4 for c in active)
        material = sum(int(np.prod(shapes[c])) * 8 for c in active if c.startswith("E"))
    psi = sum(int(np.prod(t.psi_shape(shapes[t.component]))) * 4 * banks for t in spec.h_terms)
    psi += sum(int(np.prod(t.psi_shape(shapes[t.component]))) * 4 for t in spec.e_terms)
    dft = 0
    for m in spec.monitors:
        points = max(int(np.asarray(ix).shape[0]) for ix in m.indices)
        dft += 6 * len(m.freqs) * points * 8 * 2 + 6 * points * 8 * 8 + 16 * 6 * points * 4  # + sample batch
    records = 0
    for r in spec.recorders:
        for q, c in enumerate(r.components):
            values = int(np.prod(shapes[c])) if r.indices is None else int(np.asarray(r.indices[q]).shape[0])
            plan = 0 if r.indices is None else values * np.asarray(r.indices[q]).shape[1] * 8
            records += int(r.capacity) * values * 4 + plan
        records += int(r.capacity) * 8 + 8
    return banks * field_bytes + material + psi + dft + records + 4 * max(int(spec.total_steps), 1) + (1 << 20)


class _Slot:
    """One admitted simulation: device program, state, stream and graphs."""

    def __init__(self, req: Request, program, state, stream, lib, chunk: int, nbytes: int, admitted: float):
        self.req = req
        self.program = program
        self.state = state
        self.stream = stream
        self.lib = lib
        self.nbytes = nbytes
        self.admitted = admitted
        self.remaining = req.nsteps
        self.graphs = {}
        self.events = deque()
        self.chunk = chunk

    def _graph(self, n: int):
        # Chunks of `chunk` (even) steps leave the banks in place; the last,
        # possibly odd, chunk runs once, so one graph per chunk size suffices.
        g = self.graphs.get(n)
        if g is None:
            s = self.program.fill(self.state, n)
            handle = ctypes.c_void_p()
            abi.check(self.lib.fdtd_graph_create(ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(s),
                                                 ctypes.byref(handle)), "fdtd_graph_create")
            self.graphs[n] = handle
            g = handle
        return g

    def launch(self, torch) -> bool:
        if self.remaining <= 0:
            return False
        n = min(self.chunk, self.remaining)
        g = self._graph(n)
        abi.check(self.lib.fdtd_graph_launch(ctypes.c_void_p(self.stream.cuda_stream), g), "fdtd_graph_launch")
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self.events.append(ev)
        self.remaining -= n
        if n % 2 == 1 and self.program.schedule == abi.FDTD_SCHEDULE_FUSED:
            self.state.swap_banks()
        self.state.step += n
        return True

    def retire_completed(self) -> None:
        while self.events and self.events[0].query():
            self.events.popleft()

    @property
    def done(self) -> bool:
        return self.remaining <= 0 and not self.events

    def release(self) -> None:
        for g in self.graphs.values():
            self.lib.fdtd_graph_destroy(g)
        self.graphs.clear()
        self.state = None
        self.program = None


def _collect(state, program, return_fields: bool):
    state.check()
    out = {
        "dft_re": state.dft_re.cpu().numpy(),
        "dft_im": state.dft_im.cpu().numpy(),
        "dft_w": state.dft_w.cpu().numpy(),
        "fields": None,
        "records": None,
    }
    if program.spec.recorders:
        from . import runtime

        out["records"] = [runtime.recorded(state, program, r) for r in range(len(program.spec.recorders))]
    if return_fields:
        out["fields"] = {c: state.field(c).cpu().numpy() for c in COMPONENTS if c in program.active}
    return out


class ServingEngine:
    """Admit, run and retire simulation requests with overlapping execution.

    ``hbm_budget`` bounds the bytes of all resident simulations (default: 80 %
    of the device memory free at construction); ``max_active`` bounds the
    number of resident simulations and ``max_active_cells`` their cells (32 Mi
    by default: a few large grids already fill the SMs, and more resident work
    only lengthens every request's latency); ``chunk`` is the graph length in
    steps and ``queue_depth`` the chunks kept queued per stream.
    """

    def __init__(self, device="cuda", hbm_budget: int | None = None, max_active: int = 48, chunk: int = 256,
                 return_fields: bool = False, queue_depth: int = 4, tune: bool = False,
                 max_active_cells: int | None = 32 * 1024 * 1024):
        import torch

        from . import runtime

        self.torch = torch
        self.runtime = runtime
        self.device = runtime._require_cuda(device)
        self.lib = abi.load_library()
        if hbm_budget is None:
            free, _total = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.8 * free)
        self.hbm_budget = int(hbm_budget)
        self.max_active = int(max_active)
        self.chunk = int(chunk) + (int(chunk) % 2)
        self.return_fields = return_fields
        self.queue_depth = int(queue_depth)
        self.tune = tune
        # Resident cells beyond a few large grids only share the same SMs:
        # throughput stays, latency grows.  None disables the bound.
        self.max_active_cells = max_active_cells
        self.peak_bytes = 0
        self.peak_active = 0

    def _admit(self, req: Request, now: float, nbytes: int) -> _Slot:
        torch = self.torch
        stream = torch.cuda.Stream(device=self.device)
        with torch.cuda.stream(stream):
            spec = req.spec
            program = self.runtime.compile_program(spec, device=self.device, tile="auto", z_chunk="auto",
                                                   tune=self.tune, graphs=False)
            program._times_for(req.nsteps)
            state = self.runtime.initial_state(program)
        return _Slot(req, program, state, stream, self.lib, self.chunk, nbytes, now)

    def run(self, requests: list[Request], clock=time.perf_counter) -> list[Result]:
        """Serve `requests` (arrival times relative to the call); return results by rid."""
        torch = self.torch
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        queue: deque[Request] = deque()
        active: list[_Slot] = []
        used = 0
        cells = 0
        results = {}
        t0 = clock()
        while pending or queue or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            progressed = False
            # Admission: FIFO while the budget and the slot limit allow.
            while queue and len(active) < self.max_active:
                need = estimate_bytes(queue[0].spec)
                if used + need > self.hbm_budget and active:
                    break
                if (self.max_active_cells is not None and active
                        and cells + queue[0].spec.cells > self.max_active_cells):
                    break
                req = queue.popleft()
                active.append(self._admit(req, clock() - t0, need))
                used += need
                cells += req.spec.cells
                self.peak_bytes = max(self.peak_bytes, used)
                self.peak_active = max(self.peak_active, len(active))
                progressed = True
            # Progress: keep `queue_depth` chunks queued per stream.
            for slot in active:
                slot.retire_completed()
                while len(slot.events) < self.queue_depth and slot.launch(torch):
                    progressed = True
            # Retire finished simulations.
            still = []
            for slot in active:
                if slot.done:
                    with torch.cuda.stream(slot.stream):
                        out = _collect(slot.state, slot.program, self.return_fields)
                    finished = clock() - t0
                    r = slot.req
                    results[r.rid] = Result(r.rid, r.nsteps, out["dft_re"], out["dft_im"], out["dft_w"], out["fields"],
                                            r.arrival, slot.admitted, finished, out["records"])
                    used -= slot.nbytes
                    cells -= slot.req.spec.cells
                    slot.release()
                    progressed = True
                else:
                    still.append(slot)
            active = still
            if not progressed:
                if not active and pending and not queue:
                    time.sleep(max(0.0, min(0.002, pending[0].arrival - (clock() - t0))))
                else:
                    time.sleep(0.0001)
        return [results[r.rid] for r in sorted(requests, key=lambda r: r.rid)]


def run_sequential(requests: list[Request], device="cuda", return_fields: bool = False,
                   clock=time.perf_counter) -> list[Result]:
    """The plain path one request at a time: wait for its arrival (if the GPU
    is idle), compile, run all steps, copy results back, then the next."""
    import torch

    from . import runtime

    dev = runtime._require_cuda(device)
    results = {}
    t0 = clock()
    for req in sorted(requests, key=lambda r: (r.arrival, r.rid)):
        wait = req.arrival - (clock() - t0)
        if wait > 0:
            time.sleep(wait)
        admitted = clock() - t0
        program = runtime.compile_program(req.spec, device=dev, tile="auto", z_chunk="auto")
        state = runtime.initial_state(program)
        stream = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        runtime.run_steps(state, program, req.nsteps)
        e1.record(stream)
        out = _collect(state, program, return_fields)
        torch.cuda.synchronize(dev)
        results[req.rid] = Result(req.rid, req.nsteps, out["dft_re"], out["dft_im"], out["dft_w"], out["fields"],
                                  req.arrival, admitted, clock() - t0, out["records"],
                                  gpu_s=e0.elapsed_time(e1) / 1e3)
        del state, program
    return [results[r.rid] for r in sorted(requests, key=lambda r: r.rid)]


@dataclass
class ServingStats:
    n: int
    makespan_s: float
    sims_per_s: float
    p50_s: float
    p99_s: float
    extra: dict = field(default_factory=dict)


def summarize(results: list[Result]) -> ServingStats:
    """Makespan, sims/s and latency percentiles; with per-request device
    times (the sequential path) also the GPU-busy fraction of the makespan and
    its inverse -- the most that filling the idle gaps between one request's
    steps and the next can gain, unless requests too small to fill the GPU
    also run side by side."""
    lat = np.array([r.latency for r in results])
    start = min(r.arrival for r in results)
    end = max(r.finished for r in results)
    span = max(end - start, 1e-9)
    stats = ServingStats(len(results), span, len(results) / span, float(np.percentile(lat, 50)),
                         float(np.percentile(lat, 99)))
    if all(r.gpu_s is not None for r in results):
        busy = float(sum(r.gpu_s for r in results))
        stats.extra = {"gpu_busy_s": busy, "gpu_busy_fraction": busy / span, "gap_filling_bound": span / max(busy, 1e-9)}
    return stats
