"""Per-grid-shape choice of the 3D step's tile shape and z chunk.

The class step (csrc/class_step.cu, the pitched 3D hot path) has two launch
knobs: the CTA's rows (`tile_y`: 8 or 4 rows of 128 lattice points, 8 or 4
warps) and the number of z planes one CTA marches (`z_chunk`).  Large grids
want long chunks (fewer re-read boundary planes); small grids want short
ones, so that more CTAs are resident and each CTA's plane chain is shorter.
`choose` returns the measured best for a shape class, measuring the
candidates once on the device when asked to (`tune=True`) and remembering the
result in a JSON table; without a table entry it falls back to rules fitted
to B200 measurements.

The temporal-block depth is 1 (one launch advances one step): a second step
inside the z-march would need the first step's E and H on a one- to two-cell
x / y ring around each tile (25-50 % more work on 8-row tiles) and a second
set of plane rings in shared memory, which the step's two CTAs per SM already
fill.
"""

from __future__ import annotations

import json
import os
import threading

import numpy as np

TILE_Y = (8, 4)
Z_CHUNKS = (4, 8, 16, 32)
_LOCK = threading.Lock()
_MEMO: dict = {}


def default_table_path() -> str:
    """The table lives beside the in-tree library (it describes this device's
    measurements, like the library describes this build)."""
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "_tuning.json")


def shape_class(spec) -> str:
    """Key of a tuning entry: dimensionality, grid rounded to 32 and absorber."""
    g = tuple(int(-(-int(v) // 32) * 32) for v in spec.grid_shape)
    cpml = int(bool(spec.h_terms or spec.e_terms))
    return f"{len(g)}d:" + "x".join(map(str, g)) + f":cpml{cpml}"


def heuristic(spec) -> tuple[int, int]:
    """Rules from B200 sweeps of the class step (us per step, best first):
    8-row tiles throughout; 16-plane chunks once the grid holds enough CTAs
    for many waves (512x512x256: 903 vs 946 with 8), 8-plane chunks below
    that (192^3: 247 vs 283 with 4), 4-plane chunks for grids of a few
    million cells, whose CTAs would otherwise not fill the GPU (128^3: 75 vs
    92 with 8)."""
    cells = int(np.prod(spec.grid_shape))
    if cells >= 32 * 1024 * 1024:
        return (8, 16)
    return (8, 8) if cells >= 4 * 1024 * 1024 else (8, 4)


def _load(path: str) -> dict:
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(path: str, table: dict) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def measure(spec, device="cuda", steps: int = 24, candidates=None) -> dict:
    """Time every candidate (tile_y, z_chunk) on `spec` (sources and monitors
    kept); returns {(tile_y, z_chunk): microseconds per step}."""
    import torch

    from . import runtime

    dev = runtime._require_cuda(device)
    candidates = candidates or [(ty, zc) for ty in TILE_Y for zc in Z_CHUNKS]
    out = {}
    for ty, zc in candidates:
        prog = runtime.compile_program(spec, device=dev, tile=(128, ty), z_chunk=zc, graphs=True)
        if prog.layout != "pitched":
            return {}
        prog._times_for(3 * steps + 4)
        st = runtime.initial_state(prog)
        runtime.run_steps(st, prog, steps)
        runtime.run_steps(st, prog, steps)
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        runtime.run_steps(st, prog, steps)
        b.record()
        torch.cuda.synchronize(dev)
        out[(ty, zc)] = a.elapsed_time(b) * 1e3 / steps
        del st, prog
    return out


def choose(spec, device="cuda", tune: bool = False, path: str | None = None) -> tuple[int, int]:
    """(tile_y, z_chunk) for `spec`: the table entry of its shape class, a fresh
    measurement when `tune` (stored in the table), else the heuristic."""
    if spec.ndim != 3:
        return heuristic(spec)
    key = shape_class(spec)
    path = path or default_table_path()
    with _LOCK:
        if (path, key) in _MEMO:
            return _MEMO[(path, key)]
        table = _load(path)
        if key in table:
            _MEMO[(path, key)] = tuple(table[key]["best"])
            return _MEMO[(path, key)]
    if not tune:
        return heuristic(spec)
    times = measure(spec, device=device)
    if not times:
        return heuristic(spec)
    best = min(times, key=times.get)
    with _LOCK:
        table = _load(path)
        table[key] = {"best": list(best), "us_per_step": {f"{t}x{z}": round(v, 2) for (t, z), v in times.items()}}
        _store(path, table)
        _MEMO[(path, key)] = best
    return best
