"""Golden vectors for time-domain field recorders, from the reference's own code.

Run from the repository root, in a container that has the beamz source tree:

    python -m tests.golden.make_recorder [--reference /path/to/beamz]

It drives ``_record_fields`` (``beamz/simulation/observe.py:588-646``, with
``monitor_records_on_step`` 322-324), loaded by path under the numpy stand-in
for ``jax`` (``_refload.py``), through seeded steps of random fields with
three compiled recorders: an interpolated plane of two components with a
sign, a whole-domain recorder, and one whose capacity runs out.  Writes
``tests/golden/recorder.npz``.
"""

from __future__ import annotations

import argparse
import os
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
GRID = (6, 7, 8)
STEPS = 7
RES = 20e-9
# (name, components, signs, interval, capacity, plane?)
RECORDERS = (
    ("plane", ("Ey", "Hz"), (1.0, -1.0), 2, 4, True),
    ("domain", ("Ex", "Hy"), (1.0, 1.0), 3, 3, False),
    ("full", ("Ez",), (1.0,), 1, 3, True),
)


def plane_plans(components):
    """The plane gather of the engine's planner for each component (dense flat
    offsets and weights, (V, K))."""
    from beamz_b200 import plan as P

    a = (np.arange(GRID[0] - 2) + 1.5) * RES
    b = (np.arange(GRID[1] - 2) + 1.25) * RES
    idx, w = [], []
    for c in components:
        i, ww = P.plane_gather(c, "x", 4.3 * RES, a, b, RES, GRID)
        idx.append(i.astype(np.int32))
        w.append(ww.astype(np.float32))
    return idx, w, (len(a), len(b))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("BEAMZ_REFERENCE_ROOT"),
                    help="root of the beamz source tree (or set BEAMZ_REFERENCE_ROOT)")
    ap.add_argument("--out", default=os.path.join(HERE, "recorder.npz"))
    args = ap.parse_args(argv)
    if not args.reference:
        ap.error("--reference (or BEAMZ_REFERENCE_ROOT) is required")
    os.environ["BEAMZ_REFERENCE_ROOT"] = args.reference
    from ._refload import load_reference

    ref = load_reference()
    jnp = ref.jnp
    rng = np.random.default_rng(61)
    shapes = {c: ref.lattice.component_shape_3d(c, GRID) for c in COMPONENTS}
    specs, buffers, data = [], [], {}
    for r, (name, comps, signs, interval, capacity, plane) in enumerate(RECORDERS):
        if plane:
            idx, w, shape = plane_plans(comps)
            field_shapes = (shape,) * len(comps)
        else:
            idx = [np.zeros(0, np.int32)] * len(comps)
            w = [np.zeros(0, np.float32)] * len(comps)
            field_shapes = tuple(shapes[c] for c in comps)
        start = sum(len(s.canonical_components) for s in specs)
        specs.append(types.SimpleNamespace(
            recorder_index=r, record_interval=interval, canonical_components=comps, component_signs=signs,
            field_buffer_indices=tuple(range(start, start + len(comps))), field_shapes=field_shapes,
            field_interp_flat_idx=tuple(jnp.asarray(i) for i in idx),
            field_interp_weights=tuple(jnp.asarray(x) for x in w)))
        for q, c in enumerate(comps):
            buffers.append(np.zeros((capacity, *field_shapes[q]), np.float32))
            if plane:
                data[f"{name}_idx_{c}"], data[f"{name}_w_{c}"] = idx[q], w[q]
    program = types.SimpleNamespace(monitors=tuple(specs))
    state = types.SimpleNamespace(
        recorded_fields=tuple(jnp.asarray(b) for b in buffers),
        recorded_steps=tuple(jnp.zeros(cap, dtype=np.int32) for *_, cap, _ in RECORDERS),
        recorded_times=tuple(jnp.zeros(cap, dtype=np.float32) for *_, cap, _ in RECORDERS),
        recorded_counts=tuple(jnp.zeros((), dtype=np.int32) for _ in RECORDERS))
    t = np.float32(0.0)
    dt = np.float32(3.1e-17)
    for step in range(STEPS):
        fields = {c: rng.standard_normal(shapes[c]).astype(np.float32) for c in COMPONENTS}
        for c, v in fields.items():
            data[f"step{step}_{c}"] = v
        t = np.float32(t + dt)
        update = ref.observe._record_fields(program, state, jnp.asarray(step, dtype=np.int32), t,
                                            {c: jnp.asarray(v) for c, v in fields.items()})
        state = types.SimpleNamespace(**update)
        data[f"step{step}_t"] = t
    k = 0
    for r, (name, comps, *_rest) in enumerate(RECORDERS):
        for c in comps:
            data[f"{name}_values_{c}"] = np.asarray(state.recorded_fields[k])
            k += 1
        data[f"{name}_steps"] = np.asarray(state.recorded_steps[r])
        data[f"{name}_times"] = np.asarray(state.recorded_times[r])
        data[f"{name}_count"] = np.asarray(state.recorded_counts[r])
    np.savez(args.out, **data)
    print(f"wrote {args.out}: {len(data)} arrays")


if __name__ == "__main__":
    main()
