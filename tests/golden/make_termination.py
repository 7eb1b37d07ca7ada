"""Golden vectors for automatic termination, from the reference's own code.

Run from the repository root, in a container that has the beamz source tree:

    python -m tests.golden.make_termination [--reference /path/to/beamz]

``beamz/simulation/execute.py`` imports the whole framework at module load, so
this script parses it and executes only the functions below, each from its own
source text, in a namespace holding numpy and the numpy stand-in for
``jax.numpy`` (``_jaxshim.py``, JAX's x64-disabled dtype policy):

* ``_COMPONENT_OFFSETS_2D`` (66-73) and ``_axis_integration_weights`` (77-93);
* ``_field_diagnostics`` (184-222), fed the plan ``_energy_terms`` (127-181)
  builds for scalar materials: per component (name, site material,
  integration weights / domain measure, eps0 or mu0);
* ``_remaining_source_activity`` (225-243) and ``_source_residual`` (246-251);
* ``_relative_monitor_change`` (292-316);
* ``_configured_dft_weight_sum`` (319-336).

3D component offsets come from ``beamz/lattice.py:14-21`` through the
reference loader.  Writes ``tests/golden/termination.npz``.
"""

from __future__ import annotations

import __future__
import argparse
import ast
import os
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ("_axis_integration_weights", "_field_diagnostics", "_remaining_source_activity", "_source_residual",
         "_relative_monitor_change", "_configured_dft_weight_sum")


def load_functions(root: str) -> dict:
    from . import _jaxshim
    from ._refload import load_reference

    os.environ["BEAMZ_REFERENCE_ROOT"] = root
    ref = load_reference()
    _jaxshim.install()
    import sys

    path = os.path.join(root, "beamz/simulation/execute.py")
    tree = ast.parse(open(path).read(), filename=path)
    keep = [n for n in tree.body
            if (isinstance(n, ast.FunctionDef) and n.name in NAMES)
            or (isinstance(n, ast.Assign) and any(getattr(t, "id", "") == "_COMPONENT_OFFSETS_2D" for t in n.targets))]
    module = ast.Module(body=keep, type_ignores=[])
    code = compile(module, path, "exec", flags=__future__.annotations.compiler_flag, dont_inherit=True)
    ns = {"np": np, "jnp": sys.modules["jax.numpy"], "__name__": "beamz_execute_subset"}
    exec(code, ns)
    ns["lattice"] = ref.lattice
    return ns


def _weights(fns, shape, offsets, res):
    """Physical control volumes of one component (execute.py:95-111 on a uniform grid)."""
    axes = []
    for count, off in zip(shape, offsets):
        cells = count - 1 if off == 0.0 else count
        axes.append(fns["_axis_integration_weights"](np.arange(cells + 1) * res, off, count))
    w = axes[0]
    for a in axes[1:]:
        w = np.multiply.outer(w, a)
    return w


def diagnostics_case(fns, rng, grid, polarization, res, nan=False):
    """Seeded fields and site permittivities, and the reference's result."""
    jnp = fns["jnp"]
    eps0, mu0 = 8.8541878128e-12, 1.25663706212e-6
    if len(grid) == 3:
        comps = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
        offsets = {c: tuple(fns["lattice"].component_axis_offsets_3d(c)[a] for a in "zyx") for c in comps}
    else:
        comps = ("Ez", "Hx", "Hy") if polarization == "tm" else ("Ex", "Ey", "Hz")
        offsets = {c: fns["_COMPONENT_OFFSETS_2D"][c] for c in comps}
    shapes = {c: tuple(n + (1 if off == 0.0 else 0) for n, off in zip(grid, offsets[c])) for c in comps}
    extent = [n * res for n in grid]
    domain = float(extent[0] * extent[1] * (extent[2] if len(grid) == 3 else 1.0))
    fields, mats, terms = {}, {}, []
    for c in comps:
        v = (rng.standard_normal(shapes[c]) * (1e3 if c[0] == "E" else 2.0)).astype(np.float32)
        if nan and c == comps[-1]:
            v.reshape(-1)[7] = np.nan
        fields[c] = v
        m = (rng.uniform(1.0, 12.0, shapes[c]).astype(np.float32) if c[0] == "E"
             else np.ones(shapes[c], np.float32))
        mats[c] = m
        w = _weights(fns, shapes[c], offsets[c], res)
        terms.append((c.lower(), jnp.asarray(m), jnp.asarray(w) / domain, eps0 if c[0] == "E" else mu0))
    state = types.SimpleNamespace(**{c.lower(): fields[c] for c in comps})
    energy, max_field, finite = fns["_field_diagnostics"](state, (tuple(terms), (), domain))
    return fields, mats, (energy, max_field, finite)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("BEAMZ_REFERENCE_ROOT"),
                    help="root of the beamz source tree (or set BEAMZ_REFERENCE_ROOT)")
    ap.add_argument("--out", default=os.path.join(HERE, "termination.npz"))
    args = ap.parse_args(argv)
    if not args.reference:
        ap.error("--reference (or BEAMZ_REFERENCE_ROOT) is required")
    fns = load_functions(args.reference)
    rng = np.random.default_rng(2024)
    out = {}
    res = 20e-9
    for n, off in ((1, 0.0), (1, 0.5), (5, 0.0), (5, 0.5), (8, 0.0)):
        edges = np.arange(n + 1) * res
        count = n + 1 if off == 0.0 else n
        out[f"axisw_{n}_{off}"] = fns["_axis_integration_weights"](edges, off, count)
    cases = {"3d": ((4, 5, 6), "tm", False), "3d_nan": ((3, 4, 5), "tm", True), "tm": ((6, 7), "tm", False),
             "te": ((6, 7), "te", False)}
    for name, (grid, pol, nan) in cases.items():
        fields, mats, (energy, max_field, finite) = diagnostics_case(fns, rng, grid, pol, res, nan)
        for c, v in fields.items():
            out[f"diag_{name}_field_{c}"] = v
            out[f"diag_{name}_eps_{c}"] = mats[c]
        out[f"diag_{name}_result"] = np.array([energy, max_field, float(finite)], np.float64)
        out[f"diag_{name}_grid"] = np.array(grid)
    waves = [rng.standard_normal(40).astype(np.float32), np.r_[np.hanning(20), np.zeros(5)].astype(np.float32),
             np.zeros(10, np.float32), np.r_[np.ones(5), 0.25 * np.ones(3)].astype(np.float32)]
    program = types.SimpleNamespace(sources=tuple(types.SimpleNamespace(waveform=w) for w in waves))
    activity = fns["_remaining_source_activity"](program, 60)
    for i, w in enumerate(waves):
        out[f"src_wave_{i}"] = w
    out["src_activity"] = activity
    out["src_residual"] = np.array([fns["_source_residual"](activity, s) for s in (0, 10, 30, 59, 60, 75)])
    cur = {("m", "Ez", f): (rng.standard_normal(9) + 1j * rng.standard_normal(9)) for f in range(3)}
    prev = {k: v * (1.0 + 0.01 * rng.standard_normal(9)) for k, v in cur.items()}
    cur[("m", "Hx", 0)] = np.zeros(4, complex)
    prev[("m", "Hx", 0)] = np.zeros(4, complex)
    for i, k in enumerate(sorted(cur)):
        out[f"mon_cur_{i}"] = cur[k]
        out[f"mon_prev_{i}"] = prev[k]
    out["mon_change"] = np.array([fns["_relative_monitor_change"](cur, prev)])
    sim = types.SimpleNamespace(num_steps=200, time=np.array([1e-15]), dt=3e-17)
    weight_cases = [(1, 0.0, np.inf, 0), (3, 2e-15, 5e-15, 0), (1, 1e-15, 6e-15, 1), (2, 0.0, 4e-15, 1),
                    (1, 9e-15, 1e-14, 1)]
    sums = []
    for interval, t0, t1, code in weight_cases:
        spec = types.SimpleNamespace(dft_record_interval=interval, dft_t_start=t0, dft_t_end=t1, dft_window_code=code)
        sums.append(fns["_configured_dft_weight_sum"](sim, spec))
    out["weight_cases"] = np.array(weight_cases, np.float64)
    out["weight_sums"] = np.array(sums)
    np.savez(args.out, **out)
    print(f"wrote {args.out}: {len(out)} arrays")


if __name__ == "__main__":
    main()
