"""Golden inputs for the beamz adapter, built by the reference's own compile steps.

Run from the repository root, in a container that has the beamz source tree:

    python -m tests.golden.make_adapter --reference /path/to/beamz

Everything below runs the reference's code under the numpy stand-in for
``jax.numpy`` (``_jaxshim.py``); functions of modules that import the whole
framework are executed from their own source text (parsed with ``ast``):

* CPML terms: ``beamz/simulation/kernels.py`` ``compile_cpml_term`` with the
  profiles of ``beamz/devices/_boundary_compile.py`` (``make_golden._terms_3d``);
* update coefficients as beamz compiles them for its CUDA backend
  (``beamz/simulation/compile.py:563-660``): ``precompute_h_update_coefficients``
  and ``precompute_e_update_coefficients`` (kernels.py:704-728) on the E-site
  permittivities of ``lattice.sample_voxel_grid_at_e_component_3d_centered``
  (lattice.py:732-786), then compile.py's ``_elide_uniform_grid`` (137-143),
  ``_pack_cuda_coefficient_ids`` and ``_pack_cuda_lossless_e_coefficients``
  (146-187);
* source groups: ``beamz/devices/sources/compiler.py``'s ``BatchedSlabGroup``,
  ``CompiledSourceSpec`` and ``batch_slab_specs`` (52-129), grouped per
  (timing, component) as ``execute.compiled_source_batches`` does
  (execute.py:48-52, 355-371);
* packed monitors: ``beamz/simulation/cuda/runtime.py``'s
  ``pack_dft_monitors`` (530-618) on monitor plans from
  ``lattice._component_plane_plan_3d``.

Writes ``tests/golden/adapter.npz``: the pieces beamz hands its native
program entry (``ctx``, ``coeffs``, ``groups``, ``packed_monitors``) as plain
arrays, plus the per-site E sources before packing.
"""

from __future__ import annotations

import __future__
import argparse
import ast
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

COEFF_FIELDS = ("h_decay_x", "h_source_x", "h_decay_y", "h_source_y", "h_decay_z", "h_source_z",
                "e_decay_x", "e_source_x", "e_decay_y", "e_source_y", "e_decay_z", "e_source_z")
GROUP_ORDER = (("pre_e", "Ex"), ("pre_e", "Ey"), ("pre_e", "Ez"), ("h", "Hx"), ("h", "Hy"), ("h", "Hz"),
               ("e", "Ex"), ("e", "Ey"), ("e", "Ez"))


def exec_subset(root: str, relpath: str, names, extra: dict) -> dict:
    """Execute the named top-level functions / classes of one reference file."""
    path = os.path.join(root, relpath)
    tree = ast.parse(open(path).read(), filename=path)
    keep = [n for n in tree.body if isinstance(n, (ast.FunctionDef, ast.ClassDef)) and n.name in names]
    missing = set(names) - {n.name for n in keep}
    if missing:
        raise RuntimeError(f"{relpath}: {sorted(missing)} not found")
    code = compile(ast.Module(body=keep, type_ignores=[]), path, "exec",
                   flags=__future__.annotations.compiler_flag, dont_inherit=True)
    module = types.ModuleType("beamz_subset_" + os.path.basename(relpath)[:-3])
    module.__dict__.update(extra)
    sys.modules[module.__name__] = module  # dataclasses look their module up
    exec(code, module.__dict__)
    return module.__dict__


def build(root: str) -> dict:
    from dataclasses import dataclass
    from typing import Any

    from . import _jaxshim
    from ._refload import load_reference
    from .make_golden import _monitor_ns, _terms_3d

    os.environ["BEAMZ_REFERENCE_ROOT"] = root
    ref = load_reference()
    _jaxshim.install()
    jnp = sys.modules["jax.numpy"]
    base = {"np": np, "jnp": jnp, "dataclass": dataclass, "Any": Any}
    comp = exec_subset(root, "beamz/simulation/compile.py",
                       ("_elide_uniform_grid", "_pack_cuda_coefficient_ids", "_pack_cuda_lossless_e_coefficients"),
                       base)
    src = exec_subset(root, "beamz/devices/sources/compiler.py",
                      ("BatchedSlabGroup", "CompiledSourceSpec", "batch_slab_specs"), base)
    run = exec_subset(root, "beamz/simulation/cuda/runtime.py", ("pack_dft_monitors",), base)

    rng = np.random.default_rng(11)
    grid = (8, 18, 140)
    res = 20e-9
    dt = 0.99 * res / (299792458.0 * np.sqrt(3.0))
    edges = {"back", "bottom", "top", "left", "right"}  # CPML faces; PEC on the front face
    metallic = ("front",)
    h_terms, e_terms, shapes = _terms_3d(ref, grid, dt, res, 4, edges)
    vox = np.full(grid, 2.085, np.float32)
    vox[2:6, 5:12, 20:90] = 12.11
    vox[1:3, 2:9, 100:130] = 4.0

    # Update coefficients of beamz's CUDA path.
    sigma0 = np.zeros((1, 1, 1), np.float32)
    h = [ref.kernels.precompute_h_update_coefficients(jnp.asarray(sigma0), dt) for _ in range(3)]
    e = []
    for c in ("Ex", "Ey", "Ez"):
        eps = np.asarray(ref.lattice.sample_voxel_grid_at_e_component_3d_centered(vox, c), np.float32)
        region = tuple(slice(0, n) for n in shapes[c])
        e.append(ref.kernels.precompute_e_update_coefficients(shapes[c], jnp.zeros(shapes[c], np.float32),
                                                              jnp.asarray(eps), dt, region))
    elide = comp["_elide_uniform_grid"]
    coeffs = {}
    for tag, (d, s) in zip("xyz", h):
        coeffs[f"h_decay_{tag}"], coeffs[f"h_source_{tag}"] = np.asarray(elide(d)), np.asarray(elide(s))
    e_dec = tuple(elide(d) for d, _ in e)
    e_src = tuple(np.asarray(s) for _, s in e)
    packed = comp["_pack_cuda_lossless_e_coefficients"](e_dec, e_src)
    if packed is None:
        raise RuntimeError("the scene's E material did not pack")
    tables, ids = packed
    for tag, t, i in zip("xyz", tables, ids):
        coeffs[f"e_decay_{tag}"], coeffs[f"e_source_{tag}"] = np.asarray(t), np.asarray(i)

    # Sources: CompiledSourceSpec slabs, batched per (timing, component).
    nsteps = 24
    f0 = 299792458.0 / 1.55e-6
    pulse = ref.time.GaussianPulse(freq0=f0, fwidth=0.5 * f0, offset=0.3)
    wave = np.asarray(pulse.sample((np.arange(nsteps) + 0.5) * dt)[0], np.float32)
    CSS = src["CompiledSourceSpec"]

    def slab(component, timing, start, coeff, waveform):
        coeff = np.asarray(coeff, np.float32)
        index = tuple(slice(s, s + n) for s, n in zip(start, coeff.shape))
        return CSS(component=component, timing=timing, index=index, coeff=jnp.asarray(coeff),
                   waveform=jnp.asarray(np.asarray(waveform, np.float32)), is_slab=True,
                   slab_starts=tuple(start), slab_sizes=tuple(coeff.shape))

    specs = (
        slab("Ey", "pre_e", (4, 9, 60), [[[-dt / (8.8541878128e-12 * 12.11)]]], wave),
        slab("Ey", "pre_e", (5, 10, 61), [[[-0.5 * dt / (8.8541878128e-12 * 12.11)]]], 0.5 * wave),
        slab("Hz", "h", (2, 3, 30), rng.standard_normal((1, 2, 3)), rng.standard_normal(nsteps) * 1e-3),
        slab("Ex", "e", (0, 1, 110), rng.standard_normal((grid[0] + 1, 1, 2)), rng.standard_normal(nsteps) * 1e-2),
    )
    data = {}
    for g, (timing, component) in enumerate(GROUP_ORDER):
        group, rest = src["batch_slab_specs"](tuple(s for s in specs if s.timing == timing and s.component == component))
        if rest:
            raise RuntimeError("every source must batch")
        if group is not None:
            data[f"g{g}_coeffs"] = np.asarray(group.coeffs, np.float32)
            data[f"g{g}_waves"] = np.asarray(group.waveforms, np.float32)
            data[f"g{g}_starts"] = np.asarray(group.starts, np.int32)

    # Monitors: an x-normal plane (Ey, Ez, Hy, Hz) and a z-normal plane (Ex, Ey, Hx, Hy).
    mons = []
    voff = woff = 0
    for normal, pos, comps, coords, freqs, window, norm in (
            ("x", 70.25 * res, ("Ey", "Ez", "Hy", "Hz"), ((np.arange(5) + 1.5) * res, (np.arange(12) + 3.25) * res),
             [0.9 * f0, f0, 1.1 * f0], 0, 0),
            ("z", 3.5 * res, ("Ex", "Ey", "Hx", "Hy"), ((np.arange(10) + 4.5) * res, (np.arange(40) + 40.25) * res),
             [f0, 1.2 * f0], 1, 1)):
        idx, w = [], []
        for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            fi, fw = ref.lattice._component_plane_plan_3d(c, normal_axis=normal, plane_position=pos,
                                                        coordinates=coords, resolution=res, grid_shape=grid,
                                                        field_shape=shapes[c])
            idx.append(np.asarray(fi))
            w.append(np.asarray(fw))
        k = max(a.shape[1] for a in idx)
        idx = [np.pad(a, ((0, 0), (0, k - a.shape[1]))) for a in idx]
        w = [np.pad(a, ((0, 0), (0, k - a.shape[1]))) for a in w]
        npt = idx[0].shape[0]
        mask = np.asarray([1.0 if c in comps else 0.0 for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")], np.float32)
        t0, t1 = (0.0, float("inf")) if window == 0 else (2 * dt, (nsteps - 2) * dt)
        mons.append(_monitor_ns(ref, freqs, idx, w, mask, t0, t1, 1, window, norm, 1e-6, voff, woff, npt))
        voff += 6 * len(freqs) * npt
        woff += len(freqs)
    pk = run["pack_dft_monitors"](tuple(mons))
    for name, value in zip(("indices", "weights", "freqs", "masks", "counts", "codes", "windows"), pk):
        data[f"pk_{name}"] = np.asarray(value)

    for i, t in enumerate(h_terms):
        data[f"h{i}_a"], data[f"h{i}_b"], data[f"h{i}_k"] = (np.asarray(v) for v in (t.a, t.b, t.inv_kappa))
        data[f"h{i}_meta"] = np.asarray([t.axis, t.slab.low, t.slab.high, int(t.sign)], np.int32)
        data[f"h{i}_shape"] = np.asarray(t.slab.shape, np.int64)
    for i, t in enumerate(e_terms):
        data[f"e{i}_a"], data[f"e{i}_b"], data[f"e{i}_k"] = (np.asarray(v) for v in (t.a, t.b, t.inv_kappa))
        data[f"e{i}_meta"] = np.asarray([t.axis, t.slab.low, t.slab.high, int(t.sign)], np.int32)
        data[f"e{i}_shape"] = np.asarray(t.slab.shape, np.int64)
    data.update({f"coef_{k}": v for k, v in coeffs.items()})
    data.update({f"src_{c}": s for c, s in zip(("Ex", "Ey", "Ez"), e_src)})
    data.update(grid=np.asarray(grid), dt=np.float64(dt), res=np.float64(res), nsteps=np.int32(nsteps),
                metallic=np.asarray(metallic), voxels=vox)
    return data


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("BEAMZ_REFERENCE_ROOT"),
                        help="root of the beamz source tree (or set BEAMZ_REFERENCE_ROOT)")
    args = parser.parse_args()
    if not args.reference:
        parser.error("--reference (or BEAMZ_REFERENCE_ROOT) is required")
    data = build(args.reference)
    out = os.path.join(HERE, "adapter.npz")
    np.savez_compressed(out, **data)
    print(out, sorted(data))


if __name__ == "__main__":
    main()
