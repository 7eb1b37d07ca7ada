"""Golden vectors for derivative metrics (axis-uniform and rectilinear grids),
from the reference's own code.

Run from the repository root, in a container that has the beamz source tree:

    python -m tests.golden.make_metric [--reference /path/to/beamz]

It evaluates, on seeded cell widths and fields:

* ``_compile_derivative_metrics`` (``beamz/simulation/compile.py:209-239``),
  executed from its own source text (the module imports the whole framework)
  with a stand-in material grid that carries ``metric_kind``, ``shape`` and
  ``grid.cell_widths``;
* the metric updates of ``beamz/simulation/kernels.py``:
  ``fused_update_h/e_lossy_3d_material_metric`` (293, 391),
  ``cpml_update_h_from_e_3d_metric`` (506), ``cpml_update_e_from_h_3d_metric``
  (629) and the 2D TM/TE metric curls (880-1012), loaded by path under the
  numpy stand-in for ``jax`` (``_refload.py``).

CPML terms are the uniform-grid ones of ``make_golden.py`` (the update only
reads their coefficient arrays).  Writes ``tests/golden/metric.npz``.
"""

from __future__ import annotations

import __future__
import argparse
import ast
import os
import types
from typing import NamedTuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class DerivativeMetricPlan(NamedTuple):
    """Field order of ``beamz/simulation/model.py:290-303``."""

    e_to_h_x: object
    e_to_h_y: object
    e_to_h_z: object
    h_to_e_x: object
    h_to_e_y: object
    h_to_e_z: object


def load_compile_metrics(root: str, jnp):
    path = os.path.join(root, "beamz/simulation/compile.py")
    tree = ast.parse(open(path).read(), filename=path)
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "_compile_derivative_metrics"]
    code = compile(ast.Module(body=keep, type_ignores=[]), path, "exec",
                   flags=__future__.annotations.compiler_flag, dont_inherit=True)
    ns = {"np": np, "jnp": jnp, "DerivativeMetricPlan": DerivativeMetricPlan, "__name__": "beamz_compile_subset"}
    exec(code, ns)
    return ns["_compile_derivative_metrics"]


def material_grid(kind: str, widths: dict):
    shape = tuple(len(widths[a]) for a in ("z", "y", "x") if a in widths)
    grid = types.SimpleNamespace(cell_widths=lambda axis: np.asarray(widths[axis], np.float64))
    return types.SimpleNamespace(metric_kind=kind, shape=shape, grid=grid)


def random_widths(rng, cells: dict, res: float, uniform: bool):
    out = {}
    for axis, n in cells.items():
        if uniform:
            out[axis] = np.full(n, res * float(rng.uniform(0.6, 1.4)))
        else:
            out[axis] = res * rng.uniform(0.55, 1.45, n)
    return out


def _save_metrics(data, prefix, plan):
    for name in DerivativeMetricPlan._fields:
        data[f"{prefix}_{name}"] = np.asarray(getattr(plan, name))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("BEAMZ_REFERENCE_ROOT"),
                    help="root of the beamz source tree (or set BEAMZ_REFERENCE_ROOT)")
    ap.add_argument("--out", default=os.path.join(HERE, "metric.npz"))
    args = ap.parse_args(argv)
    if not args.reference:
        ap.error("--reference (or BEAMZ_REFERENCE_ROOT) is required")
    os.environ["BEAMZ_REFERENCE_ROOT"] = args.reference
    from ._refload import load_reference
    from .make_golden import _random_fields, _term_arrays, _terms_2d, _terms_3d

    ref = load_reference()
    jnp = ref.jnp
    compile_metrics = load_compile_metrics(args.reference, jnp)
    rng = np.random.default_rng(4242)
    res = 20e-9
    data = {"res": np.float64(res)}

    # Metric plans: both kinds, 3D and 2D.
    for tag, cells in (("m3", {"z": 7, "y": 9, "x": 10}), ("m2", {"y": 12, "x": 14})):
        for kind in ("axis_uniform", "rectilinear"):
            widths = random_widths(rng, cells, res, kind == "axis_uniform")
            for axis, w in widths.items():
                data[f"{tag}_{kind}_w{axis}"] = w
            _save_metrics(data, f"{tag}_{kind}", compile_metrics(material_grid(kind, widths)))

    # 3D metric updates on a rectilinear plan.
    grid = (7, 9, 10)
    widths = random_widths(rng, {"z": 7, "y": 9, "x": 10}, res, False)
    plan = compile_metrics(material_grid("rectilinear", widths))
    for axis, w in widths.items():
        data[f"u3_w{axis}"] = w
    _save_metrics(data, "u3", plan)
    dt = 0.99 * 0.55 * res / (299792458.0 * np.sqrt(3.0))
    data.update(dt=np.float64(dt), grid=np.asarray(grid))
    h_terms, e_terms, shapes = _terms_3d(ref, grid, dt, res, 2, {"left", "right", "top", "bottom", "front", "back"})
    data.update(_term_arrays("h", h_terms))
    data.update(_term_arrays("e", e_terms))
    fields = _random_fields(rng, shapes)
    fields.update({c: fields[c] * np.float32(1.0 / 376.73) for c in ("Hx", "Hy", "Hz")})
    psi_h = [rng.standard_normal(tuple(t.slab.shape)).astype(np.float32) * np.float32(1e-3) for t in h_terms]
    psi_e = [rng.standard_normal(tuple(t.slab.shape)).astype(np.float32) * np.float32(1e-1) for t in e_terms]
    vox = rng.choice(np.asarray([2.085, 12.11], np.float32), size=grid).astype(np.float32)
    eps = [np.asarray(ref.lattice.sample_voxel_grid_at_e_component_3d_centered(vox, c)) for c in ("Ex", "Ey", "Ez")]
    data["voxels"] = vox
    data.update({f"in_{c}": v for c, v in fields.items()})
    data.update({f"in_psi_h{i}": p for i, p in enumerate(psi_h)})
    data.update({f"in_psi_e{i}": p for i, p in enumerate(psi_e)})
    jf = {c: jnp.asarray(v) for c, v in fields.items()}
    zero = jnp.asarray(np.float32(0.0))
    dt_s = jnp.asarray(dt, dtype=np.float32)
    inv = tuple(jnp.reciprocal(jnp.asarray(e)) for e in eps)
    hx, hy, hz, ph = ref.kernels.cpml_update_h_from_e_3d_metric(
        jf["Ex"], jf["Ey"], jf["Ez"], jf["Hx"], jf["Hy"], jf["Hz"], plan,
        terms=h_terms, psi_terms=[jnp.asarray(p) for p in psi_h], dt=dt_s, magnetic_conductivities=(zero, zero, zero))
    data.update(cpml_Hx=np.asarray(hx), cpml_Hy=np.asarray(hy), cpml_Hz=np.asarray(hz))
    data.update({f"cpml_psi_h{i}": np.asarray(p) for i, p in enumerate(ph)})
    for tag, metallic in (("open", frozenset()), ("pec", frozenset({"back", "bottom", "right"}))):
        ex, ey, ez, pe = ref.kernels.cpml_update_e_from_h_3d_metric(
            jf["Hx"], jf["Hy"], jf["Hz"], jf["Ex"], jf["Ey"], jf["Ez"], plan,
            terms=e_terms, psi_terms=[jnp.asarray(p) for p in psi_e], metallic_edges=metallic, dt=dt_s,
            conductivities=(zero, zero, zero), inverse_permittivities=inv)
        data.update({f"cpml_{tag}_Ex": np.asarray(ex), f"cpml_{tag}_Ey": np.asarray(ey),
                     f"cpml_{tag}_Ez": np.asarray(ez)})
        data.update({f"cpml_{tag}_psi_e{i}": np.asarray(p) for i, p in enumerate(pe)})
    metallic = frozenset({"front", "top", "left"})
    hx, hy, hz = ref.kernels.fused_update_h_lossy_3d_material_metric(
        jf["Ex"], jf["Ey"], jf["Ez"], jf["Hx"], jf["Hy"], jf["Hz"], zero, zero, zero, dt_s, plan)
    views = ref.lattice.build_h_boundary_views_for_e_3d(jf["Hx"], jf["Hy"], jf["Hz"], metallic)
    ex, ey, ez = ref.kernels.fused_update_e_lossy_3d_material_metric(
        jf["Hx"], jf["Hy"], jf["Hz"], jf["Ex"], jf["Ey"], jf["Ez"],
        zero, inv[0], zero, inv[1], zero, inv[2], dt_s, plan, boundary_views=views)
    data.update(yee_Hx=np.asarray(hx), yee_Hy=np.asarray(hy), yee_Hz=np.asarray(hz),
                yee_Ex=np.asarray(ex), yee_Ey=np.asarray(ey), yee_Ez=np.asarray(ez))

    # 2D metric curls (TM and TE) on a rectilinear plan.
    grid2 = (12, 14)
    widths2 = random_widths(rng, {"y": 12, "x": 14}, res, False)
    plan2 = compile_metrics(material_grid("rectilinear", widths2))
    for axis, w in widths2.items():
        data[f"u2_w{axis}"] = w
    _save_metrics(data, "u2", plan2)
    dt2 = 0.7 * 0.55 * res / (299792458.0 * np.sqrt(2.0))
    data.update(dt2=np.float64(dt2), grid2=np.asarray(grid2))
    for pol in ("tm", "te"):
        h_t, e_t = _terms_2d(ref, grid2, dt2, res, 3, pol)
        data.update(_term_arrays(f"{pol}h", h_t))
        data.update(_term_arrays(f"{pol}e", e_t))
        comps = ("Ez", "Hx", "Hy") if pol == "tm" else ("Ex", "Ey", "Hz")
        f = {c: rng.standard_normal(ref.lattice.component_shape_2d(c, grid2, "xy", pol)).astype(np.float32)
             for c in comps}
        p_h = [rng.standard_normal(tuple(t.slab.shape)).astype(np.float32) * np.float32(1e-2) for t in h_t]
        p_e = [rng.standard_normal(tuple(t.slab.shape)).astype(np.float32) * np.float32(1e-2) for t in e_t]
        data.update({f"{pol}_in_{c}": v for c, v in f.items()})
        data.update({f"{pol}_in_psi_h{i}": p for i, p in enumerate(p_h)})
        data.update({f"{pol}_in_psi_e{i}": p for i, p in enumerate(p_e)})
        jf2 = {c: jnp.asarray(v) for c, v in f.items()}
        metal = frozenset({"left", "top"})
        if pol == "tm":
            c0, c1, ph2 = ref.kernels.tm_xy_cpml_curl_e_to_h_2d_metric(
                jf2["Ez"], plan2, terms=h_t, psi_h_terms=[jnp.asarray(p) for p in p_h])
            ce, pe2 = ref.kernels.tm_xy_cpml_curl_h_to_e_2d_metric(
                jf2["Hx"], jf2["Hy"], plan2, jf2["Ez"].shape, metal, terms=e_t,
                psi_e_terms=[jnp.asarray(p) for p in p_e])
            data.update(tm_curl_h0=np.asarray(c0), tm_curl_h1=np.asarray(c1), tm_curl_e=np.asarray(ce))
            p0, p1 = ref.kernels.tm_xy_curl_e_to_h_2d_metric(jf2["Ez"], plan2)
            data.update(tm_plain_curl_h0=np.asarray(p0), tm_plain_curl_h1=np.asarray(p1))
            data["tm_plain_curl_e"] = np.asarray(
                ref.kernels.tm_xy_curl_h_to_e_2d_metric(jf2["Hx"], jf2["Hy"], plan2, jf2["Ez"].shape, metal))
        else:
            ch, ph2 = ref.kernels.te_xy_cpml_curl_e_to_h_2d_metric(
                jf2["Ex"], jf2["Ey"], plan2, terms=h_t, psi_h_terms=[jnp.asarray(p) for p in p_h])
            (ce0, ce1), pe2 = ref.kernels.te_xy_cpml_curl_h_to_e_2d_metric(
                jf2["Hz"], plan2, metal, terms=e_t, psi_e_terms=[jnp.asarray(p) for p in p_e])
            data.update(te_curl_h=np.asarray(ch), te_curl_e0=np.asarray(ce0), te_curl_e1=np.asarray(ce1))
            data["te_plain_curl_h"] = np.asarray(
                ref.kernels.te_xy_curl_e_to_h_2d_metric(jf2["Ex"], jf2["Ey"], plan2, jf2["Hz"].shape))
            q0, q1 = ref.kernels.te_xy_curl_h_to_e_2d_metric(jf2["Hz"], plan2, jf2["Ex"].shape, jf2["Ey"].shape,
                                                             metal)
            data.update(te_plain_curl_e0=np.asarray(q0), te_plain_curl_e1=np.asarray(q1))
        data.update({f"{pol}_psi_h{i}": np.asarray(p) for i, p in enumerate(ph2)})
        data.update({f"{pol}_psi_e{i}": np.asarray(p) for i, p in enumerate(pe2)})
    np.savez(args.out, **data)
    print(f"wrote {args.out}: {len(data)} arrays")


if __name__ == "__main__":
    main()
