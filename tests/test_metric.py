"""Derivative metrics of axis-uniform and rectilinear grids: the planner and
the oracle against the reference's own functions (``tests/golden/metric.npz``
from ``tests/golden/make_metric.py``), and the C-ABI's checks of the metric
buffers.

beamz scales each staggered difference by a per-axis inverse distance when the
grid is not isotropic (beamz/simulation/compile.py:209-239,
kernels.py:164-176, 293-455, 506-701, 880-1012); the isotropic step divides by
the cell size instead, so the two forms round differently even on equal
widths."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from beamz_b200 import abi
from beamz_b200 import plan as P
from oracle import fdtd_oracle as O
from tests.golden_io import load, terms3d, terms_from

RTOL = 2e-6


def _widths(d, tag, axes):
    return {a: d[f"{tag}_w{a}"] for a in axes}


def _metrics(d, tag):
    return {n: d[f"{tag}_{n}"] for n in P.METRIC_NAMES}


@pytest.mark.parametrize("kind", ["axis_uniform", "rectilinear"])
@pytest.mark.parametrize("tag,axes", [("m3", "zyx"), ("m2", "yx")])
def test_derivative_metrics_match_the_reference(tag, axes, kind):
    d = load("metric")
    got = P.derivative_metrics(_widths(d, f"{tag}_{kind}", axes), kind)
    for name in P.METRIC_NAMES:
        want = d[f"{tag}_{kind}_{name}"]
        have = np.asarray(getattr(got, name))
        assert have.dtype == np.float32 and have.shape == want.shape, name
        np.testing.assert_array_equal(have, want, err_msg=name)


def test_isotropic_grid_has_no_metrics_and_scalars_expand():
    assert P.derivative_metrics({"x": np.ones(3)}, "isotropic_uniform") is None
    m = P.derivative_metrics({"x": np.full(4, 2e-8), "y": np.full(3, 4e-8)}, "axis_uniform")
    np.testing.assert_array_equal(m.along("e_to_h_x", 4), np.full(4, np.float32(5e7)))
    np.testing.assert_array_equal(m.along("h_to_e_y", 4), np.full(4, np.float32(2.5e7)))
    r = P.derivative_metrics({"x": np.array([1e-8, 2e-8])}, "rectilinear")
    with pytest.raises(ValueError):
        r.along("h_to_e_x", 2)  # three backward distances for two cells
    with pytest.raises(ValueError):
        P.derivative_metrics({"x": np.array([1e-8, 0.0])}, "rectilinear")


def test_oracle_metric_3d_updates_match_the_reference():
    d = load("metric")
    grid = tuple(int(v) for v in d["grid"])
    h_terms, e_terms, _ = terms3d(d, grid)
    metrics = _metrics(d, "u3")
    f = {c: d[f"in_{c}"].copy() for c in O.COMPONENTS}
    dt, res = float(d["dt"]), float(d["res"])
    psi_h = [d[f"in_psi_h{i}"].copy() for i in range(6)]
    hx, hy, hz, ph = O.update_h_3d(f, psi_h, h_terms, dt, res, metrics=metrics)
    for name, v in (("Hx", hx), ("Hy", hy), ("Hz", hz)):
        np.testing.assert_allclose(v, d[f"cpml_{name}"], rtol=RTOL, atol=1e-9)
    for i in range(6):
        np.testing.assert_allclose(ph[i], d[f"cpml_psi_h{i}"], rtol=RTOL, atol=1e-9)
    mat = O.material_from_voxels(d["voxels"])
    for tag, metallic in (("open", set()), ("pec", {"back", "bottom", "right"})):
        psi_e = [d[f"in_psi_e{i}"].copy() for i in range(6)]
        ex, ey, ez, pe = O.update_e_3d(f, psi_e, e_terms, dt, res, mat, metallic, metrics=metrics)
        for name, v in (("Ex", ex), ("Ey", ey), ("Ez", ez)):
            np.testing.assert_allclose(v, d[f"cpml_{tag}_{name}"], rtol=RTOL, atol=1e-6)
        for i in range(6):
            np.testing.assert_allclose(pe[i], d[f"cpml_{tag}_psi_e{i}"], rtol=RTOL, atol=1e-6)
    hx, hy, hz, _ = O.update_h_3d(f, [], [], dt, res, metrics=metrics)
    for name, v in (("Hx", hx), ("Hy", hy), ("Hz", hz)):
        np.testing.assert_allclose(v, d[f"yee_{name}"], rtol=RTOL, atol=1e-9)
    ex, ey, ez, _ = O.update_e_3d(f, [], [], dt, res, mat, {"front", "top", "left"}, metrics=metrics)
    for name, v in (("Ex", ex), ("Ey", ey), ("Ez", ez)):
        np.testing.assert_allclose(v, d[f"yee_{name}"], rtol=RTOL, atol=1e-6)
    # The metric form differs from the isotropic one (which ignores the widths).
    iso, _, _, _ = O.update_h_3d(f, [], [], dt, res)
    assert not np.allclose(iso, d["yee_Hx"], rtol=1e-3)


@pytest.mark.parametrize("pol", ["tm", "te"])
def test_oracle_metric_2d_curls_match_the_reference(pol):
    d = load("metric")
    grid = tuple(int(v) for v in d["grid2"])
    res = float(d["res"])
    metrics = _metrics(d, "u2")
    (hspec, espec) = O.CPML_2D_TERMS[pol]
    shapes = O.component_shapes(grid, pol)
    h_terms = terms_from(d, f"{pol}h", [c for c, _, _ in hspec], [shapes[c][ax] for c, ax, _ in hspec])
    e_terms = terms_from(d, f"{pol}e", [c for c, _, _ in espec], [shapes[c][ax] for c, ax, _ in espec])
    comps = ("Ez", "Hx", "Hy") if pol == "tm" else ("Ex", "Ey", "Hz")
    f = {c: np.zeros((1, 1), np.float32) for c in O.COMPONENTS}
    f.update({c: d[f"{pol}_in_{c}"].copy() for c in comps})
    psi_h = [d[f"{pol}_in_psi_h{i}"].copy() for i in range(2)]
    psi_e = [d[f"{pol}_in_psi_e{i}"].copy() for i in range(2)]
    one = np.float32(1.0)
    zero_e = dict(f)
    for c in ("Ex", "Ey", "Ez"):
        zero_e[c] = np.zeros_like(f[c])
    unit = {c: (one, one) for c in ("Ex", "Ey", "Ez")}
    metallic = {"left", "top"}
    # Unit coefficients expose the curls: H_new = H - curl, E_new = 0 + curl.
    hnew, ph = O.update_h_2d(f, psi_h, h_terms, res, (one, one), pol, metrics)
    enew, pe = O.update_e_2d(zero_e, psi_e, e_terms, res, unit, metallic, pol, metrics)
    plain_h, _ = O.update_h_2d(f, [], [], res, (one, one), pol, metrics)
    plain_e, _ = O.update_e_2d(zero_e, [], [], res, unit, metallic, pol, metrics)
    if pol == "tm":
        np.testing.assert_allclose(f["Hx"] - hnew["Hx"], d["tm_curl_h0"], rtol=1e-5, atol=1e-3)
        np.testing.assert_allclose(f["Hy"] - hnew["Hy"], d["tm_curl_h1"], rtol=1e-5, atol=1e-3)
        np.testing.assert_allclose(enew["Ez"], d["tm_curl_e"], rtol=RTOL, atol=1e-6)
        np.testing.assert_allclose(f["Hx"] - plain_h["Hx"], d["tm_plain_curl_h0"], rtol=1e-5, atol=1e-3)
        np.testing.assert_allclose(f["Hy"] - plain_h["Hy"], d["tm_plain_curl_h1"], rtol=1e-5, atol=1e-3)
        np.testing.assert_allclose(plain_e["Ez"], d["tm_plain_curl_e"], rtol=RTOL, atol=1e-6)
    else:
        np.testing.assert_allclose(f["Hz"] - hnew["Hz"], d["te_curl_h"], rtol=1e-5, atol=1e-3)
        np.testing.assert_allclose(enew["Ex"], d["te_curl_e0"], rtol=RTOL, atol=1e-6)
        np.testing.assert_allclose(enew["Ey"], d["te_curl_e1"], rtol=RTOL, atol=1e-6)
        np.testing.assert_allclose(f["Hz"] - plain_h["Hz"], d["te_plain_curl_h"], rtol=1e-5, atol=1e-3)
        np.testing.assert_allclose(plain_e["Ex"], d["te_plain_curl_e0"], rtol=RTOL, atol=1e-6)
        np.testing.assert_allclose(plain_e["Ey"], d["te_plain_curl_e1"], rtol=RTOL, atol=1e-6)
    for i in range(2):
        np.testing.assert_allclose(ph[i], d[f"{pol}_psi_h{i}"], rtol=RTOL, atol=1e-6)
        np.testing.assert_allclose(pe[i], d[f"{pol}_psi_e{i}"], rtol=RTOL, atol=1e-6)


# ---- C-ABI checks of the metric buffers (no device work) -------------------


@pytest.fixture(scope="module")
def lib():
    return abi.load_library()


def _with_metrics(ndim=3):
    from tests.test_abi import _fake, _valid_program

    s = _valid_program()
    cells = (4, 5, 6)
    for a, n in enumerate(cells):
        s.metric_h[a] = _fake((n,))
        s.metric_e[a] = _fake((n + 1,))
    return s, _fake


def test_validate_accepts_metric_buffers(lib):
    s, _ = _with_metrics()
    assert lib.fdtd_validate(ctypes.byref(s)) == 0


@pytest.mark.parametrize("mutate", [
    lambda s, fk: s.metric_h.__setitem__(1, fk((6,))),          # y has 5 cells
    lambda s, fk: s.metric_e.__setitem__(2, fk((6,))),          # x needs 7 backward values
    lambda s, fk: s.metric_e.__setitem__(0, fk((5,), abi.FDTD_S32)),
    lambda s, fk: s.metric_h.__setitem__(0, abi.FdtdBuffer()),  # one axis missing
    lambda s, fk: s.metric_e.__setitem__(1, fk((2, 3))),
])
def test_validate_rejects_inconsistent_metric_buffers(lib, mutate):
    s, fk = _with_metrics()
    mutate(s, fk)
    assert lib.fdtd_validate(ctypes.byref(s)) == 1
