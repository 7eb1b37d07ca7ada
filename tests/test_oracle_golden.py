"""Pin the CPU oracle to golden vectors produced by the reference's own code.

The fixtures under ``tests/golden`` come from ``tests/golden/make_golden.py``,
which executes beamz's source files (kernels.py, lattice.py,
_boundary_compile.py, observe.py, time.py) on seeded inputs.  Every oracle
function used as a checker for the CUDA path is compared here.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import fdtd_oracle as O
from tests.golden_io import E3, H3, load, terms3d, terms_from

# Same-order float32 restatements agree to a few ulps; exp/pow/cos may differ
# by an ulp between numpy builds.
RTOL = 2e-6
ATOL = 1e-7


def test_cpml_coefficients_match_reference():
    d = load("coefficients")
    a, b, k = O.cpml_coefficients(d["sigma"], d["kappa"], d["alpha"], float(d["dt"]))
    np.testing.assert_allclose(a, d["a"], rtol=RTOL, atol=1e-9)
    np.testing.assert_allclose(b, d["b"], rtol=RTOL, atol=ATOL)
    np.testing.assert_array_equal(k, d["k"])


def test_staggered_profiles_match_reference():
    d = load("coefficients")
    assert abs(O.cpml_sigma_max(12, float(d["prof_res"])) - float(d["prof_sigma_max"])) <= 1e-12 * float(d["prof_sigma_max"])
    assert abs(O.cpml_alpha_max(float(d["prof_dt"]), True) - float(d["prof_alpha_max"])) <= 1e-12 * float(d["prof_alpha_max"])
    for kind, n in (("E", 41), ("H", 40)):
        for tag, low in (("", True), ("hi", False)):
            s, k, a = O.staggered_profile_1d(n, 12, low, True, kind, float(d["prof_sigma_max"]),
                                             float(d["prof_alpha_max"]))
            np.testing.assert_allclose(s, d[f"prof{kind}{tag}_sigma"], rtol=RTOL, atol=0)
            np.testing.assert_allclose(k, d[f"prof{kind}{tag}_kappa"], rtol=RTOL, atol=0)
            np.testing.assert_allclose(a, d[f"prof{kind}{tag}_alpha"], rtol=RTOL, atol=0)


def test_packed_recurrence_known_answer():
    d = load("coefficients")
    term = O.compile_cpml_term("Ez", 0, -1.0, np.asarray([0.8, 0.0, 0.0, 1.1], np.float32),
                               np.asarray([1.7, 1.0, 1.0, 2.2], np.float32),
                               np.asarray([0.04, 0.0, 0.0, 0.02], np.float32), 2e-13, 4)
    assert (term.low, term.high) == tuple(d["kat_slab"])
    corrected, psi = O.correct_cpml_term(d["kat_deriv"], np.zeros(term.low + term.high, np.float32), term)
    np.testing.assert_allclose(corrected, d["kat_corrected"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(psi, d["kat_psi"], rtol=RTOL, atol=ATOL)


def test_e_site_sampling_and_masks_match_reference():
    d = load("materials")
    for c in ("Ex", "Ey", "Ez"):
        np.testing.assert_array_equal(O.sample_e_site_3d(d["voxels"], c), d[f"eps_{c}"])
    for pol, comps in (("tm", ("Ez", "Hx", "Hy")), ("te", ("Ex", "Ey", "Hz"))):
        for c in comps:
            np.testing.assert_array_equal(O.sample_site_2d(d["voxels2d"], c, pol), d[f"site2d_{pol}_{c}"])
    shapes = O.component_shapes((4, 5, 6))
    masks = O.pec_masks(shapes, 3, {"front", "top", "left"})
    for c in O.COMPONENTS:
        np.testing.assert_array_equal(masks[c], d[f"mask_{c}"])
    dec, src = O.h_coefficients_2d(float(d["h2d_dt"]))
    assert dec == d["h2d_decay"] and src == d["h2d_source"]
    eps2 = O.sample_site_2d(d["voxels2d"], "Ez", "tm")
    dec, src = O.e_coefficients_2d(eps2, float(d["h2d_dt"]))
    np.testing.assert_array_equal(dec, d["e2d_decay"])
    np.testing.assert_allclose(src, d["e2d_source"], rtol=RTOL)


def test_oracle_planner_reproduces_reference_terms():
    d = load("update3d")
    grid = tuple(int(v) for v in d["grid"])
    h_ref, e_ref, _ = terms3d(d, grid)
    h, e = O.plan_cpml(grid, float(d["dt"]), float(d["res"]), pml_cells=3)
    for mine, theirs in zip(h + e, h_ref + e_ref):
        assert (mine.component, mine.axis, mine.sign, mine.low, mine.high) == (
            theirs.component, theirs.axis, theirs.sign, theirs.low, theirs.high)
        np.testing.assert_allclose(mine.a, theirs.a, rtol=RTOL, atol=1e-9)
        np.testing.assert_allclose(mine.b, theirs.b, rtol=RTOL, atol=ATOL)
        np.testing.assert_allclose(mine.inv_kappa, theirs.inv_kappa, rtol=RTOL, atol=ATOL)


def _fields3d(d):
    return {c: d[f"in_{c}"].copy() for c in O.COMPONENTS}


def test_update3d_cpml_matches_reference():
    d = load("update3d")
    grid = tuple(int(v) for v in d["grid"])
    h_terms, e_terms, _ = terms3d(d, grid)
    f = _fields3d(d)
    psi_h = [d[f"in_psi_h{i}"].copy() for i in range(6)]
    hx, hy, hz, ph = O.update_h_3d(f, psi_h, h_terms, float(d["dt"]), float(d["res"]))
    for name, v in (("Hx", hx), ("Hy", hy), ("Hz", hz)):
        np.testing.assert_allclose(v, d[f"cpml_{name}"], rtol=RTOL, atol=1e-9)
    for i in range(6):
        np.testing.assert_allclose(ph[i], d[f"cpml_psi_h{i}"], rtol=RTOL, atol=1e-9)
    mat = O.material_from_voxels(d["voxels"])
    for tag, metallic in (("open", set()), ("pec", {"back", "bottom", "right"})):
        psi_e = [d[f"in_psi_e{i}"].copy() for i in range(6)]
        ex, ey, ez, pe = O.update_e_3d(f, psi_e, e_terms, float(d["dt"]), float(d["res"]), mat, metallic)
        for name, v in (("Ex", ex), ("Ey", ey), ("Ez", ez)):
            np.testing.assert_allclose(v, d[f"cpml_{tag}_{name}"], rtol=RTOL, atol=1e-6)
        for i in range(6):
            np.testing.assert_allclose(pe[i], d[f"cpml_{tag}_psi_e{i}"], rtol=RTOL, atol=1e-6)


def test_update3d_plain_yee_matches_reference():
    d = load("update3d")
    f = _fields3d(d)
    hx, hy, hz, _ = O.update_h_3d(f, [], [], float(d["dt"]), float(d["res"]))
    for name, v in (("Hx", hx), ("Hy", hy), ("Hz", hz)):
        np.testing.assert_allclose(v, d[f"yee_{name}"], rtol=RTOL, atol=1e-9)
    mat = O.material_from_voxels(d["voxels"])
    ex, ey, ez, _ = O.update_e_3d(f, [], [], float(d["dt"]), float(d["res"]), mat, {"front", "top", "left"})
    for name, v in (("Ex", ex), ("Ey", ey), ("Ez", ez)):
        np.testing.assert_allclose(v, d[f"yee_{name}"], rtol=RTOL, atol=1e-6)


@pytest.mark.parametrize("pol", ["tm", "te"])
def test_update2d_cpml_curls_match_reference(pol):
    d = load("update2d")
    grid = tuple(int(v) for v in d["grid"])
    res, dt = float(d["res"]), float(d["dt"])
    (hspec, espec) = O.CPML_2D_TERMS[pol]
    shapes = O.component_shapes(grid, pol)
    h_terms = terms_from(d, f"{pol}h", [c for c, _, _ in hspec], [shapes[c][ax] for c, ax, _ in hspec])
    e_terms = terms_from(d, f"{pol}e", [c for c, _, _ in espec], [shapes[c][ax] for c, ax, _ in espec])
    mine_h, mine_e = O.plan_cpml(grid, dt, res, pml_cells=3, polarization=pol)
    for mine, theirs in zip(mine_h + mine_e, h_terms + e_terms):
        assert (mine.axis, mine.sign, mine.low, mine.high) == (theirs.axis, theirs.sign, theirs.low, theirs.high)
        np.testing.assert_allclose(mine.a, theirs.a, rtol=RTOL, atol=1e-9)
    comps = ("Ez", "Hx", "Hy") if pol == "tm" else ("Ex", "Ey", "Hz")
    f = {c: np.zeros((1, 1), np.float32) for c in O.COMPONENTS}
    f.update({c: d[f"{pol}_in_{c}"].copy() for c in comps})
    psi_h = [d[f"{pol}_in_psi_h{i}"].copy() for i in range(2)]
    psi_e = [d[f"{pol}_in_psi_e{i}"].copy() for i in range(2)]
    # Recover the curls from a unit-coefficient update: H_new = H - 1 * curl.
    one = np.float32(1.0)
    hnew, ph = O.update_h_2d(f, psi_h, h_terms, res, (one, one), pol)
    metallic = {"left", "top"}
    unit = {c: (one, one) for c in ("Ex", "Ey", "Ez")}
    zero_e = dict(f)
    for c in ("Ex", "Ey", "Ez"):
        zero_e[c] = np.zeros_like(f[c])
    enew, pe = O.update_e_2d(zero_e, psi_e, e_terms, res, unit, metallic, pol)
    if pol == "tm":
        np.testing.assert_allclose(f["Hx"] - hnew["Hx"], d["tm_curl_h0"], rtol=1e-5, atol=1e-3)
        np.testing.assert_allclose(f["Hy"] - hnew["Hy"], d["tm_curl_h1"], rtol=1e-5, atol=1e-3)
        np.testing.assert_allclose(enew["Ez"], d["tm_curl_e"], rtol=RTOL, atol=1e-6)
        plain, _ = O.update_e_2d(zero_e, [], [], res, unit, metallic, pol)
        np.testing.assert_allclose(plain["Ez"], d["tm_plain_curl_e"], rtol=RTOL, atol=1e-6)
    else:
        np.testing.assert_allclose(f["Hz"] - hnew["Hz"], d["te_curl_h"], rtol=1e-5, atol=1e-3)
        np.testing.assert_allclose(enew["Ex"], d["te_curl_e0"], rtol=RTOL, atol=1e-6)
        np.testing.assert_allclose(enew["Ey"], d["te_curl_e1"], rtol=RTOL, atol=1e-6)
        plain, _ = O.update_e_2d(zero_e, [], [], res, unit, metallic, pol)
        np.testing.assert_allclose(plain["Ex"], d["te_plain_curl_e0"], rtol=RTOL, atol=1e-6)
        np.testing.assert_allclose(plain["Ey"], d["te_plain_curl_e1"], rtol=RTOL, atol=1e-6)
    for i in range(2):
        np.testing.assert_allclose(ph[i], d[f"{pol}_psi_h{i}"], rtol=RTOL, atol=1e-6)
        np.testing.assert_allclose(pe[i], d[f"{pol}_psi_e{i}"], rtol=RTOL, atol=1e-6)


def test_gaussian_pulse_matches_reference():
    d = load("pulse")
    f0 = float(d["f0"])
    np.testing.assert_allclose(O.gaussian_pulse_sample(d["times"], f0, 0.2 * f0, offset=0.5), d["signal"],
                               rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(O.gaussian_pulse_sample(d["times"], f0, 0.1 * f0, amplitude=2.0, offset=4.0,
                                                       remove_dc=False), d["signal2"], rtol=1e-6, atol=1e-30)


@pytest.mark.parametrize("tag", ["plain", "hann"])
def test_dft_accumulation_matches_reference(tag):
    d = load("dft")
    grid = tuple(int(v) for v in d["grid"])
    fields = {c: d[f"f_{c}"] for c in O.COMPONENTS}
    window, norm, t0, t1, interval = d[f"{tag}_cfg"]
    mon = O.DftMonitor(d["freqs"], [d[f"idx_{i}"] for i in range(6)], [d[f"w_{i}"] for i in range(6)],
                       d["mask"], t0, t1, int(interval), int(window), int(norm), 1e-6)
    re, im, w = d["re0"].copy(), d["im0"].copy(), np.zeros(len(d["freqs"]), np.float32)
    O.accumulate_dft(mon, (re, im, w), fields, d[f"{tag}_t"], 36, float(d["dt"]))
    assert bool(d[f"{tag}_gate"])
    np.testing.assert_allclose(re, d[f"{tag}_re"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(im, d[f"{tag}_im"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(w, d[f"{tag}_w"], rtol=1e-6, atol=1e-7)


def test_plane_gather_plan_matches_reference():
    d = load("dft")
    grid = tuple(int(v) for v in d["grid"])
    res = 20e-9
    for i, c in enumerate(O.COMPONENTS):
        idx, w = O.plane_gather_plan_3d(c, "x", 3.25 * res, (np.arange(4) + 1.3) * res, (np.arange(5) + 0.7) * res,
                                        res, grid)
        k = idx.shape[1]
        np.testing.assert_array_equal(idx, d[f"idx_{i}"][:, :k])
        np.testing.assert_allclose(w, d[f"w_{i}"][:, :k], rtol=1e-7, atol=0)


def build_steps3d_program(d, dtype=np.float32):
    """The oracle program for the ``steps3d`` fixture (shared with GPU tests)."""
    grid = tuple(int(v) for v in d["grid"])
    h_terms, e_terms, shapes = terms3d(d, grid)
    mat = O.material_from_voxels(d["voxels"], dtype=dtype)
    nsteps = int(d["nsteps"])
    sources = [
        O.SlabSource("Ey", "pre_e", (5, 5, 6), d["src_coeff"], d["wave"]),
        O.SlabSource("Hz", "h", (2, 3, 4), d["h_coeff"], d["hwave"]),
    ]
    mon = O.DftMonitor(d["freqs"], [d[f"idx_{i}"] for i in range(6)], [d[f"w_{i}"] for i in range(6)], d["cmask"])
    prog = O.OracleProgram(grid, float(d["dt"]), float(d["res"]), h_terms, e_terms, mat,
                           metallic_edges=frozenset({"front"}), sources=sources, monitors=[mon])
    return prog, nsteps


def test_multistep_composition_matches_reference():
    d = load("steps3d")
    prog, nsteps = build_steps3d_program(d)
    state = O.run(O.new_state(prog), prog, nsteps)
    for c in O.COMPONENTS:
        assert O.relative_l2(state.fields[c], d[f"out_{c}"]) <= 1e-6, c
    for i in range(6):
        assert O.relative_l2(state.psi_h[i], d[f"out_psi_h{i}"]) <= 1e-5
        assert O.relative_l2(state.psi_e[i], d[f"out_psi_e{i}"]) <= 1e-5
    assert O.relative_l2(state.dft_re, d["dft_re"]) <= 1e-6
    assert O.relative_l2(state.dft_im, d["dft_im"]) <= 1e-6
    np.testing.assert_array_equal(state.dft_w, d["dft_w"])
    assert np.float32(state.t) == d["t"]


def test_fp64_oracle_tracks_fp32_oracle():
    d = load("steps3d")
    prog32, nsteps = build_steps3d_program(d)
    prog64, _ = build_steps3d_program(d, np.float64)
    s32 = O.run(O.new_state(prog32), prog32, nsteps)
    s64 = O.run(O.new_state(prog64, np.float64), prog64, nsteps)
    for c in O.COMPONENTS:
        assert O.relative_l2(s32.fields[c], s64.fields[c]) <= 1e-5, c
