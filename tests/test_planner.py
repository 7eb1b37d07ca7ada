"""The product planner (beamz_b200.plan) against the oracle's restatement."""

from __future__ import annotations

import numpy as np
import pytest

from beamz_b200 import plan as P
from oracle import fdtd_oracle as O
from tests.golden_io import load


@pytest.mark.parametrize("grid", [(9, 10, 11), (20, 16, 24), (13, 15), (40, 41)])
@pytest.mark.parametrize("pml", [3, 12])
def test_cpml_terms_match_oracle(grid, pml):
    if min(grid) <= 2 * pml:
        pytest.skip("absorber would swallow the axis")
    res = 20e-9
    dt = 0.99 * res / (P.LIGHT_SPEED * np.sqrt(len(grid)))
    pols = ("tm", "te") if len(grid) == 2 else ("tm",)
    for pol in pols:
        mh, me = P.plan_cpml(grid, dt, res, pml_cells=pml, polarization=pol)
        oh, oe = O.plan_cpml(grid, dt, res, pml_cells=pml, polarization=pol)
        for a, b in zip(mh + me, oh + oe):
            assert (a.component, a.axis, a.sign, a.low, a.high) == (b.component, b.axis, b.sign, b.low, b.high)
            np.testing.assert_array_equal(a.a, b.a)
            np.testing.assert_array_equal(a.b, b.b)
            np.testing.assert_array_equal(a.inv_kappa, b.inv_kappa)


def test_cpml_terms_on_partial_edges():
    grid = (12, 14, 16)
    res = 20e-9
    dt = 0.99 * res / (P.LIGHT_SPEED * np.sqrt(3))
    edges = ("left", "top", "back")
    mh, me = P.plan_cpml(grid, dt, res, pml_cells=4, edges=edges)
    oh, oe = O.plan_cpml(grid, dt, res, pml_cells=4, edges=edges)
    for a, b in zip(mh + me, oh + oe):
        assert (a.low, a.high) == (b.low, b.high)
        np.testing.assert_array_equal(a.a, b.a)


@pytest.mark.parametrize("explicit", [False, True])
def test_absorber_counts_and_extension(explicit):
    for grid in ((30, 32, 34), (50, 60)):
        mine = P.absorber_edge_counts(grid, 7, resolution=20e-9, explicit_thickness=explicit)
        theirs = O.cpml_material_edge_counts(grid, 7, resolution=20e-9, explicit_thickness=explicit)
        assert mine == theirs
        rng = np.random.default_rng(3)
        eps = rng.choice([2.085, 12.11], size=grid).astype(np.float32)
        np.testing.assert_array_equal(P.extend_into_absorber(eps, mine), O.extend_materials_into_absorber(eps, theirs))


def test_voxel_codebook_round_trips():
    rng = np.random.default_rng(0)
    eps = rng.choice(np.float32([1.0, 2.085, 3.5, 12.11]), size=(5, 6, 7))
    ids, table = P.voxel_codebook(eps)
    assert ids.dtype == np.uint8 and table.shape == (256,)
    np.testing.assert_array_equal(table[ids], eps)
    with pytest.raises(ValueError):
        P.voxel_codebook(np.arange(300, dtype=np.float32))


def test_site_sampling_2d_matches_oracle():
    d = load("materials")
    for pol, comps in (("tm", ("Ez", "Hx", "Hy")), ("te", ("Ex", "Ey", "Hz"))):
        for c in comps:
            np.testing.assert_array_equal(P.site_values_2d(d["voxels2d"], c, pol), d[f"site2d_{pol}_{c}"])
    eps2 = P.site_values_2d(d["voxels2d"], "Ez", "tm")
    np.testing.assert_allclose(P.e_source_2d(eps2, float(d["h2d_dt"])), d["e2d_source"], rtol=2e-7)


def test_gaussian_pulse_matches_reference():
    d = load("pulse")
    f0 = float(d["f0"])
    np.testing.assert_allclose(P.gaussian_pulse(d["times"], f0, 0.2 * f0, offset=0.5), d["signal"], rtol=1e-6,
                               atol=1e-7)


def test_plane_gather_matches_reference():
    d = load("dft")
    grid = tuple(int(v) for v in d["grid"])
    res = 20e-9
    for i, c in enumerate(P.COMPONENTS):
        idx, w = P.plane_gather(c, "x", 3.25 * res, (np.arange(4) + 1.3) * res, (np.arange(5) + 0.7) * res, res, grid)
        k = idx.shape[1]
        np.testing.assert_array_equal(idx, d[f"idx_{i}"][:, :k])
        np.testing.assert_allclose(w, d[f"w_{i}"][:, :k], rtol=1e-7, atol=0)


def test_step_times_accumulate_in_float32():
    d = load("steps3d")
    times = P.step_times(0.0, float(d["dt"]), int(d["nsteps"]))
    assert times[-1] == d["t"]
    assert times.dtype == np.float32


@pytest.mark.parametrize("grid,nmat", [((5, 6, 7), 2), ((4, 9, 3), 5), ((1, 4, 4), 1)])
def test_site_codebook_matches_oracle_sampling(grid, nmat):
    """Every E site's codebook coefficient equals fl(dt/eps0 * fl(1/eps_site))
    with eps_site sampled the oracle's way (clipped centered averages)."""
    rng = np.random.default_rng(sum(grid) + nmat)
    table = np.linspace(1.0, 12.25, nmat).astype(np.float32)
    ids = rng.integers(0, nmat, size=grid).astype(np.uint8)
    dto = np.float32(2.0e-17) / np.float32(P.EPS_0)
    words, coef = P.site_codebook(ids, table, dto)
    assert words.shape == tuple(n + 1 for n in grid)
    eps_grid = table[ids]
    for n, c in enumerate(("Ex", "Ey", "Ez")):
        eps_site = O.sample_e_site_3d(eps_grid, c).astype(np.float32)
        want = dto * (np.float32(1.0) / eps_site)
        dz, dy, dx = eps_site.shape
        got = coef[n][(words[:dz, :dy, :dx] >> (8 * n)) & 0xFF]
        np.testing.assert_array_equal(got, want)


def test_device_codebook_equals_host_build():
    """The torch (device) builder, run here on CPU tensors, equals the numpy one."""
    torch = pytest.importorskip("torch")
    from beamz_b200.runtime import device_site_codebook

    rng = np.random.default_rng(7)
    grid = (7, 10, 13)
    table = np.array([1.0, 2.25, 3.5, 12.0], np.float32)
    ids = rng.integers(0, 4, size=grid).astype(np.uint8)
    dto = np.float32(1.7e-17) / np.float32(P.EPS_0)
    words, coef = P.site_codebook(ids, table, dto)
    pitch = 16
    dev_words, dev_coef = device_site_codebook(ids, table, dto, pitch, torch.device("cpu"), z_block=3)
    dev_words = dev_words.numpy()
    np.testing.assert_array_equal(dev_words[:, :, : grid[2] + 1], words)
    assert not dev_words[:, :, grid[2] + 1:].any()
    np.testing.assert_array_equal(dev_coef.numpy(), coef)


def test_codebook_overflow_is_reported():
    ids = np.arange(60, dtype=np.uint8).reshape(3, 4, 5)
    with pytest.raises(P.CodebookOverflow):
        P.site_codebook(ids, np.linspace(1, 9, 60).astype(np.float32), np.float32(1.0))


def test_sources_clear_of_monitors():
    """The DFT sample of a step may run beside the next step only when no
    pre-E source writes a cell that a monitor gathers."""
    import dataclasses

    from beamz_b200 import workloads as W

    spec = W.scene_3d_512(total_steps=10, shape=(24, 32, 40), pml_cells=3)
    assert P.sources_clear_of_monitors(spec)
    mon = spec.monitors[0]
    ci = P.COMPONENTS.index("Ey")
    flat = int(np.asarray(mon.indices[ci])[np.asarray(mon.weights[ci]) != 0][0])
    cell = tuple(int(v) for v in np.unravel_index(flat, P.component_shape("Ey", spec.grid_shape)))

    def with_source(component, timing):
        src = P.SourcePlan(component, timing, cell, np.ones((1, 1, 1), np.float32), np.zeros(4, np.float32))
        return dataclasses.replace(spec, sources=list(spec.sources) + [src])

    assert not P.sources_clear_of_monitors(with_source("Ey", "pre_e"))
    assert P.sources_clear_of_monitors(with_source("Ey", "e"))  # written before the sample is taken
    assert P.sources_clear_of_monitors(with_source("Ex", "pre_e"))  # Ex is masked off on these planes
    # Boxes of every size, some reaching past the grid, against a brute-force scan.
    shape = P.component_shape("Ey", spec.grid_shape)
    gathered = set()
    for m in spec.monitors:
        if float(m.component_mask[ci]) != 0.0:
            gathered.update(int(v) for v in np.asarray(m.indices[ci])[np.asarray(m.weights[ci]) != 0])
    rng = np.random.default_rng(5)
    for _ in range(40):
        ext = tuple(int(v) for v in rng.integers(1, 9, 3))
        start = tuple(int(rng.integers(-3, d)) for d in shape)
        cells = {int(np.ravel_multi_index((k, j, i), shape))
                 for k in range(max(start[0], 0), min(start[0] + ext[0], shape[0]))
                 for j in range(max(start[1], 0), min(start[1] + ext[1], shape[1]))
                 for i in range(max(start[2], 0), min(start[2] + ext[2], shape[2]))}
        src = P.SourcePlan("Ey", "pre_e", start, np.ones(ext, np.float32), np.zeros(4, np.float32))
        got = P.sources_clear_of_monitors(dataclasses.replace(spec, sources=[src]))
        assert got == (not (cells & gathered)), (start, ext)


def test_affine_form_of_plane_plans():
    """The affine form (FdtdDft.affine) reproduces a plane monitor's gather
    plan exactly -- every index and weight -- and is refused when the weights
    vary from point to point."""
    torch = pytest.importorskip("torch")
    from beamz_b200 import runtime as R
    from beamz_b200 import workloads as W

    spec = W.scene_3d_512(total_steps=4, shape=(20, 36, 44), pml_cells=4)
    seen = 0
    for mon in spec.monitors:
        for c in range(6):
            if mon.component_mask[c] == 0:
                continue
            idx = np.asarray(mon.indices[c]).reshape(mon.points, -1)
            w = np.asarray(mon.weights[c]).reshape(mon.points, -1)
            words = R._affine_plan(torch.as_tensor(idx.T.copy()), torch.as_tensor(w.T.copy()))
            assert words is not None
            flag, na, nb, base, sa, sb, k = words[:7]
            assert flag == 1 and na * nb == mon.points and 1 <= k <= 4
            p = np.arange(mon.points)
            b0 = base + (p // nb) * sa + (p % nb) * sb
            for s in range(k):
                np.testing.assert_array_equal(idx[:, s], b0 + words[8 + s])
                wk = np.array([words[16 + s]], np.int32).view(np.float32)[0]
                np.testing.assert_array_equal(w[:, s], np.full(mon.points, wk, np.float32))
            assert not np.any(w[:, k:])
            seen += 1
            w2 = w.copy()
            w2[5, 0] *= 2.0
            assert R._affine_plan(torch.as_tensor(idx.T.copy()), torch.as_tensor(w2.T.copy())) is None
    assert seen == 16  # four planes, four sampled components each

