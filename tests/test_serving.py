"""Serving loop: results identical alone and in the mix; request stream and stats."""

from __future__ import annotations

import numpy as np
import pytest

from beamz_b200 import plan as P
from beamz_b200 import serve, workloads as W


def _mix():
    specs = [
        W.scene_2d(total_steps=300, seed=1, shape=(96, 96), n_monitors=2),
        W.scene_3d_512(total_steps=260, seed=2, shape=(24, 40, 64), n_monitors=2, n_freqs=3, pml_cells=4),
        W.scene_2d(total_steps=150, seed=3, shape=(128, 160), n_monitors=1),
        W.scene_3d_512(total_steps=131, seed=4, shape=(20, 33, 45), n_monitors=1, n_freqs=3, pml_cells=4),
        W.scene_2d(total_steps=401, seed=5, shape=(64, 64), n_monitors=4),
        W.scene_3d_512(total_steps=200, seed=6, shape=(32, 32, 32), n_monitors=3, n_freqs=3, pml_cells=4),
    ]
    arrivals = [0.0, 0.0, 0.005, 0.01, 0.02, 0.02]
    return [serve.Request(i, s, s.total_steps, a) for i, (s, a) in enumerate(zip(specs, arrivals))]


def test_request_stream_is_seeded_and_mixed():
    a = W.serving_requests(12, rate=100.0, seed=3, steps=(50, 80), sizes_2d=(64, 128),
                           shapes_3d=((16, 24, 32),))
    b = W.serving_requests(12, rate=100.0, seed=3, steps=(50, 80), sizes_2d=(64, 128),
                           shapes_3d=((16, 24, 32),))
    assert [t for t, _ in a] == [t for t, _ in b]
    assert all(np.array_equal(x.voxel_ids, y.voxel_ids) for (_, x), (_, y) in zip(a, b) if x.ndim == 3)
    times = [t for t, _ in a]
    assert times == sorted(times) and times[0] > 0
    assert {s.ndim for _, s in a} == {2, 3}
    assert all(50 <= s.total_steps <= 80 and 1 <= len(s.monitors) <= 4 for _, s in a)


def test_estimate_grows_with_the_grid():
    small = W.scene_3d_512(total_steps=10, shape=(16, 24, 32), n_monitors=1, n_freqs=3, pml_cells=4)
    big = W.scene_3d_512(total_steps=10, shape=(48, 96, 128), n_monitors=1, n_freqs=3, pml_cells=4)
    assert serve.estimate_bytes(big) > 4 * serve.estimate_bytes(small) > 0
    nz, ny, nx = big.grid_shape
    assert serve.estimate_bytes(big) >= 12 * (nz + 1) * (ny + 1) * (nx + 1) * 4


def test_summary_percentiles():
    res = [serve.Result(i, 1, None, None, None, None, arrival=0.1 * i, admitted=0.1 * i, finished=0.1 * i + 1.0 + i)
           for i in range(10)]
    st = serve.summarize(res)
    assert st.n == 10
    assert st.p50_s == pytest.approx(np.percentile([1.0 + i for i in range(10)], 50))
    assert st.makespan_s == pytest.approx(0.9 + 10.0 - 0.0)


@pytest.mark.gpu
def test_results_identical_alone_and_in_the_mix():
    reqs = _mix()
    engine = serve.ServingEngine(max_active=3, chunk=64, return_fields=True)
    mixed = engine.run(reqs)
    alone = serve.run_sequential(reqs, return_fields=True)
    assert engine.peak_active >= 2
    for m, a in zip(mixed, alone):
        assert m.rid == a.rid
        np.testing.assert_array_equal(m.dft_re, a.dft_re)
        np.testing.assert_array_equal(m.dft_im, a.dft_im)
        np.testing.assert_array_equal(m.dft_w, a.dft_w)
        for c in a.fields:
            np.testing.assert_array_equal(m.fields[c], a.fields[c], err_msg=f"request {m.rid} {c}")
        assert m.finished >= m.admitted >= m.arrival


@pytest.mark.gpu
def test_recorders_identical_alone_and_in_the_mix():
    import dataclasses

    reqs = _mix()
    for r in (reqs[1], reqs[4]):
        spec = r.spec
        rec = P.domain_recorder(spec.grid_shape, P.active_components(spec.ndim, spec.polarization)[:2], 25,
                                r.nsteps, spec.polarization)
        r.spec = dataclasses.replace(spec, recorders=[rec])
    mixed = serve.ServingEngine(max_active=3, chunk=64).run(reqs)
    alone = serve.run_sequential(reqs)
    for m, a in zip(mixed, alone):
        assert (m.records is None) == (a.records is None) == (m.rid not in (1, 4))
        for rm, ra in zip(m.records or [], a.records or []):
            assert len(ra["steps"]) == reqs[m.rid].nsteps // 25
            for k in ra:
                np.testing.assert_array_equal(rm[k], ra[k], err_msg=f"request {m.rid} {k}")


@pytest.mark.gpu
def test_budget_limits_residency():
    reqs = _mix()
    one = max(serve.estimate_bytes(r.spec) for r in reqs)
    engine = serve.ServingEngine(hbm_budget=one, chunk=64)
    res = engine.run(reqs)
    assert len(res) == len(reqs)
    assert engine.peak_bytes <= one or engine.peak_active == 1


def test_autotune_table_and_heuristic(tmp_path):
    from beamz_b200 import autotune

    small = W.scene_3d_512(total_steps=10, shape=(16, 24, 40), n_monitors=1, n_freqs=3, pml_cells=4)
    assert autotune.shape_class(small) == "3d:32x32x64:cpml1"
    assert autotune.choose(small, path=str(tmp_path / "t.json")) == autotune.heuristic(small)
    table = {autotune.shape_class(small): {"best": [4, 32], "us_per_step": {}}}
    autotune._store(str(tmp_path / "u.json"), table)
    assert autotune.choose(small, path=str(tmp_path / "u.json")) == (4, 32)
    big = W.scene_3d_512(total_steps=1, shape=(256, 512, 512), monitors=False, sources=False)
    assert autotune.heuristic(big) == (8, 16)
