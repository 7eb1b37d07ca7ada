"""CUDA path (through the C ABI) against the CPU oracle and the golden vectors.

Tolerances: the step is float32 arithmetic in the reference's order of
operations, so fields are expected to agree to a few ulps; the accuracy bar
is relative L2 <= 1e-5 for fields and <= 1e-4 for DFT accumulators, and both
are asserted here.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from beamz_b200 import plan as P  # noqa: E402
from beamz_b200 import runtime as R  # noqa: E402
from oracle import fdtd_oracle as O  # noqa: E402
from tests.golden_io import load, terms3d  # noqa: E402
from tests.scenarios import oracle_state, random_initial_fields, scenario_2d, scenario_3d, to_oracle  # noqa: E402

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5
DFT_TOL = 1e-4


def _compare(gpu: dict, st: O.OracleState, active, tol=FIELD_TOL, dft_tol=DFT_TOL):
    for c in active:
        err = O.relative_l2(gpu[c], st.fields[c])
        assert err <= tol, f"{c}: rel L2 {err:.3e}"
    for i, p in enumerate(st.psi_h):
        if p.size:
            assert O.relative_l2(gpu["psi_h"][i], p) <= max(tol, 1e-5), f"psi_h{i}"
    for i, p in enumerate(st.psi_e):
        if p.size:
            assert O.relative_l2(gpu["psi_e"][i], p) <= max(tol, 1e-5), f"psi_e{i}"
    if st.dft_re is not None and st.dft_re.size:
        assert O.relative_l2(gpu["dft_re"], st.dft_re) <= dft_tol
        assert O.relative_l2(gpu["dft_im"], st.dft_im) <= dft_tol
        np.testing.assert_allclose(gpu["dft_w"], st.dft_w, rtol=1e-6, atol=1e-6)
    assert np.float32(gpu["t"]) == np.float32(st.t)


@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_golden_steps3d(schedule):
    """16 steps of the reference-composed fixture (CPML on 5 faces, PEC front)."""
    d = load("steps3d")
    grid = tuple(int(v) for v in d["grid"])
    h_terms, e_terms, shapes = terms3d(d, grid)
    to_plan = lambda ts: [P.CpmlTermPlan(t.component, t.axis, t.sign, t.low, t.high, t.a, t.b, t.inv_kappa) for t in ts]  # noqa: E731
    ids, table = P.voxel_codebook(d["voxels"])
    mon = P.DftMonitorPlan(d["freqs"], [d[f"idx_{i}"] for i in range(6)], [d[f"w_{i}"] for i in range(6)], d["cmask"])
    spec = P.ProgramSpec(grid, float(d["dt"]), float(d["res"]), voxel_ids=ids, eps_table=table,
                         h_terms=to_plan(h_terms), e_terms=to_plan(e_terms), metallic_edges=frozenset({"front"}),
                         sources=[P.SourcePlan("Ey", "pre_e", (5, 5, 6), d["src_coeff"], d["wave"]),
                                  P.SourcePlan("Hz", "h", (2, 3, 4), d["h_coeff"], d["hwave"])],
                         monitors=[mon], total_steps=int(d["nsteps"]))
    prog = R.compile_program(spec, schedule=schedule)
    state = R.run_steps(R.initial_state(prog), prog, int(d["nsteps"]))
    out = state.numpy()
    for c in P.COMPONENTS:
        assert O.relative_l2(out[c], d[f"out_{c}"]) <= FIELD_TOL, c
    assert O.relative_l2(out["dft_re"], d["dft_re"]) <= DFT_TOL
    assert O.relative_l2(out["dft_im"], d["dft_im"]) <= DFT_TOL
    np.testing.assert_array_equal(out["dft_w"], d["dft_w"])
    assert np.float32(out["t"]) == d["t"]


def test_golden_single_phases():
    """One H and one E phase from the update3d fixture (random fields and psi)."""
    d = load("update3d")
    grid = tuple(int(v) for v in d["grid"])
    h_terms, e_terms, _ = terms3d(d, grid)
    to_plan = lambda ts: [P.CpmlTermPlan(t.component, t.axis, t.sign, t.low, t.high, t.a, t.b, t.inv_kappa) for t in ts]  # noqa: E731
    ids, table = P.voxel_codebook(d["voxels"])
    for tag, metallic in (("open", frozenset()), ("pec", frozenset({"back", "bottom", "right"}))):
        spec = P.ProgramSpec(grid, float(d["dt"]), float(d["res"]), voxel_ids=ids, eps_table=table,
                             h_terms=to_plan(h_terms), e_terms=to_plan(e_terms), metallic_edges=metallic)
        prog = R.compile_program(spec, schedule="phases")
        fields = {c: d[f"in_{c}"] for c in P.COMPONENTS}
        state = R.initial_state(prog, fields=fields, psi_h=[d[f"in_psi_h{i}"] for i in range(6)],
                                psi_e=[d[f"in_psi_e{i}"] for i in range(6)])
        R.update_h(state, prog)
        torch.cuda.synchronize()
        out = state.numpy()
        if tag == "open":
            for c in ("Hx", "Hy", "Hz"):
                np.testing.assert_allclose(out[c], d[f"cpml_{c}"], rtol=2e-6, atol=1e-9)
            for i in range(6):
                np.testing.assert_allclose(out["psi_h"][i], d[f"cpml_psi_h{i}"], rtol=2e-6, atol=1e-9)
        # E from the fixture's input H, not the updated one.
        for i, c in enumerate(("Hx", "Hy", "Hz")):
            state.fields[3 + i].copy_(torch.as_tensor(d[f"in_{c}"], device="cuda"))
        R.update_e(state, prog)
        out = state.numpy()
        masks = O.pec_masks({c: d[f"in_{c}"].shape for c in P.COMPONENTS}, 3, metallic)
        for c in ("Ex", "Ey", "Ez"):
            expected = np.where(masks[c], 0.0, d[f"cpml_{tag}_{c}"])
            np.testing.assert_allclose(out[c], expected, rtol=2e-6, atol=1e-6)
        for i in range(6):
            np.testing.assert_allclose(out["psi_e"][i], d[f"cpml_{tag}_psi_e{i}"], rtol=2e-6, atol=1e-6)


CASES_3D = [
    dict(grid=(9, 10, 11), metallic=()),
    dict(grid=(7, 13, 5), metallic=("front", "top", "left")),
    dict(grid=(12, 9, 40), metallic=("back", "right", "bottom"), pml_cells=4),
    dict(grid=(6, 8, 37), cpml_edges=(), metallic=("front", "back", "bottom", "top", "left", "right")),
    dict(grid=(10, 35, 9), cpml_edges=("left", "top", "back"), metallic=("right",)),
    dict(grid=(9, 17, 64), metallic=("right", "bottom")),
]


@pytest.mark.parametrize("case", range(len(CASES_3D)))
@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_random_3d_against_oracle(case, schedule):
    kw = dict(CASES_3D[case])
    nsteps = 11
    spec = scenario_3d(seed=case, nsteps=nsteps, **kw)
    fields = random_initial_fields(spec, seed=case + 10)
    prog = R.compile_program(spec, schedule=schedule)
    state = R.run_steps(R.initial_state(prog, fields=fields), prog, nsteps)
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog, fields), oprog, nsteps)
    _compare(state.numpy(), st, P.COMPONENTS)


@pytest.mark.parametrize("step_kernel", ["classes", "codebook"])
@pytest.mark.parametrize("tile", [(32, 4), (32, 8), (32, 16), (64, 4), (64, 8)])
@pytest.mark.parametrize("z_chunk", [0, 3])
def test_fused_tiles_and_z_chunks_are_bitwise_identical(tile, z_chunk, step_kernel):
    spec = scenario_3d(grid=(11, 21, 70), seed=4, nsteps=6, metallic=("front",))
    fields = random_initial_fields(spec, seed=5)
    ref_prog = R.compile_program(spec, schedule="phases")
    ref = R.run_steps(R.initial_state(ref_prog, fields=fields), ref_prog, 6).numpy()
    prog = R.compile_program(spec, schedule="fused", tile=tile, z_chunk=z_chunk, step_kernel=step_kernel)
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 6).numpy()
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(out[c], ref[c], err_msg=c)
    np.testing.assert_array_equal(out["dft_re"], ref["dft_re"])


def test_lossy_uniform_h_matches_the_scalar_schedule():
    """A uniform H decay below one (magnetic loss) through the pitched
    straight path, whose interior tiles pair two components per instruction:
    every field equals the dense scalar schedule's bit for bit (each product
    and difference rounded on its own, none fused)."""
    import dataclasses

    spec = scenario_3d(grid=(24, 24, 192), seed=6, nsteps=6, metallic=("front",))
    loss = np.float32(0.9996)
    site = {c: (np.float32(0.9993), np.float32(np.float32(s) * loss)) for c, (_d, s) in spec.h_coefficients().items()}
    spec = dataclasses.replace(spec, h_site=site)
    fields = random_initial_fields(spec, seed=7)
    ref_prog = R.compile_program(spec, schedule="phases")
    ref = R.run_steps(R.initial_state(ref_prog, fields=fields), ref_prog, 6).numpy()
    prog = R.compile_program(spec, schedule="fused", layout="pitched", tile=(32, 8), z_chunk=8)
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 6).numpy()
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(out[c], ref[c], err_msg=c)


# Grids whose x extent is a multiple of the 32-wide tile: the last tile owns the
# face column x = X; low faces take the straight path with per-lane ghosts.
FACE_CASES = [
    dict(grid=(9, 17, 64), metallic=("right", "front")),
    dict(grid=(7, 24, 32), metallic=("left", "right", "bottom", "top"), pml_cells=5),
    dict(grid=(13, 16, 96), cpml_edges=("right", "back", "bottom"), metallic=("left",)),
    dict(grid=(6, 40, 64), cpml_edges=(), metallic=()),
]


@pytest.mark.parametrize("case", range(len(FACE_CASES)))
@pytest.mark.parametrize("tile_y", [4, 8, 16])
def test_fused_face_columns_are_bitwise_identical(case, tile_y):
    spec = scenario_3d(seed=20 + case, nsteps=7, **FACE_CASES[case])
    fields = random_initial_fields(spec, seed=30 + case)
    ref_prog = R.compile_program(spec, schedule="phases")
    ref = R.run_steps(R.initial_state(ref_prog, fields=fields), ref_prog, 7).numpy()
    prog = R.compile_program(spec, schedule="fused", tile=(32, tile_y), z_chunk=4)
    assert prog.layout == "pitched"
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 7).numpy()
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(out[c], ref[c], err_msg=c)
    for a, b in zip(out["psi_h"] + out["psi_e"], ref["psi_h"] + ref["psi_e"]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(out["dft_re"], ref["dft_re"])


@pytest.mark.parametrize("pol", ["tm", "te"])
@pytest.mark.parametrize("schedule", ["fused", "phases"])
@pytest.mark.parametrize("metallic", [(), ("left", "top")])
def test_2d_against_oracle(pol, schedule, metallic):
    nsteps = 25
    spec = scenario_2d(grid=(17, 23), polarization=pol, metallic=metallic, nsteps=nsteps)
    fields = random_initial_fields(spec, seed=3)
    prog = R.compile_program(spec, schedule=schedule)
    state = R.run_steps(R.initial_state(prog, fields=fields), prog, nsteps)
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog, fields), oprog, nsteps)
    _compare(state.numpy(), st, P.active_components(2, pol))


def test_phase_entries_compose_to_the_program():
    """pre-E sources, H, H sources, E, E sources, DFT through the phase-level ABI."""
    spec = scenario_3d(grid=(8, 9, 10), seed=7, nsteps=5, metallic=("top",))
    fields = random_initial_fields(spec, seed=8)
    prog = R.compile_program(spec, schedule="phases")
    a = R.initial_state(prog, fields=fields)
    for _ in range(5):
        R.step_by_phases(a, prog)
    b = R.run_steps(R.initial_state(prog, fields=fields), prog, 5)
    oa, ob = a.numpy(), b.numpy()
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(oa[c], ob[c])
    np.testing.assert_array_equal(oa["dft_re"], ob["dft_re"])


def test_chunked_runs_resume_exactly():
    """Graph chunks, odd chunk lengths and continuation give the same state."""
    spec = scenario_3d(grid=(8, 9, 33), seed=9, nsteps=40)
    fields = random_initial_fields(spec, seed=2)
    prog = R.compile_program(spec, schedule="fused")
    one = R.run_steps(R.initial_state(prog, fields=fields), prog, 40).numpy()
    st = R.initial_state(prog, fields=fields)
    for n in (7, 1, 13, 19):
        R.run_steps(st, prog, n, chunk=5)
    two = st.numpy()
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(one[c], two[c])
    np.testing.assert_array_equal(one["dft_im"], two["dft_im"])
    assert one["step"] == two["step"] == 40


def test_deterministic_across_runs():
    spec = scenario_3d(grid=(10, 30, 41), seed=11, nsteps=8)
    fields = random_initial_fields(spec, seed=12)
    prog = R.compile_program(spec, schedule="fused", z_chunk=4)
    a = R.run_steps(R.initial_state(prog, fields=fields), prog, 8).numpy()
    b = R.run_steps(R.initial_state(prog, fields=fields), prog, 8).numpy()
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(a[c], b[c])


def test_fp64_error_is_reported_and_small():
    """The FP32 CUDA result against the FP64 oracle (reported, loose bound)."""
    spec = scenario_3d(grid=(10, 12, 14), seed=13, nsteps=30)
    prog = R.compile_program(spec)
    out = R.run_steps(R.initial_state(prog), prog, 30).numpy()
    oprog = to_oracle(spec, np.float64)
    st = O.run(oracle_state(oprog, dtype=np.float64), oprog, 30)
    for c in ("Ex", "Ey", "Ez"):
        assert O.relative_l2(out[c], st.fields[c]) <= 1e-4


BITWISE_CASES = {
    "3d_cpml_sources_pec": lambda: scenario_3d(grid=(9, 12, 40), seed=3, nsteps=4, metallic=("front", "left")),
    "3d_cpml_face_column": lambda: scenario_3d(grid=(10, 17, 64), seed=5, nsteps=4, metallic=("right",)),
    "2d_tm": lambda: scenario_2d(grid=(17, 23), polarization="tm", nsteps=4),
    "2d_te": lambda: scenario_2d(grid=(17, 23), polarization="te", nsteps=4),
}


@pytest.mark.parametrize("case", sorted(BITWISE_CASES))
@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_fields_are_bit_identical_to_the_fp32_oracle(case, schedule):
    """Every field after 4 steps equals the float32 oracle bit for bit (each
    product and sum rounded once, in the reference's order); the DFT arena,
    whose phases come from CUDA's sincosf, stays within its tolerance."""
    spec = BITWISE_CASES[case]()
    fields = random_initial_fields(spec, seed=4)
    prog = R.compile_program(spec, schedule=schedule)
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 4).numpy()
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog, fields), oprog, 4)
    for c in P.active_components(spec.ndim, spec.polarization):
        np.testing.assert_array_equal(out[c], st.fields[c], err_msg=c)
    for mine, ref in ((out["dft_re"], st.dft_re), (out["dft_im"], st.dft_im)):
        assert O.relative_l2(mine, ref) <= DFT_TOL


WAVEFRONT_CASES = {
    "3d_pitched": (lambda: scenario_3d(grid=(12, 16, 40), seed=8, nsteps=40, metallic=("top",)), "fused"),
    "3d_dense": (lambda: scenario_3d(grid=(12, 16, 40), seed=8, nsteps=40, metallic=("top",)), "phases"),
    "2d_tm": (lambda: scenario_2d(grid=(31, 37), polarization="tm", nsteps=40), "fused"),
    "2d_te": (lambda: scenario_2d(grid=(31, 37), polarization="te", nsteps=40), "phases"),
}


@pytest.mark.parametrize("case", sorted(WAVEFRONT_CASES))
def test_wavefronts_from_zero_fields_are_bit_identical(case):
    """Fields grown from zero by the sources: ahead of each wavefront the
    values fall through the subnormal range, where the division of a tiny
    difference by the cell size must still round as the oracle's does."""
    build, schedule = WAVEFRONT_CASES[case]
    spec = build()
    prog = R.compile_program(spec, schedule=schedule)
    assert (prog.layout == "pitched") == (case == "3d_pitched")
    out = R.run_steps(R.initial_state(prog), prog, 40).numpy()
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog), oprog, 40)
    tiny = 0
    for c in P.active_components(spec.ndim, spec.polarization):
        np.testing.assert_array_equal(out[c], st.fields[c], err_msg=c)
        v = np.abs(st.fields[c])
        tiny += int(np.count_nonzero((v > 0) & (v < 2.0**-100)))
    assert tiny > 0  # the case reaches the tiny range


@pytest.mark.parametrize("graphs", [True, False])
def test_dft_sampling_beside_the_next_step_is_bit_identical(graphs):
    """Samples taken on a side stream while the next step runs give the same
    arena and fields, bit for bit, as samples taken in line, over two calls."""
    from beamz_b200 import workloads as W

    spec = W.scene_3d_512(total_steps=60, shape=(40, 48, 96), pml_cells=6)
    outs = []
    for overlap in (False, True):
        prog = R.compile_program(spec, dft_overlap=overlap, graphs=graphs)
        assert prog.dft_overlap == overlap
        st = R.initial_state(prog)
        R.run_steps(st, prog, 23)
        R.run_steps(st, prog, 18)
        st.check()
        outs.append(st.numpy())
    for key in ("dft_re", "dft_im", "dft_w", "Ey", "Hz"):
        np.testing.assert_array_equal(outs[1][key], outs[0][key], err_msg=key)
    assert np.abs(outs[1]["dft_re"]).max() > 0


@pytest.mark.parametrize("case", ["pitched", "dense3d", "tm", "te"])
def test_device_packed_gather_plans_equal_the_host_packing(case):
    """fdtd_pack_gather builds the [M, 6, K, P] plan (nonzero weights first,
    device-layout offsets) bit for bit as the host restatement does,
    including monitors of different sizes and zero weights between nonzero ones."""
    from beamz_b200 import workloads as W
    from tests.scenarios import pack_dft_monitors_host

    if case in ("pitched", "dense3d"):
        spec = W.scene_3d_512(total_steps=10, shape=(24, 40, 56), pml_cells=4, n_monitors=3, n_freqs=2)
        schedule = "fused" if case == "pitched" else "phases"
    else:
        spec = scenario_2d(grid=(17, 23), polarization=case, nsteps=10)
        schedule = "fused"
    mon = spec.monitors[0]
    w = [np.asarray(a, np.float32).copy() for a in mon.weights]
    for a in w:  # a zero between nonzero slots, so the reorder moves something
        if a.shape[1] > 2:
            a[::3, 0] = 0.0
    spec.monitors[0] = P.DftMonitorPlan(mon.freqs, mon.indices, w, mon.component_mask)
    prog = R.compile_program(spec, schedule=schedule)
    assert (prog.layout == "pitched") == (case == "pitched")
    idx, wts = pack_dft_monitors_host(spec.monitors, [prog.shapes[c] for c in P.COMPONENTS], prog._strides)
    np.testing.assert_array_equal(prog.arena.indices.cpu().numpy(), idx)
    np.testing.assert_array_equal(prog.arena.weights.cpu().numpy(), wts)


def test_device_voxel_histogram_counts_every_id():
    ids = np.random.default_rng(3).integers(0, 7, size=(33, 17, 29)).astype(np.uint8)
    ids[0, 0, :5] = 250
    got = R.voxel_histogram(torch.as_tensor(ids, device="cuda"), torch.device("cuda"))
    np.testing.assert_array_equal(got, np.bincount(ids.reshape(-1), minlength=256))


@pytest.mark.parametrize("dims", [3, 2])
def test_dft_step_batching_is_bit_identical(dims):
    """Samples buffered and flushed every few steps (and at every call's end)
    give the same arena, bit for bit, as per-step accumulation."""
    spec = (scenario_3d(grid=(9, 12, 40), seed=8, nsteps=37) if dims == 3
            else scenario_2d(grid=(17, 23), polarization="tm", nsteps=37))
    fields = random_initial_fields(spec, seed=2)
    outs = []
    for batch in (1, 8, 5, 16):
        prog = R.compile_program(spec, dft_batch=batch)
        st = R.initial_state(prog, fields=fields)
        R.run_steps(st, prog, 20)
        R.run_steps(st, prog, 17)
        outs.append(st.numpy())
    for out in outs[1:]:
        for key in ("dft_re", "dft_im", "dft_w"):
            np.testing.assert_array_equal(out[key], outs[0][key], err_msg=key)


@pytest.mark.parametrize("layout", ["pitched", "dense"])
def test_affine_dft_sampling_equals_the_gather_plan(layout):
    """Plane monitors on uniform coordinates get the affine form of their
    plans, and sampling through it (no plan read per point) gives the arena of
    the packed gather plan bit for bit."""
    from beamz_b200 import workloads as W

    spec = W.scene_3d_512(total_steps=40, shape=(28, 40, 128), pml_cells=4)
    outs = []
    for affine in (True, False):
        prog = R.compile_program(spec, schedule="fused" if layout == "pitched" else "phases")
        assert prog.dft_batch > 1
        flags = prog.arena.affine[..., 0].cpu().numpy()
        masks = prog.arena.masks.cpu().numpy()
        np.testing.assert_array_equal(flags, (masks != 0).astype(np.int32))  # every sampled plan
        if not affine:
            prog.arena.affine.zero_()  # the gather plans instead
        st = R.initial_state(prog)
        R.run_steps(st, prog, 21)
        R.run_steps(st, prog, 19)
        outs.append(st.numpy())
    for key in ("dft_re", "dft_im", "dft_w"):
        np.testing.assert_array_equal(outs[0][key], outs[1][key], err_msg=key)
    assert np.abs(outs[0]["dft_re"]).max() > 0


@pytest.mark.parametrize("pol", ["tm", "te"])
def test_2d_pre_e_sources_inside_the_fused_step(pol):
    """2D fused programs add pre-E sources to the staged E planes instead of
    the bank: overlapping boxes that cross tile edges (8-row, 32-column tiles)
    give the oracle's fields bit for bit, like the phase schedule."""
    import dataclasses

    base = scenario_2d(grid=(37, 70), polarization=pol, nsteps=12)
    rng = np.random.default_rng(8)
    comp = "Ez" if pol == "tm" else "Ey"
    extra = [P.SourcePlan(comp, "pre_e", (5, 20), rng.standard_normal((11, 30)).astype(np.float32),
                          rng.standard_normal(12).astype(np.float32)),
             P.SourcePlan(comp, "pre_e", (7, 25), rng.standard_normal((9, 14)).astype(np.float32),
                          rng.standard_normal(12).astype(np.float32))]
    if pol == "te":
        extra.append(P.SourcePlan("Ex", "pre_e", (15, 30), rng.standard_normal((2, 5)).astype(np.float32),
                                  rng.standard_normal(12).astype(np.float32)))
    spec = dataclasses.replace(base, sources=list(base.sources) + extra)
    fields = random_initial_fields(spec, seed=3)
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog, fields), oprog, 12)
    for schedule in ("fused", "phases"):
        prog = R.compile_program(spec, schedule=schedule)
        out = R.run_steps(R.initial_state(prog, fields=fields), prog, 12).numpy()
        for c in P.active_components(2, pol):
            np.testing.assert_array_equal(out[c], st.fields[c], err_msg=f"{schedule} {c}")
