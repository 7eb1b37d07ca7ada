"""The class step (FDTD_FLAG_CLASSES, the engine's 3D hot path) against the
float32 oracle: bit for bit in its default arithmetic, and within the
accuracy target (relative L2 <= 1e-5 for fields and CPML memories, <= 1e-4
for the DFT arena) with the opt-in tolerance arithmetic (FDTD_FLAG_FAST_MATH:
1/dx folded into the coefficients, fused multiply-adds) over short runs.
Grids are wide enough in x (>= 128 lattice points) that the straight tile
bodies run, with column X updated by the column kernel after the tiles (X a
multiple of 128) and with a partial last tile (X not a multiple)."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from beamz_b200 import abi  # noqa: E402
from beamz_b200 import plan as P  # noqa: E402
from beamz_b200 import runtime as R  # noqa: E402
from oracle import fdtd_oracle as O  # noqa: E402
from tests.scenarios import oracle_state, random_initial_fields, scenario_3d, to_oracle  # noqa: E402

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5
DFT_TOL = 1e-4

CASES = [
    dict(grid=(10, 20, 256), pml_cells=6),                                         # column X: the column kernel
    dict(grid=(9, 17, 300), pml_cells=5, metallic=("front", "left", "top")),       # partial last tile, PEC
    dict(grid=(12, 24, 130), pml_cells=4, metallic=("right", "bottom", "back")),
    dict(grid=(11, 16, 256), cpml_edges=(), metallic=("front", "back", "bottom", "top", "left", "right")),
    dict(grid=(13, 40, 128), cpml_edges=("left", "top", "back"), metallic=("right",)),
    dict(grid=(12, 40, 384), pml_cells=4),                                          # interior tiles
]


def _bitwise(gpu, st):
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(gpu[c], st.fields[c], err_msg=c)
    for ours, ref in ((gpu["psi_h"], st.psi_h), (gpu["psi_e"], st.psi_e)):
        for i, p in enumerate(ref):
            if p.size:
                np.testing.assert_array_equal(ours[i], p)


def _compare(gpu, st, tol=FIELD_TOL, dft_tol=DFT_TOL):
    for c in P.COMPONENTS:
        err = O.relative_l2(gpu[c], st.fields[c])
        assert err <= tol, f"{c}: rel L2 {err:.3e}"
    for name, ours, ref in (("psi_h", gpu["psi_h"], st.psi_h), ("psi_e", gpu["psi_e"], st.psi_e)):
        for i, p in enumerate(ref):
            if p.size:
                err = O.relative_l2(ours[i], p)
                assert err <= tol, f"{name}{i}: rel L2 {err:.3e}"
    if st.dft_re is not None and st.dft_re.size:
        assert O.relative_l2(gpu["dft_re"], st.dft_re) <= dft_tol
        assert O.relative_l2(gpu["dft_im"], st.dft_im) <= dft_tol
        np.testing.assert_allclose(gpu["dft_w"], st.dft_w, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("tile_y", [8, 4])
@pytest.mark.parametrize("z_chunk", [16, 4, 0])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_class_step_is_bit_identical_to_the_fp32_oracle(case, z_chunk, tile_y):
    nsteps = 12
    spec = scenario_3d(seed=case, nsteps=nsteps, **CASES[case])
    fields = random_initial_fields(spec, seed=case + 30)
    prog = R.compile_program(spec, z_chunk=z_chunk, tile=(128, tile_y), step_kernel="classes")
    assert prog.layout == "pitched" and prog.step_kernel == "classes" and prog.arithmetic == "exact"
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, nsteps).numpy()
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog, fields), oprog, nsteps)
    _bitwise(out, st)
    _compare(out, st)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_fast_math_within_tolerance_of_the_fp32_oracle(case):
    nsteps = 12
    spec = scenario_3d(seed=case, nsteps=nsteps, **CASES[case])
    fields = random_initial_fields(spec, seed=case + 30)
    prog = R.compile_program(spec, arithmetic="fast", step_kernel="classes")
    assert prog.arithmetic == "fast"
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, nsteps).numpy()
    oprog = to_oracle(spec)
    _compare(out, O.run(oracle_state(oprog, fields), oprog, nsteps))


@pytest.mark.parametrize("case", [0, 1, 5])
def test_class_step_from_zero_fields_with_sources(case):
    """Wavefronts grown from zero fields by the sources (the leading edges pass
    through the subnormal range) still bit for bit."""
    nsteps = 40
    spec = scenario_3d(seed=case + 7, nsteps=nsteps, **CASES[case])
    prog = R.compile_program(spec, step_kernel="classes")
    out = R.run_steps(R.initial_state(prog), prog, nsteps).numpy()
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog), oprog, nsteps)
    _bitwise(out, st)
    _compare(out, st)


@pytest.mark.parametrize("metallic", [(), ("right", "front", "top")])
def test_column_x_with_an_h_source_on_it(metallic):
    """The column kernel (x = X when X is a multiple of 128) applies H-timing
    sources on Hx there, the x = X wall and the CPML terms of the column, bit
    for bit, over chunks of several planes and rows."""
    nsteps = 10
    spec = scenario_3d(grid=(19, 41, 128), seed=11, pml_cells=4, nsteps=nsteps, metallic=metallic)
    rng = np.random.default_rng(5)
    nz, ny, nx = spec.grid_shape
    spec.sources.append(P.SourcePlan("Hx", "h", (3, 5, nx - 1), rng.standard_normal((9, 33, 2)).astype(np.float32),
                                     (rng.standard_normal(nsteps) * 1e-3).astype(np.float32)))
    fields = random_initial_fields(spec, seed=6)
    prog = R.compile_program(spec, step_kernel="classes")
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, nsteps).numpy()
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog, fields), oprog, nsteps)
    _bitwise(out, st)
    _compare(out, st)


def test_class_and_codebook_steps_agree_bitwise():
    spec = scenario_3d(seed=3, nsteps=20, **CASES[5])
    fields = random_initial_fields(spec, seed=9)
    a_prog = R.compile_program(spec, step_kernel="classes")
    b_prog = R.compile_program(spec, step_kernel="codebook")
    assert a_prog.step_kernel == "classes" and b_prog.step_kernel == "codebook"
    a = R.run_steps(R.initial_state(a_prog, fields=fields), a_prog, 20).numpy()
    b = R.run_steps(R.initial_state(b_prog, fields=fields), b_prog, 20).numpy()
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(a[c], b[c], err_msg=c)
    np.testing.assert_array_equal(a["dft_re"], b["dft_re"])


def test_fast_math_and_exact_steps_agree_within_tolerance():
    spec = scenario_3d(seed=3, nsteps=20, **CASES[5])
    fields = random_initial_fields(spec, seed=9)
    fast = R.compile_program(spec, arithmetic="fast", step_kernel="classes")
    exact = R.compile_program(spec, step_kernel="classes")
    assert fast.arithmetic == "fast" and exact.arithmetic == "exact"
    a = R.run_steps(R.initial_state(fast, fields=fields), fast, 20).numpy()
    b = R.run_steps(R.initial_state(exact, fields=fields), exact, 20).numpy()
    for c in P.COMPONENTS:
        assert O.relative_l2(a[c], b[c]) <= FIELD_TOL, c
    assert O.relative_l2(a["dft_re"], b["dft_re"]) <= DFT_TOL


def test_class_step_is_deterministic_and_chunk_invariant():
    spec = scenario_3d(seed=2, nsteps=9, **CASES[0])
    fields = random_initial_fields(spec, seed=3)
    outs = []
    for zc in (16, 16, 3):
        prog = R.compile_program(spec, z_chunk=zc, step_kernel="classes")
        outs.append(R.run_steps(R.initial_state(prog, fields=fields), prog, 9).numpy())
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(outs[0][c], outs[1][c], err_msg=c)
        np.testing.assert_array_equal(outs[0][c], outs[2][c], err_msg=c)


def test_bounded_wait_expiry_sets_the_status_and_the_context_stays_usable():
    """A test-only flag arms the first copy barrier of the pitched step without
    issuing its copies: every CTA's bounded wait runs out (2 ms), the kernel
    records the expiry in the status word and returns, nothing is left in
    flight; the host raises, and a following normal run is correct."""
    spec = scenario_3d(grid=(6, 9, 140), seed=3, nsteps=2, sources=False, monitors=False)
    stalled = R.compile_program(spec, graphs=False, wait_limit_ns=2_000_000, test_stall=True, step_kernel="classes")
    st = R.initial_state(stalled)
    R.run_steps(st, stalled, 1)
    torch.cuda.synchronize()
    with pytest.raises(abi.FdtdError):
        st.check()
    fields = random_initial_fields(spec, seed=4)
    prog = R.compile_program(spec, step_kernel="classes")
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 2).numpy()
    oprog = to_oracle(spec)
    _compare(out, O.run(oracle_state(oprog, fields), oprog, 2))
