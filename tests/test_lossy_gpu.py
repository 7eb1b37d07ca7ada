"""Conductive 3D materials on the device: the class step with (decay, source)
classes (fused schedule) and the dense per-site step (phases) bit for bit
against the oracle's restatement of beamz's CUDA form, and within the field
tolerance against its JAX form (see tests/test_lossy.py)."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from beamz_b200 import plan as P  # noqa: E402
from beamz_b200 import runtime as R  # noqa: E402
from oracle import fdtd_oracle as O  # noqa: E402
from tests.scenarios import oracle_state, random_initial_fields  # noqa: E402
from tests.test_lossy import assert_family_close, lossy_scene  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_lossy_step_matches_the_cuda_form_bit_for_bit(schedule):
    spec, oprog, e_site, h_site, _ = lossy_scene(nsteps=12, seed=2)
    fields = random_initial_fields(spec, seed=9)
    prog = R.compile_program(spec, schedule=schedule)
    assert prog.layout == ("pitched" if schedule == "fused" else "dense")
    assert prog.lossy == (schedule == "fused")
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 12).numpy()
    jax_form = O.run(oracle_state(oprog, fields), oprog, 12)
    oprog.e_coeffs, oprog.h_coeffs_3d = e_site, h_site
    cuda_form = O.run(oracle_state(oprog, fields), oprog, 12)
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(out[c], cuda_form.fields[c], err_msg=c)
    for a, b in zip(out["psi_h"] + out["psi_e"], cuda_form.psi_h + cuda_form.psi_e):
        np.testing.assert_array_equal(a, b)
    assert O.relative_l2(out["dft_re"], cuda_form.dft_re) <= 1e-4
    assert_family_close(out, jax_form.fields, 1e-5)


LOSSY_CASES = [
    dict(grid=(9, 12, 128), metallic=()),                   # one full tile, column X by the column kernel
    dict(grid=(10, 14, 150), metallic=("right", "top")),    # a partial last tile, PEC on x = X
    dict(grid=(8, 20, 256), metallic=("left", "front")),
]


@pytest.mark.parametrize("tile_y", [8, 4])
@pytest.mark.parametrize("case", range(len(LOSSY_CASES)))
def test_lossy_class_step_matches_the_cuda_form_bit_for_bit(case, tile_y):
    """The class step with E and H (decay, source) classes: fields and CPML
    memories of beamz's CUDA form bit for bit over two chunked calls, the DFT
    arena within 1e-4."""
    spec, oprog, e_site, h_site, _ = lossy_scene(nsteps=14, seed=case + 11, **LOSSY_CASES[case])
    fields = random_initial_fields(spec, seed=case + 4)
    prog = R.compile_program(spec, tile=(128, tile_y))
    assert prog.lossy and prog.step_kernel == "classes" and prog.layout == "pitched"
    st = R.initial_state(prog, fields=fields)
    R.run_steps(st, prog, 9)
    out = R.run_steps(st, prog, 5).numpy()
    oprog.e_coeffs, oprog.h_coeffs_3d = e_site, h_site
    ref = O.run(oracle_state(oprog, fields), oprog, 14)
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(out[c], ref.fields[c], err_msg=c)
    for a, b in zip(out["psi_h"] + out["psi_e"], ref.psi_h + ref.psi_e):
        np.testing.assert_array_equal(a, b)
    assert O.relative_l2(out["dft_re"], ref.dft_re) <= 1e-4  # device phases: sincosf
    assert O.relative_l2(out["dft_im"], ref.dft_im) <= 1e-4


def test_lossy_classes_fall_back_to_the_dense_step():
    """More (decay, source) classes than the class step's tables hold: the
    dense per-site step runs instead, with the same result."""
    rng = np.random.default_rng(1)
    spec, oprog, e_site, h_site, _ = lossy_scene(
        grid=(8, 10, 24), nsteps=6, seed=2, sigma_of=lambda s: rng.uniform(0.0, 5e4, s.shape).astype(np.float32))
    prog = R.compile_program(spec)
    assert not prog.lossy and prog.layout == "dense"
    fields = random_initial_fields(spec, seed=3)
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 6).numpy()
    oprog.e_coeffs, oprog.h_coeffs_3d = e_site, h_site
    ref = O.run(oracle_state(oprog, fields), oprog, 6)
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(out[c], ref.fields[c], err_msg=c)


def test_lossy_fields_decay_faster_than_lossless():
    """Sanity of the physics: the same scene without its conductivity keeps
    more field energy after the pulse."""
    import dataclasses

    spec, _, _, _, (eps, _sigma) = lossy_scene(nsteps=60, seed=3)
    prog = R.compile_program(spec)
    lossy = R.field_diagnostics(R.run_steps(R.initial_state(prog), prog, 60), prog).energy
    e0, h0, ee0 = P.lossy_site_coefficients_3d(eps, np.zeros(spec.grid_shape, np.float32), spec.dt)
    plain = dataclasses.replace(spec, e_site=e0, h_site=h0, e_site_eps=ee0)
    prog0 = R.compile_program(plain)
    lossless = R.field_diagnostics(R.run_steps(R.initial_state(prog0), prog0, 60), prog0).energy
    assert 0.0 < lossy < lossless


@pytest.mark.parametrize("pol", ["tm", "te"])
@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_lossy_2d_step_matches_the_oracle_bit_for_bit(pol, schedule):
    from tests.test_lossy import lossy_scene_2d

    spec, oprog = lossy_scene_2d(polarization=pol, seed=4)
    fields = random_initial_fields(spec, seed=10)
    prog = R.compile_program(spec, schedule=schedule)
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 12).numpy()
    st = O.run(oracle_state(oprog, fields), oprog, 12)
    for c in P.active_components(2, pol):
        np.testing.assert_array_equal(out[c], st.fields[c], err_msg=c)
    assert O.relative_l2(out["dft_re"], st.dft_re) <= 1e-4
