"""Conductive 3D materials on the device: the dense per-site step (both
schedules) bit for bit against the oracle's restatement of beamz's CUDA form,
and within the field tolerance against its JAX form (see tests/test_lossy.py)."""

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
    assert prog.layout == "dense"
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
