"""Sponge absorbers on the device: a 3D scene whose only boundary is a
graded-conductivity sponge runs through the dense per-site step bit for bit
against the oracle (both schedules), and the sponge absorbs an outgoing
pulse that the bare box keeps."""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from beamz_b200 import plan as P  # noqa: E402
from beamz_b200 import runtime as R  # noqa: E402
from oracle import fdtd_oracle as O  # noqa: E402
from tests.scenarios import oracle_state, random_initial_fields  # noqa: E402
from tests.test_lossy import lossy_scene  # noqa: E402

pytestmark = pytest.mark.gpu

GRID = (14, 16, 22)
RES = 20e-9


def _sponge(sigma):
    return P.sponge_conductivity(GRID, RES, base_sigma=sigma, thickness=4 * RES)


@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_sponge_step_matches_the_oracle_bit_for_bit(schedule):
    spec, oprog, e_site, h_site, _ = lossy_scene(grid=GRID, seed=5, pml_cells=0, nsteps=12, sigma_of=_sponge)
    oprog.e_coeffs, oprog.h_coeffs_3d = e_site, h_site
    fields = random_initial_fields(spec, seed=3)
    prog = R.compile_program(spec, schedule=schedule)
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 12).numpy()
    st = O.run(oracle_state(oprog, fields), oprog, 12)
    for c in P.COMPONENTS:
        np.testing.assert_array_equal(out[c], st.fields[c], err_msg=c)
    assert O.relative_l2(out["dft_re"], st.dft_re) <= 1e-4


def _pulse_2d(sponge: bool):
    """The reference's pulse-convergence scene (80 x 80 vacuum at 10 cells per
    wavelength, an Ez pulse that ends at step 65) with a 1 um sponge on every
    edge in place of its CPML, or with no absorber at all."""
    from tests.test_termination_gpu import _pulse_scene

    spec = _pulse_scene(total=420)
    n = spec.grid_shape[0]
    sigma = P.sponge_conductivity((n, n), spec.resolution, thickness=1e-6) if sponge else np.zeros((n, n), np.float32)
    e, h, eps = P.lossy_site_coefficients_2d(np.ones((n, n), np.float32), sigma, spec.dt, "tm")
    return dataclasses.replace(spec, h_terms=[], e_terms=[], e_site=e, h_site=h, e_site_eps=eps)


@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_sponge_2d_step_matches_the_oracle_bit_for_bit(schedule):
    from tests.scenarios import to_oracle

    spec = _pulse_2d(True)
    prog = R.compile_program(spec, schedule=schedule)
    out = R.run_steps(R.initial_state(prog), prog, 90).numpy()
    oprog = to_oracle(spec)
    oprog.h_coeffs = spec.h_site
    st = O.run(O.new_state(oprog), oprog, 90)
    for c in ("Ez", "Hx", "Hy"):
        np.testing.assert_array_equal(out[c], st.fields[c], err_msg=c)
    assert O.relative_l2(out["dft_re"], st.dft_re) <= 1e-4


def test_sponge_absorbs_the_outgoing_pulse():
    """After the pulse, the bare box keeps its energy (lossless reflecting
    edges); the sponge drains it by orders of magnitude (the oracle gives
    6.5e-35 J against 1.4e-41 J at step 420)."""
    energy = {}
    for sponge in (False, True):
        spec = _pulse_2d(sponge)
        prog = R.compile_program(spec)
        energy[sponge] = R.field_diagnostics(R.run_steps(R.initial_state(prog), prog, 420), prog).energy
    assert energy[False] > 0.0
    assert energy[True] < 1e-4 * energy[False]
