"""Axis-uniform and rectilinear grids on the device: the dense step kernels
(both schedules, 3D voxel and conductive per-site material, 2D TM/TE) bit for
bit against the oracle's metric form (pinned to beamz's metric updates in
tests/test_metric.py)."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from beamz_b200 import plan as P  # noqa: E402
from beamz_b200 import runtime as R  # noqa: E402
from oracle import fdtd_oracle as O  # noqa: E402
from tests.scenarios import (oracle_state, random_initial_fields, scenario_2d, scenario_3d, to_oracle,  # noqa: E402
                             with_metrics)

pytestmark = pytest.mark.gpu


def _assert_bitwise(out, st, comps):
    for c in comps:
        np.testing.assert_array_equal(out[c], st.fields[c], err_msg=c)
    for a, b in zip(out["psi_h"] + out["psi_e"], st.psi_h + st.psi_e):
        np.testing.assert_array_equal(a, b)
    if st.dft_re.size:
        assert O.relative_l2(out["dft_re"], st.dft_re) <= 1e-4
        assert O.relative_l2(out["dft_im"], st.dft_im) <= 1e-4


@pytest.mark.parametrize("kind", ["rectilinear", "axis_uniform"])
@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_metric_3d_step_matches_the_oracle_bit_for_bit(schedule, kind):
    base = scenario_3d(grid=(10, 13, 37), seed=6, metallic=("back", "top"), nsteps=10)
    spec = with_metrics(base, kind, seed=1)
    fields = random_initial_fields(spec, seed=4)
    prog = R.compile_program(spec, schedule=schedule)
    assert prog.layout == "dense"
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 10).numpy()
    st = O.run(oracle_state(to_oracle(spec), fields), to_oracle(spec), 10)
    _assert_bitwise(out, st, P.COMPONENTS)
    # and the metric mattered: the isotropic program ends elsewhere
    iso = R.compile_program(base, schedule=schedule, layout="dense")
    other = R.run_steps(R.initial_state(iso, fields=fields), iso, 10).numpy()
    assert not np.array_equal(other["Ey"], out["Ey"])


@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_metric_lossy_3d_step_matches_the_cuda_form(schedule):
    from tests.test_lossy import lossy_scene

    spec, oprog, e_site, h_site, _ = lossy_scene(nsteps=12, seed=2)
    spec = with_metrics(spec, "rectilinear", seed=3)
    oprog.metrics = spec.metrics.as_dict()
    oprog.e_coeffs, oprog.h_coeffs_3d = e_site, h_site
    fields = random_initial_fields(spec, seed=9)
    prog = R.compile_program(spec, schedule=schedule)
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 12).numpy()
    st = O.run(oracle_state(oprog, fields), oprog, 12)
    _assert_bitwise(out, st, P.COMPONENTS)


@pytest.mark.parametrize("pol", ["tm", "te"])
@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_metric_2d_step_matches_the_oracle_bit_for_bit(pol, schedule):
    spec = with_metrics(scenario_2d(grid=(19, 26), polarization=pol, metallic=("left",), nsteps=14), seed=5)
    fields = random_initial_fields(spec, seed=8)
    prog = R.compile_program(spec, schedule=schedule)
    out = R.run_steps(R.initial_state(prog, fields=fields), prog, 14).numpy()
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog, fields), oprog, 14)
    _assert_bitwise(out, st, P.active_components(2, pol))


def test_metric_programs_take_the_dense_layout():
    spec = with_metrics(scenario_3d(grid=(8, 9, 10), seed=1, nsteps=2))
    assert R.compile_program(spec).layout == "dense"
    with pytest.raises(ValueError, match="isotropic"):
        R.compile_program(spec, layout="pitched")
