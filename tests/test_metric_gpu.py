"""Axis-uniform and rectilinear grids on the device: the class step (3D voxel
programs, fused schedule) and the dense step kernels (phases, conductive
per-site material, 2D TM/TE) bit for bit against the oracle's metric form
(pinned to beamz's metric updates in tests/test_metric.py)."""

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
    assert prog.layout == ("pitched" if schedule == "fused" else "dense")
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


METRIC_CASES = [
    dict(grid=(10, 13, 128), metallic=("back", "top"), kind="rectilinear"),       # one full tile
    dict(grid=(9, 20, 150), metallic=("right", "bottom"), kind="rectilinear"),    # a partial last tile, PEC on x = X
    dict(grid=(28, 30, 140), metallic=("left", "front"), kind="axis_uniform", pml_cells=12),  # staged x psi
]


@pytest.mark.parametrize("tile_y", [8, 4])
@pytest.mark.parametrize("case", range(len(METRIC_CASES)))
def test_metric_class_step_matches_the_oracle_bit_for_bit(case, tile_y):
    """The class step with per-axis inverse distances: fields and CPML
    memories bit for bit over two chunked calls, the DFT arena within 1e-4."""
    kw = dict(METRIC_CASES[case])
    kind = kw.pop("kind")
    spec = with_metrics(scenario_3d(seed=case + 3, nsteps=14, **kw), kind, seed=case + 1)
    fields = random_initial_fields(spec, seed=case + 7)
    prog = R.compile_program(spec, tile=(128, tile_y))
    assert prog.layout == "pitched" and prog.step_kernel == "classes"
    st = R.initial_state(prog, fields=fields)
    R.run_steps(st, prog, 9)
    out = R.run_steps(st, prog, 5).numpy()
    ost = O.run(oracle_state(to_oracle(spec), fields), to_oracle(spec), 14)
    _assert_bitwise(out, ost, P.COMPONENTS)


def test_metric_programs_layouts():
    """Metric programs take the class step; the tolerance arithmetic and the
    codebook step carry no metrics, so those go to the dense step (and refuse
    the pitched layout when it is asked for)."""
    spec = with_metrics(scenario_3d(grid=(8, 9, 10), seed=1, nsteps=2))
    prog = R.compile_program(spec)
    assert prog.layout == "pitched" and prog.step_kernel == "classes"
    assert R.compile_program(spec, arithmetic="fast").layout == "dense"
    assert R.compile_program(spec, step_kernel="codebook").layout == "dense"
    with pytest.raises(ValueError, match="non-isotropic"):
        R.compile_program(spec, layout="pitched", step_kernel="codebook")
