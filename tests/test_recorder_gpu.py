"""Field recorders on the device (fdtd_record_fields and the recorder launch
inside fdtd_launch_program) against the oracle's restatement of beamz's
_record_fields (pinned in tests/test_recorder.py): plane and whole-domain
recorders, a capacity that runs out, chunked runs, pitched and dense layouts."""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from beamz_b200 import plan as P  # noqa: E402
from beamz_b200 import runtime as R  # noqa: E402
from oracle import fdtd_oracle as O  # noqa: E402
from tests.scenarios import oracle_state, random_initial_fields, scenario_2d, scenario_3d, to_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def _with_recorders(spec, nsteps):
    g, res = spec.grid_shape, spec.resolution
    if spec.ndim == 3:
        a = (np.arange(g[0] - 2) + 1.5) * res
        b = (np.arange(g[1] - 3) + 1.25) * res
        recs = [P.plane_recorder(g, res, "x", 0.45 * g[2] * res, a, b, ("Ey", "Hz"), interval=3, num_steps=nsteps),
                P.domain_recorder(g, ("Ex", "Hy"), interval=4, num_steps=nsteps),
                dataclasses.replace(P.domain_recorder(g, ("Ez",), interval=1, num_steps=nsteps), capacity=5,
                                    signs=(-1.0,))]
    else:
        comps = P.active_components(2, spec.polarization)
        recs = [P.domain_recorder(g, comps, interval=2, num_steps=nsteps, polarization=spec.polarization)]
    return dataclasses.replace(spec, recorders=recs)


def _check(spec, out_state, prog, st):
    for r, rec in enumerate(spec.recorders):
        got = R.recorded(out_state, prog, r)
        store = st.records[r]
        n = store["count"]
        assert len(got["steps"]) == n
        np.testing.assert_array_equal(got["steps"], store["steps"][:n])
        np.testing.assert_array_equal(got["times"], store["times"][:n])
        for q, c in enumerate(rec.components):
            np.testing.assert_array_equal(got[c].reshape(n, -1), store["values"][q][:n], err_msg=f"{r} {c}")


@pytest.mark.parametrize("schedule", ["fused", "phases"])
def test_recorders_match_the_oracle(schedule):
    steps = 14
    spec = _with_recorders(scenario_3d(grid=(10, 13, 36), seed=2, nsteps=steps), steps)
    fields = random_initial_fields(spec, seed=5)
    prog = R.compile_program(spec, schedule=schedule)
    assert prog.layout == ("pitched" if schedule == "fused" else "dense")
    st_dev = R.run_steps(R.initial_state(prog, fields=fields), prog, steps, chunk=5)  # three graph chunks
    oprog = to_oracle(spec)
    st = O.run(oracle_state(oprog, fields), oprog, steps)
    assert [s["count"] for s in st.records] == [4, 3, 5]
    _check(spec, st_dev, prog, st)


def test_recorders_through_the_phase_entries():
    steps = 6
    spec = _with_recorders(scenario_3d(grid=(8, 9, 12), seed=3, nsteps=steps), steps)
    fields = random_initial_fields(spec, seed=6)
    prog = R.compile_program(spec, schedule="phases")
    st_dev = R.initial_state(prog, fields=fields)
    for _ in range(steps):
        R.step_by_phases(st_dev, prog)
    oprog = to_oracle(spec)
    _check(spec, st_dev, prog, O.run(oracle_state(oprog, fields), oprog, steps))


@pytest.mark.parametrize("pol", ["tm", "te"])
def test_2d_domain_recorder(pol):
    steps = 9
    spec = _with_recorders(scenario_2d(grid=(15, 19), polarization=pol, nsteps=steps), steps)
    fields = random_initial_fields(spec, seed=7)
    prog = R.compile_program(spec)
    st_dev = R.run_steps(R.initial_state(prog, fields=fields), prog, steps)
    oprog = to_oracle(spec)
    _check(spec, st_dev, prog, O.run(oracle_state(oprog, fields), oprog, steps))
