"""The C restatement (CPU baseline) against the numpy oracle."""

from __future__ import annotations

import numpy as np
import pytest

from beamz_b200 import plan as P
from oracle import cpu_port
from oracle import fdtd_oracle as O
from tests.scenarios import oracle_state, random_initial_fields, scenario_2d, scenario_3d, to_oracle


@pytest.mark.parametrize("kw", [dict(grid=(9, 10, 11)), dict(grid=(7, 13, 5), metallic=("front", "top", "left")),
                                dict(grid=(10, 35, 9), cpml_edges=("left", "top", "back"), metallic=("right",))])
def test_c_port_matches_oracle_3d(kw):
    spec = scenario_3d(nsteps=9, **kw)
    fields = random_initial_fields(spec, seed=4)
    run = cpu_port.HostRun(spec, fields).run(9, threads=2)
    prog = to_oracle(spec)
    st = O.run(oracle_state(prog, fields), prog, 9)
    for c in P.COMPONENTS:
        assert O.relative_l2(run.fields[c], st.fields[c]) <= 1e-6, c
    assert O.relative_l2(run.dft_re, st.dft_re) <= 1e-5
    np.testing.assert_allclose(run.dft_w, st.dft_w, rtol=1e-6)


@pytest.mark.parametrize("pol", ["tm", "te"])
def test_c_port_matches_oracle_2d(pol):
    spec = scenario_2d(grid=(17, 23), polarization=pol, metallic=("left",), nsteps=15)
    fields = random_initial_fields(spec, seed=5)
    run = cpu_port.HostRun(spec, fields).run(15, threads=2)
    prog = to_oracle(spec)
    st = O.run(oracle_state(prog, fields), prog, 15)
    for c in P.active_components(2, pol):
        assert O.relative_l2(run.fields[c], st.fields[c]) <= 1e-6, c
    assert O.relative_l2(run.dft_im, st.dft_im) <= 1e-5
