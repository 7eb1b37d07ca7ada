"""S-parameter assembly against golden vectors from the reference's own
``s_parameters`` (tests/golden/make_sparams.py): wave selection by port axis
and direction, the incident floor, the ratios, the power balance and the
monitor-flux checks, bit for bit (float64 numpy on both sides)."""

from __future__ import annotations

import os

import numpy as np
import pytest

from beamz_b200 import sparameters as S
from tests.golden.make_sparams import CASES, DIAG_KEYS, FLUX_KEYS

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sparams.npz")


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_s_parameters_match_the_reference(case):
    tag, is_3d, ports, source, outputs, floor = case
    g = np.load(GOLDEN)
    specs = [S.PortSpec(name, axis, d) for name, axis, d in ports]
    waves = {name: {f"a_{br}": g[f"{tag}_{name}_a_{br}"] for br in ("plus", "minus")} for name, _a, _d in ports}
    flux = {name: g[f"{tag}_{name}_flux"] for name, _a, _d in ports}
    res = S.s_parameters(waves, specs, source, output_ports=outputs, frequencies=g[f"{tag}_freqs"],
                         min_incident_db=floor, is_3d=is_3d, monitor_flux=flux)
    names = [p[0] for p in ports] if outputs is None else list(outputs)
    assert sorted(res.s_matrix) == sorted((o, source) for o in names)
    for o in names:
        np.testing.assert_array_equal(res.s_matrix[(o, source)], g[f"{tag}_S_{o}_{source}"], err_msg=o)
    for key in DIAG_KEYS:
        np.testing.assert_array_equal(res.diagnostics[key], g[f"{tag}_{key}"], err_msg=key)
    for name, entry in res.diagnostics["monitor_flux_checks"].items():
        for key in FLUX_KEYS:
            np.testing.assert_array_equal(entry[key], g[f"{tag}_{name}_{key}"], err_msg=f"{name} {key}")
        assert entry["incident_wave"] == str(g[f"{tag}_{name}_incident"])
    # the planted weak incident sample is masked out
    if floor <= -40.0 and names:
        assert not res.diagnostics["valid_mask"].all()


def test_wave_selectors():
    """In 3D an x- or y-normal port's positive-axis wave is the minus branch;
    a "-" port swaps incident and scattered."""
    sel = S.wave_selectors
    assert sel(S.PortSpec("p", "x", "+"), True) == ("minus", "plus")
    assert sel(S.PortSpec("p", "y", "-"), True) == ("plus", "minus")
    assert sel(S.PortSpec("p", "z", "+"), True) == ("plus", "minus")
    assert sel(S.PortSpec("p", "x", "+"), False) == ("plus", "minus")
    with pytest.raises(ValueError):
        S.PortSpec("p", "w")
    with pytest.raises(ValueError):
        S.s_parameters({}, [S.PortSpec("a", "x")], "b", frequencies=[1.0])


@pytest.mark.parametrize("case", ["pu", "pw"])
def test_port_projection_matches_the_reference(case):
    """The 2D port projection after the mode solve (power normalisation, mode
    matrix, pseudo-inverse, sqrt-measure weighting) and the coefficient step,
    against the reference's ``_build_port_projection_2d`` run on the same
    seeded profiles (the pseudo-inverse is an SVD: 1e-12 relative)."""
    g = np.load(GOLDEN)
    dl = g[f"{case}_dl"]
    sign = -1.0 if case == "pu" else 1.0
    proj = S.port_projection(g[f"{case}_e"], g[f"{case}_h"], dl if dl.ndim else float(dl), sign)
    np.testing.assert_array_equal(proj["mode_matrix"], g[f"{case}_mode_matrix"])
    np.testing.assert_allclose(proj["pinv"], g[f"{case}_pinv"], rtol=1e-12, atol=0)
    assert proj["condition_number"] == pytest.approx(float(g[f"{case}_cond"]), rel=1e-12)
    assert ("projection_weights" in proj) == (case == "pw")
    n = g[f"{case}_e"].size
    field = g[f"{case}_field"]
    a_plus, a_minus = S.project_waves(proj, field[:n], field[n:])
    np.testing.assert_allclose([a_plus, a_minus], g[f"{case}_coeff"], rtol=1e-12, atol=0)


def test_monitor_projection_phase():
    f = np.array([1.9e14, 2.0e14])
    np.testing.assert_array_equal(S.monitor_projection_phase("Ez", f, 3e-17), np.ones(2))
    np.testing.assert_array_equal(S.monitor_projection_phase("Hy", f, 3e-17), np.exp(-1j * np.pi * f * 3e-17))
