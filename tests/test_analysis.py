"""Monitor analysis: the oracle's DFT flux and modal overlap against beamz's
own functions (``tests/golden/analysis.npz`` from
``tests/golden/make_analysis.py``: observe.py:166-234 and
devices/modes/fields.py:76-129)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import fdtd_oracle as O
from tests.golden.make_analysis import FLUX_CASES, OVERLAP_CASES
from tests.golden_io import load


@pytest.mark.parametrize("case", FLUX_CASES, ids=[c[0] for c in FLUX_CASES])
def test_monitor_flux_matches_the_reference(case):
    tag, axis, sign, base_dt, with_iw = case
    d = load("analysis")
    fields = {c: O.flux_component(d[f"{tag}_re"][i] + 1j * d[f"{tag}_im"][i].astype(np.float64),
                                  d[f"{tag}_wsum"], c, d[f"{tag}_freqs"], base_dt)
              for i, c in enumerate(O.COMPONENTS)}
    got = O.monitor_dft_flux(fields, axis, sign, d[f"{tag}_iw"] if with_iw else None,
                             measure=float(d[f"{tag}_power_scale"]))
    np.testing.assert_allclose(got, d[f"{tag}_flux"], rtol=1e-13, atol=0.0)


@pytest.mark.parametrize("case", OVERLAP_CASES, ids=[c[0] for c in OVERLAP_CASES])
def test_modal_overlap_matches_the_reference(case):
    tag, axis, direction, kind = case
    d = load("analysis")
    names = O.TANGENTIAL_COMPONENTS[axis]
    fields = {c: d[f"{tag}_field_{c}"] for c in names}
    mode = {c: d[f"{tag}_mode_{c}"] for c in names}
    measure = ({c: d[f"{tag}_measure_{c}"] for c in names[:2]} if kind == "mapping"
               else d[f"{tag}_measure"] if kind == "array" else float(d[f"{tag}_measure"]))
    got = O.modal_overlap(fields, mode, axis, measure, direction)
    want = complex(d[f"{tag}_overlap"])
    assert got == want  # same operations in the same order
