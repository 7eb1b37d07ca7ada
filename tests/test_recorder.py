"""Time-domain field recorders: the oracle's restatement against beamz's own
``_record_fields`` (``tests/golden/recorder.npz`` from
``tests/golden/make_recorder.py``), and the planner's recorder plans."""

from __future__ import annotations

import numpy as np

from beamz_b200 import plan as P
from oracle import fdtd_oracle as O
from tests.golden.make_recorder import GRID, RECORDERS, STEPS
from tests.golden_io import load


def test_oracle_records_match_the_reference():
    d = load("recorder")
    recs = []
    for name, comps, signs, interval, capacity, plane in RECORDERS:
        idx = [d[f"{name}_idx_{c}"] for c in comps] if plane else None
        w = [d[f"{name}_w_{c}"] for c in comps] if plane else None
        recs.append(O.FieldRecorder(comps, interval, capacity, idx, w, signs))
    shapes = O.component_shapes(GRID)
    records = O.new_records(recs, shapes)
    for step in range(STEPS):
        fields = {c: d[f"step{step}_{c}"] for c in O.COMPONENTS}
        O.record_fields(recs, records, fields, step, d[f"step{step}_t"])
    for (name, comps, _signs, _i, capacity, plane), store in zip(RECORDERS, records):
        n = int(d[f"{name}_count"])
        assert store["count"] == n
        np.testing.assert_array_equal(store["steps"], d[f"{name}_steps"])
        np.testing.assert_array_equal(store["times"], d[f"{name}_times"])
        for q, c in enumerate(comps):
            want = d[f"{name}_values_{c}"].reshape(capacity, -1)
            if plane:  # beamz sums the slots with jnp.sum, the oracle in slot order
                np.testing.assert_allclose(store["values"][q], want, rtol=1e-6, atol=1e-7)
            else:
                np.testing.assert_array_equal(store["values"][q], want)


def test_recorder_plans():
    r = P.domain_recorder((4, 5, 6), ("Ex", "Hz"), interval=3, num_steps=10)
    assert r.capacity == 4 and r.shapes == ((5, 6, 6), (5, 5, 6)) and r.indices is None
    a, b = (np.arange(3) + 1.5) * 2e-8, (np.arange(4) + 1.25) * 2e-8
    p = P.plane_recorder((6, 7, 8), 2e-8, "x", 8.6e-8, a, b, ("Ey",), interval=2, num_steps=7)
    assert p.capacity == 4 and p.shapes == ((3, 4),)
    assert p.indices[0].shape[0] == 12 and np.allclose(p.weights[0].sum(axis=1), 1.0, atol=1e-6)
