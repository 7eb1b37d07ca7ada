"""Time-domain field recorders: the oracle's restatement against beamz's own
``_record_fields`` (``tests/golden/recorder.npz`` from
``tests/golden/make_recorder.py``), and the planner's recorder plans."""

from __future__ import annotations

import numpy as np
import pytest

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


# ---- C-ABI checks of recorder buffers (fake pointers, no device work) -------


def _program_with_recorder():
    from beamz_b200 import abi
    from tests.test_abi import _fake, _valid_program

    s = _valid_program()  # 3D 4 x 5 x 6 cells
    s.recorder_count = 1
    r = s.recorders[0]
    r.interval, r.capacity, r.component_count = 2, 3, 2
    r.components[0], r.components[1] = 1, 5       # Ey (5, 5, 7) whole; Hz gathered
    r.signs[0] = r.signs[1] = 1.0
    r.values[0] = _fake((3, 5 * 5 * 7))
    r.indices[1], r.weights[1] = _fake((4, 10), abi.FDTD_S32), _fake((4, 10))
    r.values[1] = _fake((3, 10))
    r.steps, r.times, r.count = _fake((3,), abi.FDTD_S32), _fake((3,)), _fake((2,), abi.FDTD_S32)
    return s, _fake, abi


def test_validate_accepts_recorders():
    import ctypes

    from beamz_b200 import abi

    s, _, _ = _program_with_recorder()
    assert abi.load_library().fdtd_validate(ctypes.byref(s)) == 0


@pytest.mark.parametrize("mutate", [
    lambda s, fk, abi: setattr(s.recorders[0], "interval", 0),
    lambda s, fk, abi: setattr(s, "recorder_count", 5),
    lambda s, fk, abi: s.recorders[0].components.__setitem__(0, 6),
    lambda s, fk, abi: s.recorders[0].values.__setitem__(0, fk((3, 5 * 5 * 6))),       # wrong whole size
    lambda s, fk, abi: s.recorders[0].values.__setitem__(1, fk((2, 10))),             # capacity mismatch
    lambda s, fk, abi: s.recorders[0].weights.__setitem__(1, abi.FdtdBuffer()),       # indices without weights
    lambda s, fk, abi: s.recorders[0].indices.__setitem__(1, fk((33, 10), abi.FDTD_S32)),  # K > 32
    lambda s, fk, abi: setattr(s.recorders[0], "count", fk((1,), abi.FDTD_S32)),
    lambda s, fk, abi: setattr(s.recorders[0], "steps", fk((3,))),                    # not S32
])
def test_validate_rejects_inconsistent_recorders(mutate):
    import ctypes

    s, fk, abi = _program_with_recorder()
    mutate(s, fk, abi)
    assert abi.load_library().fdtd_validate(ctypes.byref(s)) == 1
