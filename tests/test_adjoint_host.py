"""Host logic of the adjoint's curl recording (no GPU): the recorder plan
reads H over the design box grown by one cell towards lower coordinates, and
the curls formed from a record equal fdtd_adjoint_curl's differences and
divisions (beamz/lattice.py Yee layout) evaluated directly."""

from __future__ import annotations

import types

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from beamz_b200 import adjoint as A  # noqa: E402
from beamz_b200.plan import active_components, component_shape  # noqa: E402


def _problem(ndim, grid, box, nsteps, pol="tm", metrics=None):
    """An AdjointProblem shell with the attributes the curl helpers read."""
    pr = object.__new__(A.AdjointProblem)
    lo, hi = box
    if ndim == 2:
        lo, hi = (0, *lo), (1, *hi)
    pr.box_lo, pr.box_hi = tuple(lo), tuple(hi)
    pr.box_shape = tuple(h - l for l, h in zip(pr.box_lo, pr.box_hi))
    pr.nsteps = nsteps
    pr.active = active_components(ndim, pol)
    pr.e_active = [c for c in ("Ex", "Ey", "Ez") if c in pr.active]
    pr.device = torch.device("cpu")
    spec = types.SimpleNamespace(ndim=ndim, grid_shape=grid, polarization=pol, recorders=[], resolution=2e-8,
                                 metrics=metrics)
    pr.spec = spec
    return pr, spec


def _curl_direct(h, c, k, j, i, res, me=(None, None, None)):
    """fdtd_adjoint_curl at E site (k, j, i) of component c, float32: each
    backward difference divided by the cell size, or times the metric."""
    r = np.float32(res)

    def sc(d, axis, at):
        return np.float32(d / r) if me[axis] is None else np.float32(d * me[axis][at])

    if c == 0:
        v = sc(h["Hz"][k, j, i] - h["Hz"][k, j - 1, i], 1, j)
        if "Hy" in h:
            v = v - sc(h["Hy"][k, j, i] - h["Hy"][k - 1, j, i], 0, k)
    elif c == 1:
        v = -sc(h["Hz"][k, j, i] - h["Hz"][k, j, i - 1], 2, i)
        if "Hx" in h:
            v = v + sc(h["Hx"][k, j, i] - h["Hx"][k - 1, j, i], 0, k)
    else:
        v = sc(h["Hy"][k, j, i] - h["Hy"][k, j, i - 1], 2, i) - sc(h["Hx"][k, j, i] - h["Hx"][k, j - 1, i], 1, j)
    return np.float32(v)


@pytest.mark.parametrize("ndim,pol,grid_kind", [(3, "tm", None), (2, "tm", None), (2, "te", None),
                                               (3, "tm", "rectilinear"), (2, "tm", "rectilinear")])
def test_recorded_curls_equal_the_curl_kernel_formula(ndim, pol, grid_kind):
    from beamz_b200.plan import derivative_metrics

    grid = (9, 10, 12) if ndim == 3 else (10, 12)
    box = ((2, 3, 4), (6, 8, 9)) if ndim == 3 else ((3, 4), (8, 9))
    metrics = None
    if grid_kind is not None:
        wrng = np.random.default_rng(9)
        axes = ("z", "y", "x") if ndim == 3 else ("y", "x")
        metrics = derivative_metrics({a: 2e-8 * wrng.uniform(1.0, 1.6, n) for a, n in zip(axes, grid)}, grid_kind)
    pr, spec = _problem(ndim, grid, box, nsteps=3, pol=pol, metrics=metrics)
    pr.curl_record = pr._curl_recorder(spec, 1 << 30)
    plan, margin, ext = pr.curl_record
    assert margin == ((1, 1, 1) if ndim == 3 else (0, 1, 1))
    rng = np.random.default_rng(4)
    fields = {}
    for c in plan.components:
        shape = component_shape(c, spec.grid_shape, pol)
        fields[c] = rng.standard_normal((3, *shape)).astype(np.float32)
    # the recorder's records: field[indices] for every step (weights are 1)
    values = [torch.as_tensor(np.stack([fields[c][s].reshape(-1)[plan.indices[q][:, 0]] for s in range(3)]))
              for q, c in enumerate(plan.components)]
    state = types.SimpleNamespace(records=[{"values": values}])
    curls = pr._curls(state, 0, 3)
    lo = pr.box_lo
    cells = (1, *grid) if ndim == 2 else grid
    me = [None, None, None]
    if metrics is not None:
        for a, name in enumerate(("z", "y", "x")):
            if ndim == 3 or a > 0:
                me[a] = metrics.along(f"h_to_e_{name}", cells[a] + 1)
    for ci, c in enumerate(("Ex", "Ey", "Ez")):
        if c not in pr.e_active:
            assert curls[ci] is None
            continue
        got = curls[ci].numpy()
        for s in range(3):
            h = {n: (fields[n][s] if ndim == 3 else fields[n][s][None]) for n in plan.components}
            for kb, jb, ib in np.ndindex(*pr.box_shape):
                want = _curl_direct(h, ci, lo[0] + kb, lo[1] + jb, lo[2] + ib, spec.resolution, me)
                assert got[s, kb, jb, ib] == want, (c, s, kb, jb, ib)


def test_curl_recording_falls_back_to_checkpoints():
    pr, spec = _problem(3, (9, 10, 12), ((2, 3, 4), (6, 8, 9)), nsteps=100)
    assert pr._curl_recorder(spec, 1 << 30) is not None
    assert pr._curl_recorder(spec, 1000) is None  # over the byte limit
    spec.recorders = [object()] * 4  # no recorder slot left
    assert pr._curl_recorder(spec, 1 << 30) is None
    pr2, spec2 = _problem(3, (9, 10, 12), ((0, 3, 4), (6, 8, 9)), nsteps=10)
    assert pr2._curl_recorder(spec2, 1 << 30) is None  # no plane below the box
