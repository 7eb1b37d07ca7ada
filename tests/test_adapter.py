"""The beamz adapter (beamz_b200/beamz_adapter.py) on the pieces beamz's own
compile steps produce (``tests/golden/adapter.npz``, written by
``tests/golden/make_adapter.py`` from the reference's functions).

CPU: the adapter decodes beamz's packed lossless coefficients back to the
reference's per-site sources bit for bit, and maps CPML terms, batched slab
sources and packed DFT monitors onto the planner's structures.  GPU: a run
through ``run_program_steps`` equals the float32 oracle in beamz's CUDA-path
coefficient form bit for bit (fields, CPML memories, DFT arena), on the
pitched class step, and two chunked calls equal one call."""

from __future__ import annotations

from types import SimpleNamespace
from typing import NamedTuple

import numpy as np
import pytest

from beamz_b200 import beamz_adapter as A
from beamz_b200 import plan as P
from tests.golden_io import load

GOLD = load("adapter")


class PackedSlab(NamedTuple):  # field names of beamz's CpmlPackedSlabSpec
    axis: int
    low: int
    high: int
    shape: tuple
    logical_stop: int = -1


class Term(NamedTuple):  # field names of beamz's CpmlTerm
    component: str
    axis: int
    sign: float
    a: np.ndarray
    b: np.ndarray
    inv_kappa: np.ndarray
    slab: PackedSlab


class State(NamedTuple):  # the SimulationState fields the native entry reads and writes
    hx: np.ndarray
    hy: np.ndarray
    hz: np.ndarray
    ex: np.ndarray
    ey: np.ndarray
    ez: np.ndarray
    cpml_psi_h_terms: tuple
    cpml_psi_e_terms: tuple
    dft_vec_re: np.ndarray
    dft_vec_im: np.ndarray
    dft_weight_sum: np.ndarray
    t: np.float32
    current_step: np.int32


H_NAMES = ("Hx", "Hx", "Hy", "Hy", "Hz", "Hz")
E_NAMES = ("Ex", "Ex", "Ey", "Ey", "Ez", "Ez")


def beamz_pieces():
    d = GOLD

    def terms(prefix, names):
        out = []
        for i, c in enumerate(names):
            axis, low, high, sign = (int(v) for v in d[f"{prefix}{i}_meta"])
            out.append(Term(c, axis, float(sign), d[f"{prefix}{i}_a"], d[f"{prefix}{i}_b"], d[f"{prefix}{i}_k"],
                            PackedSlab(axis, low, high, tuple(int(v) for v in d[f"{prefix}{i}_shape"]))))
        return out

    h_terms, e_terms = terms("h", H_NAMES), terms("e", E_NAMES)
    ctx = SimpleNamespace(
        dt=float(d["dt"]), resolution=float(d["res"]), metrics=None,
        config=SimpleNamespace(metric_kind="isotropic_uniform", cuda_flags=0, backend="cuda_streamed"),
        boundary=SimpleNamespace(cpml=SimpleNamespace(enabled=True, metallic_edges=frozenset(str(v) for v in d["metallic"]),
                                                      h_terms=h_terms, e_terms=e_terms)))
    coeffs = SimpleNamespace(**{k[5:]: d[k] for k in d if k.startswith("coef_")})
    groups = tuple(
        SimpleNamespace(coeffs=d[f"g{g}_coeffs"], waveforms=d[f"g{g}_waves"], starts=d[f"g{g}_starts"],
                        n=int(d[f"g{g}_coeffs"].shape[0])) if f"g{g}_coeffs" in d else None
        for g in range(9))
    packed = tuple(d[f"pk_{n}"] for n in ("indices", "weights", "freqs", "masks", "counts", "codes", "windows"))
    grid = tuple(int(v) for v in d["grid"])
    shapes = {c: P.component_shape(c, grid) for c in P.COMPONENTS}
    rng = np.random.default_rng(3)
    f = {c: (rng.standard_normal(shapes[c]) * (1.0 if c[0] == "E" else 1 / 376.73)).astype(np.float32)
         for c in P.COMPONENTS}
    nv = int(sum(6 * c[0] * c[1] for c in packed[4]))
    nw = int(sum(c[0] for c in packed[4]))
    state = State(f["Hx"], f["Hy"], f["Hz"], f["Ex"], f["Ey"], f["Ez"],
                  tuple(np.zeros(t.slab.shape, np.float32) for t in h_terms),
                  tuple(np.zeros(t.slab.shape, np.float32) for t in e_terms),
                  np.zeros(nv, np.float32), np.zeros(nv, np.float32), np.zeros(nw, np.float32),
                  np.float32(0.0), np.int32(0))
    return state, ctx, coeffs, groups, packed


def test_packed_lossless_coefficients_decode_to_the_reference_sources():
    state, ctx, coeffs, groups, packed = beamz_pieces()
    grid = A.grid_shape(state)
    shapes = {c: P.component_shape(c, grid) for c in P.COMPONENTS}
    e_site = A.e_site_coefficients(coeffs, shapes)
    for c in ("Ex", "Ey", "Ez"):
        dec, src = e_site[c]
        assert np.float32(dec) == np.float32(1.0)
        np.testing.assert_array_equal(src, GOLD[f"src_{c}"], err_msg=c)


def test_program_spec_maps_terms_sources_and_monitors():
    state, ctx, coeffs, groups, packed = beamz_pieces()
    spec = A.program_spec(state, ctx, coeffs, groups, packed, total_steps=24)
    assert spec.grid_shape == tuple(int(v) for v in GOLD["grid"])
    assert spec.metallic_edges == frozenset({"front"})
    for ours, theirs in zip(spec.h_terms + spec.e_terms, ctx.boundary.cpml.h_terms + ctx.boundary.cpml.e_terms):
        assert (ours.component, ours.axis, ours.sign, ours.low, ours.high) == (
            theirs.component, theirs.axis, theirs.sign, theirs.slab.low, theirs.slab.high)
        np.testing.assert_array_equal(ours.a, np.ravel(theirs.a))
        np.testing.assert_array_equal(ours.inv_kappa, np.ravel(theirs.inv_kappa))
    # The two pre-E Ey slabs were batched into one group by beamz; they come back as two sources.
    assert [(s.component, s.timing, s.start) for s in spec.sources] == [
        ("Ey", "pre_e", (4, 9, 60)), ("Ey", "pre_e", (5, 10, 61)), ("Hz", "h", (2, 3, 30)), ("Ex", "e", (0, 1, 110))]
    assert len(spec.monitors) == 2
    counts = packed[4]
    for m, mon in enumerate(spec.monitors):
        nf, npt = int(counts[m][0]), int(counts[m][1])
        assert mon.points == npt and mon.freqs.shape == (nf,)
        for c in range(6):
            np.testing.assert_array_equal(mon.indices[c], packed[0][m, c, :npt])
    assert (spec.monitors[1].window_code, spec.monitors[1].normalization_code) == (1, 1)
    h = spec.h_coefficients()
    assert all(np.ndim(v) == 0 for pair in h.values() for v in pair)


@pytest.mark.gpu
def test_run_program_steps_matches_the_oracle_bitwise():
    pytest.importorskip("torch")
    from oracle import fdtd_oracle as O
    from oracle.from_spec import oracle_program

    state, ctx, coeffs, groups, packed = beamz_pieces()
    nsteps = int(GOLD["nsteps"])
    out = A.run_program_steps(state, ctx, coeffs, groups, packed, nsteps, step_kernel="classes")
    prog = A.compile_program(state, ctx, coeffs, groups, packed, total_steps=nsteps, step_kernel="classes")
    assert prog.layout == "pitched" and prog.step_kernel == "classes"
    spec = A.program_spec(state, ctx, coeffs, groups, packed, total_steps=nsteps)
    oprog = oracle_program(spec)
    st = O.new_state(oprog)
    for c, name in A._STATE_FIELDS:
        st.fields[c] = np.asarray(getattr(state, name)).copy()
    st = O.run(st, oprog, nsteps)
    for c, name in A._STATE_FIELDS:
        np.testing.assert_array_equal(getattr(out, name), st.fields[c], err_msg=c)
    for ours, ref in zip(out.cpml_psi_h_terms + out.cpml_psi_e_terms, st.psi_h + st.psi_e):
        np.testing.assert_array_equal(ours, ref)
    assert O.relative_l2(out.dft_vec_re, st.dft_re) <= 1e-6
    assert O.relative_l2(out.dft_vec_im, st.dft_im) <= 1e-6
    np.testing.assert_array_equal(out.dft_weight_sum, st.dft_w)
    assert int(out.current_step) == nsteps and np.float32(out.t) == np.float32(st.t)


@pytest.mark.gpu
def test_chunked_calls_equal_one_call():
    pytest.importorskip("torch")
    state, ctx, coeffs, groups, packed = beamz_pieces()
    one = A.run_program_steps(state, ctx, coeffs, groups, packed, 24)
    half = A.run_program_steps(state, ctx, coeffs, groups, packed, 10)
    two = A.run_program_steps(half, ctx, coeffs, groups, packed, 14)
    for name in ("hx", "hy", "hz", "ex", "ey", "ez", "dft_vec_re", "dft_vec_im", "dft_weight_sum"):
        np.testing.assert_array_equal(getattr(two, name), getattr(one, name), err_msg=name)
    for a, b in zip(two.cpml_psi_h_terms + two.cpml_psi_e_terms, one.cpml_psi_h_terms + one.cpml_psi_e_terms):
        np.testing.assert_array_equal(a, b)
