"""fdtd_adjoint_step_noalloc against fdtd_adjoint_step (collected last):
bit for bit over two consecutive adjoint steps, on a 2D TM program and on a
3D program with CPML on every face and a DFT plane."""

from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import pytest

from beamz_b200 import abi
from beamz_b200 import plan as P
from beamz_b200 import workloads as W

pytestmark = pytest.mark.gpu

_E_SRC = (5, 4, 3, 5, 4, 3)
_H_SRC = (2, 1, 0, 2, 1, 0)


def _adjoint_state(prog, seed):
    import torch

    from beamz_b200 import runtime as R

    rng = np.random.default_rng(seed)
    lam = R.initial_state(prog)
    for t in list(lam.fields) + list(lam.psi_h) + list(lam.psi_e):
        if t.numel():
            t.copy_(torch.as_tensor(rng.standard_normal(tuple(t.shape)).astype(np.float32)))
    return lam


def _step(prog, n, scratch, g):
    a = abi.FdtdAdjointStep()
    a.abi_version = abi.FDTD_ABI_VERSION
    a.step = n
    if scratch is not None:
        for t, buf in scratch["e"].items():
            a.scratch_e[t] = abi.buffer_of(buf)
        for t, buf in scratch["h"].items():
            a.scratch_h[t] = abi.buffer_of(buf)
    a.dft_grad_re = abi.buffer_of(g[0])
    a.dft_grad_im = abi.buffer_of(g[1])
    return a


def _spec(kind):
    if kind == "2d":
        spec = W.scene_2d(total_steps=64, seed=9, shape=(72, 80), pml_cells=6, n_monitors=2)
        return dataclasses.replace(spec, metallic_edges=frozenset({"bottom", "right"}))
    # 3D: all twelve derivative terms live, CPML on every axis (psi transposed
    # on all three), Ex/Ey/Ez of different extents, a DFT plane.
    import torch

    from beamz_b200 import adjoint as AD

    spec = W.scene_3d_512(total_steps=64, seed=3, shape=(22, 24, 26), pml_cells=4, n_monitors=1, n_freqs=3)
    eps = torch.as_tensor(np.asarray(spec.eps_table, np.float32)[spec.voxel_ids])
    coefs = AD.eps_to_coefficients_3d(eps, spec.dt, P.EPS_0)
    spec = AD.site_spec(spec, {c: v.cpu().numpy() for c, v in zip(("Ex", "Ey", "Ez"), coefs)})
    return dataclasses.replace(spec, metallic_edges=frozenset({"front"}))


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_noalloc_adjoint_step_matches_the_allocating_entry_point(kind):
    import torch

    from beamz_b200 import runtime as R

    spec = _spec(kind)
    prog = R.compile_program(spec, schedule="phases", layout="dense")
    active = P.active_components(spec.ndim, spec.polarization)
    scratch = {"e": {}, "h": {}}
    for t in range(6):
        ec, hs = P.COMPONENTS[t // 2], P.COMPONENTS[_E_SRC[t]]
        if ec in active and hs in active:
            scratch["e"][t] = torch.zeros(prog.shapes[ec], device="cuda")
        hc, es = P.COMPONENTS[3 + t // 2], P.COMPONENTS[_H_SRC[t]]
        if hc in active and es in active:
            scratch["h"][t] = torch.zeros(prog.shapes[hc], device="cuda")
    rng = np.random.default_rng(4)
    n_arena = prog.arena.value_count
    g = (torch.as_tensor(rng.standard_normal(n_arena).astype(np.float32), device="cuda"),
         torch.as_tensor(rng.standard_normal(n_arena).astype(np.float32), device="cuda"))
    ref = _adjoint_state(prog, 7)
    out = _adjoint_state(prog, 7)
    stream = R._stream(prog)
    for n in (40, 39):  # two calls in a row
        a = _step(prog, n, scratch, g)
        s = prog.fill(ref, 0)
        abi.check(prog.lib.fdtd_adjoint_step(stream, ctypes.byref(s), ctypes.byref(a)), "fdtd_adjoint_step")
        b = _step(prog, n, None, g)
        s = prog.fill(out, 0)
        abi.check(prog.lib.fdtd_adjoint_step_noalloc(stream, ctypes.byref(s), ctypes.byref(b)),
                  "fdtd_adjoint_step_noalloc")
        torch.cuda.synchronize()
        for x, y in zip(list(ref.fields) + ref.psi_h + ref.psi_e, list(out.fields) + out.psi_h + out.psi_e):
            assert torch.equal(x, y)


def test_noalloc_rejects_programs_beyond_its_scratch():
    from beamz_b200 import runtime as R

    spec = W.scene_2d(total_steps=4, seed=1, shape=(1100, 1100), pml_cells=6, n_monitors=1)
    prog = R.compile_program(spec, schedule="phases", layout="dense")
    lam = R.initial_state(prog)
    a = abi.FdtdAdjointStep()
    a.abi_version = abi.FDTD_ABI_VERSION
    s = prog.fill(lam, 0)
    assert prog.lib.fdtd_adjoint_step_noalloc(R._stream(prog), ctypes.byref(s), ctypes.byref(a)) == 1
