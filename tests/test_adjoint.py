"""Adjoint step: exact transpose of the forward step, and gradients against
central finite differences."""

from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import pytest

from beamz_b200 import abi
from beamz_b200 import plan as P
from beamz_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _site_3d(shape, seed, pml=4, metallic=()):
    torch = _torch()
    from beamz_b200 import adjoint as A

    spec = W.scene_3d_512(total_steps=200, seed=seed, shape=shape, pml_cells=pml, n_monitors=1, n_freqs=2)
    eps = torch.as_tensor(spec.eps_table[spec.voxel_ids], device="cuda")
    coefs = A.eps_to_coefficients_3d(eps, spec.dt, P.EPS_0)
    spec = A.site_spec(spec, {c: v.cpu().numpy() for c, v in zip(("Ex", "Ey", "Ez"), coefs)})
    return dataclasses.replace(spec, metallic_edges=frozenset(metallic))


def _site_2d(shape, seed, metallic=()):
    spec = W.scene_2d(total_steps=300, seed=seed, shape=shape, pml_cells=6, n_monitors=1)
    return dataclasses.replace(spec, metallic_edges=frozenset(metallic))


def _dot(a_list, b_list):
    return sum(float(np.dot(a.detach().double().cpu().numpy().ravel(), b.detach().double().cpu().numpy().ravel()))
               for a, b in zip(a_list, b_list))


@pytest.mark.parametrize("case", ["2d", "2d_pec", "3d", "3d_pec", "2d_metric", "3d_metric"])
def test_adjoint_step_is_the_exact_transpose(case):
    """<lambda', A u> == <A^T lambda', u> over fields and CPML memories
    (isotropic and rectilinear grids)."""
    torch = _torch()
    from beamz_b200 import runtime as R
    from tests.scenarios import with_metrics

    metallic = ("left", "top", "front") if case.endswith("pec") else ()
    spec = _site_2d((40, 48), 3, metallic) if case.startswith("2d") else _site_3d((14, 20, 36), 4, 3, metallic)
    spec = dataclasses.replace(spec, sources=[], monitors=[])
    if case.endswith("metric"):
        spec = with_metrics(spec, "rectilinear", seed=2)
    fprog = R.compile_program(spec, schedule="fused", layout="dense")
    aprog = R.compile_program(spec, schedule="phases", layout="dense")
    rng = np.random.default_rng(11)
    active = P.active_components(spec.ndim, spec.polarization)
    fields = {c: rng.standard_normal(fprog.shapes[c]).astype(np.float32) for c in active}
    st = R.initial_state(fprog, fields=fields)
    for p in st.psi_h + st.psi_e:
        p.copy_(torch.as_tensor(rng.standard_normal(tuple(p.shape)).astype(np.float32)))
    u0 = [f.clone() for f in st.fields] + [p.clone() for p in st.psi_h + st.psi_e]
    R.run_steps(st, fprog, 1)
    u1 = list(st.fields) + list(st.psi_h + st.psi_e)

    lam = R.initial_state(aprog)
    for f in lam.fields:
        if f.numel():
            f.copy_(torch.as_tensor(rng.standard_normal(tuple(f.shape)).astype(np.float32)))
    for p in lam.psi_h + lam.psi_e:
        p.copy_(torch.as_tensor(rng.standard_normal(tuple(p.shape)).astype(np.float32)))
    l1 = [f.clone() for f in lam.fields] + [p.clone() for p in lam.psi_h + lam.psi_e]

    a = abi.FdtdAdjointStep()
    a.abi_version = abi.FDTD_ABI_VERSION
    a.step = 0
    keep = []
    for t in range(6):
        ec, hs = P.COMPONENTS[t // 2], P.COMPONENTS[(5, 4, 3, 5, 4, 3)[t]]
        if ec in active and hs in active:
            keep.append(torch.zeros(aprog.shapes[ec], device="cuda"))
            a.scratch_e[t] = abi.buffer_of(keep[-1])
        hc, es = P.COMPONENTS[3 + t // 2], P.COMPONENTS[(2, 1, 0, 2, 1, 0)[t]]
        if hc in active and es in active:
            keep.append(torch.zeros(aprog.shapes[hc], device="cuda"))
            a.scratch_h[t] = abi.buffer_of(keep[-1])
    s = aprog.fill(lam, 0)
    abi.check(aprog.lib.fdtd_adjoint_step(R._stream(aprog), ctypes.byref(s), ctypes.byref(a)), "adjoint")
    l0 = list(lam.fields) + list(lam.psi_h + lam.psi_e)
    lhs = _dot(l1, u1)
    rhs = _dot(l0, u0)
    assert abs(lhs - rhs) <= 2e-5 * (abs(lhs) + abs(rhs) + 1.0), (lhs, rhs)


def _richardson(objective, x, direction, h):
    """Central differences at h and h/2 combined to cancel the h^2 term."""
    torch = _torch()
    with torch.no_grad():
        def central(step):
            return (float(objective(x + step * direction)) - float(objective(x - step * direction))) / (2 * step)
        return (4.0 * central(h / 2) - central(h)) / 3.0


def _objective_2d(spec):
    """|sum_p w_p D_Ez(p, f1)|^2 at the line monitor, Gaussian port weights."""
    torch = _torch()
    mon = spec.monitors[0]
    npts = np.asarray(mon.indices[0]).shape[0]
    nf = len(mon.freqs)
    prof = np.exp(-0.5 * ((np.arange(npts) - npts / 2) / (npts / 8)) ** 2).astype(np.float32)
    w = torch.as_tensor(prof, device="cuda")
    ez = P.COMPONENT_INDEX["Ez"]

    def J(re, im):
        f = nf // 2
        sl = slice((ez * nf + f) * npts, (ez * nf + f + 1) * npts)
        o_re = (w * re[sl]).sum()
        o_im = (w * im[sl]).sum()
        return o_re * o_re + o_im * o_im

    return J


@pytest.mark.parametrize("grid", ["uniform", "rectilinear"])
def test_gradient_2d_matches_finite_differences(grid):
    torch = _torch()
    from beamz_b200 import adjoint as A
    from tests.scenarios import with_metrics

    ny = nx = 64
    spec = W.scene_2d(total_steps=420, seed=5, shape=(ny, nx), pml_cells=8, n_monitors=1)
    if grid != "uniform":
        spec = with_metrics(spec, grid, seed=4)
    box = ((24, 20), (40, 36))  # Ez sites (y, x), interior, clear of the absorber
    eps_bg = torch.full((ny, nx), W.OXIDE, device="cuda")
    gen = torch.Generator(device="cpu").manual_seed(0)
    rho = torch.rand((16, 16), generator=gen).cuda().requires_grad_(True)
    problem = A.AdjointProblem(spec, 420, box, checkpoint_every=50)
    J = _objective_2d(spec)

    def objective(r):
        eps = eps_bg.clone()
        eps[24:40, 20:36] = W.OXIDE + r * (W.SI - W.OXIDE)
        c = A.eps_to_coefficients_2d(eps, spec.dt, P.EPS_0)
        re, im = A.simulate(problem, [c])
        return J(re, im)

    val = objective(rho)
    val.backward()
    g = rho.grad.detach().clone()
    direction = torch.randn((16, 16), generator=gen).cuda()
    fd = _richardson(objective, rho, direction, 2e-2)
    ad = float((g * direction).sum())
    assert abs(fd - ad) <= 1e-3 * abs(fd), (fd, ad)


def test_gradient_3d_matches_finite_differences():
    torch = _torch()
    from beamz_b200 import adjoint as A

    shape = (20, 28, 40)
    spec = W.scene_3d_512(total_steps=260, seed=6, shape=shape, pml_cells=4, n_monitors=1, n_freqs=2)
    base = torch.as_tensor(spec.eps_table[spec.voxel_ids], device="cuda")
    coefs0 = A.eps_to_coefficients_3d(base, spec.dt, P.EPS_0)
    sspec = A.site_spec(spec, {c: v.cpu().numpy() for c, v in zip(("Ex", "Ey", "Ez"), coefs0)})
    box = ((7, 9, 12), (13, 19, 28))
    problem = A.AdjointProblem(sspec, 260, box, checkpoint_every=40)
    mon = spec.monitors[0]
    npts = max(np.asarray(ix).shape[0] for ix in mon.indices)
    nf = len(mon.freqs)
    gen = torch.Generator(device="cpu").manual_seed(1)
    w = torch.randn(npts, generator=gen).cuda()
    ey = P.COMPONENT_INDEX["Ey"]

    def objective(r):
        eps = base.clone()
        eps[8:12, 10:18, 13:27] = W.OXIDE + r * (W.SI - W.OXIDE)
        coefs = A.eps_to_coefficients_3d(eps, spec.dt, P.EPS_0)
        re, im = A.simulate(problem, coefs)
        sl = slice((ey * nf) * npts, (ey * nf + 1) * npts)
        o_re, o_im = (w * re[sl]).sum(), (w * im[sl]).sum()
        return o_re * o_re + o_im * o_im

    rho = torch.rand((4, 8, 14), generator=gen).cuda().requires_grad_(True)
    objective(rho).backward()
    g = rho.grad.detach().clone()
    direction = torch.randn((4, 8, 14), generator=gen).cuda()
    fd = _richardson(objective, rho, direction, 2e-2)
    ad = float((g * direction).sum())
    assert abs(fd - ad) <= 1e-3 * abs(fd), (fd, ad)


@pytest.mark.parametrize("dims", ["2d", "3d", "3d_metric"])
def test_recorded_curls_give_the_recomputed_gradient(dims):
    """The backward pass that reads the forward curl from H recorded over the
    box every step (no forward steps in the backward) returns the gradient of
    the checkpoint-and-recompute pass bit for bit."""
    torch = _torch()
    from beamz_b200 import adjoint as A

    gen = torch.Generator(device="cpu").manual_seed(3)
    if dims == "2d":
        spec = W.scene_2d(total_steps=300, seed=5, shape=(64, 64), pml_cells=8, n_monitors=1)
        nsteps, box = 300, ((24, 20), (40, 36))
        eps = torch.full((64, 64), W.OXIDE, device="cuda")
        eps[24:40, 20:36] = W.SI
        coefs = [A.eps_to_coefficients_2d(eps, spec.dt, P.EPS_0)]
    else:
        spec = _site_3d((20, 28, 40), 6)
        if dims == "3d_metric":
            from tests.scenarios import with_metrics

            spec = with_metrics(spec, "rectilinear", seed=5)
        nsteps, box = 200, ((7, 9, 12), (13, 19, 28))
        coefs = [torch.as_tensor(spec.e_site[c][1], device="cuda") for c in ("Ex", "Ey", "Ez")]
    grads = []
    for limit in (4 << 30, 0):
        problem = A.AdjointProblem(spec, nsteps, box, checkpoint_every=70, curl_store_bytes=limit)
        assert (problem.curl_record is not None) == (limit > 0)
        problem.set_coefficients(dict(zip(problem.e_active, coefs)))
        re, im = problem.forward()
        g_re = torch.randn(re.shape, generator=gen).cuda()
        g_im = torch.randn(im.shape, generator=gen).cuda()
        gen.manual_seed(3)
        grads.append(problem.backward(g_re, g_im))
    for c in grads[0]:
        assert float(grads[0][c].abs().max()) > 0
        np.testing.assert_array_equal(grads[0][c].cpu().numpy(), grads[1][c].cpu().numpy(), err_msg=c)
