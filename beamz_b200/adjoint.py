"""Adjoint (time-reversed) FDTD and permittivity gradients.

:class:`AdjointProblem` runs one simulation forward and back-propagates
gradients of any function of its DFT arena to the per-site E update
coefficients c = dt / (eps0 eps_site) inside a design box:

* forward: the plain fused step (``run_steps``).  A field recorder in the
  forward program keeps H over the box (and a one-cell margin) after every
  step when that fits ``curl_store_bytes``; otherwise the forward saves
  (fields, CPML memories) every ``checkpoint_every`` steps;
* backward, from the last step: the curl of each active E component over the
  box comes from the recorded H (256 steps at a time), or, with checkpoints,
  segment by segment from the last: restore the checkpoint and recompute the
  segment's steps while ``fdtd_adjoint_curl`` stores the curl after every
  step (the same differences and divisions, so the same bits).  Then
  ``fdtd_adjoint_step`` runs for the steps in reverse.  Each adjoint step
  injects the DFT adjoint source of that step's sample, transposes the E and
  H updates exactly (CPML memories, ghost planes and metallic walls included)
  and accumulates dJ/dc += mu * curl over the box.

:func:`simulate` wraps it in a ``torch.autograd.Function`` whose inputs are
the coefficient arrays (one per active E component, beamz's dense component
shapes) and whose outputs are the DFT arena's real and imaginary parts, so a
design parametrisation (density -> permittivity -> c) and an objective (a
mode overlap) are ordinary differentiable torch code around it.  beamz takes
its gradients with JAX through the whole solver; this is the hand-written
discrete adjoint of the engine's own step.  Gradients outside the box are
returned as zeros.
"""

from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import abi
from .plan import COMPONENT_INDEX, COMPONENTS, ProgramSpec, active_components, component_shape

# E component each E term differentiates the H of (3D term order), and vice versa.
_E_TERM_SRC = (5, 4, 3, 5, 4, 3)
_H_TERM_SRC = (2, 1, 0, 2, 1, 0)


def _torch():
    import torch

    return torch


class AdjointProblem:
    """One differentiable simulation (dense layout, per-site E material)."""

    def __init__(self, spec: ProgramSpec, nsteps: int, box, checkpoint_every: int = 100, device="cuda",
                 curl_store_bytes: int = 4 << 30):
        from . import runtime

        torch = _torch()
        if spec.e_site is None:
            raise ValueError("the adjoint needs a per-site E material (ProgramSpec.e_site)")
        self.runtime = runtime
        self.spec = spec
        self.nsteps = int(nsteps)
        self.every = max(1, int(checkpoint_every))
        self.lib = abi.load_library()
        self.active = active_components(spec.ndim, spec.polarization)
        self.e_active = [c for c in ("Ex", "Ey", "Ez") if c in self.active]
        # The box in the 3D lattice frame (2D TM is the z = 1 slab).
        lo, hi = (tuple(int(v) for v in b) for b in box)
        if spec.ndim == 2:
            lo, hi = (0, *lo), (1, *hi)
        self.box_lo, self.box_hi = lo, hi
        self.box_shape = tuple(h - l for l, h in zip(lo, hi))
        # The gradient needs the forward curl over the box after every step.
        # When H over the box (and a one-cell margin) for every step fits in
        # `curl_store_bytes`, a field recorder inside the forward program
        # keeps it and the backward pass runs no forward steps; otherwise the
        # backward recomputes each checkpoint segment (``checkpoint_every``).
        self.curl_record = self._curl_recorder(spec, curl_store_bytes)
        fspec = spec if self.curl_record is None else dataclasses.replace(
            spec, recorders=[*spec.recorders, self.curl_record[0]])
        self.forward_program = runtime.compile_program(fspec, device=device, schedule="fused", layout="dense")
        self.adjoint_program = runtime.compile_program(spec, device=device, schedule="phases", layout="dense")
        self.forward_program._times_for(self.nsteps + 1)
        self.adjoint_program._times_for(self.nsteps + 1)
        self.device = self.forward_program.device
        self.checkpoints = []
        self.dft = None

    def _curl_recorder(self, spec: ProgramSpec, limit: int):
        """(RecorderPlan, margin, extended shape) recording every active H
        component on the box grown by one cell towards lower coordinates (z
        only in 3D), or None when it does not fit `limit` bytes (with the curls
        computed from it), a recorder slot, or the components' extents."""
        from .plan import RecorderPlan

        if len(spec.recorders) >= abi.FDTD_MAX_RECORDERS or self.nsteps < 1:
            return None
        h_active = [c for c in ("Hx", "Hy", "Hz") if c in self.active]
        margin = (1 if spec.ndim == 3 else 0, 1, 1)
        ext_lo = tuple(l - m for l, m in zip(self.box_lo, margin))
        ext = tuple(h - l for l, h in zip(ext_lo, self.box_hi))
        values = int(np.prod(ext))
        need = 4 * self.nsteps * (values * len(h_active) + int(np.prod(self.box_shape)) * len(self.e_active))
        if need > limit or min(ext_lo) < 0:
            return None
        kk, jj, ii = np.meshgrid(*(np.arange(l, h) for l, h in zip(ext_lo, self.box_hi)), indexing="ij")
        idx, w = [], []
        for c in h_active:
            shape = component_shape(c, spec.grid_shape, spec.polarization)
            shape = (1, *shape) if spec.ndim == 2 else tuple(shape)
            if any(h > n for h, n in zip(self.box_hi, shape)):
                return None
            flat = (kk * shape[1] + jj) * shape[2] + ii
            idx.append(flat.reshape(-1, 1).astype(np.int32))
            w.append(np.ones((values, 1), np.float32))
        plan = RecorderPlan(tuple(h_active), 1, self.nsteps, idx, w, shapes=(ext,) * len(h_active))
        return plan, margin, ext

    def _curls(self, state, s0: int, s1: int):
        """The forward curl of every active E component over the box after
        steps s0 .. s1-1, from the recorded H: fdtd_adjoint_curl's
        differences and divisions in its order (a device-tensor divisor, so
        every quotient is a correctly rounded division)."""
        torch = _torch()
        plan, margin, ext = self.curl_record
        bufs = state.records[len(state.records) - 1]["values"]
        h = {c: bufs[q][s0:s1].reshape((s1 - s0, *ext)) for q, c in enumerate(plan.components)}
        res = torch.tensor(np.float32(self.spec.resolution), device=self.device)
        bz, by, bx = self.box_shape
        mz = margin[0]
        C, Y, X = slice(mz, mz + bz), slice(1, 1 + by), slice(1, 1 + bx)
        Cm, Ym, Xm = slice(mz - 1, mz - 1 + bz) if mz else None, slice(0, by), slice(0, bx)
        me = self._box_metrics()

        def sc(diff, axis):  # divided by the cell size, or times the box's E-side inverse distances
            return diff / res if me[axis] is None else diff * me[axis]

        out = [None] * 3
        if "Ex" in self.e_active:
            cu = sc(h["Hz"][:, C, Y, X] - h["Hz"][:, C, Ym, X], 1)
            if "Hy" in h:
                cu = cu - sc(h["Hy"][:, C, Y, X] - h["Hy"][:, Cm, Y, X], 0)
            out[0] = cu
        if "Ey" in self.e_active:
            cu = -sc(h["Hz"][:, C, Y, X] - h["Hz"][:, C, Y, Xm], 2)
            if "Hx" in h:
                cu = cu + sc(h["Hx"][:, C, Y, X] - h["Hx"][:, Cm, Y, X], 0)
            out[1] = cu
        if "Ez" in self.e_active:
            out[2] = sc(h["Hy"][:, C, Y, X] - h["Hy"][:, C, Y, Xm], 2) - sc(h["Hx"][:, C, Y, X] - h["Hx"][:, C, Ym, X], 1)
        return [None if c is None else c.contiguous() for c in out]

    def _box_metrics(self):
        """Per axis (z, y, x) the E-side inverse distances of a derivative
        metric over the box, shaped to broadcast against [steps, z, y, x], or
        None (the isotropic grid, or z in 2D)."""
        torch = _torch()
        out = [None, None, None]
        metrics = self.spec.metrics
        if metrics is None:
            return out
        cells = tuple(int(v) for v in self.spec.grid_shape)
        names = ("z", "y", "x") if self.spec.ndim == 3 else (None, "y", "x")
        if self.spec.ndim == 2:
            cells = (1, *cells)
        for a, name in enumerate(names):
            if name is None:
                continue
            m = np.asarray(metrics.along(f"h_to_e_{name}", cells[a] + 1), np.float32)[self.box_lo[a]:self.box_hi[a]]
            shape = [1, 1, 1, 1]
            shape[1 + a] = m.size
            out[a] = torch.as_tensor(m.reshape(shape), device=self.device)
        return out

    # -- coefficients ---------------------------------------------------------
    def set_coefficients(self, coefs: dict) -> None:
        """Copy per-site c arrays (component -> tensor in beamz's shape) into both programs."""
        for c, value in coefs.items():
            for prog in (self.forward_program, self.adjoint_program):
                dst = prog.e_source[c]
                if dst.dim() == 0:
                    raise ValueError(f"{c}: the program was compiled with a uniform coefficient")
                dst.copy_(value.detach().reshape(dst.shape).to(dst.dtype))

    # -- forward --------------------------------------------------------------
    def _snapshot(self, state):
        return ([f.clone() for f in state.fields], [p.clone() for p in state.psi_h], [p.clone() for p in state.psi_e],
                state.step)

    def _restore(self, state, snap):
        fields, psi_h, psi_e, step = snap
        for dst, src in zip(state.fields, fields):
            dst.copy_(src)
        for dst, src in zip(state.psi_h, psi_h):
            dst.copy_(src)
        for dst, src in zip(state.psi_e, psi_e):
            dst.copy_(src)
        state.counter.fill_(int(step))
        state.step = int(step)

    def forward(self):
        rt = self.runtime
        state = rt.initial_state(self.forward_program)
        self.checkpoints = []
        done = 0
        while done < self.nsteps:
            if self.curl_record is None:  # the backward pass recomputes from these
                self.checkpoints.append(self._snapshot(state))
            n = min(self.every, self.nsteps - done)
            rt.run_steps(state, self.forward_program, n)
            done += n
        state.check()
        self.dft = (state.dft_re.clone(), state.dft_im.clone(), state.dft_w.clone())
        self._state = state
        return self.dft[0], self.dft[1]

    # -- backward -------------------------------------------------------------
    def _step_struct(self, step: int, scratch_e, scratch_h, g_re, g_im, curls, grads):
        a = abi.FdtdAdjointStep()
        a.abi_version = abi.FDTD_ABI_VERSION
        a.step = int(step)
        for t in range(6):
            if scratch_e[t] is not None:
                a.scratch_e[t] = abi.buffer_of(scratch_e[t])
            if scratch_h[t] is not None:
                a.scratch_h[t] = abi.buffer_of(scratch_h[t])
        if g_re is not None:
            a.dft_grad_re = abi.buffer_of(g_re)
            a.dft_grad_im = abi.buffer_of(g_im)
        for c in self.e_active:
            i = COMPONENT_INDEX[c]
            if curls is not None:
                a.curl[i] = abi.buffer_of(curls[i])
            if grads is not None:
                a.grad[i] = abi.buffer_of(grads[i])
        a.box_lo[:] = list(self.box_lo)
        a.box_hi[:] = list(self.box_hi)
        return a

    def backward(self, g_re=None, g_im=None):
        """dJ/dc per active E component (beamz shapes; zero outside the box)
        for dJ/d(dft re) = g_re and dJ/d(dft im) = g_im."""
        torch = _torch()
        rt = self.runtime
        dev = self.device
        if self.dft is None:
            raise RuntimeError("run forward() first")
        shapes = self.adjoint_program.shapes
        lam = rt.initial_state(self.adjoint_program)  # adjoint fields and memories, zero
        prog = self.adjoint_program
        scratch_e = [None] * 6
        scratch_h = [None] * 6
        for t in range(6):
            ec, hs = COMPONENTS[t // 2], COMPONENTS[_E_TERM_SRC[t]]
            if ec in self.active and hs in self.active:
                scratch_e[t] = torch.zeros(shapes[ec], dtype=torch.float32, device=dev)
            hc, es = COMPONENTS[3 + t // 2], COMPONENTS[_H_TERM_SRC[t]]
            if hc in self.active and es in self.active:
                scratch_h[t] = torch.zeros(shapes[hc], dtype=torch.float32, device=dev)
        if g_re is not None or g_im is not None:
            g_re = torch.zeros_like(self.dft[0]) if g_re is None else g_re.detach().float().contiguous()
            g_im = torch.zeros_like(self.dft[1]) if g_im is None else g_im.detach().float().contiguous()
        grads = [None] * 3
        for c in self.e_active:
            grads[COMPONENT_INDEX[c]] = torch.zeros(self.box_shape, dtype=torch.float32, device=dev)
        stream = rt._stream(prog)
        if self.curl_record is not None:  # curls from the forward's recorded H, 256 steps at a time
            for s1 in range(self.nsteps, 0, -256):
                s0 = max(0, s1 - 256)
                curl_all = self._curls(self._state, s0, s1)
                for n in reversed(range(s0, s1)):
                    curls = [None if c is None else c[n - s0] for c in curl_all]
                    a = self._step_struct(n, scratch_e, scratch_h, g_re, g_im, curls, grads)
                    s = prog.fill(lam, 0)
                    abi.check(self.lib.fdtd_adjoint_step(stream, ctypes.byref(s), ctypes.byref(a)),
                              "fdtd_adjoint_step")
                del curl_all
            return self._finish(lam, grads)
        fprog = self.forward_program
        rstate = rt.initial_state(fprog)
        nseg = len(self.checkpoints)
        for seg in reversed(range(nseg)):
            s0 = seg * self.every
            s1 = min(s0 + self.every, self.nsteps)
            self._restore(rstate, self.checkpoints[seg])
            curls = [[None] * 3 for _ in range(s1 - s0)]
            for n in range(s0, s1):
                rt.run_steps(rstate, fprog, 1)
                for c in self.e_active:
                    curls[n - s0][COMPONENT_INDEX[c]] = torch.empty(self.box_shape, dtype=torch.float32, device=dev)
                a = self._step_struct(n, [None] * 6, [None] * 6, None, None, curls[n - s0], None)
                s = fprog.fill(rstate, 0)
                abi.check(self.lib.fdtd_adjoint_curl(stream, ctypes.byref(s), ctypes.byref(a)), "fdtd_adjoint_curl")
            for n in reversed(range(s0, s1)):
                a = self._step_struct(n, scratch_e, scratch_h, g_re, g_im, curls[n - s0], grads)
                s = prog.fill(lam, 0)
                abi.check(self.lib.fdtd_adjoint_step(stream, ctypes.byref(s), ctypes.byref(a)), "fdtd_adjoint_step")
            del curls
        rstate.check()
        return self._finish(lam, grads)

    def _finish(self, lam, grads):
        torch = _torch()
        shapes = self.adjoint_program.shapes
        dev = self.device
        lam.check()
        self.lambda_state = lam
        out = {}
        lo, hi = self.box_lo, self.box_hi
        for c in self.e_active:
            full = torch.zeros(shapes[c], dtype=torch.float32, device=dev)
            view = full.reshape((1, *shapes[c])) if self.spec.ndim == 2 else full
            view[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = grads[COMPONENT_INDEX[c]]
            out[c] = full
        return out


class _FdtdFunction:
    """Built lazily so importing this module does not import torch."""

    cls = None

    @classmethod
    def get(cls):
        if cls.cls is None:
            torch = _torch()

            class Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, problem, *coefs):
                    problem.set_coefficients(dict(zip(problem.e_active, coefs)))
                    re, im = problem.forward()
                    ctx.problem = problem
                    return re.clone(), im.clone()

                @staticmethod
                def backward(ctx, g_re, g_im):
                    grads = ctx.problem.backward(g_re, g_im)
                    return (None, *[grads[c] for c in ctx.problem.e_active])

            cls.cls = Fn
        return cls.cls


def simulate(problem: AdjointProblem, coefs):
    """(dft_re, dft_im) of `problem` with E coefficients `coefs` (one tensor per
    active E component, in order Ex, Ey, Ez), differentiable w.r.t. them."""
    return _FdtdFunction.get().apply(problem, *coefs)


# -- design parametrisation helpers -------------------------------------------------

def eps_to_coefficients_2d(eps_voxels, dt, eps0):
    """TM Ez coefficient c = dt / (eps0 eps_site), the site taking its owning
    voxel (beamz/lattice.py:935-972), as differentiable torch ops."""
    torch = _torch()
    ny, nx = eps_voxels.shape
    rows = torch.clamp(torch.arange(ny + 1, device=eps_voxels.device), max=ny - 1)
    cols = torch.clamp(torch.arange(nx + 1, device=eps_voxels.device), max=nx - 1)
    site = eps_voxels[rows][:, cols]
    return torch.tensor(np.float32(dt), device=eps_voxels.device) / (
        torch.tensor(np.float32(eps0), device=eps_voxels.device) * site)


def eps_to_coefficients_3d(eps_voxels, dt, eps0):
    """Ex/Ey/Ez coefficients from a voxel permittivity grid: centered averages
    of the four voxels sharing each edge with clipped indices
    (beamz/lattice.py:732-786), c = fl(dt)/fl(eps0) * (1/eps_site)."""
    torch = _torch()
    nz, ny, nx = eps_voxels.shape
    dev = eps_voxels.device

    def clip_idx(n, m):
        return torch.clamp(torch.arange(-1, n, device=dev), 0, m - 1), torch.clamp(torch.arange(0, n + 1, device=dev), 0, m - 1)

    zlo, zhi = clip_idx(nz, nz)
    ylo, yhi = clip_idx(ny, ny)
    xlo, xhi = clip_idx(nx, nx)
    v = eps_voxels
    half = 0.5
    # Ex (nz+1, ny+1, nx): average z then y.
    az = half * (v[zlo] + v[zhi])
    ex = half * (az[:, ylo] + az[:, yhi])
    # Ey (nz+1, ny, nx+1): average z then x.
    ey = half * (az[:, :, xlo] + az[:, :, xhi])
    # Ez (nz, ny+1, nx+1): average y then x.
    ay = half * (v[:, ylo] + v[:, yhi])
    ez = half * (ay[:, :, xlo] + ay[:, :, xhi])
    dto = torch.tensor(np.float32(np.float32(dt) / np.float32(eps0)), device=dev)
    return [dto * (1.0 / ex), dto * (1.0 / ey), dto * (1.0 / ez)]


def site_spec(spec: ProgramSpec, coefs: dict) -> ProgramSpec:
    """`spec` with a per-site E material (decay 1, source = coefs[c] on the host)."""
    e_site = {c: (np.float32(1.0), np.asarray(v, np.float32)) for c, v in coefs.items()}
    return dataclasses.replace(spec, voxel_ids=None, eps_table=None, e_site=e_site)


def component_shapes(spec: ProgramSpec) -> dict:
    return {c: component_shape(c, spec.grid_shape, spec.polarization) for c in COMPONENTS}
