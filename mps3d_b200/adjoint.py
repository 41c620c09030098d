"""Differentiable solves over the C ABI, and the electron-flux adjoint.

:class:`LinearSolve` is x = A(vel, dcoeff)^{-1} rhs as a
``torch.autograd.Function``: the forward pass is one ``mps_linsolve_dev``;
the backward pass is one transposed solve (``opts.transpose``; for the
symmetric diffusion class the same V-cycle) for lam = A^{-T} dL/dx, and
``mps_operator_vjp_dev`` for dL/d(vel, dcoeff) = -d(lam^T A x)/d(vel, dcoeff).
Every solve stores only its output for the backward pass (step
checkpointing: the iterate history of the solver is not kept).

:class:`ElectronFluxAdjoint` is the implicit electron transport model of the
benchmark's adjoint configuration: a plasma Poisson solve whose FRONT
Dirichlet value is the electrode voltage V, drift v = mu grad(phi) and
diffusivity D = mu Te, ``steps`` implicit Scharfetter-Gummel steps
n_{k+1} = A(v, D)^{-1} n_k / dt, and the loss = electron flux through the
z = L face, sum over the top cells of v_z n h_x h_y.  The reference has no
adjoint; its forward pieces are poisson_solve (poissoneq.f90:387-477),
update_efield (poissoneq.f90:565-680) and eden_solve (edeneq.f90:446-525).
The solve is a parameter (``solve_fn``), so that a test can run the same
model over a different implementation of the solves.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import capi, solver
from .problem import BC_CODES, Problem


@dataclass
class OperatorSpec:
    """The fixed part of an operator: grid, boundary codes, flux, time term and
    the solver settings of its forward and transposed solves."""
    lx: int
    ly: int
    lz: int
    llen: tuple
    bc: tuple                  # six MPS_BC_* integers
    flux: int = 0
    timederiv: bool = False
    dt: float = 1.0
    tol: float = 1e-12
    precision: str = "fp64"
    krylov: Optional[str] = None
    maxit: int = 100
    handle: Optional[capi.Handle] = None
    handle_t: Optional[capi.Handle] = None  # for the transposed solves (None: ``handle``)


def _ghosted(t):
    import torch

    return torch.nn.functional.pad(t, (1, 1, 1, 1, 1, 1))


def _faces(spec: OperatorSpec, device):
    import torch

    sizes = [spec.ly * spec.lz] * 2 + [spec.lx * spec.lz] * 2 + [spec.lx * spec.ly] * 2
    return [torch.zeros(s, dtype=torch.float64, device=device) for s in sizes]


def _grid(spec: OperatorSpec):
    return capi.Grid(spec.lx, spec.ly, spec.lz, *[float(v) for v in spec.llen])


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def device_solve(spec: OperatorSpec, rhs, vel_g, dc_g, transpose: bool):
    """x = A^{-1} rhs (or A^{-T} rhs): interior rhs in, interior x out; the
    right-hand side enters as mgridsterm with zero source and zero boundary
    values."""
    import torch

    h = (spec.handle_t if transpose and spec.handle_t is not None else spec.handle) or solver.default_handle()
    dev = rhs.device
    shape = (spec.lz + 2, spec.ly + 2, spec.lx + 2)
    src = torch.zeros(shape, dtype=torch.float64, device=dev)
    x = torch.zeros(shape, dtype=torch.float64, device=dev)
    faces = _faces(spec, dev)
    bcv = (C.c_void_p * 6)(*[C.c_void_p(f.data_ptr()) for f in faces])
    bcc = (C.c_int * 6)(*spec.bc)
    krylov = spec.krylov if spec.krylov is not None else ("fgmres" if spec.flux == 1 else None)
    o = solver.make_opts(tol=spec.tol, precision=spec.precision, krylov=krylov, transpose=transpose,
                         flux=spec.flux, maxit=spec.maxit)
    info = capi.Info()
    r = rhs.contiguous()
    st = h._lib.mps_linsolve_dev(h.h, C.byref(_grid(spec)), int(spec.timederiv), float(spec.dt), _ptr(vel_g),
                                 _ptr(dc_g), None, _ptr(src), bcc, bcv, _ptr(r), _ptr(x), C.byref(o),
                                 C.byref(info), C.c_void_p(capi.stream_arg(torch.cuda.current_stream(dev))))
    if st != 0:
        raise capi.SolverError(st, h.last_error())
    return x[1:-1, 1:-1, 1:-1].contiguous()


def device_vjp(spec: OperatorSpec, vel_g, dc_g, lam, u):
    """d(lam^T A u)/d(vel, dcoeff) through mps_operator_vjp_dev."""
    import torch

    dev = lam.device
    gv = torch.zeros((3, spec.lz, spec.ly, spec.lx), dtype=torch.float64, device=dev)
    gd = torch.zeros((spec.lz, spec.ly, spec.lx), dtype=torch.float64, device=dev)
    o = solver.make_opts(flux=spec.flux)
    lam = lam.contiguous()
    u = u.contiguous()
    st = capi.load().mps_operator_vjp_dev(C.byref(_grid(spec)), _ptr(vel_g), _ptr(dc_g), (C.c_int * 6)(*spec.bc),
                                          _ptr(lam), _ptr(u), C.byref(o), _ptr(gv), _ptr(gd), None,
                                          C.c_void_p(capi.stream_arg(torch.cuda.current_stream(dev))))
    if st != 0:
        raise capi.SolverError(st, "mps_operator_vjp_dev")
    return gv, gd


def _make_linear_solve():
    import torch

    class LinearSolve(torch.autograd.Function):
        """x = A(vel, dcoeff)^{-1} rhs; vel (3, lz, ly, lx) or None, dcoeff (lz, ly, lx)."""

        @staticmethod
        def forward(ctx, rhs, vel, dcoeff, spec):
            vel_g = None if vel is None else _ghosted(vel.to(torch.float64)).contiguous()
            dc_g = _ghosted(dcoeff.to(torch.float64)).contiguous()
            x = device_solve(spec, rhs.to(torch.float64), vel_g, dc_g, transpose=False)
            ctx.spec = spec
            ctx.has_vel = vel is not None
            ctx.save_for_backward(x, vel_g if vel_g is not None else x.new_zeros(0), dc_g)
            return x

        @staticmethod
        def backward(ctx, gx):
            x, vel_g, dc_g = ctx.saved_tensors
            vel_g = vel_g if ctx.has_vel else None
            lam = device_solve(ctx.spec, gx.to(torch.float64), vel_g, dc_g, transpose=True)
            gvel = gdc = None
            if ctx.needs_input_grad[1] or ctx.needs_input_grad[2]:
                gv, gd = device_vjp(ctx.spec, vel_g, dc_g, lam, x)
                gvel = -gv if ctx.needs_input_grad[1] else None
                gdc = -gd if ctx.needs_input_grad[2] else None
            return lam, gvel, gdc, None

    return LinearSolve


_LinearSolve = None


def linear_solve(rhs, vel, dcoeff, spec: OperatorSpec):
    """Differentiable x = A(vel, dcoeff)^{-1} rhs on the device (see :class:`LinearSolve`)."""
    global _LinearSolve
    if _LinearSolve is None:
        _LinearSolve = _make_linear_solve()
    return _LinearSolve.apply(rhs, vel, dcoeff, spec)


class ElectronFluxAdjoint:
    """The electron-flux loss L(V, mu) and its gradients (see the module text).

    ``case`` is :func:`mps3d_b200.workloads.electron_adjoint_case`; the
    right-hand side of the Poisson solve is b0 + V b1, with b0 = find_bvec of
    the space charge at V = 0 and b1 = find_bvec of a unit FRONT voltage (the
    Dirichlet term is linear in V).  ``solve_fn(rhs, vel, dcoeff, spec)`` and
    ``bvec_fn(problem)`` default to the device implementations."""

    def __init__(self, case, device="cuda", handle=None, tol=1e-12, poisson_precision="fp64",
                 sg_precision="fp64", solve_fn=None, bvec_fn=None):
        import torch

        self.case = case
        self.device = device
        n = case["n"]
        L = case["length"]
        self.n = n
        self.h = L / n
        self.dt = case["dt"]
        self.steps = case["steps"]
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device)  # noqa: E731
        self.eps = t(case["eps"][1:-1, 1:-1, 1:-1])
        self.te = t(case["te"])
        self.n_old = t(case["n_old"])
        bc_p = tuple(BC_CODES[c] for c in ["PERI", "PERI", "PERI", "PERI", "DIRC", "DIRC"])
        bc_s = tuple(BC_CODES[c] for c in ["PERI", "PERI", "PERI", "PERI", "ZGRD", "ZGRD"])
        # A handle keeps the workspace and the captured graphs of one operator
        # signature; a solve of another signature replaces them.  The device
        # solves therefore take one handle per operator kind -- Poisson
        # (``handle``, forward and transposed: the operator is symmetric), SG
        # forward, SG transposed -- and every solve of a gradient replays its
        # own graphs.
        hp = hs = hst = handle
        if solve_fn is None:
            d = torch.device(device)
            di = d.index if d.index is not None else torch.cuda.current_device()
            hp = handle or capi.Handle(di)
            hs, hst = capi.Handle(di), capi.Handle(di)
        self.pspec = OperatorSpec(n, n, n, (L, L, L), bc_p, flux=0, tol=tol, precision=poisson_precision,
                                  handle=hp)
        self.sspec = OperatorSpec(n, n, n, (L, L, L), bc_s, flux=1, timederiv=True, dt=self.dt, tol=tol,
                                  precision=sg_precision, krylov="fgmres", handle=hs, handle_t=hst)
        self.solve_fn = solve_fn or linear_solve
        bvec = bvec_fn or self._device_bvec
        zero = np.zeros_like(case["rho"])
        p0 = Problem(n, n, n, (L, L, L), dcoeff=case["eps"], source=case["rho"],
                     bc=["PERI", "PERI", "PERI", "PERI", "DIRC", "DIRC"], bcvals=[None, None, None, None, 0.0, 0.0])
        p1 = Problem(n, n, n, (L, L, L), dcoeff=case["eps"], source=zero,
                     bc=["PERI", "PERI", "PERI", "PERI", "DIRC", "DIRC"], bcvals=[None, None, None, None, 0.0, 1.0])
        self.b0 = t(bvec(p0))
        self.b1 = t(bvec(p1))

    def _device_bvec(self, prob):
        dp = solver.DeviceProblem(prob, device=self.device)
        return solver.find_bvec_dev(dp, handle=self.pspec.handle).cpu().numpy()

    def potential_ghosted(self, phi, V):
        """Ghost layer of phi: periodic in x and y, Dirichlet 0 at z = 0 and V at z = L."""
        import torch

        p = torch.cat([phi[:, :, -1:], phi, phi[:, :, :1]], dim=2)
        p = torch.cat([p[:, -1:, :], p, p[:, :1, :]], dim=1)
        bottom = -p[:1]
        top = 2.0 * V - p[-1:]
        return torch.cat([bottom, p, top], dim=0)

    def fields(self, V, mu):
        """Drift velocity (3, n, n, n) and diffusivity of mobility mu at voltage V."""
        import torch

        b = self.b0 + V * self.b1
        phi = self.solve_fn(b, None, self.eps, self.pspec)
        pg = self.potential_ghosted(phi, V)
        h2 = 2.0 * self.h
        gx = (pg[1:-1, 1:-1, 2:] - pg[1:-1, 1:-1, :-2]) / h2
        gy = (pg[1:-1, 2:, 1:-1] - pg[1:-1, :-2, 1:-1]) / h2
        gz = (pg[2:, 1:-1, 1:-1] - pg[:-2, 1:-1, 1:-1]) / h2
        m = mu.to(torch.float64)
        vel = torch.stack([m * gx, m * gy, m * gz])
        return vel, m * self.te

    def loss(self, V, mu):
        vel, D = self.fields(V, mu)
        ne = self.n_old
        for _ in range(self.steps):
            ne = self.solve_fn(ne / self.dt, vel, D, self.sspec)
        return (vel[2, -1] * ne[-1]).sum() * (self.h * self.h)

    def gradient(self, V: float, mu):
        """(L, dL/dV, dL/dmu) at (V, mu); mu float32 (n, n, n) tensor, gradient in its dtype."""
        import torch

        Vt = torch.tensor(float(V), dtype=torch.float64, device=self.device, requires_grad=True)
        m = mu.detach().clone().requires_grad_(True)
        L = self.loss(Vt, m)
        gV, gmu = torch.autograd.grad(L, (Vt, m))
        return float(L.detach()), float(gV), gmu
