"""FP64 reference implementation of the differentiable solve, for tests:
the same :class:`mps3d_b200.adjoint.ElectronFluxAdjoint` model run on the CPU
with the oracle's solves (forward and transposed FGMRES over its V-cycle) and
the oracle's operator VJP in place of the CUDA library."""
import numpy as np
import torch

from mps3d_b200.problem import BC_NAMES, Problem
from oracle import oracle as O


def _problem(spec, vel, dcoeff):
    pad = lambda a: np.pad(a, 1)  # noqa: E731
    v = None if vel is None else np.stack([pad(vel[a]) for a in range(3)])
    return Problem(spec.lx, spec.ly, spec.lz, tuple(spec.llen), dcoeff=pad(dcoeff), source=np.zeros(
        (spec.lz + 2, spec.ly + 2, spec.lx + 2)), vel=v, bc=[BC_NAMES[c] for c in spec.bc], bcvals=[0.0] * 6,
        timederiv=spec.timederiv, dt=spec.dt, flux=spec.flux)


class OracleSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rhs, vel, dcoeff, spec):
        v = None if vel is None else vel.detach().cpu().numpy()
        d = dcoeff.detach().cpu().numpy()
        p = _problem(spec, v, d)
        x, hist = O.RowsMG(p).fgmres(rhs.detach().cpu().numpy(), m=40, maxit=400, tol=1e-14)
        ctx.p = p
        ctx.has_vel = vel is not None
        xt = torch.from_numpy(np.ascontiguousarray(x))
        ctx.save_for_backward(xt)
        return xt

    @staticmethod
    def backward(ctx, gx):
        (x,) = ctx.saved_tensors
        p = ctx.p
        lam, hist = O.RowsMG(p, transpose=True).fgmres(gx.detach().cpu().numpy(), m=40, maxit=400, tol=1e-14)
        gv, gd, _ = O.operator_vjp(p, lam, x.numpy())
        gvel = torch.from_numpy(-gv) if (ctx.has_vel and ctx.needs_input_grad[1]) else None
        gdc = torch.from_numpy(-gd) if ctx.needs_input_grad[2] else None
        return torch.from_numpy(np.ascontiguousarray(lam)), gvel, gdc, None


def oracle_solve(rhs, vel, dcoeff, spec):
    return OracleSolve.apply(rhs, vel, dcoeff, spec)


def oracle_bvec(prob):
    return O.build_rhs(prob)
