"""Python front end of the solver, mirroring the reference's solver interface.

``vcycle_once`` has the meaning of one ``perform_vcycle`` call
(mgridlib/mgridsteps.f90:384-417): ghosted solution in/out and the RMS
residual norm of the post-smoothing residual out.  ``linsolve`` replaces the
equation modules' loop ``do i=1,nvcycles; call perform_vcycle(...);
if(resnorm .le. err_tol) exit`` (e.g. plasma_pde/poissoneq.f90:427-450) and
adds the relative-residual stop, mixed precision and FGMRES.

Host numpy arrays go through ``mps_linsolve`` (copies inside the call);
``DeviceProblem`` holds the same fields as torch CUDA tensors for the
device-pointer entry points.  Every path calls the CUDA library; errors
raise :class:`mps3d_b200.capi.SolverError` with the library's status.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import capi
from .problem import Problem

_PREC = {"fp64": capi.PREC_FP64, "mixed": capi.PREC_MIXED}
_HIER = {"cell": capi.HIER_CELL, "geom": capi.HIER_GEOM}
_KRY = {None: capi.KRYLOV_NONE, "none": capi.KRYLOV_NONE, "fgmres": capi.KRYLOV_FGMRES}
_TOLK = {"rms": capi.TOL_RMS_ABS, "rel": capi.TOL_REL_L2}

_default_handle = None


def default_handle() -> capi.Handle:
    global _default_handle
    if _default_handle is None:
        _default_handle = capi.Handle()
    return _default_handle


def make_opts(tol=1e-10, tol_kind="rel", maxit=50, precision="fp64", hierarchy="geom", ranks=(1, 1, 1),
              krylov=None, restart=30, nu1=2, nu2=2, fill_ghosts=False, inner_cycles=0, transpose=False,
              flux=None, max_coarse=125, use_graph=True):
    return capi.default_opts(
        tol=float(tol), tol_kind=_TOLK[tol_kind], maxit=int(maxit), precision=_PREC[precision],
        hierarchy=_HIER[hierarchy], ranks=tuple(int(r) for r in ranks), krylov=_KRY[krylov], restart=int(restart),
        nu1=int(nu1), nu2=int(nu2), fill_ghosts=int(bool(fill_ghosts)), inner_cycles=int(inner_cycles),
        transpose=int(bool(transpose)), flux=int(flux or 0), max_coarse=int(max_coarse),
        use_graph=int(bool(use_graph)))


def _grid(p: Problem) -> capi.Grid:
    return capi.Grid(p.lx, p.ly, p.lz, p.llen[0], p.llen[1], p.llen[2])


def _np_ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


def _bc(p: Problem):
    return (C.c_int * 6)(*p.bc)


def _check(h: capi.Handle, st: int, info: capi.Info, allow_not_converged=True):
    if st == capi.MPS_ERR_NOT_CONVERGED and allow_not_converged:
        return
    if st != 0:
        raise capi.SolverError(st, h.last_error())


def linsolve(prob: Problem, soln: Optional[np.ndarray] = None, handle: Optional[capi.Handle] = None,
             mgridsterm: Optional[np.ndarray] = None, raise_not_converged=False, **kw):
    """Solve on host arrays. Returns (soln, info dict)."""
    h = handle or default_handle()
    o = make_opts(flux=prob.flux, **kw)
    x = prob.zeros_ghosted() if soln is None else np.ascontiguousarray(soln, dtype=np.float64).copy()
    bcv = (C.c_void_p * 6)(*[C.c_void_p(v.ctypes.data) for v in prob.bcvals])
    info = capi.Info()
    vel = prob.vel if np.any(prob.vel) else None
    reac = prob.reac if np.any(prob.reac) else None
    st = h._lib.mps_linsolve(h.h, C.byref(_grid(prob)), int(prob.timederiv), float(prob.dt), _np_ptr(vel),
                             _np_ptr(prob.dcoeff), _np_ptr(reac), _np_ptr(prob.source), _bc(prob), bcv,
                             _np_ptr(None if mgridsterm is None else np.ascontiguousarray(mgridsterm)),
                             _np_ptr(x), C.byref(o), C.byref(info))
    _check(h, st, info, allow_not_converged=not raise_not_converged)
    return x, info.as_dict()


def vcycle_once(prob: Problem, soln: np.ndarray, handle: Optional[capi.Handle] = None, ranks=(1, 1, 1),
                hierarchy="cell", mgridsterm=None, nu1=2, nu2=2):
    """One perform_vcycle call on host arrays: returns (soln, resnorm)."""
    h = handle or default_handle()
    o = make_opts(hierarchy=hierarchy, ranks=ranks, nu1=nu1, nu2=nu2, flux=prob.flux)
    x = np.ascontiguousarray(soln, dtype=np.float64).copy()
    bcv = (C.c_void_p * 6)(*[C.c_void_p(v.ctypes.data) for v in prob.bcvals])
    rn = C.c_double(0.0)
    vel = prob.vel if np.any(prob.vel) else None
    reac = prob.reac if np.any(prob.reac) else None
    st = h._lib.mps_vcycle_once(h.h, C.byref(_grid(prob)), int(prob.timederiv), float(prob.dt), _np_ptr(vel),
                                _np_ptr(prob.dcoeff), _np_ptr(reac), _np_ptr(prob.source), _bc(prob), bcv,
                                _np_ptr(None if mgridsterm is None else np.ascontiguousarray(mgridsterm)),
                                _np_ptr(x), C.byref(rn), C.byref(o))
    if st != 0:
        raise capi.SolverError(st, h.last_error())
    return x, rn.value


class DeviceProblem:
    """The fields of a :class:`Problem` resident on a CUDA device (torch tensors)."""

    def __init__(self, prob: Problem, device="cuda"):
        import torch

        self.prob = prob
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        self.vel = t(prob.vel) if np.any(prob.vel) else None
        self.dcoeff = t(prob.dcoeff)
        self.reac = t(prob.reac) if np.any(prob.reac) else None
        self.source = t(prob.source)
        self.bcvals = [t(v) for v in prob.bcvals]
        self.device = device

    @staticmethod
    def ptr(x):
        return None if x is None else C.c_void_p(x.data_ptr())

    def bcv(self):
        return (C.c_void_p * 6)(*[C.c_void_p(v.data_ptr()) for v in self.bcvals])


def linsolve_dev(dp: DeviceProblem, soln, handle: Optional[capi.Handle] = None, stream=None, mgridsterm=None,
                 **kw):
    """Solve with device tensors (soln: ghosted float64 CUDA tensor, updated in place)."""
    import torch

    h = handle or default_handle()
    p = dp.prob
    o = make_opts(flux=p.flux, **kw)
    info = capi.Info()
    s = capi.stream_arg(stream)
    st = h._lib.mps_linsolve_dev(h.h, C.byref(_grid(p)), int(p.timederiv), float(p.dt), dp.ptr(dp.vel),
                                 dp.ptr(dp.dcoeff), dp.ptr(dp.reac), dp.ptr(dp.source), _bc(p), dp.bcv(),
                                 dp.ptr(mgridsterm), dp.ptr(soln), C.byref(o), C.byref(info), C.c_void_p(s))
    _check(h, st, info)
    return soln, info.as_dict()


def linsolve_batched_dev(dps, solns, handle: Optional[capi.Handle] = None, stream=None, **kw):
    """Solve independent problems together through mps_linsolve_batched_dev.

    dps: list of :class:`DeviceProblem` (diffusion class: no convection);
    solns: matching ghosted float64 CUDA tensors (initial guesses, updated in
    place).  Returns the list of per-problem info dicts.  Options as for
    :func:`linsolve` (stationary iteration; precision "mixed" or "fp64")."""
    import torch

    h = handle or default_handle()
    n = len(dps)
    assert n == len(solns) and n >= 1
    descs = (capi.ProblemDesc * n)()
    keep = []
    for i, (dp, x) in enumerate(zip(dps, solns)):
        p = dp.prob
        d = descs[i]
        d.g = _grid(p)
        d.timederiv = int(p.timederiv)
        d.dt = float(p.dt)
        ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        d.vel = ptr(dp.vel)
        d.dcoeff = ptr(dp.dcoeff)
        d.reac = ptr(dp.reac)
        d.source = ptr(dp.source)
        d.bc_code[:] = list(p.bc)
        for f in range(6):
            d.bcval[f] = dp.bcvals[f].data_ptr()
        d.mgridsterm = None
        d.soln = x.data_ptr()
        keep.append((dp, x))
    o = make_opts(**kw)
    infos = (capi.Info * n)()
    s = capi.stream_arg(stream)
    st = h._lib.mps_linsolve_batched_dev(h.h, n, descs, C.byref(o), infos, C.c_void_p(s))
    if st not in (0, capi.MPS_ERR_NOT_CONVERGED):
        raise capi.SolverError(st, h.last_error())
    return [infos[i].as_dict() for i in range(n)]


def apply_A_dev(dp: DeviceProblem, soln, handle: Optional[capi.Handle] = None, transpose=False):
    """AX = A soln (interior (lz,ly,lx) float64 CUDA tensor) through mps_apply_A_dev."""
    import torch

    h = handle or default_handle()
    p = dp.prob
    out = torch.empty(p.shape, dtype=torch.float64, device=soln.device)
    o = make_opts(flux=p.flux, transpose=transpose)
    st = h._lib.mps_apply_A_dev(h.h, C.byref(_grid(p)), int(p.timederiv), float(p.dt), dp.ptr(dp.vel),
                                dp.ptr(dp.dcoeff), dp.ptr(dp.reac), _bc(p), dp.ptr(soln), dp.ptr(out), C.byref(o),
                                C.c_void_p(capi.stream_arg()))
    if st != 0:
        raise capi.SolverError(st, h.last_error())
    return out


def apply_A_noalloc(dp: DeviceProblem, soln, out=None, transpose=False, stream=None):
    """AX = A soln through mps_apply_A_noalloc: no handle and no device allocation
    inside the call (its scratch is the library's static device array).  The
    caller provides ``out`` (interior (lz,ly,lx) float64 on the device) when it
    must not allocate either; the work is queued on ``stream`` (default: torch's
    current stream) and is not waited for."""
    import torch

    p = dp.prob
    if out is None:
        out = torch.empty(p.shape, dtype=torch.float64, device=soln.device)
    o = make_opts(flux=p.flux, transpose=transpose)
    s = capi.stream_arg(stream)
    st = capi.load().mps_apply_A_noalloc(C.byref(_grid(p)), int(p.timederiv), float(p.dt), dp.ptr(dp.vel),
                                         dp.ptr(dp.dcoeff), dp.ptr(dp.reac), _bc(p), dp.ptr(soln), dp.ptr(out),
                                         C.byref(o), C.c_void_p(s))
    if st != 0:
        raise capi.SolverError(st, "mps_apply_A_noalloc: " + capi.STATUS_NAMES.get(st, str(st)))
    return out


def find_bvec_dev(dp: DeviceProblem, handle: Optional[capi.Handle] = None, mgridsterm=None):
    import torch

    h = handle or default_handle()
    p = dp.prob
    out = torch.empty(p.shape, dtype=torch.float64, device=dp.dcoeff.device)
    o = make_opts(flux=p.flux)
    st = h._lib.mps_find_bvec_dev(h.h, C.byref(_grid(p)), dp.ptr(dp.vel), dp.ptr(dp.dcoeff), dp.ptr(dp.source),
                                  _bc(p), dp.bcv(), dp.ptr(mgridsterm), dp.ptr(out), C.byref(o),
                                  C.c_void_p(capi.stream_arg()))
    if st != 0:
        raise capi.SolverError(st, h.last_error())
    return out


def fill_ghosts_dev(dp: DeviceProblem, soln, handle: Optional[capi.Handle] = None):
    import torch

    h = handle or default_handle()
    p = dp.prob
    st = h._lib.mps_fill_ghosts_dev(h.h, C.byref(_grid(p)), _bc(p), dp.bcv(), dp.ptr(soln),
                                    C.c_void_p(capi.stream_arg()))
    if st != 0:
        raise capi.SolverError(st, h.last_error())
    return soln
