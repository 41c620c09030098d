"""On-device operator assembly and the implicit plasma step, over the C ABI.

The reference assembles every equation's operator on the host before its
solve (update_efield, plasma_pde/poissoneq.f90:565-680;
eden_update_transport, plasma_pde/edeneq.f90:360-444;
poisson_update_transport, plasma_pde/poissoneq.f90:335-385) and chains the
solves in its time loop (plasma_pde/solve_manager.f90:363-502).  These
wrappers run the device versions (mps_efield_dev, mps_eden_transport_dev,
mps_poisson_source_dev) and the whole potential + electron step
(mps_plasma_step_dev) on torch CUDA tensors in the reference's ghosted layout
(numpy/torch shape (nz+2, ny+2, nx+2), i fastest; vector fields with a
leading axis of 3).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import capi, solver
from .problem import bc_code

ECHARGE = 1.602176634e-19  # C
EPS0 = 8.8541878128e-12    # F/m


def _grid(shape_xyz, llen):
    nx, ny, nz = shape_xyz
    return capi.Grid(int(nx), int(ny), int(nz), *[float(v) for v in llen])


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _check(st, what):
    if st != 0:
        raise capi.SolverError(st, what)


def _faces(bcvals, device):
    import torch

    out = []
    for v in bcvals:
        out.append(None if v is None else torch.from_numpy(np.array(v, dtype=np.float64, order="C")).to(device))
    return out


def efield_dev(phi, llen, bc: Sequence, bcvals=None, scale: float = 1.0, limiter: bool = False, stream=None):
    """E = -scale * grad(phi) (mps_efield_dev).  phi: ghosted float64 CUDA
    tensor; its ghosts are set in place by the potential's boundary rules
    first, as update_efield does.  Returns E, shape (3,) + phi.shape."""
    import torch

    nz, ny, nx = (s - 2 for s in phi.shape)
    codes = (C.c_int * 6)(*[bc_code(c) for c in bc])
    faces = _faces(bcvals or [None] * 6, phi.device)
    fv = (C.c_void_p * 6)(*[_ptr(f) for f in faces])
    e = torch.empty((3,) + tuple(phi.shape), dtype=torch.float64, device=phi.device)
    st = capi.load().mps_efield_dev(C.byref(_grid((nx, ny, nz), llen)), codes, fv, _ptr(phi), float(scale),
                                    int(bool(limiter)), _ptr(e), C.c_void_p(capi.stream_arg(stream)))
    _check(st, "mps_efield_dev")
    return e


def eden_transport_dev(efield, llen, mu, d=None, te=None, prod=None, n_old=None, dt: Optional[float] = None,
                       scaling=(1.0, 1.0, 1.0), stream=None):
    """(vel, dcoeff, source) of the electron operator (mps_eden_transport_dev)
    from E and the signed mobility; D = d, or |mu| te when d is None; a time
    derivative (n_old / dt in the source) when dt is given."""
    import torch

    shape = tuple(mu.shape)
    nz, ny, nx = (s - 2 for s in shape)
    vel = torch.empty((3,) + shape, dtype=torch.float64, device=mu.device)
    dc = torch.empty(shape, dtype=torch.float64, device=mu.device)
    src = torch.empty(shape, dtype=torch.float64, device=mu.device)
    sc = (C.c_double * 3)(*[float(v) for v in scaling])
    st = capi.load().mps_eden_transport_dev(C.byref(_grid((nx, ny, nz), llen)), _ptr(efield), _ptr(mu), _ptr(d),
                                            _ptr(te), _ptr(prod), _ptr(n_old), int(dt is not None),
                                            float(dt or 0.0), sc, _ptr(vel), _ptr(dc), _ptr(src),
                                            C.c_void_p(capi.stream_arg(stream)))
    _check(st, "mps_eden_transport_dev")
    return vel, dc, src


def poisson_source_dev(n_e, llen, n_ion=None, charge=None, scale: float = ECHARGE / EPS0, phi_old=None,
                       dt: float = 1.0, stream=None):
    """The space-charge source (mps_poisson_source_dev): n_ion is a
    (nspec,) + ghosted tensor, charge a float64 tensor of nspec charge
    numbers on the device."""
    import torch

    shape = tuple(n_e.shape)
    nz, ny, nx = (s - 2 for s in shape)
    nspec = 0 if n_ion is None else int(n_ion.shape[0])
    src = torch.empty(shape, dtype=torch.float64, device=n_e.device)
    st = capi.load().mps_poisson_source_dev(C.byref(_grid((nx, ny, nz), llen)), _ptr(n_e), nspec, _ptr(n_ion),
                                            _ptr(charge), float(scale), _ptr(phi_old), float(dt), _ptr(src),
                                            C.c_void_p(capi.stream_arg(stream)))
    _check(st, "mps_poisson_source_dev")
    return src


class PlasmaStep:
    """The potential + electron part of one implicit time step on the device
    (mps_plasma_step_dev): Poisson source, potential solve, E field, electron
    operator, implicit Scharfetter-Gummel electron solve from n_old, floor and
    ghosts.  Two handles keep both solvers' workspaces resident."""

    def __init__(self, case: dict, device="cuda", phi_opts=None, e_opts=None):
        import torch

        self.case = case
        self.device = device
        t = lambda a: None if a is None else torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(device)  # noqa: E731
        n = case["shape"]
        self.llen = case["llen"]
        self.eps = t(case["eps"])
        self.mu_e = t(case["mu_e"])
        self.d_e = t(case.get("d_e"))
        self.te = t(case.get("te"))
        self.prod = t(case.get("prod_e"))
        self.n_ion = t(case["n_ion"])
        self.charge = t(np.asarray(case["ion_charge"], dtype=np.float64))
        self.phi_faces = _faces(case["phi_bcvals"], device)
        self.ne_faces = _faces(case["ne_bcvals"], device)
        g = tuple(self.eps.shape)
        z = lambda *s: torch.zeros(s, dtype=torch.float64, device=device)  # noqa: E731
        self.phi_source = z(*g)
        self.efield = z(3, *g)
        self.vel = z(3, *g)
        self.dcoeff = z(*g)
        self.source = z(*g)
        self.hp = capi.Handle(torch.device(device).index or 0)
        self.he = capi.Handle(torch.device(device).index or 0)
        self.phi_opts = solver.make_opts(**(phi_opts or {"precision": "mixed", "tol": 1e-10, "maxit": 60}))
        self.e_opts = solver.make_opts(**(e_opts or {"precision": "mixed", "krylov": "fgmres", "flux": 1,
                                                     "tol": 1e-10, "maxit": 60}))
        S = capi.PlasmaStep()
        S.g = _grid(n, self.llen)
        S.phi_bc[:] = [bc_code(c) for c in case["phi_bc"]]
        S.phi_bcval[:] = [f.data_ptr() if f is not None else None for f in self.phi_faces]
        S.eps = self.eps.data_ptr()
        S.rho_scale = float(case.get("rho_scale", ECHARGE / EPS0))
        S.nion = int(self.n_ion.shape[0])
        S.n_ion = self.n_ion.data_ptr()
        S.ion_charge = self.charge.data_ptr()
        S.phi_source = self.phi_source.data_ptr()
        S.ne_bc[:] = [bc_code(c) for c in case["ne_bc"]]
        S.ne_bcval[:] = [f.data_ptr() if f is not None else None for f in self.ne_faces]
        S.mu_e = self.mu_e.data_ptr()
        S.d_e = self.d_e.data_ptr() if self.d_e is not None else None
        S.te = self.te.data_ptr() if self.te is not None else None
        S.prod_e = self.prod.data_ptr() if self.prod is not None else None
        S.dt = float(case["dt"])
        S.nemin = float(case["nemin"])
        S.efield_scale = float(case.get("efield_scale", 1.0))
        S.limiter = int(bool(case.get("limiter", False)))
        S.vel_scaling, S.dcoeff_scaling, S.source_scaling = [float(v) for v in case.get("scaling", (1, 1, 1))]
        S.efield = self.efield.data_ptr()
        S.vel = self.vel.data_ptr()
        S.dcoeff = self.dcoeff.data_ptr()
        S.source = self.source.data_ptr()
        self.S = S

    def step(self, phi, n_e, stream=None):
        """One step in place: phi (guess in, potential out) and n_e (n_old in,
        n_new out), ghosted float64 CUDA tensors.  Returns the two solves'
        info dicts."""
        self.S.phi = phi.data_ptr()
        self.S.n_e = n_e.data_ptr()
        ip, ie = capi.Info(), capi.Info()
        st = capi.load().mps_plasma_step_dev(self.hp.h, self.he.h, C.byref(self.S), C.byref(self.phi_opts),
                                             C.byref(self.e_opts), C.byref(ip), C.byref(ie),
                                             C.c_void_p(capi.stream_arg(stream)))
        if st not in (0, capi.MPS_ERR_NOT_CONVERGED):
            raise capi.SolverError(st, "mps_plasma_step_dev: " + self.hp.last_error() + " " + self.he.last_error())
        return ip.as_dict(), ie.as_dict()

    def close(self):
        self.hp.close()
        self.he.close()
