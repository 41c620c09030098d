"""Restatement of the reference's operator producers and of the potential +
electron part of its implicit time step (TEST INFRASTRUCTURE ONLY: the
checker of mps_efield_dev, mps_eden_transport_dev, mps_poisson_source_dev and
mps_plasma_step_dev).

Arrays are ghosted, numpy shape (nz+2, ny+2, nx+2) (Fortran order, i
fastest); vector fields carry a leading axis of 3.  The solves are the FP64
oracle's (oracle.RowsMG), converged to 1e-13.
"""
from __future__ import annotations

import numpy as np

from mps3d_b200.problem import Problem, bc_code

from . import oracle as O

PERI = 4


def ghost_copy(f, bc):
    """update_boundary_ghostvalues with every face 'ZGRD' (ghost = first
    interior value), periodic faces wrapping: the ghost rule update_efield
    applies to E (plasma_pde/poissoneq.f90:580-583, 672-679)."""
    g = f.copy()
    per = [bc_code(bc[2 * a]) == PERI for a in range(3)]
    # x faces over interior (j, k)
    if per[0]:
        g[1:-1, 1:-1, 0], g[1:-1, 1:-1, -1] = f[1:-1, 1:-1, -2], f[1:-1, 1:-1, 1]
    else:
        g[1:-1, 1:-1, 0], g[1:-1, 1:-1, -1] = f[1:-1, 1:-1, 1], f[1:-1, 1:-1, -2]
    if per[1]:
        g[1:-1, 0, 1:-1], g[1:-1, -1, 1:-1] = f[1:-1, -2, 1:-1], f[1:-1, 1, 1:-1]
    else:
        g[1:-1, 0, 1:-1], g[1:-1, -1, 1:-1] = f[1:-1, 1, 1:-1], f[1:-1, -2, 1:-1]
    if per[2]:
        g[0, 1:-1, 1:-1], g[-1, 1:-1, 1:-1] = f[-2, 1:-1, 1:-1], f[1, 1:-1, 1:-1]
    else:
        g[0, 1:-1, 1:-1], g[-1, 1:-1, 1:-1] = f[1, 1:-1, 1:-1], f[-2, 1:-1, 1:-1]
    return g


def _minmod(ntr, dtr):
    """minmodlimiter, plasma_pde/poissoneq.f90:549-563 (elementwise)."""
    out = np.ones_like(ntr)
    nz = dtr != 0
    r = np.zeros_like(ntr)
    r[nz] = ntr[nz] / dtr[nz]
    out[nz] = np.maximum(0.0, np.minimum(1.0, r[nz]))
    return out


def efield(phi, llen, bc, scale=1.0, limiter=False):
    """update_efield (plasma_pde/poissoneq.f90:565-680) on a potential whose
    ghosts are already set: central differences (:593-611), the optional
    minmod limiter (:614-662), E = -scale * grad (:667), ghosts by
    ghost_copy."""
    nz, ny, nx = (s - 2 for s in phi.shape)
    h = (llen[0] / nx, llen[1] / ny, llen[2] / nz)
    c = phi[1:-1, 1:-1, 1:-1]
    xm, xp = phi[1:-1, 1:-1, :-2], phi[1:-1, 1:-1, 2:]
    ym, yp = phi[1:-1, :-2, 1:-1], phi[1:-1, 2:, 1:-1]
    zm, zp = phi[:-2, 1:-1, 1:-1], phi[2:, 1:-1, 1:-1]
    g = [0.5 * (xp - xm) / h[0], 0.5 * (yp - ym) / h[1], 0.5 * (zp - zm) / h[2]]
    if limiter:
        g = [g[0] * _minmod(c - xm, xp - c), g[1] * _minmod(c - ym, yp - c), g[2] * _minmod(c - zm, zp - c)]
    E = np.zeros((3,) + phi.shape)
    for a in range(3):
        E[a][1:-1, 1:-1, 1:-1] = -g[a] * scale
        E[a] = ghost_copy(E[a], bc)
    return E


def eden_transport(E, mu, d=None, te=None, prod=None, n_old=None, dt=None, scaling=(1.0, 1.0, 1.0)):
    """eden_update_transport (plasma_pde/edeneq.f90:360-444) with the mobility
    and diffusivity given as fields: vel = mu E, dcoeff = D (or |mu| te),
    source = production, all scaled (:435-438), + n_old/dt (:441); ghosts
    zero."""
    vel = np.zeros_like(E)
    dc = np.zeros_like(mu)
    src = np.zeros_like(mu)
    I = (slice(1, -1),) * 3
    for a in range(3):
        vel[a][I] = mu[I] * E[a][I] * scaling[0]
    dc[I] = (d[I] if d is not None else np.abs(mu[I]) * te[I]) * scaling[1]
    if prod is not None:
        src[I] = prod[I] * scaling[2]
    if dt is not None:
        src[I] += n_old[I] / dt
    return vel, dc, src


def poisson_source(n_e, n_ion, charge, scale):
    """poisson_update_transport (plasma_pde/poissoneq.f90:335-385): (sum_s
    q_s n_s - n_e) * scale; ghosts zero."""
    src = np.zeros_like(n_e)
    I = (slice(1, -1),) * 3
    q = np.zeros_like(n_e[I])
    for s in range(len(charge)):
        q += charge[s] * n_ion[s][I]
    src[I] = (q - n_e[I]) * scale
    return src


def _ghosted(interior):
    out = np.zeros(tuple(s + 2 for s in interior.shape))
    out[1:-1, 1:-1, 1:-1] = interior
    return out


def plasma_step(case, n_e):
    """One potential + electron step (plasma_pde/solve_manager.f90:363-502:
    poisson_solve, update_efield, eden_solve with its floor and ghosts,
    edeneq.f90:446-525) over the oracle's FP64 solves.  Returns the ghosted
    phi, E, vel, dcoeff, source and the new ghosted n_e."""
    nx, ny, nz = case["shape"]
    llen = case["llen"]
    psrc = poisson_source(n_e, case["n_ion"], case["ion_charge"], case["rho_scale"])
    P = Problem(nx, ny, nz, llen, dcoeff=case["eps"], source=psrc, bc=list(case["phi_bc"]),
                bcvals=list(case["phi_bcvals"]))
    x, hist = O.RowsMG(P, hier=O.HIER_GEOM).solve(O.build_rhs(P), maxit=80, tol=1e-13)
    assert hist[-1] <= 1e-13, hist[-3:]
    phi = _ghosted(x)
    O.fill_ghosts(P, phi)
    E = efield(phi, llen, case["phi_bc"], case.get("efield_scale", 1.0), case.get("limiter", False))
    vel, dc, src = eden_transport(E, case["mu_e"], case.get("d_e"), case.get("te"), case.get("prod_e"), n_e,
                                  case["dt"], case.get("scaling", (1.0, 1.0, 1.0)))
    Pe = Problem(nx, ny, nz, llen, dcoeff=dc, source=src, vel=vel, bc=list(case["ne_bc"]),
                 bcvals=list(case["ne_bcvals"]), timederiv=True, dt=case["dt"], flux=1)
    ne, hist = O.RowsMG(Pe, hier=O.HIER_GEOM).fgmres(O.build_rhs(Pe), m=30, maxit=200, tol=1e-13)
    assert hist[-1] <= 1e-13, hist[-3:]
    ne = np.maximum(ne, case["nemin"])
    neg = _ghosted(ne)
    O.fill_ghosts(Pe, neg)
    return phi, E, vel, dc, src, neg
