"""Restatement of the reference's 1D manufactured-solution driver with the
Scharfetter-Gummel flux (TEST INFRASTRUCTURE ONLY: the known answer that pins
the oracle's 3D SG operator, and through it the CUDA SG kernels).

The reference program, mps1d/source/pde_driver/mms1/mms.f90:29-124, solves

    d/dx(c u) = d/dx(k du/dx) + r u + s,  c = -1, k = 0.5, r = 2, s = -x^2

on [0, 1] with u = 0 at both ends; the exact solution is 0.5 (x^2 - x).  It
discretises on np = 2^n + 1 vertices (dx = 1/(np - 1)) with findAX
(mps1d/source/convdiff.f90:236-314): per face i, i+1 the SG weights of
find_sg_exponential_flux (convdiff.f90:10-64), AX(i) += flux/dx,
AX(i+1) -= flux/dx, no separate diffusion for scheme 4 (:289), AX -= reac X,
Dirichlet rows AX(1) = X(1), AX(np) = X(np); the right-hand side is findrhs
(:316-341): b = source, b(1) = b(np) = the Dirichlet values.  The reference
solves that system with GMRES to 1e-9 (mms.f90:99-106); here it is solved
exactly (dense), and the reported figure is the same L2 error,
sqrt(sum (phi - exact)^2 / np) (mms.f90:113-121).
"""
from __future__ import annotations

import math

import numpy as np


def sg_face(cL, cR, DL, DR, dx):
    """find_sg_exponential_flux (mps1d/source/convdiff.f90:10-64): (wL, wR)."""
    eps = 1.0e-10
    c_half = 0.5 * (cL + cR)
    D_half = 2.0 * DL * DR / (DL + DR + eps)
    sign_c = -1.0 if c_half <= 0.0 else 1.0
    if abs(D_half) < eps:
        return cL * 0.5 * (1.0 + sign_c), cR * 0.5 * (1.0 - sign_c)
    Pe = c_half * dx / D_half
    if abs(Pe) < eps:
        return D_half / dx, -D_half / dx
    if Pe > 0.0:
        e = math.exp(-Pe)
        return c_half / (1.0 - e), -c_half * e / (1.0 - e)
    e = math.exp(Pe)
    return c_half * e / (e - 1.0), -c_half / (e - 1.0)


def mms_sg(np_points: int):
    """(x, phi, exact, l2err) of the reference's MMS problem with flux scheme
    4 on ``np_points`` vertices."""
    n = int(np_points)
    dx = 1.0 / (n - 1)
    x = np.arange(n) * dx
    vel = np.full(n, -1.0)
    dco = np.full(n, 0.5)
    reac = np.full(n, 2.0)
    src = -(x ** 2)
    A = np.zeros((n, n))
    for i in range(n - 1):  # faces (convdiff.f90:258-290)
        wL, wR = sg_face(vel[i], vel[i + 1], dco[i], dco[i + 1], dx)
        A[i, i] += wL / dx
        A[i, i + 1] += wR / dx
        A[i + 1, i] -= wL / dx
        A[i + 1, i + 1] -= wR / dx
    A[np.arange(n), np.arange(n)] -= reac  # reaction (:293-295)
    A[0, :] = 0.0                          # Dirichlet rows (:298-303)
    A[0, 0] = 1.0
    A[-1, :] = 0.0
    A[-1, -1] = 1.0
    b = src.copy()                         # findrhs (:330-341)
    b[0] = 0.0
    b[-1] = 0.0
    phi = np.linalg.solve(A, b)
    exact = 0.5 * (x ** 2 - x)
    l2 = math.sqrt(float(np.sum((phi - exact) ** 2)) / n)
    return x, phi, exact, l2


def quasi_1d_problem(n_cells: int, ny: int = 2, nz: int = 2):
    """The same problem on the 3D cell-centred operator: ``n_cells`` cells in
    x over [0, 1], Dirichlet 0 on both x faces, zero-flux y and z faces
    (ZGRD with no velocity across them: every field is uniform in y and z),
    SG faces."""
    from mps3d_b200.problem import Problem

    g = (nz + 2, ny + 2, n_cells + 2)
    xc = (np.arange(n_cells) + 0.5) / n_cells
    vel = np.zeros((3,) + g)
    vel[0][...] = -1.0
    dc = np.full(g, 0.5)
    re = np.full(g, 2.0)
    src = np.zeros(g)
    src[1:-1, 1:-1, 1:-1] = -(xc ** 2)[None, None, :]
    return Problem(n_cells, ny, nz, (1.0, ny / n_cells, nz / n_cells), dcoeff=dc, source=src, vel=vel, reac=re,
                   bc=["DIRC", "DIRC", "ZGRD", "ZGRD", "ZGRD", "ZGRD"], bcvals=[0.0] * 6, flux=1)


def l2_error_cells(prob, phi_interior):
    """The reference's L2 error measure on the cell centres of the quasi-1D
    problem (every y/z cell; they are equal)."""
    xc = (np.arange(prob.lx) + 0.5) / prob.lx
    exact = 0.5 * (xc ** 2 - xc)
    d = np.asarray(phi_interior) - exact[None, None, :]
    return math.sqrt(float(np.mean(d ** 2)))
