"""Seeded synthetic inputs for the benchmark configurations.

The reference publishes no datasets for this path; each configuration is a
seeded synthetic stand-in with the shapes, sizes and value distributions the
configuration names (numpy PCG64 generators, seed 1000+c plus a per-field
offset).  All fields are returned as a :class:`Problem` with ghosted
Fortran-order arrays.
"""
from __future__ import annotations

import numpy as np

from .problem import Problem

ECHARGE = 1.602176634e-19  # C
EPS0 = 8.8541878128e-12    # F/m


def _rng(config: int, field: int):
    return np.random.default_rng(1000 + config + 7919 * field)


def poisson_dirichlet(n: int, seed_config: int = 1, length: float = 1.0, nz=None, ny=None) -> Problem:
    """Config 1: -lap u = f on the unit cube, n^3 cells, coefficient 1,
    Dirichlet 0 on all faces, f ~ U[-1,1] (Laplace_test-style operator)."""
    nx = n
    ny = ny or n
    nz = nz or n
    g = (nz + 2, ny + 2, nx + 2)
    dc = np.zeros(g)
    dc[1:-1, 1:-1, 1:-1] = 1.0
    src = np.zeros(g)
    src[1:-1, 1:-1, 1:-1] = _rng(seed_config, 0).uniform(-1.0, 1.0, size=(nz, ny, nx))
    return Problem(nx, ny, nz, (length, length, length), dcoeff=dc, source=src,
                   bc=["DIRC"] * 6, bcvals=[0.0] * 6)


def plasma_poisson(n: int = 257, slab_cells: int = 10, eps_slab: float = 4.0, v_front: float = 1000.0,
                   length: float = 0.01, seed_config: int = 2) -> Problem:
    """Config 2: plasma Poisson on an n^3 grid over a 1 cm cube.

    Permittivity 1 in the gas and ``eps_slab`` in a dielectric slab of
    ``slab_cells`` cells at z=0; Dirichlet 0 V at z=0 (BACK) and ``v_front`` at
    z=1 (FRONT); periodic x/y; right-hand side e(n_i - n_e)/eps0 with n_i, n_e
    lognormal(mu=ln 1e16 m^-3, sigma=1) (the sign of poissoneq.f90:372,377).
    """
    g = (n + 2, n + 2, n + 2)
    eps = np.zeros(g)
    eps[1:-1, 1:-1, 1:-1] = 1.0
    eps[1:1 + slab_cells, 1:-1, 1:-1] = eps_slab
    ni = _rng(seed_config, 1).lognormal(mean=np.log(1e16), sigma=1.0, size=(n, n, n))
    ne = _rng(seed_config, 2).lognormal(mean=np.log(1e16), sigma=1.0, size=(n, n, n))
    src = np.zeros(g)
    src[1:-1, 1:-1, 1:-1] = ECHARGE * (ni - ne) / EPS0
    return Problem(n, n, n, (length, length, length), dcoeff=eps, source=src,
                   bc=["PERI", "PERI", "PERI", "PERI", "DIRC", "DIRC"],
                   bcvals=[None, None, None, None, 0.0, v_front])


def laplace_test(n: int = 128) -> Problem:
    """tests/Laplace_test deck: lap(phi)=0, DIRC 0/1 on x faces, ZGRD elsewhere;
    the discrete solution is phi_i = x_i exactly."""
    g = (n + 2, n + 2, n + 2)
    dc = np.zeros(g)
    dc[1:-1, 1:-1, 1:-1] = 1.0
    return Problem(n, n, n, (1.0, 1.0, 1.0), dcoeff=dc, source=np.zeros(g),
                   bc=["DIRC", "DIRC", "ZGRD", "ZGRD", "ZGRD", "ZGRD"], bcvals=[0.0, 1.0, 0, 0, 0, 0])


def gpde_step(nx=80, ny=48, nz=32, phi=None, dt=0.1) -> Problem:
    """tests/gpde_test deck, one implicit step: dphi/dt + div(-x phi) =
    div(0.5 grad phi) + 2 phi - x^2 (generic_pde/pdedefs.f90:244-278)."""
    g = (nz + 2, ny + 2, nx + 2)
    x = (np.arange(nx) + 0.5) / nx
    vel = np.zeros((3,) + g)
    vel[0][1:-1, 1:-1, 1:-1] = -1.0
    dc = np.zeros(g)
    dc[1:-1, 1:-1, 1:-1] = 0.5
    re = np.zeros(g)
    re[1:-1, 1:-1, 1:-1] = 2.0
    src = np.zeros(g)
    src[1:-1, 1:-1, 1:-1] = -(x ** 2)[None, None, :]
    if phi is not None:
        src = src + phi / dt
    return Problem(nx, ny, nz, (1.0, 0.6, 0.4), dcoeff=dc, source=src, vel=vel, reac=re,
                   bc=["DIRC", "FLUX", "ZGRD", "ZGRD", "ZGRD", "ZGRD"], bcvals=[0.0, -0.25, 0, 0, 0, 0],
                   timederiv=True, dt=dt)


def random_operator(nx, ny, nz, bc, seed=0, vel=True, reac=True, timederiv=False, dt=1e-2, flux=0,
                    llen=(1.0, 0.8, 1.2)) -> Problem:
    """Random positive coefficients/velocities for operator parity tests."""
    rng = np.random.default_rng(seed)
    g = (nz + 2, ny + 2, nx + 2)
    dc = rng.uniform(0.5, 2.0, size=g)
    v = rng.uniform(-3.0, 3.0, size=(3,) + g) if vel else None
    r = rng.uniform(-1.0, 0.0, size=g) if reac else None
    src = rng.uniform(-1.0, 1.0, size=g)
    shapes = [(nz, ny), (nz, ny), (nz, nx), (nz, nx), (ny, nx), (ny, nx)]
    bcv = [rng.uniform(-1, 1, size=s) for s in shapes]
    return Problem(nx, ny, nz, llen, dcoeff=dc, source=src, vel=v, reac=r, bc=bc, bcvals=bcv,
                   timederiv=timederiv, dt=dt, flux=flux)
