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


def inject_potential(phi_fine: np.ndarray, n: int) -> np.ndarray:
    """Cell 2I of a ghosted (2n-1)^3 potential becomes cell I of an n^3 one
    (injection: 257^3 -> 129^3 keeps cells 0, 2, ..., 256)."""
    nf = 2 * n - 1
    assert phi_fine.shape == (nf + 2,) * 3
    out = np.zeros((n + 2,) * 3)
    out[1:-1, 1:-1, 1:-1] = phi_fine[1:-1:2, 1:-1:2, 1:-1:2]
    return out


def electron_sg_step(n: int = 129, phi: np.ndarray = None, v_front: float = 1000.0, length: float = 0.01,
                     dt: float = 1e-11, seed_config: int = 3) -> Problem:
    """Config 3: one implicit electron drift-diffusion step with
    Scharfetter-Gummel faces on an n^3 grid over a 1 cm cube.

    mobility mu = 0.03 (1 + 0.5 U[0,1]) m^2/Vs, D = mu Te with Te ~ U[1,4] eV,
    drift v = -mu E with E = -grad(phi) (electrons; the reference stores the
    signed mobility, ion_elec_chem.f90:234-235), n_old lognormal(ln 1e16, 1)
    m^-3, time derivative 1/dt on the diagonal and n_old/dt in the source
    (edeneq.f90:441).  phi is the ghosted potential of the plasma Poisson
    problem (a (2n-1)^3 solve injected onto n^3, :func:`inject_potential`);
    None gives the linear ramp 0 -> v_front V along z.  x/y periodic, z ZGRD
    (zero diffusive flux, convective outflow).
    """
    g = (n + 2, n + 2, n + 2)
    h = length / n
    if phi is None:
        z = (np.arange(n) + 0.5) * h
        phi = np.zeros(g)
        phi[1:-1, 1:-1, 1:-1] = (v_front * z / length)[:, None, None]
    ph = np.array(phi, dtype=np.float64, copy=True)
    # ghosts of phi: periodic in x/y, Dirichlet 0 / v_front at z=0 / z=L
    ph[1:-1, 1:-1, 0] = ph[1:-1, 1:-1, -2]
    ph[1:-1, 1:-1, -1] = ph[1:-1, 1:-1, 1]
    ph[1:-1, 0, 1:-1] = ph[1:-1, -2, 1:-1]
    ph[1:-1, -1, 1:-1] = ph[1:-1, 1, 1:-1]
    ph[0, 1:-1, 1:-1] = -ph[1, 1:-1, 1:-1]
    ph[-1, 1:-1, 1:-1] = 2.0 * v_front - ph[-2, 1:-1, 1:-1]
    c = ph[1:-1, 1:-1, 1:-1]
    gx = (ph[1:-1, 1:-1, 2:] - ph[1:-1, 1:-1, :-2]) / (2 * h)
    gy = (ph[1:-1, 2:, 1:-1] - ph[1:-1, :-2, 1:-1]) / (2 * h)
    gz = (ph[2:, 1:-1, 1:-1] - ph[:-2, 1:-1, 1:-1]) / (2 * h)
    del c
    mu = 0.03 * (1.0 + 0.5 * _rng(seed_config, 1).uniform(0.0, 1.0, size=(n, n, n)))
    te = _rng(seed_config, 2).uniform(1.0, 4.0, size=(n, n, n))
    nold = _rng(seed_config, 3).lognormal(mean=np.log(1e16), sigma=1.0, size=(n, n, n))

    def ghosted(a):
        out = np.zeros(g)
        out[1:-1, 1:-1, 1:-1] = a
        out[1:-1, 1:-1, 0] = a[:, :, -1]
        out[1:-1, 1:-1, -1] = a[:, :, 0]
        out[1:-1, 0, 1:-1] = a[:, -1, :]
        out[1:-1, -1, 1:-1] = a[:, 0, :]
        out[0, 1:-1, 1:-1] = a[0]
        out[-1, 1:-1, 1:-1] = a[-1]
        return out

    # v = -mu E = mu grad(phi)
    vel = np.stack([ghosted(mu * gx), ghosted(mu * gy), ghosted(mu * gz)])
    dc = ghosted(mu * te)
    src = ghosted(nold / dt)
    return Problem(n, n, n, (length, length, length), dcoeff=dc, source=src, vel=vel,
                   bc=["PERI", "PERI", "PERI", "PERI", "ZGRD", "ZGRD"], bcvals=[None] * 6,
                   timederiv=True, dt=dt, flux=1)


BATCH_SIZES = (33, 49, 65, 97, 129)


def batch_sizes(count: int = 64, sizes=BATCH_SIZES, seed_config: int = 4):
    """The cubic sizes of :func:`batch_poisson` (without building the fields)."""
    return [int(n) for n in _rng(seed_config, 0).choice(np.asarray(sizes), size=count)]


def batch_poisson(count: int = 64, sizes=BATCH_SIZES, seed_config: int = 4):
    """Config 4: ``count`` independent constant-coefficient Poisson problems on
    the unit cube, cubic sizes drawn uniformly from ``sizes``, Dirichlet 0,
    right-hand sides U[-1,1] (a seed per problem)."""
    ns = batch_sizes(count, sizes, seed_config)
    out = []
    for q, n in enumerate(ns):
        n = int(n)
        g = (n + 2, n + 2, n + 2)
        dc = np.zeros(g)
        dc[1:-1, 1:-1, 1:-1] = 1.0
        src = np.zeros(g)
        src[1:-1, 1:-1, 1:-1] = _rng(seed_config, 1 + q).uniform(-1.0, 1.0, size=(n, n, n))
        out.append(Problem(n, n, n, (1.0, 1.0, 1.0), dcoeff=dc, source=src, bc=["DIRC"] * 6, bcvals=[0.0] * 6))
    return out


def electron_adjoint_case(n: int = 129, v_front: float = 1000.0, length: float = 0.01, dt: float = 1e-11,
                          steps: int = 5, slab_cells: int = None):
    """Config 5: the fields of the electron-flux adjoint on an n^3 grid.

    The plasma Poisson problem of config 2 at n^3 (dielectric slab of
    ``slab_cells`` cells, default 10 n / 257 rounded, so the same 0.39 mm),
    whose FRONT Dirichlet value is the electrode voltage, and the electron
    step of config 3 (mobility, Te, n_old) repeated ``steps`` times.  Returns
    a dict of numpy arrays; ``mu`` is float32 (the differentiated field).
    """
    if slab_cells is None:
        slab_cells = max(1, int(round(10 * n / 257)))
    pp = plasma_poisson(n, slab_cells=slab_cells, v_front=v_front, length=length)
    mu = (0.03 * (1.0 + 0.5 * _rng(3, 1).uniform(0.0, 1.0, size=(n, n, n)))).astype(np.float32)
    te = _rng(3, 2).uniform(1.0, 4.0, size=(n, n, n))
    nold = _rng(3, 3).lognormal(mean=np.log(1e16), sigma=1.0, size=(n, n, n))
    return {"n": n, "length": length, "dt": dt, "steps": steps, "v_front": v_front, "eps": pp.dcoeff,
            "rho": pp.source, "mu": mu, "te": te, "n_old": nold}


def plasma_step_case(n: int = 129, slab_cells: int = None, v_front: float = 1000.0, length: float = 0.01,
                     dt: float = 1e-11, nemin: float = 1e7):
    """The potential + electron part of one implicit step on an n^3 grid
    over a 1 cm cube: the plasma Poisson problem of config 2 (dielectric slab,
    Dirichlet 0 / v_front on z, periodic x/y) with one singly charged ion
    species, and the electrons of config 3 (signed mobility
    -0.03 (1 + 0.5 U[0,1]) m^2/Vs, Te ~ U[1,4] V, D = |mu| Te, dt, periodic
    x/y and ZGRD z, floor nemin).  Returns a dict of ghosted numpy arrays and
    settings, and the initial electron density under ``n_e0``."""
    if slab_cells is None:
        slab_cells = max(1, int(round(10 * n / 257)))
    pp = plasma_poisson(n, slab_cells=slab_cells, v_front=v_front, length=length)
    g = (n + 2,) * 3

    def ghosted(a):
        out = np.zeros(g)
        out[1:-1, 1:-1, 1:-1] = a
        return out

    ni = ghosted(_rng(2, 1).lognormal(mean=np.log(1e16), sigma=1.0, size=(n, n, n)))
    ne = ghosted(_rng(2, 2).lognormal(mean=np.log(1e16), sigma=1.0, size=(n, n, n)))
    mu = ghosted(-0.03 * (1.0 + 0.5 * _rng(3, 1).uniform(0.0, 1.0, size=(n, n, n))))
    te = ghosted(_rng(3, 2).uniform(1.0, 4.0, size=(n, n, n)))
    return {"shape": (n, n, n), "llen": (length,) * 3, "eps": pp.dcoeff, "phi_bc": list(pp.bc),
            "phi_bcvals": [None, None, None, None, pp.bcvals[4], pp.bcvals[5]], "n_ion": ni[None], "ion_charge": [1.0],
            "rho_scale": ECHARGE / EPS0, "ne_bc": ["PERI", "PERI", "PERI", "PERI", "ZGRD", "ZGRD"],
            "ne_bcvals": [None] * 6, "mu_e": mu, "te": te, "d_e": None, "prod_e": None, "dt": dt, "nemin": nemin,
            "efield_scale": 1.0, "limiter": False, "scaling": (1.0, 1.0, 1.0), "n_e0": ne}
