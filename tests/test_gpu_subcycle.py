"""The small levels of the V-cycle in one thread block (k_subcycle) against
the per-level launches.

From the first level of at most 8192 cells down to the coarsest, the solver
runs one launch of one block with the fields in shared memory instead of one
launch per colour pass, transfer and coarsest solve.  Both forms evaluate the
same operators and transfers, so a V-cycle from the same iterate must agree to
rounding, and solves must take the same iterations.  A handle created with
MPS_SUBCYCLE=0 in the environment runs the per-level launches only.  Cases:
variable and uniform coefficients, a reaction field with 1/dt, periodic,
Dirichlet and zero-gradient faces, merged (odd) cells on the small levels,
elongated shapes, and hierarchies the block form leaves alone (odd periodic
sizes among its levels).  Convergence at the benchmark sizes is checked
against the FP64 oracle by test_gpu_configs.py.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import capi, solver, workloads as W  # noqa: E402
from mps3d_b200.problem import Problem  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handles():
    assert torch.cuda.is_available()
    old = os.environ.get("MPS_SUBCYCLE")
    os.environ["MPS_SUBCYCLE"] = "0"
    try:
        per_level = capi.Handle(0)
    finally:
        if old is None:
            del os.environ["MPS_SUBCYCLE"]
        else:
            os.environ["MPS_SUBCYCLE"] = old
    block = capi.Handle(0)
    yield per_level, block
    per_level.close()
    block.close()


def diffusion(nx, ny, nz, bc, seed, reac=False, dt=None, llen=(1.0, 0.8, 1.2)):
    """Random positive coefficient field, random source and face values;
    optionally a negative reaction field (diagonal -reac) and 1/dt."""
    rng = np.random.default_rng(seed)
    g = (nz + 2, ny + 2, nx + 2)
    dc = rng.uniform(0.5, 2.0, size=g)
    src = rng.uniform(-1.0, 1.0, size=g)
    shapes = [(nz, ny), (nz, ny), (nz, nx), (nz, nx), (ny, nx), (ny, nx)]
    bcv = [rng.uniform(-1, 1, size=s) for s in shapes]
    kw = {}
    if reac:
        kw["reac"] = -rng.uniform(0.5, 3.0, size=g)
    if dt is not None:
        kw["timederiv"] = True
        kw["dt"] = dt
    return Problem(nx, ny, nz, llen, dcoeff=dc, source=src, bc=bc, bcvals=bcv, **kw)


# (name, problem, whether the one-block sub-cycle applies)
CASES = [
    ("plasma-65", lambda: W.plasma_poisson(65), True),
    ("poisson-const-41", lambda: W.poisson_dirichlet(41), True),
    ("peri-x-32x24x16", lambda: diffusion(32, 24, 16, ["PERI", "PERI", "DIRC", "DIRC", "ZGRD", "DIRC"], 2), True),
    ("reac-dt-zgrd-36x28x20", lambda: diffusion(36, 28, 20, ["ZGRD"] * 6, 3, reac=True, dt=0.05), True),
    ("elongated-70x20x9", lambda: diffusion(70, 20, 9, ["DIRC", "ZGRD", "DIRC", "DIRC", "ZGRD", "DIRC"], 4,
                                             llen=(7.0, 2.0, 0.9)), True),
    ("plasma-48-odd-periodic-coarse", lambda: W.plasma_poisson(48), False),
]


def _run_pair(handles, p, **kw):
    per_level, block = handles
    xr, ir = solver.linsolve(p, handle=per_level, **kw)
    xb, ib = solver.linsolve(p, handle=block, **kw)
    return xr, ir, xb, ib


@pytest.mark.parametrize("name,make,applies", CASES, ids=[c[0] for c in CASES])
def test_vcycle_matches_per_level_launches(handles, name, make, applies):
    per_level, block = handles
    p = make()
    rng = np.random.default_rng(11)
    x0 = rng.uniform(-1.0, 1.0, size=p.zeros_ghosted().shape)
    xr, _ = solver.vcycle_once(p, x0, handle=per_level, hierarchy="geom")
    xb, _ = solver.vcycle_once(p, x0, handle=block, hierarchy="geom")
    scale = np.abs(xr).max()
    diff = np.abs(xb - xr).max() / scale
    print(f"{name}: one FP64 V-cycle, block vs per-level, max relative difference {diff:.3e}")
    # the same operators and transfers in another summation order: rounding
    assert diff <= 1e-11, (name, diff)
    if not applies:
        assert diff == 0.0, (name, diff)


@pytest.mark.parametrize("name,make,applies", CASES, ids=[c[0] for c in CASES])
def test_fixed_iterations_match(handles, name, make, applies):
    p = make()
    for precision, bound in (("fp64", 1e-11), ("mixed", 1e-5)):
        xr, ir, xb, ib = _run_pair(handles, p, precision=precision, maxit=2, tol=1e-30)
        assert ir["iters"] == ib["iters"] == 2
        diff = np.abs(xb - xr).max() / np.abs(xr).max()
        print(f"{name} {precision}: two iterations, max relative difference {diff:.3e}; "
              f"launches {ir['launches']} per level, {ib['launches']} block")
        assert diff <= bound, (name, precision, diff)
        if applies:
            assert ib["launches"] < ir["launches"], (name, precision)
        else:
            assert ib["launches"] == ir["launches"], (name, precision)


@pytest.mark.parametrize("name,make,applies", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solves_converge_alike(handles, name, make, applies, precision):
    p = make()
    xr, ir, xb, ib = _run_pair(handles, p, precision=precision, tol=1e-10, raise_not_converged=True)
    assert ir["rel_res"] <= 1e-10 and ib["rel_res"] <= 1e-10
    assert abs(ir["iters"] - ib["iters"]) <= 1, (ir["iters"], ib["iters"])
    diff = np.abs(xb - xr).max() / np.abs(xr).max()
    assert diff <= 1e-8, (name, precision, diff)
