"""The finest level's red/black colour pass staged in shared memory by the
Tensor Memory Accelerator (k_colour_tma, FP32: the mixed solve's V-cycle)
against the register-fed pass (k_colourv_split).

Both forms evaluate every cell with the same operation order, so solves run
for a fixed number of iterations must give the same iterate.  A handle
created with MPS_TMA=0 in the environment runs the register-fed pass only.  Cases: variable and constant coefficients, periodic seams of odd and
even length, Dirichlet / zero-gradient faces, shapes whose rows and planes do
not divide into the tiles.  Convergence at the benchmark sizes is checked
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
    old = os.environ.get("MPS_TMA")
    os.environ["MPS_TMA"] = "0"
    try:
        reg = capi.Handle(0)
    finally:
        if old is None:
            del os.environ["MPS_TMA"]
        else:
            os.environ["MPS_TMA"] = old
    tma = capi.Handle(0)
    yield reg, tma
    reg.close()
    tma.close()


def diffusion(nx, ny, nz, bc, seed):
    """Random positive coefficient field (diffusion only), random source and
    face values."""
    rng = np.random.default_rng(seed)
    g = (nz + 2, ny + 2, nx + 2)
    dc = rng.uniform(0.5, 2.0, size=g)
    src = rng.uniform(-1.0, 1.0, size=g)
    shapes = [(nz, ny), (nz, ny), (nz, nx), (nz, nx), (ny, nx), (ny, nx)]
    bcv = [rng.uniform(-1, 1, size=s) for s in shapes]
    return Problem(nx, ny, nz, (1.0, 0.8, 1.2), dcoeff=dc, source=src, bc=bc, bcvals=bcv)


CASES = [
    ("plasma-65", lambda: W.plasma_poisson(65)),
    ("plasma-48", lambda: W.plasma_poisson(48)),
    ("poisson-const-41", lambda: W.poisson_dirichlet(41)),
    ("peri-odd-45x37x29", lambda: diffusion(45, 37, 29, ["PERI"] * 6, 1)),
    ("mixed-bc-40x36x24", lambda: diffusion(40, 36, 24, ["PERI", "PERI", "DIRC", "DIRC", "ZGRD", "DIRC"], 2)),
    ("rows-50x70x19", lambda: diffusion(50, 70, 19, ["ZGRD", "DIRC", "DIRC", "ZGRD", "PERI", "PERI"], 4)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_tma_colour_pass_matches_register_pass(handles, name, make):
    reg, tma = handles
    p = make()
    precision = "mixed"
    kw = dict(precision=precision, maxit=2, tol=1e-30)
    xr, ir = solver.linsolve(p, handle=reg, **kw)
    xt, it = solver.linsolve(p, handle=tma, **kw)
    assert ir["iters"] == it["iters"] == 2
    diff = np.abs(xt - xr).max() / np.abs(xr).max()
    print(f"{name}: TMA vs register colour pass, max relative difference {diff:.3e}")
    # the same arithmetic per cell: equal iterates (measured: bit-identical;
    # the bound at FP32 rounding of the V-cycle correction allows for the
    # compiler's contraction choices)
    assert diff <= 1e-6, (name, diff)
