"""The CUDA SG path on the reference's SG known answer: the manufactured
solution of mps1d/source/pde_driver/mms1/mms.f90 (flux scheme 4) laid along x
of the 3D operator (oracle/mms1d.py).  The GPU solve (FGMRES with a V-cycle
preconditioner, FP64 and mixed) must agree with the oracle's solution and so
converge to 0.5 (x^2 - x) at second order with the oracle's error constant."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import capi, solver  # noqa: E402
from oracle import mms1d as M  # noqa: E402
from oracle import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_gpu_sg_solves_converge_to_mms_solution(prec):
    h = capi.Handle(0)
    errs = []
    for n in (16, 32, 64, 128):
        p = M.quasi_1d_problem(n)
        mg = O.RowsMG(p, hier=O.HIER_GEOM)
        xo, hist = mg.fgmres(O.build_rhs(p), m=30, maxit=200, tol=1e-12)
        x, info = solver.linsolve(p, handle=h, tol=1e-12, precision=prec, krylov="fgmres", restart=30, maxit=100)
        assert info["status"] == 0, info
        xi = x[1:-1, 1:-1, 1:-1]
        assert np.linalg.norm(xi - xo) / np.linalg.norm(xo) <= 1e-9
        e = M.l2_error_cells(p, xi)
        assert e == pytest.approx(M.l2_error_cells(p, xo), rel=1e-6)
        assert e <= 0.25 / n ** 2
        errs.append(e)
    orders = [math.log2(a / b) for a, b in zip(errs, errs[1:])]
    assert all(1.95 <= o <= 2.05 for o in orders), errs
    h.close()
