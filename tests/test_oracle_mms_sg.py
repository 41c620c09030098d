"""The oracle's Scharfetter-Gummel operator pinned to the reference's SG known
answer: the 1D manufactured solution of mps1d/source/pde_driver/mms1/mms.f90
(d/dx(-u) = d/dx(0.5 du/dx) + 2u - x^2 on [0, 1], u = 0 at both ends, exact
0.5 (x^2 - x)) with flux scheme 4 (convdiff.f90:10-64).

* The restatement of the reference program (oracle/mms1d.py) converges to
  the exact solution at second order, as the reference's L2-error output
  (mms.f90:113-121) does for scheme 4.
* Its SG face weights equal the oracle's C restatement (orc_sg_face) over
  every branch (upwind when D ~ 0, central when Pe ~ 0, both signs of Pe).
* The oracle's 3D SG operator on the same problem laid along x (cell-centred,
  zero-flux y/z faces) converges to the same exact solution at second order.
"""
import math

import pytest

from oracle import mms1d as M
from oracle import oracle as O


def _orders(errs):
    return [math.log2(a / b) for a, b in zip(errs, errs[1:])]


def test_reference_mms_sg_converges_second_order():
    errs = [M.mms_sg(2 ** k + 1)[3] for k in range(4, 9)]  # 17 .. 257 points
    for o in _orders(errs):
        assert 1.95 <= o <= 2.05, errs
    # the error constant: l2 ~ C dx^2 with C ~ 0.045 for this problem
    for k, e in zip(range(4, 9), errs):
        assert e <= 0.05 * (1.0 / 2 ** k) ** 2


@pytest.mark.parametrize("c", [-1.0, 1.0, -37.0, 37.0, 1e-12, -1e-12, 0.0])
@pytest.mark.parametrize("D", [0.5, 2.0, 1e-12])
def test_sg_weights_agree_with_reference_restatement(c, D):
    dx = 1.0 / 64
    for cL, cR, DL, DR in ((c, c, D, D), (c, 0.5 * c, D, 3.0 * D), (0.3 * c, c, 2.0 * D, D)):
        wl, wr = M.sg_face(cL, cR, DL, DR, dx)
        ol, orr = O.sg_face(cL, cR, DL, DR, dx)
        assert ol == pytest.approx(wl, rel=1e-14, abs=1e-300)
        assert orr == pytest.approx(wr, rel=1e-14, abs=1e-300)


def test_oracle_3d_sg_operator_converges_to_mms_solution():
    errs = []
    for n in (16, 32, 64, 128):
        p = M.quasi_1d_problem(n)
        mg = O.RowsMG(p, hier=O.HIER_GEOM)
        x, hist = mg.fgmres(O.build_rhs(p), m=30, maxit=200, tol=1e-12)
        assert hist[-1] <= 1e-12
        errs.append(M.l2_error_cells(p, x))
        assert errs[-1] <= 0.25 / n ** 2, (n, errs[-1])
    for o in _orders(errs):
        assert 1.95 <= o <= 2.05, errs
