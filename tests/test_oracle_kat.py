"""The oracle against the reference's own known-answer decks.

tests/Laplace_test (128^3, 2x2x2 ranks, DIRC 0/1 on x, ZGRD elsewhere): the
cell-centred operator reproduces phi = x exactly.  tests/gpde_test (80x48x32,
5x1x2 ranks): the implicit march converges to 0.5(x^2-x) up to the first-order
upwind error.  Reduced sizes keep the CPU suite fast; the rank layouts are the
decks' own.
"""
import numpy as np
import pytest

from mps3d_b200 import workloads as W
from oracle import oracle as O


@pytest.mark.parametrize("n,ranks", [(16, (2, 2, 2)), (32, (2, 2, 2)), (24, (1, 1, 1))])
def test_laplace_known_answer(n, ranks):
    p = W.laplace_test(n)
    s, rel, rms = O.solve(p, ranks=ranks, maxit=30, tol=1e-11, tol_kind=0)
    x = (np.arange(n) + 0.5) / n
    assert rms[-1] <= 1e-11
    np.testing.assert_allclose(s[1:-1, 1:-1, 1:-1], np.broadcast_to(x, (n, n, n)), atol=1e-11)


def _march(nx, ny, nz, ranks, steps=200, dt=0.1, nv=10):
    phi = np.zeros((nz + 2, ny + 2, nx + 2))
    for _ in range(steps):
        p = W.gpde_step(nx, ny, nz, phi=phi, dt=dt)
        phi, rel, rms = O.solve(p, soln=phi, ranks=ranks, maxit=nv, tol=1e-14, tol_kind=0)
    x = (np.arange(nx) + 0.5) / nx
    return np.abs(phi[1:-1, 1:-1, 1:-1] - 0.5 * (x ** 2 - x)[None, None, :]).max()


def test_gpde_known_answer_first_order():
    e1 = _march(20, 12, 8, (5, 1, 2))
    e2 = _march(40, 24, 16, (5, 1, 2))
    assert e1 < 0.15 * (1 / 20)
    assert e2 < 0.15 * (1 / 40)
    assert 1.5 < e1 / e2 < 2.5  # first-order upwind convergence


def test_cell_hierarchy_rate_matches_reference_behaviour():
    # 2 pre / 2 post RB-GS V-cycle on Laplace: ~0.17 per cycle, monotone
    p = W.laplace_test(32)
    s, rel, rms = O.solve(p, ranks=(2, 2, 2), maxit=8, tol=0, tol_kind=1)
    rates = rel[1:] / rel[:-1]
    assert np.all(rates < 0.25)
