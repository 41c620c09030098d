"""Self-consistency of the oracle's two layers (restatement vs rows machinery)."""
import numpy as np
import pytest

from mps3d_b200 import workloads as W
from oracle import oracle as O

BCS = [
    ["DIRC", "DIRC", "ZGRD", "FLUX", "DIRC", "ZGRD"],
    ["PERI", "PERI", "DIRC", "ZGRD", "PERI", "PERI"],
    ["ZGRD", "DIRC", "PERI", "PERI", "FLUX", "DIRC"],
]


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("shape", [(5, 6, 7), (8, 8, 8), (9, 4, 6)])
def test_rows_match_find_AX(bc, shape):
    p = W.random_operator(*shape, bc=bc, seed=3, timederiv=True)
    u = np.random.default_rng(1).standard_normal(p.ghost_shape)
    AX, d, o = O.find_AX(p, u)
    rows = O.build_rows(p, flux=0)
    Au = O.rows_apply(p, rows, np.ascontiguousarray(u[1:-1, 1:-1, 1:-1]))
    np.testing.assert_allclose(Au, AX, rtol=1e-12, atol=1e-12 * np.abs(AX).max())
    np.testing.assert_allclose(rows[0], d, rtol=1e-12)


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("flux", [0, 1])
def test_transpose_identity(bc, flux):
    p = W.random_operator(6, 5, 7, bc=bc, seed=5, flux=flux)
    rows = O.build_rows(p)
    rT = O.rows_transpose(p, rows)
    rng = np.random.default_rng(2)
    x = rng.standard_normal(p.shape)
    y = rng.standard_normal(p.shape)
    lhs = np.vdot(O.rows_apply(p, rows, x), y)
    rhs = np.vdot(x, O.rows_apply(p, rT, y))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


def test_rows_mg_matches_fas_vcycle_cell():
    # the correction-scheme V-cycle over rows equals the reference FAS V-cycle
    p = W.random_operator(16, 16, 16, bc=["DIRC", "DIRC", "ZGRD", "ZGRD", "DIRC", "FLUX"], seed=7, vel=False,
                          reac=False)
    mg = O.RowsMG(p, hier=O.HIER_CELL)
    b = O.find_bvec(p)
    x_fas = p.zeros_ghosted()
    x_cs = np.zeros(p.shape)
    for _ in range(3):
        O.vcycle(p, x_fas)
        r = b - O.rows_apply(p, mg.rows(0), x_cs)
        e = mg.vcycle(np.zeros(p.shape), r)
        x_cs = x_cs + e
        np.testing.assert_allclose(x_cs, x_fas[1:-1, 1:-1, 1:-1], rtol=1e-10,
                                   atol=1e-10 * np.abs(x_fas).max())


@pytest.mark.parametrize("n,bc,bound", [
    (17, ["DIRC"] * 6, 0.15), (33, ["DIRC"] * 6, 0.15), (32, ["DIRC"] * 6, 0.15),
    (33, ["PERI"] * 4 + ["DIRC", "DIRC"], 0.22), (33, ["PERI"] * 4 + ["DIRC", "ZGRD"], 0.22)])
def test_geom_hierarchy_levels_and_rate(n, bc, bound):
    # odd sizes coarsen by merging the odd cell (33 -> 16 -> 8 -> 4) and keep
    # the even-size rate (trilinear prolongation at the true cell centres)
    p = W.poisson_dirichlet(n)
    p = type(p)(p.lx, p.ly, p.lz, p.llen, dcoeff=p.dcoeff, source=p.source, bc=bc, bcvals=[0.0] * 6)
    mg = O.RowsMG(p, hier=O.HIER_GEOM)
    lv = mg.levels()
    assert lv[0] == (n, n, n)
    assert lv[-1][0] * lv[-1][1] * lv[-1][2] <= 125
    b = O.find_bvec(p)
    x, hist = mg.solve(b, maxit=30, tol=1e-12)
    assert hist[-1] <= 1e-12
    assert np.all(hist[2:] / hist[1:-1] < bound)


def test_periodic_odd_solve_and_fgmres():
    p = W.plasma_poisson(n=17, slab_cells=3)
    mg = O.RowsMG(p, hier=O.HIER_GEOM)
    b = O.find_bvec(p)
    x1, h1 = mg.solve(b, maxit=40, tol=1e-12)
    x2, h2 = mg.fgmres(b, m=30, maxit=60, tol=1e-12)
    assert h1[-1] <= 1e-12 and h2[-1] <= 1e-12
    np.testing.assert_allclose(x1, x2, rtol=1e-9, atol=1e-9 * np.abs(x1).max())


def test_sg_face_limits():
    # SG reduces to central diffusion at Pe -> 0 and to upwinding at large Pe
    wL, wR = O.sg_face(0.0, 0.0, 1.0, 1.0, 0.1)
    assert np.isclose(wL, 10.0, rtol=1e-9) and np.isclose(wR, -10.0, rtol=1e-9)
    wL, wR = O.sg_face(100.0, 100.0, 1e-3, 1e-3, 0.1)
    assert np.isclose(wL, 100.0, rtol=1e-9) and abs(wR) < 1e-12
    wL, wR = O.sg_face(-100.0, -100.0, 1e-3, 1e-3, 0.1)
    assert abs(wL) < 1e-12 and np.isclose(wR, -100.0, rtol=1e-9)
