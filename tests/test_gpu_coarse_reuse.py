"""The coarsest-level inverse is kept with its matrix and reused by the next
solve whose assembled coarsest matrix is the same (repeated solves with one
operator, as in time stepping with a fixed permittivity); any change of the
matrix recomputes it.  Solves on a handle that reuses or recomputes must give
the same answer, bit for bit, as the same solve on a fresh handle."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import capi, solver, workloads as W  # noqa: E402

pytestmark = pytest.mark.gpu

BC = ["DIRC", "ZGRD", "PERI", "PERI", "DIRC", "FLUX"]


def _fresh(p, **kw):
    return solver.linsolve(p, handle=capi.Handle(0), **kw)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_reused_and_recomputed_inverse_match_a_fresh_handle(prec):
    h = capi.Handle(0)
    p = W.random_operator(17, 15, 13, bc=BC, seed=51, vel=False, reac=True)
    x1, i1 = solver.linsolve(p, handle=h, tol=1e-11, precision=prec)
    x2, i2 = solver.linsolve(p, handle=h, tol=1e-11, precision=prec)  # same matrix: reused
    assert i1["status"] == i2["status"] == 0
    assert np.array_equal(x1, x2) and i1["iters"] == i2["iters"]
    # same grid and signature, another coefficient field: recomputed
    q = W.random_operator(17, 15, 13, bc=BC, seed=52, vel=False, reac=True)
    xq, iq = solver.linsolve(q, handle=h, tol=1e-11, precision=prec)
    xr, ir = _fresh(q, tol=1e-11, precision=prec)
    assert iq["status"] == ir["status"] == 0
    assert np.array_equal(xq, xr) and iq["iters"] == ir["iters"]
    # and back to the first operator
    x3, i3 = solver.linsolve(p, handle=h, tol=1e-11, precision=prec)
    assert np.array_equal(x3, x1)


def test_singular_coarsest_operator_reused():
    """A pure Neumann operator has a singular coarsest matrix (its constant
    direction is pinned to zero); the second solve reuses that inverse."""
    base = W.poisson_dirichlet(9)
    src = np.random.default_rng(53).standard_normal(base.ghost_shape)
    src -= src[1:-1, 1:-1, 1:-1].mean()  # a consistent right-hand side
    p = type(base)(9, 9, 9, (1, 1, 1), dcoeff=base.dcoeff, source=src, bc=["ZGRD"] * 6, bcvals=[0.0] * 6)
    h = capi.Handle(0)
    xa, ia = solver.linsolve(p, handle=h, maxit=8)
    xb, ib = solver.linsolve(p, handle=h, maxit=8)
    xc, ic = _fresh(p, maxit=8)
    assert ia["status"] == ib["status"] == ic["status"]
    assert np.array_equal(xa, xb) and np.array_equal(xb, xc)
