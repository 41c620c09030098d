"""GPU parity: the CUDA library (through its C ABI) against the FP64 oracle.

Operator-level checks are exact up to floating-point reassociation (relative
1e-13); solves must reach relative residual <= 1e-10 and relative solution
error <= 1e-9 against the oracle's converged FP64 solution.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import capi, solver, workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

OP_TOL = 1e-13
BCS = [
    ["DIRC", "DIRC", "ZGRD", "FLUX", "DIRC", "ZGRD"],
    ["PERI", "PERI", "DIRC", "ZGRD", "PERI", "PERI"],
    ["ZGRD", "DIRC", "PERI", "PERI", "FLUX", "DIRC"],
    ["DIRC"] * 6,
]
SHAPES = [(5, 6, 7), (8, 8, 8), (9, 4, 6), (17, 16, 15)]


@pytest.fixture(scope="module")
def handle():
    assert torch.cuda.is_available()
    return capi.Handle(0)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kind", ["poisson", "varcoef", "convection"])
def test_apply_A_matches_find_AX(handle, bc, shape, kind):
    p = W.random_operator(*shape, bc=bc, seed=11, vel=(kind == "convection"), reac=(kind != "poisson"),
                          timederiv=(kind == "convection"))
    if kind == "poisson":
        p.dcoeff[...] = 1.7
    u = np.random.default_rng(4).standard_normal(p.ghost_shape)
    AX, _, _ = O.find_AX(p, u)
    dp = solver.DeviceProblem(p)
    out = solver.apply_A_dev(dp, torch.from_numpy(u).cuda(), handle=handle).cpu().numpy()
    assert _rel(out, AX) <= OP_TOL


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("shape", SHAPES[:3])
def test_apply_A_sg_and_transpose(handle, bc, shape):
    p = W.random_operator(*shape, bc=bc, seed=12, vel=True, reac=True, timederiv=True, flux=1)
    rows = O.build_rows(p)
    u = np.random.default_rng(5).standard_normal(p.ghost_shape)
    ui = np.ascontiguousarray(u[1:-1, 1:-1, 1:-1])
    dp = solver.DeviceProblem(p)
    out = solver.apply_A_dev(dp, torch.from_numpy(u).cuda(), handle=handle).cpu().numpy()
    assert _rel(out, O.rows_apply(p, rows, ui)) <= OP_TOL
    outT = solver.apply_A_dev(dp, torch.from_numpy(u).cuda(), handle=handle, transpose=True).cpu().numpy()
    assert _rel(outT, O.rows_apply(p, O.rows_transpose(p, rows), ui)) <= OP_TOL


@pytest.mark.parametrize("bc", BCS)
def test_find_bvec_and_ghosts(handle, bc):
    p = W.random_operator(7, 6, 5, bc=bc, seed=13, vel=True)
    dp = solver.DeviceProblem(p)
    b = solver.find_bvec_dev(dp, handle=handle).cpu().numpy()
    assert _rel(b, O.find_bvec(p)) <= OP_TOL
    u = np.random.default_rng(6).standard_normal(p.ghost_shape)
    ref = O.fill_ghosts(p, u.copy())
    got = solver.fill_ghosts_dev(dp, torch.from_numpy(u.copy()).cuda(), handle=handle).cpu().numpy()
    # faces only (edges/corners are not touched by either)
    for sl in [(slice(1, -1), slice(1, -1), slice(None)), (slice(1, -1), slice(None), slice(1, -1)),
               (slice(None), slice(1, -1), slice(1, -1))]:
        np.testing.assert_allclose(got[sl], ref[sl], rtol=1e-15, atol=0)


@pytest.mark.parametrize("case", ["laplace16_222", "varcoef16", "gpde_512", "odd15"])
def test_vcycle_once_iterates_match_reference(handle, case):
    """mps_vcycle_once == perform_vcycle (CELL hierarchy) cycle by cycle."""
    ranks = (1, 1, 1)
    if case == "laplace16_222":
        p, ranks = W.laplace_test(16), (2, 2, 2)
    elif case == "varcoef16":
        p = W.random_operator(16, 16, 16, bc=["DIRC", "DIRC", "ZGRD", "ZGRD", "DIRC", "FLUX"], seed=14,
                              vel=False, reac=True)
    elif case == "gpde_512":
        p, ranks = W.gpde_step(20, 12, 8, dt=0.1), (5, 1, 2)
    else:
        p = W.random_operator(15, 15, 15, bc=["DIRC"] * 6, seed=15, vel=True, reac=True, timederiv=True)
    xo = p.zeros_ghosted()
    xg = p.zeros_ghosted()
    for it in range(3):
        rn_o = O.vcycle(p, xo, ranks=ranks)
        xg, rn_g = solver.vcycle_once(p, xg, handle=handle, ranks=ranks)
        scale = np.abs(xo[1:-1, 1:-1, 1:-1]).max()
        d = np.abs(xg[1:-1, 1:-1, 1:-1] - xo[1:-1, 1:-1, 1:-1]).max() / scale
        assert d <= 1e-10, (it, d)
        assert abs(rn_g - rn_o) <= 1e-8 * max(rn_o, 1e-300) + 1e-14 * scale, (it, rn_g, rn_o)


def _oracle_solution(p, flux=0):
    mg = O.RowsMG(p, hier=O.HIER_GEOM)
    b = O.build_rhs(p)
    x, hist = mg.fgmres(b, m=40, maxit=300, tol=1e-14)
    assert hist[-1] <= 1e-13
    return x, b


@pytest.mark.parametrize("case", ["config1_33", "config2_33", "config2_17", "gpde_odd", "aniso"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("krylov", [None, "fgmres"])
def test_solve_matches_oracle(handle, case, prec, krylov):
    if case == "config1_33":
        p = W.poisson_dirichlet(33)
    elif case == "config2_33":
        p = W.plasma_poisson(33, slab_cells=4)
    elif case == "config2_17":
        p = W.plasma_poisson(17, slab_cells=3)
    elif case == "gpde_odd":
        p = W.gpde_step(21, 13, 9)
    else:
        p = W.random_operator(24, 13, 18, bc=["DIRC", "ZGRD", "PERI", "PERI", "DIRC", "FLUX"], seed=16, vel=False,
                              reac=True, llen=(1.0, 0.5, 0.8))
    ref, b = _oracle_solution(p)
    x, info = solver.linsolve(p, handle=handle, tol=1e-11, precision=prec, krylov=krylov, maxit=80)
    assert info["status"] == 0, info
    xi = x[1:-1, 1:-1, 1:-1]
    rel_res = np.linalg.norm(b - O.rows_apply(p, O.build_rows(p), np.ascontiguousarray(xi))) / np.linalg.norm(b)
    err = np.linalg.norm(xi - ref) / np.linalg.norm(ref)
    assert rel_res <= 1e-10, rel_res
    assert err <= 1e-9, err


def test_sg_fgmres_matches_oracle(handle):
    p = W.random_operator(20, 18, 16, bc=["PERI", "PERI", "PERI", "PERI", "ZGRD", "ZGRD"], seed=17, vel=True,
                          reac=False, timederiv=True, dt=1e-2, flux=1)
    ref, b = _oracle_solution(p)
    for prec in ("fp64", "mixed"):
        x, info = solver.linsolve(p, handle=handle, tol=1e-11, precision=prec, krylov="fgmres", maxit=100)
        assert info["status"] == 0, info
        err = np.linalg.norm(x[1:-1, 1:-1, 1:-1] - ref) / np.linalg.norm(ref)
        assert err <= 1e-9, (prec, err)


def test_failures_return_status(handle):
    p = W.poisson_dirichlet(9)
    p.source[3, 3, 3] = np.nan
    with pytest.raises(capi.SolverError) as e:
        solver.linsolve(p, handle=handle)
    assert e.value.status == capi.MPS_ERR_NAN
    # pure Neumann operator with a non-zero-mean right-hand side: inconsistent
    q = W.poisson_dirichlet(9)
    q = type(q)(9, 9, 9, (1, 1, 1), dcoeff=q.dcoeff, source=np.ones(q.ghost_shape), bc=["ZGRD"] * 6,
                bcvals=[0.0] * 6)
    x, info = solver.linsolve(q, handle=handle, maxit=5)
    assert info["status"] in (capi.MPS_ERR_NOT_CONVERGED, capi.MPS_ERR_BREAKDOWN)
    # bad arguments
    r = W.poisson_dirichlet(8)
    with pytest.raises(capi.SolverError) as e:
        solver.linsolve(r, handle=handle, hierarchy="cell", ranks=(3, 1, 1))
    assert e.value.status == capi.MPS_ERR_BAD_ARG
    # the handle stays usable after errors
    x, info = solver.linsolve(r, handle=handle)
    assert info["status"] == 0


def test_workspace_allocation_failure_is_a_clean_status(monkeypatch):
    """A handle whose workspace cap (MPS_WORKSPACE_LIMIT_BYTES, read by
    mps_create) is too small for the grid fails the set-up with
    MPS_ERR_NOMEM before any kernel runs, and stays usable for a grid that
    fits."""
    monkeypatch.setenv("MPS_WORKSPACE_LIMIT_BYTES", str(4 << 20))
    h = capi.Handle(0)
    monkeypatch.delenv("MPS_WORKSPACE_LIMIT_BYTES")
    for prec in ("fp64", "mixed"):
        with pytest.raises(capi.SolverError) as e:
            solver.linsolve(W.poisson_dirichlet(65), handle=h, precision=prec)
        assert e.value.status == capi.MPS_ERR_NOMEM
    x, info = solver.linsolve(W.poisson_dirichlet(9), handle=h)
    assert info["status"] == 0
    h.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_electron_sg_step_matches_oracle(handle, prec):
    """Implicit SG electron step (potential: a 33^3 plasma Poisson solve
    injected onto 17^3), FGMRES(30) with a V-cycle preconditioner."""
    pp = W.plasma_poisson(33, slab_cells=4)
    phi_i, _ = _oracle_solution(pp)
    phi = np.zeros((35, 35, 35))
    phi[1:-1, 1:-1, 1:-1] = phi_i
    p = W.electron_sg_step(17, phi=W.inject_potential(phi, 17))
    ref, b = _oracle_solution(p)
    x, info = solver.linsolve(p, handle=handle, tol=1e-11, precision=prec, krylov="fgmres", restart=30, maxit=60)
    assert info["status"] == 0, info
    xi = x[1:-1, 1:-1, 1:-1]
    rel_res = np.linalg.norm(b - O.rows_apply(p, O.build_rows(p), np.ascontiguousarray(xi))) / np.linalg.norm(b)
    assert rel_res <= 1e-10, rel_res
    assert np.linalg.norm(xi - ref) / np.linalg.norm(ref) <= 1e-9
