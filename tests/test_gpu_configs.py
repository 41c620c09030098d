"""GPU parity at the benchmark configurations' own sizes.

Every workload the benchmark reports is solved here through the C ABI with
the benchmark's own settings (zero initial guess, stop at relative residual
1e-10) and compared with the FP64 oracle on the same seeded inputs:

* the relative residual ||b - A x|| / ||b|| is evaluated by the oracle
  (its own rows and right-hand side, not the GPU's residual kernel) and must
  be <= 1e-10;
* the relative solution error against the oracle's FP64 solve, converged to
  1e-13 or below, must be <= 1e-9.

Workloads: plasma Poisson at 257^3 (mixed and FP64), Poisson at 65^3, the
implicit Scharfetter-Gummel electron step at 129^3 whose potential is the
257^3 oracle solution injected onto 129^3 (FGMRES, mixed and FP64), the
64-problem batch of sizes 33..129 (batched mixed and FP64), and the
electron-flux gradient at 33^3 against the same model over the FP64 oracle.
The oracle runs on the host cores (OpenMP); the 257^3 reference solve takes
tens of seconds.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import capi, solver, workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-10        # the benchmark's stop test (relative residual)
RES_BAR = 1e-10    # oracle-evaluated relative residual
ERR_BAR = 1e-9     # relative solution error against the converged FP64 oracle solve


@pytest.fixture(scope="module")
def handle():
    assert torch.cuda.is_available()
    h = capi.Handle(0)
    yield h
    h.close()


def oracle_reference(p, krylov=False):
    """(x, b, rows): the oracle's FP64 solution converged to <= 1e-13, its
    right-hand side and its fine-level rows."""
    mg = O.RowsMG(p, hier=O.HIER_GEOM)
    b = O.build_rhs(p)
    if krylov:
        x, hist = mg.fgmres(b, m=30, maxit=200, tol=1e-13)
    else:
        x, hist = mg.solve(b, maxit=80, tol=1e-13)
    assert hist[-1] <= 1e-13, hist[-3:]
    return x, b, mg.rows(0)


def check(p, x_ghosted, ref):
    x_ref, b, rows = ref
    xi = np.ascontiguousarray(x_ghosted[1:-1, 1:-1, 1:-1])
    rel_res = np.linalg.norm(b - O.rows_apply(p, rows, xi)) / np.linalg.norm(b)
    err = np.linalg.norm(xi - x_ref) / np.linalg.norm(x_ref)
    assert rel_res <= RES_BAR, rel_res
    assert err <= ERR_BAR, err
    return rel_res, err


def device_solve(p, handle, **kw):
    dp = solver.DeviceProblem(p)
    x = torch.zeros(p.ghost_shape, dtype=torch.float64, device="cuda")
    _, info = solver.linsolve_dev(dp, x, handle=handle, tol=TOL, maxit=60, **kw)
    assert info["status"] == 0, info
    return x.cpu().numpy(), info


@pytest.fixture(scope="module")
def plasma257():
    p = W.plasma_poisson(257)
    return p, oracle_reference(p)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_config2_plasma_poisson_257(handle, plasma257, prec):
    p, ref = plasma257
    x, info = device_solve(p, handle, precision=prec)
    check(p, x, ref)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_config1_poisson_65(handle, prec):
    p = W.poisson_dirichlet(65)
    x, _ = device_solve(p, handle, precision=prec)
    check(p, x, oracle_reference(p))


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_config3_sg_step_129(handle, plasma257, prec):
    _, (phi_i, _, _) = plasma257
    phi = np.zeros((259, 259, 259))
    phi[1:-1, 1:-1, 1:-1] = phi_i
    p = W.electron_sg_step(129, phi=W.inject_potential(phi, 129))
    ref = oracle_reference(p, krylov=True)
    x, _ = device_solve(p, handle, precision=prec, krylov="fgmres", restart=30)
    check(p, x, ref)


@pytest.fixture(scope="module")
def batch64():
    ps = W.batch_poisson(64)
    return ps, [oracle_reference(p) for p in ps]


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_config4_batch_of_64(handle, batch64, prec):
    ps, refs = batch64
    assert sorted({p.lx for p in ps}) == [33, 49, 65, 97, 129]
    dps = [solver.DeviceProblem(p) for p in ps]
    xs = [torch.zeros(p.ghost_shape, dtype=torch.float64, device="cuda") for p in ps]
    infos = solver.linsolve_batched_dev(dps, xs, handle=handle, tol=TOL, precision=prec, maxit=60)
    for p, x, info, ref in zip(ps, xs, infos, refs):
        assert info["status"] == 0, info
        check(p, x.cpu().numpy(), ref)


@pytest.mark.parametrize("n", [33, 129])
def test_config5_gradient_matches_fp64_oracle(n):
    """The electron-flux gradient (5 implicit SG steps, V and the FP32
    mobility field) at 33^3 and at the configuration's 129^3 against the same
    model over the FP64 oracle."""
    from adjoint_oracle import oracle_bvec, oracle_solve
    from mps3d_b200.adjoint import ElectronFluxAdjoint

    case = W.electron_adjoint_case(n)
    V = case["v_front"]
    mu = torch.from_numpy(case["mu"])
    gpu = ElectronFluxAdjoint(case, device="cuda", tol=1e-12)
    ref = ElectronFluxAdjoint(case, device="cpu", solve_fn=oracle_solve, bvec_fn=oracle_bvec)
    # FP64 mobility on both sides: the gradients themselves in FP64
    L, gV, gmu = gpu.gradient(V, mu.double().cuda())
    L_r, gV_r, gmu_r = ref.gradient(V, mu.double())
    assert abs(L - L_r) <= 1e-9 * abs(L_r), (L, L_r)
    assert abs(gV - gV_r) <= 1e-9 * abs(gV_r), (gV, gV_r)
    g, gr = gmu.cpu().numpy(), gmu_r.numpy()
    assert np.linalg.norm(g - gr) / np.linalg.norm(gr) <= 1e-9
    # the FP32 mobility field of the configuration: its gradient is the FP64
    # one rounded to FP32
    _, _, g32 = gpu.gradient(V, mu.cuda())
    assert g32.dtype == torch.float32
    assert np.linalg.norm(g32.cpu().double().numpy() - gr) / np.linalg.norm(gr) <= 1e-7
