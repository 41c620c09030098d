"""Adjoint on the GPU: mps_operator_vjp_dev against the oracle's VJP; the
electron-flux gradient (transposed SG solves + VJP + symmetric Poisson
adjoint, torch autograd) against the same model over the FP64 oracle and
against central finite differences (h = 1e-4 relative)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import workloads as W  # noqa: E402
from mps3d_b200.adjoint import ElectronFluxAdjoint, OperatorSpec, device_vjp  # noqa: E402
from mps3d_b200.problem import BC_CODES  # noqa: E402
from oracle import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

BCS = [["PERI", "PERI", "PERI", "PERI", "ZGRD", "ZGRD"], ["DIRC", "ZGRD", "DIRC", "FLUX", "DIRC", "DIRC"],
       ["ZGRD", "DIRC", "PERI", "PERI", "FLUX", "ZGRD"]]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("flux", [0, 1])
@pytest.mark.parametrize("bc", BCS)
def test_operator_vjp_matches_oracle(flux, bc):
    p = W.random_operator(13, 9, 7, bc=bc, seed=51, vel=True, reac=True, timederiv=True, flux=flux,
                          llen=(1.0, 0.6, 0.9))
    rng = np.random.default_rng(52)
    lam, u = rng.standard_normal(p.shape), rng.standard_normal(p.shape)
    gv, gd, _ = O.operator_vjp(p, lam, u)
    spec = OperatorSpec(p.lx, p.ly, p.lz, p.llen, tuple(p.bc), flux=flux)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    gv_d, gd_d = device_vjp(spec, t(p.vel), t(p.dcoeff), t(lam), t(u))
    torch.cuda.synchronize()
    assert _rel(gv_d.cpu().numpy(), gv) <= 1e-11
    assert _rel(gd_d.cpu().numpy(), gd) <= 1e-11


def test_electron_flux_gradient_matches_fp64_oracle_gradient():
    from adjoint_oracle import oracle_bvec, oracle_solve

    case = W.electron_adjoint_case(9)
    mu = torch.from_numpy(case["mu"])
    gpu = ElectronFluxAdjoint(case, device="cuda", tol=1e-13)
    L, gV, gmu = gpu.gradient(case["v_front"], mu.cuda())
    ref = ElectronFluxAdjoint(case, device="cpu", solve_fn=oracle_solve, bvec_fn=oracle_bvec)
    L_r, gV_r, gmu_r = ref.gradient(case["v_front"], mu)
    assert abs(L - L_r) <= 1e-10 * abs(L_r)
    assert abs(gV - gV_r) <= 1e-9 * abs(gV_r), (gV, gV_r)
    assert _rel(gmu.cpu().double().numpy(), gmu_r.double().numpy()) <= 1e-9


def test_electron_flux_gradient_matches_central_differences():
    case = W.electron_adjoint_case(17)
    model = ElectronFluxAdjoint(case, device="cuda", tol=1e-13)
    V = case["v_front"]
    mu = torch.from_numpy(case["mu"]).cuda()
    L0, gV, gmu = model.gradient(V, mu)
    assert gmu.dtype == torch.float32
    mu64 = mu.double()
    f = lambda v, m: float(model.loss(torch.tensor(v, dtype=torch.float64, device="cuda"), m))  # noqa: E731
    h = 1e-4 * V
    fd_V = (f(V + h, mu64) - f(V - h, mu64)) / (2 * h)
    assert abs(fd_V - gV) <= 1e-6 * abs(gV), (fd_V, gV)
    # mobility: derivative along a random relative perturbation of every cell
    d = torch.from_numpy(np.random.default_rng(53).uniform(-1.0, 1.0, size=case["mu"].shape)).cuda() * mu64 * 1e-4
    fd_mu = (f(V, mu64 + d) - f(V, mu64 - d)) / 2.0
    an = float((gmu.double() * d).sum())
    assert abs(fd_mu - an) <= 1e-6 * abs(an), (fd_mu, an)
