"""The CUDA path (through the C ABI) against the committed golden fixtures:
operator and right-hand side to 1e-13, perform_vcycle iterates to 1e-10,
converged solutions to 1e-9 relative error, the SG operator VJP to 1e-11."""
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as G  # noqa: E402
from mps3d_b200 import capi, solver  # noqa: E402
from mps3d_b200.adjoint import OperatorSpec, device_vjp  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", "golden.npz"))


@pytest.fixture(scope="module")
def handle():
    return capi.Handle(0)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_operator_and_rhs(gold, handle):
    p = G.operator_case()
    dp = solver.DeviceProblem(p)
    AX = solver.apply_A_dev(dp, torch.from_numpy(gold["op_u"]).cuda(), handle=handle).cpu().numpy()
    assert _rel(AX, gold["op_AX"]) <= 1e-13
    b = solver.find_bvec_dev(dp, handle=handle).cpu().numpy()
    assert _rel(b, gold["op_b"]) <= 1e-13


def test_vcycle_iterates(gold, handle):
    q = G.vcycle_case()
    x = q.zeros_ghosted()
    for it in range(3):
        x, rn = solver.vcycle_once(q, x, handle=handle, ranks=(2, 2, 2))
        assert _rel(x[1:-1, 1:-1, 1:-1], gold[f"vc_x{it}"]) <= 1e-10
        assert abs(rn - float(gold[f"vc_res{it}"])) <= 1e-8 * abs(float(gold[f"vc_res{it}"]))


@pytest.mark.parametrize("name", ["poisson", "sg"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_solutions(gold, handle, name, prec):
    p = G.poisson_case() if name == "poisson" else G.sg_case()
    krylov = "fgmres" if name == "sg" else None
    x, info = solver.linsolve(p, handle=handle, tol=1e-12, precision=prec, krylov=krylov, maxit=80)
    assert info["status"] == 0, info
    ref = gold[f"{name}_x"]
    assert np.linalg.norm(x[1:-1, 1:-1, 1:-1] - ref) / np.linalg.norm(ref) <= 1e-9


def test_operator_vjp(gold):
    v = G.vjp_case()
    spec = OperatorSpec(v.lx, v.ly, v.lz, v.llen, tuple(v.bc), flux=1)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    gv, gd = device_vjp(spec, t(v.vel), t(v.dcoeff), t(gold["vjp_lam"]), t(gold["vjp_u"]))
    torch.cuda.synchronize()
    assert _rel(gv.cpu().numpy(), gold["vjp_gvel"]) <= 1e-11
    assert _rel(gd.cpu().numpy(), gold["vjp_gd"]) <= 1e-11
