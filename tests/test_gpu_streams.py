"""Calls from torch's default stream are ordered with the work queued on it.

torch's default stream is the legacy default stream; the handle's own stream
is non-blocking.  Inputs written on the default stream behind a long-running
kernel must be read only after they are written, and outputs must be complete
when the default stream reads them: each entry point here runs right after a
delay kernel on the default stream whose end releases the input, and its
result is compared with the same call on inputs that were ready in advance."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import capi, solver, workloads as W  # noqa: E402

pytestmark = pytest.mark.gpu

DELAY_CYCLES = 200_000_000  # about 0.1 s of GPU time: longer than a host call takes to reach its first launch


def _rel(a, b):
    return (a - b).abs().max().item() / max(b.abs().max().item(), 1e-300)


def test_linsolve_dev_waits_for_inputs_on_the_default_stream():
    p = W.random_operator(20, 18, 16, bc=["DIRC", "DIRC", "PERI", "PERI", "ZGRD", "DIRC"], seed=41, vel=False,
                          reac=True)
    dp = solver.DeviceProblem(p)
    ref = torch.zeros(p.ghost_shape, dtype=torch.float64, device="cuda")
    solver.linsolve_dev(dp, ref, handle=capi.Handle(0), tol=1e-12, maxit=60)
    torch.cuda.synchronize()
    src = dp.source.clone()
    dp.source.zero_()
    torch.cuda.synchronize()
    h = capi.Handle(0)
    x = torch.zeros(p.ghost_shape, dtype=torch.float64, device="cuda")
    assert torch.cuda.current_stream().cuda_stream == 0  # the legacy default stream
    torch.cuda._sleep(DELAY_CYCLES)
    dp.source.copy_(src)  # the right-hand side exists only once the delay has passed
    solver.linsolve_dev(dp, x, handle=h, tol=1e-12, maxit=60)
    out = x.clone()  # read on the default stream
    torch.cuda.synchronize()
    assert _rel(out, ref) <= 1e-10


def test_apply_A_dev_waits_for_inputs_on_the_default_stream():
    p = W.random_operator(15, 14, 13, bc=["PERI", "PERI", "DIRC", "FLUX", "ZGRD", "DIRC"], seed=42, vel=True,
                          reac=False)
    dp = solver.DeviceProblem(p)
    h = capi.Handle(0)
    u = torch.from_numpy(np.random.default_rng(43).standard_normal(p.ghost_shape)).cuda()
    ref = solver.apply_A_dev(dp, u, handle=h)
    torch.cuda.synchronize()
    v = torch.zeros_like(u)
    torch.cuda._sleep(DELAY_CYCLES)
    v.copy_(u)
    got = solver.apply_A_dev(dp, v, handle=h).clone()
    torch.cuda.synchronize()
    assert _rel(got, ref) <= 1e-13
