"""mps_apply_A_noalloc: A soln with no device allocation inside the call.

This entry point is for callers that cannot allocate device memory when they
need the operator applied -- a time stepper whose memory pool already holds
the free HBM, or one that cannot let cudaFree stall its streams.  Its scratch
is a static device array shared by every call, so the test makes two calls in
a row with different grids (the second smaller, so the first call's data is
still in the array) and checks each against the handle-based mps_apply_A_dev
at the operator tolerance of the other parity tests.  It also checks that a
call leaves the device's free memory unchanged and that a grid past the limit
is refused before anything runs.  The file name makes pytest collect it last;
it passes alone in a fresh process as well.
"""
import gc

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import capi, solver, workloads as W  # noqa: E402

pytestmark = pytest.mark.gpu

OP_TOL = 1e-13  # relative, as for every operator-level parity check


def _rel(a, b):
    return (a - b).abs().max().item() / max(b.abs().max().item(), 1e-300)


def _cases():
    first = W.random_operator(17, 16, 15, bc=["PERI", "PERI", "DIRC", "ZGRD", "DIRC", "FLUX"], seed=21, vel=True,
                              reac=True, timederiv=True, flux=1)
    second = W.random_operator(9, 4, 6, bc=["DIRC", "FLUX", "PERI", "PERI", "ZGRD", "DIRC"], seed=22, vel=True,
                               reac=False)
    return [(first, False), (second, True)]


def test_noalloc_matches_apply_A_dev_on_consecutive_calls():
    h = capi.Handle(0)
    rng = np.random.default_rng(23)
    for p, transpose in _cases():
        dp = solver.DeviceProblem(p)
        u = torch.from_numpy(rng.standard_normal(p.ghost_shape)).cuda()
        ref = solver.apply_A_dev(dp, u, handle=h, transpose=transpose)
        out = torch.full(p.shape, float("nan"), dtype=torch.float64, device="cuda")
        solver.apply_A_noalloc(dp, u, out=out, transpose=transpose)
        torch.cuda.synchronize()
        assert torch.isfinite(out).all()
        assert _rel(out, ref) <= OP_TOL


def test_noalloc_leaves_free_memory_unchanged():
    p, transpose = _cases()[0]
    dp = solver.DeviceProblem(p)
    u = torch.from_numpy(np.random.default_rng(24).standard_normal(p.ghost_shape)).cuda()
    out = torch.empty(p.shape, dtype=torch.float64, device="cuda")
    solver.apply_A_noalloc(dp, u, out=out, transpose=transpose)  # the device's first call sets up, if not done yet
    gc.collect()  # handles left by earlier tests free their workspaces now, not during the calls
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        solver.apply_A_noalloc(dp, u, out=out, transpose=transpose)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # other owners may still hand memory back meanwhile; nothing may be taken
    assert free1 >= free0


def test_noalloc_refuses_grids_past_the_limit():
    # round_up(64, 16) * 64 * 65 = 266240 > 262144 cells: refused before any launch
    p = W.random_operator(64, 64, 65, bc=["DIRC"] * 6, seed=25, vel=False, reac=False)
    dp = solver.DeviceProblem(p)
    u = torch.zeros(p.ghost_shape, dtype=torch.float64, device="cuda")
    out = torch.zeros(p.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(capi.SolverError) as e:
        solver.apply_A_noalloc(dp, u, out=out)
    assert e.value.status == capi.MPS_ERR_TOO_LARGE
    torch.cuda.synchronize()
    assert bool((out == 0).all())
    # exactly at the limit (64^3) the call runs and matches
    q = W.random_operator(64, 64, 64, bc=["DIRC"] * 6, seed=26, vel=False, reac=True)
    dq = solver.DeviceProblem(q)
    v = torch.from_numpy(np.random.default_rng(27).standard_normal(q.ghost_shape)).cuda()
    ref = solver.apply_A_dev(dq, v, handle=capi.Handle(0))
    got = solver.apply_A_noalloc(dq, v)
    torch.cuda.synchronize()
    assert _rel(got, ref) <= OP_TOL
