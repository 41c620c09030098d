"""mps_apply_A_noalloc: A soln with no device allocation inside the call.

This entry point is for callers that cannot allocate device memory when they
need the operator applied -- a time stepper whose memory pool already holds
the free HBM, or one that cannot let cudaFree stall its streams.  Its scratch
is a static device array shared by every call, so the test makes two calls in
a row with different grids (the second smaller, so the first call's data is
still in the array) and checks each against the handle-based mps_apply_A_dev
at the operator tolerance of the other parity tests.  It also checks that a
call leaves the device's free memory unchanged and that a grid past the limit
is refused before anything runs, and, in a fresh process, that the first
call on a device takes no more device memory than the static array itself
(the CUDA runtime reserves the array when that call loads the library's code
on the device) while later calls take none.  The file name makes pytest
collect it last; it passes alone in a fresh process as well.
"""
import gc
import json
import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import capi, solver, workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

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
        # and against the FP64 oracle's rows directly (upwind or SG, A or A^T)
        rows = O.build_rows(p)
        if transpose:
            rows = O.rows_transpose(p, rows)
        ui = np.ascontiguousarray(u.cpu().numpy()[1:-1, 1:-1, 1:-1])
        want = torch.from_numpy(O.rows_apply(p, rows, ui))
        assert _rel(out.cpu(), want) <= OP_TOL


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


_FIRST_CALL = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, %r)
from mps3d_b200 import solver, workloads as W
p = W.random_operator(17, 16, 15, bc=["PERI", "PERI", "DIRC", "ZGRD", "DIRC", "FLUX"], seed=21, vel=True,
                      reac=True, timederiv=True, flux=1)
dp = solver.DeviceProblem(p)
u = torch.from_numpy(np.random.default_rng(28).standard_normal(p.ghost_shape)).cuda()
out = torch.empty(p.shape, dtype=torch.float64, device="cuda")
torch.cuda.synchronize()
free0, _ = torch.cuda.mem_get_info()
solver.apply_A_noalloc(dp, u, out=out)
torch.cuda.synchronize()
free1, _ = torch.cuda.mem_get_info()
for _ in range(3):
    solver.apply_A_noalloc(dp, u, out=out)
torch.cuda.synchronize()
free2, _ = torch.cuda.mem_get_info()
print(json.dumps({"free0": free0, "free1": free1, "free2": free2, "finite": bool(torch.isfinite(out).all())}))
"""


def test_noalloc_first_call_in_fresh_process_reserves_only_the_scratch():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    env.pop("CUDA_MODULE_LOADING", None)  # the default: lazy loading
    r = subprocess.run([sys.executable, "-c", _FIRST_CALL % root], capture_output=True, text=True, env=env,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["finite"]
    # the first call loads the library's module on the device: the 32 MiB
    # array plus the module's code (a few MiB at most)
    taken = d["free0"] - d["free1"]
    assert taken <= capi.NOALLOC_SCRATCH_BYTES + (16 << 20), taken
    # from then on no call takes device memory
    assert d["free2"] >= d["free1"]
