"""Batched solves (mps_linsolve_batched_dev) against the FP64 oracle and the
single-problem path: every problem of a batch of uneven sizes must reach the
same accuracy as if it were solved alone (relative residual <= 1e-10,
relative solution error <= 1e-9 against the oracle)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import capi, solver, workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def handle():
    return capi.Handle(0)


def _mixed_batch():
    """Uneven sizes (hierarchies of different depths), a variable-coefficient
    problem with reaction and a time derivative, periodic faces, a zero
    right-hand side."""
    ps = W.batch_poisson(count=5, sizes=(9, 13, 17, 11, 7))
    ps.append(W.random_operator(14, 10, 12, bc=["DIRC", "ZGRD", "PERI", "PERI", "DIRC", "FLUX"], seed=31, vel=False,
                                reac=True, timederiv=True, llen=(1.0, 0.7, 0.9)))
    ps.append(W.plasma_poisson(17, slab_cells=3))
    z = W.poisson_dirichlet(6)
    z.source[...] = 0.0
    ps.append(z)
    return ps


def _oracle(p):
    mg = O.RowsMG(p, hier=O.HIER_GEOM)
    b = O.build_rhs(p)
    x, hist = mg.fgmres(b, m=40, maxit=300, tol=1e-14)
    return x, b


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_batched_matches_oracle(handle, prec):
    ps = _mixed_batch()
    dps = [solver.DeviceProblem(p) for p in ps]
    xs = [torch.zeros(p.ghost_shape, dtype=torch.float64, device="cuda") for p in ps]
    infos = solver.linsolve_batched_dev(dps, xs, handle=handle, tol=1e-11, precision=prec, maxit=60)
    for p, x, info in zip(ps, xs, infos):
        assert info["status"] == 0, info
        xi = x.cpu().numpy()[1:-1, 1:-1, 1:-1]
        ref, b = _oracle(p)
        bn = np.linalg.norm(b)
        if bn == 0.0:
            assert np.abs(xi).max() == 0.0
            continue
        rel_res = np.linalg.norm(b - O.rows_apply(p, O.build_rows(p), np.ascontiguousarray(xi))) / bn
        assert rel_res <= 1e-10, (p.shape, rel_res)
        assert np.linalg.norm(xi - ref) / np.linalg.norm(ref) <= 1e-9


def test_batched_equals_single_solves(handle):
    """The iteration counts of solving each problem alone (within one: the two
    paths round the FP32 V-cycle differently), and the same solution."""
    ps = W.batch_poisson(count=4, sizes=(9, 17, 13))
    dps = [solver.DeviceProblem(p) for p in ps]
    xs = [torch.zeros(p.ghost_shape, dtype=torch.float64, device="cuda") for p in ps]
    infos = solver.linsolve_batched_dev(dps, xs, handle=handle, tol=1e-11, precision="mixed", maxit=40)
    for dp, x, info in zip(dps, xs, infos):
        x1 = torch.zeros_like(x)
        _, i1 = solver.linsolve_dev(dp, x1, handle=handle, tol=1e-11, precision="mixed", maxit=40)
        assert abs(info["iters"] - i1["iters"]) <= 1, (info, i1)
        d = (x - x1)[1:-1, 1:-1, 1:-1].abs().max().item() / x1.abs().max().item()
        assert d <= 1e-9, d


def test_batched_limits_and_repeats(handle):
    ps = W.batch_poisson(count=3, sizes=(9, 15))
    dps = [solver.DeviceProblem(p) for p in ps]
    xs = [torch.zeros(p.ghost_shape, dtype=torch.float64, device="cuda") for p in ps]
    infos = solver.linsolve_batched_dev(dps, xs, handle=handle, tol=1e-14, precision="mixed", maxit=1)
    assert all(i["status"] == capi.MPS_ERR_NOT_CONVERGED and i["iters"] == 1 for i in infos), infos
    # the same batch again (graph replay), now to convergence, from the
    # previous iterates as initial guesses
    infos = solver.linsolve_batched_dev(dps, xs, handle=handle, tol=1e-10, precision="mixed", maxit=40)
    assert all(i["status"] == 0 for i in infos), infos
    # unsupported option and operator class are refused
    with pytest.raises(capi.SolverError) as e:
        solver.linsolve_batched_dev(dps, xs, handle=handle, krylov="fgmres")
    assert e.value.status == capi.MPS_ERR_BAD_ARG
    q = W.random_operator(8, 8, 8, bc=["DIRC"] * 6, seed=32, vel=True, reac=False)
    with pytest.raises(capi.SolverError) as e:
        solver.linsolve_batched_dev([solver.DeviceProblem(q)], [torch.zeros(q.ghost_shape, dtype=torch.float64,
                                                                             device="cuda")], handle=handle)
    assert e.value.status == capi.MPS_ERR_BAD_ARG
    # the handle still solves single problems afterwards
    x, info = solver.linsolve(ps[0], handle=handle)
    assert info["status"] == 0


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_repeated_batch_replays_setup_with_new_data(prec):
    """A repeated batch (same problems and buffers) runs its set-up eagerly,
    then captures it as a CUDA graph, then replays it.  New right-hand sides
    and initial guesses written into the same buffers must be picked up by
    the replayed set-up: every solve equals an eager solve of the same data on
    a fresh handle (the same kernels, so to rounding of the FP64 sums)."""
    ps = _mixed_batch()
    dps = [solver.DeviceProblem(p) for p in ps]
    xs = [torch.zeros(p.ghost_shape, dtype=torch.float64, device="cuda") for p in ps]
    rep = capi.Handle(0)
    rng = np.random.default_rng(7)
    try:
        for call in range(5):
            if call >= 3:  # new data in the same device buffers
                for dp, p in zip(dps, ps):
                    if np.abs(p.source).max() == 0.0:
                        continue
                    dp.source.copy_(torch.from_numpy(rng.uniform(-1.0, 1.0, size=p.ghost_shape)))
            for x in xs:
                x.zero_()
            if call == 4:  # and a non-zero initial guess
                for x in xs:
                    x.copy_(torch.from_numpy(rng.uniform(-0.1, 0.1, size=tuple(x.shape))))
            x0 = [x.clone() for x in xs]
            infos = solver.linsolve_batched_dev(dps, xs, handle=rep, tol=1e-11, precision=prec, maxit=60)
            fresh = capi.Handle(0)
            try:
                ys = [x.clone() for x in x0]
                ref = solver.linsolve_batched_dev(dps, ys, handle=fresh, tol=1e-11, precision=prec, maxit=60)
            finally:
                fresh.close()
            for x, y, a, b in zip(xs, ys, infos, ref):
                assert a["status"] == b["status"] == 0, (call, a, b)
                assert a["iters"] == b["iters"], (call, a["iters"], b["iters"])
                scale = max(float(y.abs().max()), 1e-300)
                assert float((x - y).abs().max()) <= 1e-12 * scale, call
    finally:
        rep.close()
