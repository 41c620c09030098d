"""Adjoint pieces on the CPU: the oracle's operator VJP against central
differences of lam^T A(theta) u, and the electron-flux model's gradient
(oracle solves, torch autograd) against central differences of its loss."""
import numpy as np
import pytest

from mps3d_b200 import workloads as W
from oracle import oracle as O

BCS = [["PERI", "PERI", "PERI", "PERI", "ZGRD", "ZGRD"], ["DIRC", "ZGRD", "DIRC", "FLUX", "DIRC", "DIRC"],
       ["ZGRD", "DIRC", "PERI", "PERI", "FLUX", "ZGRD"]]


@pytest.mark.parametrize("flux", [0, 1])
@pytest.mark.parametrize("bc", BCS)
def test_operator_vjp_matches_central_differences(flux, bc):
    p = W.random_operator(6, 5, 4, bc=bc, seed=41, vel=True, reac=True, timederiv=True, flux=flux)
    rng = np.random.default_rng(42)
    lam, u = rng.standard_normal(p.shape), rng.standard_normal(p.shape)
    gv, gd, gr = O.operator_vjp(p, lam, u)

    def s_of(vel, dc, re):
        q = type(p)(p.lx, p.ly, p.lz, p.llen, dcoeff=dc, source=p.source, vel=vel, reac=re, bc=p.bc,
                    bcvals=p.bcvals, timederiv=p.timederiv, dt=p.dt, flux=p.flux)
        return float(np.sum(lam * O.rows_apply(q, O.build_rows(q), u)))

    # directional derivatives along random perturbations of each field
    # (interior cells; the ghost layer does not enter the operator)
    for field in ("vel", "dcoeff", "reac"):
        base = {"vel": p.vel, "dcoeff": p.dcoeff, "reac": p.reac}
        d = np.zeros_like(base[field])
        sl = (Ellipsis, slice(1, -1), slice(1, -1), slice(1, -1))
        d[sl] = rng.uniform(-1.0, 1.0, size=d[sl].shape)
        h = 1e-4  # truncation ~h^2 stays below the rounding of s (|s| eps / h)
        args_p = dict(base); args_p[field] = base[field] + h * d
        args_m = dict(base); args_m[field] = base[field] - h * d
        fd = (s_of(args_p["vel"], args_p["dcoeff"], args_p["reac"]) -
              s_of(args_m["vel"], args_m["dcoeff"], args_m["reac"])) / (2 * h)
        g = {"vel": gv, "dcoeff": gd, "reac": gr}[field]
        an = float(np.sum(g * d[sl]))
        s0 = abs(s_of(p.vel, p.dcoeff, p.reac))
        assert abs(fd - an) <= 1e-7 * max(abs(an), 1.0) + 100 * 2.2e-16 * s0 / h, (field, fd, an)


def test_sg_face_derivatives_cover_every_branch():
    """Central differences of the SG weights in the upwind limit (D ~ 0), the
    central limit (Pe ~ 0) and both signs of Pe."""
    cases = [(0.3, 0.5, 1e-13, 1e-13, 0.1), (2.0, -1.0, 0.4, 0.6, 0.05), (-3.0, -2.0, 0.2, 0.1, 0.1),
             (1e-4, 2e-4, 0.5, 0.5, 0.1), (40.0, 30.0, 0.01, 0.02, 0.1)]
    for cL, cR, DL, DR, dx in cases:
        dwL, dwR = O.sg_face_d(cL, cR, DL, DR, dx)
        x = [cL, cR, DL, DR]
        for q in range(4):
            # velocities: an absolute step (the forward formula cancels at small
            # Pe, so tiny steps measure its rounding); diffusivities: relative,
            # which keeps the upwind-limit case (D ~ 0) in its branch
            h = 1e-5 * max(abs(x[q]), 1.0) if q < 2 else 1e-4 * x[q]
            xp = list(x); xp[q] += h
            xm = list(x); xm[q] -= h
            wp, wm = O.sg_face(*xp, dx), O.sg_face(*xm, dx)
            for side in (0, 1):
                fd = (wp[side] - wm[side]) / (2 * h)
                an = (dwL, dwR)[side][q]
                assert abs(fd - an) <= 1e-6 * max(abs(an), 1.0), (cL, cR, DL, DR, q, side, fd, an)


def test_electron_flux_gradient_oracle_matches_central_differences():
    torch = pytest.importorskip("torch")
    from adjoint_oracle import oracle_bvec, oracle_solve
    from mps3d_b200.adjoint import ElectronFluxAdjoint

    case = W.electron_adjoint_case(7, steps=2)
    model = ElectronFluxAdjoint(case, device="cpu", solve_fn=oracle_solve, bvec_fn=oracle_bvec)
    V = case["v_front"]
    mu = torch.from_numpy(case["mu"])
    L0, gV, gmu = model.gradient(V, mu)
    mu64 = mu.to(torch.float64)
    h = 1e-4 * V
    fd_V = (float(model.loss(torch.tensor(V + h, dtype=torch.float64), mu64)) -
            float(model.loss(torch.tensor(V - h, dtype=torch.float64), mu64))) / (2 * h)
    assert abs(fd_V - gV) <= 1e-6 * abs(gV), (fd_V, gV)
    d = torch.from_numpy(np.random.default_rng(43).uniform(-1.0, 1.0, size=mu.shape)) * mu64 * 1e-4
    Vt = torch.tensor(V, dtype=torch.float64)
    fd_mu = (float(model.loss(Vt, mu64 + d)) - float(model.loss(Vt, mu64 - d))) / 2.0
    an = float((gmu.to(torch.float64) * d).sum())
    assert abs(fd_mu - an) <= 1e-6 * abs(an), (fd_mu, an)


def test_sg_face_derivatives_match_extended_precision():
    """The oracle's SG weight derivatives against the Bernoulli form evaluated
    with 50-digit decimals, including |Pe| down to 1e-9 where closed forms
    cancel."""
    from decimal import Decimal, getcontext

    getcontext().prec = 50

    def exact(cL, cR, DL, DR, dx):
        c = (Decimal(cL) + Decimal(cR)) / 2
        D = 2 * Decimal(DL) * Decimal(DR) / (Decimal(DL) + Decimal(DR) + Decimal("1e-10"))
        Pe = c * Decimal(dx) / D

        def B(x):
            return x / (x.exp() - 1)

        def dB(x):
            e = x.exp()
            return (e - 1 - x * e) / ((e - 1) ** 2)

        return [float(-dB(-Pe)), float(-dB(Pe)), float((B(-Pe) + Pe * dB(-Pe)) / Decimal(dx)),
                float(-(B(Pe) - Pe * dB(Pe)) / Decimal(dx))]

    rng = np.random.default_rng(44)
    for t in range(400):
        cL, cR = rng.uniform(-3.0, 3.0, 2)
        DL, DR = rng.uniform(0.5, 2.0, 2)
        if t % 2 == 0:
            cR = -cL + rng.uniform(-0.1, 0.1) * 10.0 ** (-int(rng.integers(0, 8)))
        if abs(0.5 * (cL + cR) * 0.077 / (2 * DL * DR / (DL + DR + 1e-10))) < 1e-10:
            continue  # the |Pe| < 1e-10 branch (central weights, no c dependence) is its own definition
        dwL, dwR = O.sg_face_d(cL, cR, DL, DR, 0.077)
        dD = 2 * DR * (DR + 1e-10) / (DL + DR + 1e-10) ** 2
        got = [2 * dwL[0], 2 * dwR[0], dwL[2] / dD, dwR[2] / dD]
        ref = exact(cL, cR, DL, DR, 0.077)
        for q in range(4):
            assert abs(got[q] - ref[q]) <= 1e-11 * max(abs(ref[q]), 1.0), (cL, cR, DL, DR, q, got[q], ref[q])
