"""On-device operator assembly and the implicit plasma step against the
oracle's restatement of the reference's producers (oracle/step_oracle.py):

* mps_efield_dev == update_efield (plasma_pde/poissoneq.f90:565-680), with
  and without the minmod limiter, for Dirichlet, zero-gradient and periodic
  faces, ghosts included;
* mps_eden_transport_dev == eden_update_transport (edeneq.f90:360-444);
* mps_poisson_source_dev == poisson_update_transport (poissoneq.f90:335-385);
* mps_plasma_step_dev == the potential + electron part of the time step
  (solve_manager.f90:363-502) over the FP64 oracle's solves: potential, E and
  the new electron density to 1e-9 relative.
Producers are exact up to rounding (1e-13 relative)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import step as ST  # noqa: E402
from mps3d_b200 import workloads as W  # noqa: E402
from mps3d_b200.problem import Problem  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import step_oracle as SO  # noqa: E402

pytestmark = pytest.mark.gpu

OP_TOL = 1e-13
BCS = [["PERI", "PERI", "PERI", "PERI", "DIRC", "DIRC"], ["DIRC", "ZGRD", "FLUX", "DIRC", "PERI", "PERI"],
       ["ZGRD", "ZGRD", "DIRC", "DIRC", "ZGRD", "FLUX"]]


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _problem(nx, ny, nz, llen, bc, bcvals):
    g = (nz + 2, ny + 2, nx + 2)
    return Problem(nx, ny, nz, llen, dcoeff=np.ones(g), source=np.zeros(g), bc=bc, bcvals=bcvals)


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("limiter", [False, True])
def test_efield_matches_update_efield(bc, limiter):
    nx, ny, nz, llen = 13, 9, 11, (0.01, 0.008, 0.012)
    rng = np.random.default_rng(71)
    bcvals = [rng.uniform(-5, 5, size=s) for s in [(nz, ny)] * 2 + [(nz, nx)] * 2 + [(ny, nx)] * 2]
    P = _problem(nx, ny, nz, llen, bc, bcvals)
    phi = rng.standard_normal(P.ghost_shape) * 100.0
    phi_o = O.fill_ghosts(P, phi.copy())
    E_o = SO.efield(phi_o, llen, bc, scale=2.5, limiter=limiter)
    phi_d = _t(phi)
    E_d = ST.efield_dev(phi_d, llen, bc, P.bcvals, scale=2.5, limiter=limiter)
    torch.cuda.synchronize()
    assert _rel(E_d.cpu().numpy(), E_o) <= OP_TOL
    # the potential's face ghosts were set in place, as update_efield does
    got = phi_d.cpu().numpy()
    for sl in [(slice(1, -1), slice(1, -1), slice(None)), (slice(1, -1), slice(None), slice(1, -1)),
               (slice(None), slice(1, -1), slice(1, -1))]:
        np.testing.assert_allclose(got[sl], phi_o[sl], rtol=1e-15, atol=0)


@pytest.mark.parametrize("variant", ["d_field", "einstein_prod_dt", "scaled"])
def test_eden_transport_matches(variant):
    rng = np.random.default_rng(72)
    g = (9, 8, 12)
    E = rng.standard_normal((3,) + g) * 1e4
    mu = -rng.uniform(0.01, 0.05, size=g)
    d = rng.uniform(0.01, 0.2, size=g)
    te = rng.uniform(1.0, 4.0, size=g)
    prod = rng.uniform(0.0, 1e20, size=g)
    nold = rng.lognormal(np.log(1e16), 1.0, size=g)
    kw = {"d_field": dict(d=d), "einstein_prod_dt": dict(te=te, prod=prod, n_old=nold, dt=1e-11),
          "scaled": dict(d=d, prod=prod, n_old=nold, dt=1e-9, scaling=(2.0, 0.5, 3.0))}[variant]
    ref = SO.eden_transport(E, mu, kw.get("d"), kw.get("te"), kw.get("prod"), kw.get("n_old"), kw.get("dt"),
                            kw.get("scaling", (1.0, 1.0, 1.0)))
    dev = ST.eden_transport_dev(_t(E), (0.01, 0.01, 0.01), _t(mu), d=_t(kw["d"]) if "d" in kw else None,
                                te=_t(kw["te"]) if "te" in kw else None, prod=_t(kw["prod"]) if "prod" in kw else None,
                                n_old=_t(kw["n_old"]) if "n_old" in kw else None, dt=kw.get("dt"),
                                scaling=kw.get("scaling", (1.0, 1.0, 1.0)))
    torch.cuda.synchronize()
    for a, b in zip(dev, ref):
        assert _rel(a.cpu().numpy(), b) <= OP_TOL


def test_poisson_source_matches():
    rng = np.random.default_rng(73)
    g = (7, 10, 9)
    ne = rng.lognormal(np.log(1e16), 1.0, size=g)
    ni = rng.lognormal(np.log(1e16), 1.0, size=(2,) + g)
    q = [1.0, 2.0]
    ref = SO.poisson_source(ne, ni, q, ST.ECHARGE / ST.EPS0)
    dev = ST.poisson_source_dev(_t(ne), (0.01,) * 3, n_ion=_t(ni), charge=_t(np.array(q)))
    torch.cuda.synchronize()
    assert _rel(dev.cpu().numpy(), ref) <= OP_TOL


@pytest.mark.parametrize("n", [17, 65, 129])
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_plasma_step_matches_oracle(n, prec):
    case = W.plasma_step_case(n)
    phi_o, E_o, vel_o, dc_o, src_o, ne_o = SO.plasma_step(case, case["n_e0"])
    stp = ST.PlasmaStep(case, phi_opts={"precision": prec, "tol": 1e-12, "maxit": 80},
                        e_opts={"precision": prec, "krylov": "fgmres", "flux": 1, "tol": 1e-12, "maxit": 80})
    phi = torch.zeros(case["eps"].shape, dtype=torch.float64, device="cuda")
    ne = _t(case["n_e0"])
    ip, ie = stp.step(phi, ne)
    torch.cuda.synchronize()
    assert ip["status"] == 0 and ie["status"] == 0, (ip, ie)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    assert rel(phi.cpu().numpy(), phi_o) <= 1e-9
    assert rel(stp.efield.cpu().numpy(), E_o) <= 1e-9
    assert rel(stp.dcoeff.cpu().numpy(), dc_o) <= OP_TOL
    assert rel(stp.source.cpu().numpy(), src_o) <= OP_TOL
    assert rel(ne.cpu().numpy(), ne_o) <= 1e-9
    assert float(ne[1:-1, 1:-1, 1:-1].min()) >= case["nemin"]
    stp.close()
