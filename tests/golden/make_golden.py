"""Writes the golden fixtures of this folder from the FP64 oracle (seeded
inputs; run from the repository root: python tests/golden/make_golden.py).

The reference (Fortran/MPI) cannot be built or imported here, so the oracle --
pinned by tests/test_oracle_kat.py against the reference's own known-answer
decks -- produces the vectors: find_AX / find_bvec of a random operator,
three perform_vcycle iterates (reference CELL hierarchy, 2x2x2 rank layout),
converged solutions of small plasma Poisson and SG electron-step problems, and
an SG operator VJP.  The fixtures pin the CUDA path (tests/test_gpu_golden.py)
and the oracle itself (tests/test_oracle_golden.py) to fixed numbers.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mps3d_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def operator_case():
    return W.random_operator(9, 7, 6, bc=["DIRC", "ZGRD", "PERI", "PERI", "DIRC", "FLUX"], seed=61, vel=True,
                             reac=True, timederiv=True)


def vcycle_case():
    return W.laplace_test(16)


def poisson_case():
    return W.plasma_poisson(17, slab_cells=3)


def sg_case():
    return W.electron_sg_step(13)


def vjp_case():
    return W.random_operator(8, 6, 5, bc=["PERI", "PERI", "PERI", "PERI", "ZGRD", "ZGRD"], seed=62, vel=True,
                             reac=True, timederiv=True, flux=1)


def make():
    out = {}
    p = operator_case()
    u = np.random.default_rng(63).standard_normal(p.ghost_shape)
    AX, _, _ = O.find_AX(p, u)
    out["op_u"] = u
    out["op_AX"] = AX
    out["op_b"] = O.find_bvec(p)
    q = vcycle_case()
    x = q.zeros_ghosted()
    for it in range(3):
        rn = O.vcycle(q, x, ranks=(2, 2, 2))
        out[f"vc_x{it}"] = x[1:-1, 1:-1, 1:-1].copy()
        out[f"vc_res{it}"] = np.array(rn)
    for name, case in (("poisson", poisson_case()), ("sg", sg_case())):
        mg = O.RowsMG(case, hier=O.HIER_GEOM)
        b = O.build_rhs(case)
        xs, hist = mg.fgmres(b, m=40, maxit=300, tol=1e-14)
        out[f"{name}_x"] = xs
    v = vjp_case()
    rng = np.random.default_rng(64)
    lam, uu = rng.standard_normal(v.shape), rng.standard_normal(v.shape)
    gv, gd, gr = O.operator_vjp(v, lam, uu)
    out.update(vjp_lam=lam, vjp_u=uu, vjp_gvel=gv, vjp_gd=gd)
    return out


if __name__ == "__main__":
    data = make()
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **data)
    print({k: v.shape for k, v in data.items()})
