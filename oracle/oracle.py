"""ctypes front end of the FP64 CPU oracle (oracle/mps_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker the CUDA library is compared against.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It takes the same :class:`mps3d_b200.problem.Problem` the
product API takes, so both sides read identical inputs.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_build", "libmps_oracle.so")
# the -march=native build used for CPU-baseline timings: compiled on the host
# that runs it, into a folder named after that host's CPU, never shipped
NATIVE_ENV = "MPS_ORACLE_NATIVE"

HIER_CELL = 0
HIER_GEOM = 1


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def cpu_model() -> str:
    """The host CPU's model name (as lscpu prints it)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _native_path():
    import hashlib
    import platform

    tag = hashlib.sha1((cpu_model() + platform.machine()).encode()).hexdigest()[:10]
    return os.path.join(HERE, "_build", "native-" + tag)


def build_native() -> str:
    d = _native_path()
    subprocess.check_call(["make", "-s", "-C", HERE, "native", f"NATIVE_DIR={d}"])
    return os.path.join(d, "libmps_oracle.so")


class _Grid(C.Structure):
    _fields_ = [
        ("lx", C.c_int), ("ly", C.c_int), ("lz", C.c_int),
        ("llenx", C.c_double), ("lleny", C.c_double), ("llenz", C.c_double),
        ("px", C.c_int), ("py", C.c_int), ("pz", C.c_int),
        ("hier", C.c_int), ("max_coarse", C.c_int), ("nu1", C.c_int), ("nu2", C.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if os.environ.get(NATIVE_ENV) == "1":
            path = build_native()  # make rebuilds it only when the sources changed
        else:
            path = LIBPATH
            if not os.path.exists(path):
                build()
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        gp = C.POINTER(_Grid)
        L.orc_find_AX.argtypes = [gp, dp, C.c_int, C.c_double, dp, dp, dp, ip, dp, dp, dp]
        L.orc_find_bvec.argtypes = [gp, dp, dp, dp, ip, C.POINTER(dp), dp, C.c_int, dp]
        L.orc_vcycle.argtypes = [gp, dp, C.c_int, C.c_double, dp, dp, dp, dp, ip, C.POINTER(dp), dp, dp]
        L.orc_vcycle.restype = C.c_int
        L.orc_solve.argtypes = [gp, dp, C.c_int, C.c_double, dp, dp, dp, dp, ip, C.POINTER(dp),
                                C.c_int, C.c_double, C.c_int, dp, dp]
        L.orc_solve.restype = C.c_int
        L.orc_rel_residual.argtypes = [gp, dp, C.c_int, C.c_double, dp, dp, dp, dp, ip, C.POINTER(dp), dp]
        L.orc_rel_residual.restype = C.c_double
        L.orc_fill_ghosts.argtypes = [gp, dp, ip, C.POINTER(dp)]
        L.orc_build_rows.argtypes = [gp, C.c_int, C.c_int, C.c_double, dp, dp, dp, ip, dp]
        L.orc_build_rhs.argtypes = [gp, C.c_int, dp, dp, dp, ip, C.POINTER(dp), dp]
        L.orc_rows_apply.argtypes = [gp, ip, dp, dp, dp]
        L.orc_rows_transpose.argtypes = [gp, ip, dp, dp]
        L.orc_sg_face.argtypes = [C.c_double] * 5 + [dp, dp]
        L.orc_sg_face_d.argtypes = [C.c_double] * 5 + [dp, dp]
        L.orc_operator_vjp.argtypes = [gp, C.c_int, dp, dp, ip, dp, dp, dp, dp, dp]
        L.orc_mg_create.argtypes = [gp, C.c_int, C.c_int, C.c_double, dp, dp, dp, ip, C.c_int]
        L.orc_mg_create.restype = C.c_void_p
        L.orc_mg_destroy.argtypes = [C.c_void_p]
        L.orc_mg_levels.argtypes = [C.c_void_p, ip]
        L.orc_mg_levels.restype = C.c_int
        L.orc_mg_vcycle.argtypes = [C.c_void_p, dp, dp]
        L.orc_mg_rows.argtypes = [C.c_void_p, C.c_int]
        L.orc_mg_rows.restype = dp
        L.orc_fgmres.argtypes = [C.c_void_p, dp, dp, C.c_int, C.c_int, C.c_double, dp]
        L.orc_fgmres.restype = C.c_int
        L.orc_mg_solve.argtypes = [C.c_void_p, dp, dp, C.c_int, C.c_double, dp]
        L.orc_mg_solve.restype = C.c_int
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        _lib = L
    return _lib


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return lib().orc_get_threads()


def native_loaded() -> bool:
    """True when the -march=native build is the one loaded."""
    return _lib is not None and os.environ.get(NATIVE_ENV) == "1"


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _grid(prob, hier=HIER_CELL, ranks=(1, 1, 1), max_coarse=125, nu1=2, nu2=2):
    return _Grid(prob.lx, prob.ly, prob.lz, prob.llen[0], prob.llen[1], prob.llen[2],
                 ranks[0], ranks[1], ranks[2], hier, max_coarse, nu1, nu2)


def _bc(prob):
    return (C.c_int * 6)(*prob.bc)


def _bcv(prob):
    arr = (C.POINTER(C.c_double) * 6)()
    for f in range(6):
        arr[f] = _p(prob.bcvals[f])
    return arr


def find_AX(prob, soln):
    g = _grid(prob)
    n = prob.shape
    AX, d, o = np.zeros(n), np.zeros(n), np.zeros(n)
    soln = np.ascontiguousarray(soln, dtype=np.float64)
    lib().orc_find_AX(C.byref(g), _p(soln), int(prob.timederiv), prob.dt, _p(prob.vel), _p(prob.dcoeff),
                      _p(prob.reac), _bc(prob), _p(AX), _p(d), _p(o))
    return AX, d, o


def find_bvec(prob, mgridsource=None, applybc=True):
    g = _grid(prob)
    b = np.zeros(prob.shape)
    ms = None if mgridsource is None else _p(np.ascontiguousarray(mgridsource, dtype=np.float64))
    lib().orc_find_bvec(C.byref(g), _p(prob.vel), _p(prob.dcoeff), _p(prob.source), _bc(prob), _bcv(prob),
                        ms, int(applybc), _p(b))
    return b


def vcycle(prob, soln, hier=HIER_CELL, ranks=(1, 1, 1), max_coarse=125, nu1=2, nu2=2):
    """One perform_vcycle call in place on the ghosted ``soln``; returns the
    reference's RMS residual norm."""
    g = _grid(prob, hier, ranks, max_coarse, nu1, nu2)
    rn = C.c_double(0.0)
    st = lib().orc_vcycle(C.byref(g), _p(soln), int(prob.timederiv), prob.dt, _p(prob.vel), _p(prob.dcoeff),
                          _p(prob.reac), _p(prob.source), _bc(prob), _bcv(prob), None, C.byref(rn))
    if st:
        raise RuntimeError(f"oracle vcycle status {st}")
    return rn.value


def solve(prob, soln=None, hier=HIER_CELL, ranks=(1, 1, 1), maxit=20, tol=1e-10, tol_kind=1,
          max_coarse=125, nu1=2, nu2=2):
    """Caller loop of repeated V-cycles; returns (soln, rel_hist, rms_hist)."""
    g = _grid(prob, hier, ranks, max_coarse, nu1, nu2)
    soln = prob.zeros_ghosted() if soln is None else np.ascontiguousarray(soln, dtype=np.float64).copy()
    rel = np.zeros(maxit + 1)
    rms = np.zeros(maxit + 1)
    it = lib().orc_solve(C.byref(g), _p(soln), int(prob.timederiv), prob.dt, _p(prob.vel), _p(prob.dcoeff),
                         _p(prob.reac), _p(prob.source), _bc(prob), _bcv(prob), maxit, tol, tol_kind,
                         _p(rel), _p(rms))
    if it < 0:
        raise RuntimeError(f"oracle solve status {-it}")
    return soln, rel[:it], rms[:it]


def rel_residual(prob, soln):
    g = _grid(prob)
    rms = C.c_double(0.0)
    r = lib().orc_rel_residual(C.byref(g), _p(np.ascontiguousarray(soln, dtype=np.float64)), int(prob.timederiv),
                               prob.dt, _p(prob.vel), _p(prob.dcoeff), _p(prob.reac), _p(prob.source), _bc(prob),
                               _bcv(prob), C.byref(rms))
    return r, rms.value


def fill_ghosts(prob, soln):
    g = _grid(prob)
    lib().orc_fill_ghosts(C.byref(g), _p(soln), _bc(prob), _bcv(prob))
    return soln


def build_rows(prob, flux=None):
    g = _grid(prob)
    rows = np.zeros((7,) + prob.shape)
    fl = prob.flux if flux is None else flux
    lib().orc_build_rows(C.byref(g), fl, int(prob.timederiv), prob.dt, _p(prob.vel), _p(prob.dcoeff),
                         _p(prob.reac), _bc(prob), _p(rows))
    return rows


def build_rhs(prob, flux=None):
    g = _grid(prob)
    b = np.zeros(prob.shape)
    fl = prob.flux if flux is None else flux
    lib().orc_build_rhs(C.byref(g), fl, _p(prob.vel), _p(prob.dcoeff), _p(prob.source), _bc(prob), _bcv(prob),
                        _p(b))
    return b


def rows_apply(prob, rows, u):
    g = _grid(prob)
    out = np.zeros(prob.shape)
    lib().orc_rows_apply(C.byref(g), _bc(prob), _p(np.ascontiguousarray(rows)), _p(np.ascontiguousarray(u)),
                         _p(out))
    return out


def rows_transpose(prob, rows):
    g = _grid(prob)
    out = np.zeros_like(rows)
    lib().orc_rows_transpose(C.byref(g), _bc(prob), _p(np.ascontiguousarray(rows)), _p(out))
    return out


def sg_face(cL, cR, DL, DR, dx):
    wL, wR = C.c_double(), C.c_double()
    lib().orc_sg_face(cL, cR, DL, DR, dx, C.byref(wL), C.byref(wR))
    return wL.value, wR.value


def operator_vjp(prob, lam, u, flux=None):
    """Gradients of lam^T A u with respect to vel (3, lz, ly, lx), dcoeff and
    reac (lz, ly, lx) for interior lam, u (uniform grid)."""
    g = _grid(prob)
    fl = prob.flux if flux is None else flux
    gv = np.zeros((3,) + prob.shape)
    gd = np.zeros(prob.shape)
    gr = np.zeros(prob.shape)
    vel = prob.vel if prob.vel is not None else np.zeros((3,) + prob.ghost_shape)
    lib().orc_operator_vjp(C.byref(g), fl, _p(np.ascontiguousarray(vel)), _p(prob.dcoeff), _bc(prob),
                           _p(np.ascontiguousarray(lam)), _p(np.ascontiguousarray(u)), _p(gv), _p(gd), _p(gr))
    return gv, gd, gr


def sg_face_d(cL, cR, DL, DR, dx):
    dwL, dwR = (C.c_double * 4)(), (C.c_double * 4)()
    lib().orc_sg_face_d(cL, cR, DL, DR, dx, dwL, dwR)
    return list(dwL), list(dwR)


class RowsMG:
    """Correction-scheme V-cycle over explicit 7-point rows (extension layer)."""

    def __init__(self, prob, hier=HIER_GEOM, ranks=(1, 1, 1), max_coarse=125, nu1=2, nu2=2,
                 transpose=False, flux=None):
        self.prob = prob
        self._g = _grid(prob, hier, ranks, max_coarse, nu1, nu2)
        fl = prob.flux if flux is None else flux
        self.h = lib().orc_mg_create(C.byref(self._g), fl, int(prob.timederiv), prob.dt, _p(prob.vel),
                                     _p(prob.dcoeff), _p(prob.reac), _bc(prob), int(transpose))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_mg_destroy(self.h)
            self.h = None

    def levels(self):
        dims = (C.c_int * 96)()
        n = lib().orc_mg_levels(self.h, dims)
        return [(dims[3 * i], dims[3 * i + 1], dims[3 * i + 2]) for i in range(n)]

    def rows(self, level=0):
        lx, ly, lz = self.levels()[level]
        p = lib().orc_mg_rows(self.h, level)
        return np.ctypeslib.as_array(p, shape=(7, lz, ly, lx)).copy()

    def vcycle(self, u, f):
        u = np.ascontiguousarray(u, dtype=np.float64)
        lib().orc_mg_vcycle(self.h, _p(u), _p(np.ascontiguousarray(f, dtype=np.float64)))
        return u

    def solve(self, b, x=None, maxit=50, tol=1e-10):
        x = np.zeros(self.prob.shape) if x is None else np.ascontiguousarray(x, dtype=np.float64).copy()
        hist = np.zeros(maxit + 2)
        it = lib().orc_mg_solve(self.h, _p(np.ascontiguousarray(b, dtype=np.float64)), _p(x), maxit, tol,
                                _p(hist))
        return x, hist[: it + 1]

    def fgmres(self, b, x=None, m=30, maxit=200, tol=1e-10):
        x = np.zeros(self.prob.shape) if x is None else np.ascontiguousarray(x, dtype=np.float64).copy()
        hist = np.zeros(maxit + 2)
        it = lib().orc_fgmres(self.h, _p(np.ascontiguousarray(b, dtype=np.float64)), _p(x), m, maxit, tol,
                              _p(hist))
        return x, hist[: it + 1]
