"""ctypes binding of the C ABI declared in include/mps_linsolve.h.

This is the only route from Python into the solver: every call goes through
the in-tree CUDA library mps3d_b200/_lib/libmps3d_b200.so.  There is no CPU
fallback; a missing library raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

LIBPATH = _build.LIB

# status codes (enum mps_status)
MPS_OK = 0
MPS_ERR_NOT_CONVERGED = 1
MPS_ERR_NAN = 2
MPS_ERR_BREAKDOWN = 3
MPS_ERR_BAD_ARG = 4
MPS_ERR_TIMEOUT = 5
MPS_ERR_CUDA = 6
MPS_ERR_NOMEM = 7
MPS_ERR_TOO_LARGE = 8
STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", 2: "NAN", 3: "BREAKDOWN", 4: "BAD_ARG", 5: "TIMEOUT", 6: "CUDA",
                7: "NOMEM", 8: "TOO_LARGE"}
# mps_apply_A_noalloc: round_up(lx, 16) * ly * lz limit and its static scratch
NOALLOC_MAX_CELLS = 262144
NOALLOC_SCRATCH_BYTES = 16 * 8 * NOALLOC_MAX_CELLS

HIER_CELL, HIER_GEOM = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
KRYLOV_NONE, KRYLOV_FGMRES = 0, 1
FLUX_UPWIND, FLUX_SG = 0, 1
TOL_RMS_ABS, TOL_REL_L2 = 0, 1

# every symbol include/mps_linsolve.h declares
EXPORTS = [
    "mps_default_opts", "mps_version", "mps_create", "mps_destroy", "mps_stream", "mps_last_error",
    "mps_linsolve", "mps_linsolve_dev", "mps_vcycle_once", "mps_apply_A_dev", "mps_find_bvec_dev",
    "mps_fill_ghosts_dev", "mps_set_profile", "mps_get_profile", "mps_apply_A_noalloc",
    "mps_linsolve_batched_dev", "mps_operator_vjp_dev",
    "mps_efield_dev", "mps_eden_transport_dev", "mps_poisson_source_dev", "mps_plasma_step_dev",
    "mps_write_vtr_dev", "mps_write_vtr_piece_dev", "mps_write_pvtr",
]

PROF_SMOOTH, PROF_RESTRICT, PROF_PROLONG, PROF_RESID, PROF_NCLASS = 0, 1, 2, 3, 8


class Profile(C.Structure):
    _fields_ = [("count", C.c_int * 8), ("ms", C.c_double * 8), ("precision_bytes", C.c_int),
                ("coeff_field", C.c_int), ("cells", C.c_longlong)]


class Grid(C.Structure):
    _fields_ = [("lx", C.c_int), ("ly", C.c_int), ("lz", C.c_int),
                ("llenx", C.c_double), ("lleny", C.c_double), ("llenz", C.c_double)]


class Opts(C.Structure):
    _fields_ = [
        ("tol", C.c_double), ("tol_kind", C.c_int), ("maxit", C.c_int),
        ("nu1", C.c_int), ("nu2", C.c_int), ("hierarchy", C.c_int), ("ranks", C.c_int * 3),
        ("max_coarse", C.c_int), ("precision", C.c_int), ("inner_cycles", C.c_int),
        ("krylov", C.c_int), ("restart", C.c_int), ("fill_ghosts", C.c_int), ("use_graph", C.c_int),
        ("transpose", C.c_int), ("flux", C.c_int),
    ]


class Info(C.Structure):
    _fields_ = [("status", C.c_int), ("iters", C.c_int), ("vcycles", C.c_int), ("levels", C.c_int),
                ("rel_res", C.c_double), ("rms_res", C.c_double), ("rel_res0", C.c_double),
                ("time_ms", C.c_double), ("launches", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ProblemDesc(C.Structure):
    """struct mps_problem: one problem of a batched call (device pointers)."""
    _fields_ = [("g", Grid), ("timederiv", C.c_int), ("dt", C.c_double), ("vel", C.c_void_p),
                ("dcoeff", C.c_void_p), ("reac", C.c_void_p), ("source", C.c_void_p), ("bc_code", C.c_int * 6),
                ("bcval", C.c_void_p * 6), ("mgridsterm", C.c_void_p), ("soln", C.c_void_p)]


class PlasmaStep(C.Structure):
    """struct mps_plasma_step: the fields of one implicit potential + electron
    step (device pointers, ghosted Fortran layout)."""
    _fields_ = [("g", Grid), ("phi_bc", C.c_int * 6), ("phi_bcval", C.c_void_p * 6), ("eps", C.c_void_p),
                ("phi", C.c_void_p), ("rho_scale", C.c_double), ("nion", C.c_int), ("n_ion", C.c_void_p),
                ("ion_charge", C.c_void_p), ("phi_source", C.c_void_p), ("ne_bc", C.c_int * 6),
                ("ne_bcval", C.c_void_p * 6), ("n_e", C.c_void_p), ("mu_e", C.c_void_p), ("d_e", C.c_void_p),
                ("te", C.c_void_p), ("prod_e", C.c_void_p), ("dt", C.c_double), ("nemin", C.c_double),
                ("efield_scale", C.c_double), ("limiter", C.c_int), ("vel_scaling", C.c_double),
                ("dcoeff_scaling", C.c_double), ("source_scaling", C.c_double), ("efield", C.c_void_p),
                ("vel", C.c_void_p), ("dcoeff", C.c_void_p), ("source", C.c_void_p)]


BATCH_MAX = 4096

_lib = None


def load(build_if_missing: bool = False):
    """Load the CUDA library; raises if it is absent (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        if build_if_missing:
            _build.build()
        else:
            raise RuntimeError(f"CUDA library {LIBPATH} is not built (run __graft_entry__.build())")
    L = C.CDLL(LIBPATH)
    dp = C.POINTER(C.c_double)
    vp = C.c_void_p
    ip = C.POINTER(C.c_int)
    L.mps_default_opts.argtypes = [C.POINTER(Opts)]
    L.mps_version.restype = C.c_char_p
    L.mps_create.argtypes = [C.POINTER(vp), C.c_int]
    L.mps_destroy.argtypes = [vp]
    L.mps_stream.argtypes = [vp]
    L.mps_stream.restype = vp
    L.mps_last_error.argtypes = [vp]
    L.mps_last_error.restype = C.c_char_p
    common = [vp, C.POINTER(Grid), C.c_int, C.c_double, vp, vp, vp, vp, ip, C.POINTER(vp), vp, vp,
              C.POINTER(Opts), C.POINTER(Info)]
    L.mps_linsolve.argtypes = common
    L.mps_linsolve_dev.argtypes = common + [vp]
    L.mps_vcycle_once.argtypes = [vp, C.POINTER(Grid), C.c_int, C.c_double, vp, vp, vp, vp, ip, C.POINTER(vp), vp,
                                  vp, dp, C.POINTER(Opts)]
    L.mps_apply_A_dev.argtypes = [vp, C.POINTER(Grid), C.c_int, C.c_double, vp, vp, vp, ip, vp, vp,
                                  C.POINTER(Opts), vp]
    L.mps_find_bvec_dev.argtypes = [vp, C.POINTER(Grid), vp, vp, vp, ip, C.POINTER(vp), vp, vp, C.POINTER(Opts), vp]
    L.mps_fill_ghosts_dev.argtypes = [vp, C.POINTER(Grid), ip, C.POINTER(vp), vp, vp]
    L.mps_set_profile.argtypes = [vp, C.c_int]
    L.mps_get_profile.argtypes = [vp, C.POINTER(Profile), C.c_int]
    L.mps_linsolve_batched_dev.argtypes = [vp, C.c_int, C.POINTER(ProblemDesc), C.POINTER(Opts), C.POINTER(Info), vp]
    L.mps_operator_vjp_dev.argtypes = [C.POINTER(Grid), vp, vp, ip, vp, vp, C.POINTER(Opts), vp, vp, vp, vp]
    L.mps_apply_A_noalloc.argtypes = [C.POINTER(Grid), C.c_int, C.c_double, vp, vp, vp, ip, vp, vp, C.POINTER(Opts),
                                      vp]
    L.mps_efield_dev.argtypes = [C.POINTER(Grid), ip, C.POINTER(vp), vp, C.c_double, C.c_int, vp, vp]
    L.mps_eden_transport_dev.argtypes = [C.POINTER(Grid), vp, vp, vp, vp, vp, vp, C.c_int, C.c_double, dp, vp, vp,
                                         vp, vp]
    L.mps_poisson_source_dev.argtypes = [C.POINTER(Grid), vp, C.c_int, vp, vp, C.c_double, vp, C.c_double, vp, vp]
    L.mps_plasma_step_dev.argtypes = [vp, vp, C.POINTER(PlasmaStep), C.POINTER(Opts), C.POINTER(Opts),
                                      C.POINTER(Info), C.POINTER(Info), vp]
    cp = C.POINTER(C.c_char_p)
    L.mps_write_vtr_dev.argtypes = [C.c_char_p, C.POINTER(Grid), dp, C.c_int, cp, C.POINTER(vp), vp]
    L.mps_write_vtr_piece_dev.argtypes = [C.c_char_p, C.c_int, ip, C.POINTER(Grid), dp, C.c_int, cp, C.POINTER(vp),
                                          vp]
    L.mps_write_pvtr.argtypes = [C.c_char_p, ip, ip, C.c_int, cp]
    for name in ("mps_write_vtr_dev", "mps_write_vtr_piece_dev", "mps_write_pvtr", "mps_efield_dev", "mps_eden_transport_dev", "mps_poisson_source_dev", "mps_plasma_step_dev",
                 "mps_set_profile", "mps_get_profile", "mps_create", "mps_destroy", "mps_linsolve", "mps_linsolve_dev", "mps_vcycle_once",
                 "mps_apply_A_dev", "mps_find_bvec_dev", "mps_fill_ghosts_dev", "mps_apply_A_noalloc",
                 "mps_linsolve_batched_dev", "mps_operator_vjp_dev"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def default_opts(**kw) -> Opts:
    o = Opts()
    load().mps_default_opts(C.byref(o))
    for k, v in kw.items():
        if k == "ranks":
            o.ranks[:] = list(v)
        else:
            if not hasattr(o, k):
                raise KeyError(k)
            setattr(o, k, v)
    return o


class SolverError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__(f"mps status {status} ({STATUS_NAMES.get(status, '?')}): {msg}")
        self.status = status


# cudaStreamLegacy: the legacy default stream, named by a handle that is not NULL
CUDA_STREAM_LEGACY = 1


def stream_arg(stream=None) -> int:
    """The ``stream`` argument of the *_dev entry points for a torch stream (or
    its ``cuda_stream`` integer; None = torch's current stream).

    torch's default stream is the legacy default stream, whose ``cuda_stream``
    is 0.  The library reads NULL as "the handle's own stream", a non-blocking
    stream that is ordered with no other stream, so a call given 0 would read
    inputs that torch has not finished writing and return before its outputs
    are written as torch sees them.  0 is therefore passed as cudaStreamLegacy,
    which the library orders its work after and before like any caller stream."""
    if stream is None:
        import torch

        stream = torch.cuda.current_stream()
    s = stream if isinstance(stream, int) else int(stream.cuda_stream)
    return s if s != 0 else CUDA_STREAM_LEGACY


class Handle:
    """Owns an mps_handle (a CUDA stream and a device workspace)."""

    def __init__(self, device: int = -1):
        self._lib = load()
        h = C.c_void_p()
        st = self._lib.mps_create(C.byref(h), int(device))
        if st != 0:
            raise SolverError(st, "mps_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self._lib.mps_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return self._lib.mps_stream(self.h) or 0

    def set_profile(self, on):
        """False: off; True or 1: time the finest level; 1 + l: time level l."""
        self._lib.mps_set_profile(self.h, int(on))

    def get_profile(self, reset=True) -> Profile:
        p = Profile()
        self._lib.mps_get_profile(self.h, C.byref(p), int(bool(reset)))
        return p

    def last_error(self) -> str:
        r = self._lib.mps_last_error(self.h)
        return r.decode() if r else ""
