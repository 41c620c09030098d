"""Build the CUDA library in-tree: mps3d_b200/_lib/libmps3d_b200.so (sm_100a).

    python -m mps3d_b200.build          # or __graft_entry__.build()
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libmps3d_b200.so")
SOURCES = ["mps_solver.cu", "mps_kernels.cu", "mps_noalloc.cu", "mps_adjoint.cu", "mps_step.cu", "mps_vtk.cu"]
HEADERS = ["mps_core.cuh", "mps_kernels.cuh", "mps_batch.cuh", "mps_tma.cuh", "mps_subcycle.cuh", os.path.join("..", "..", "include", "mps_linsolve.h")]

ARCH_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-static-global-template-stub=false",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    """Compile every source to an object in parallel (one nvcc per file),
    then link the shared library."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    cc = nvcc()
    jobs = []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [cc] + ARCH_FLAGS + list(extra or []) + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        jobs.append((subprocess.Popen(cmd, cwd=CSRC, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True),
                     obj))
    errors = []
    for proc, _ in jobs:
        out, _ = proc.communicate()
        if proc.returncode != 0:
            errors.append(out)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    tmp = LIB + ".tmp"
    link = [cc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp] + [o for _, o in jobs]
    if verbose:
        print(" ".join(link))
    r = subprocess.run(link, cwd=CSRC, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
