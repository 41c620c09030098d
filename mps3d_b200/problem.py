"""Operator / boundary-condition description shared by the solver API.

The fields mirror the arguments of ``perform_vcycle`` (mgridlib/mgridsteps.f90:384-417):
ghosted ``real*8`` arrays of shape ``(-g_nglayers+1 : l+g_nglayers)`` per
direction in Fortran order, ``vel`` with a trailing ``NDIM`` axis, six face
arrays of boundary values and six 4-character BC codes in the order LEFT,
RIGHT, BOTTOM, TOP, BACK, FRONT (mgridlib/globalvars.f90:11-17, 57-66).

In numpy the Fortran ``(lx+2, ly+2, lz+2)`` array is held as a C-ordered
``(lz+2, ly+2, lx+2)`` array: the same bytes, i fastest.  Face arrays are
``left/right: (lz, ly)``, ``bottom/top: (lz, lx)``, ``back/front: (ly, lx)``
in C order, i.e. Fortran ``(ly,lz)``, ``(lx,lz)``, ``(lx,ly)``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

# face order, mgridlib/globalvars.f90:11-17
LEFT, RIGHT, BOTTOM, TOP, BACK, FRONT = range(6)
# BC codes: 'DIRC','FLUX','ZGRD' are the reference's (discretepde.f90:428-606,
# 798-1100); 'DZGD' appears in plasma_pde/poissoneq.f90:259 and is treated by
# find_AX/find_bvec like a zero-flux face; 'PERI' (periodic) is an extension.
BC_CODES = {"DIRC": 1, "FLUX": 2, "ZGRD": 3, "PERI": 4, "DZGD": 5}
BC_NAMES = {v: k for k, v in BC_CODES.items()}


def bc_code(c) -> int:
    if isinstance(c, str):
        return BC_CODES[c.upper()]
    return int(c)


@dataclass
class Problem:
    """One linear system ``A u = b`` in the reference's operator form

    du/dt + div(vel u) = div(dcoeff grad u) + reac u + source

    discretised by finite volumes on ``lx*ly*lz`` cells of a box of size
    ``llen``.  ``timederiv`` adds ``1/dt`` to the diagonal (find_AX,
    discretepde.f90:1106); the caller folds ``u_old/dt`` into ``source`` as the
    reference's equation modules do (e.g. plasma_pde/edeneq.f90:441).
    """

    lx: int
    ly: int
    lz: int
    llen: Sequence[float]
    dcoeff: np.ndarray
    source: np.ndarray
    bc: List[int]
    bcvals: List[np.ndarray]
    vel: np.ndarray = None
    reac: np.ndarray = None
    timederiv: bool = False
    dt: float = 1.0
    flux: int = 0  # 0 upwind (reference 3D), 1 Scharfetter-Gummel (extension)

    def __post_init__(self):
        g = self.ghost_shape
        self.bc = [bc_code(c) for c in self.bc]
        if len(self.bc) != 6:
            raise ValueError("six BC codes required")
        for a, b in ((0, 1), (2, 3), (4, 5)):
            if (self.bc[a] == 4) != (self.bc[b] == 4):
                raise ValueError("PERI must be set on both faces of a direction")
        if self.vel is None:
            self.vel = np.zeros((3,) + g)
        if self.reac is None:
            self.reac = np.zeros(g)
        self.vel = np.ascontiguousarray(self.vel, dtype=np.float64)
        self.dcoeff = np.ascontiguousarray(self.dcoeff, dtype=np.float64)
        self.reac = np.ascontiguousarray(self.reac, dtype=np.float64)
        self.source = np.ascontiguousarray(self.source, dtype=np.float64)
        if self.vel.shape != (3,) + g:
            raise ValueError(f"vel shape {self.vel.shape} != {(3,) + g}")
        for name in ("dcoeff", "reac", "source"):
            if getattr(self, name).shape != g:
                raise ValueError(f"{name} shape {getattr(self, name).shape} != {g}")
        shapes = self.face_shapes
        vals = []
        for f in range(6):
            v = self.bcvals[f] if self.bcvals is not None and self.bcvals[f] is not None else 0.0
            v = np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), shapes[f]))
            vals.append(v)
        self.bcvals = vals
        self.llen = tuple(float(x) for x in self.llen)

    @property
    def ghost_shape(self):
        return (self.lz + 2, self.ly + 2, self.lx + 2)

    @property
    def shape(self):
        return (self.lz, self.ly, self.lx)

    @property
    def ncells(self):
        return self.lx * self.ly * self.lz

    @property
    def face_shapes(self):
        return [(self.lz, self.ly)] * 2 + [(self.lz, self.lx)] * 2 + [(self.ly, self.lx)] * 2

    def zeros_ghosted(self):
        return np.zeros(self.ghost_shape)


def ghosted(interior: np.ndarray) -> np.ndarray:
    """Embed an interior ``(lz, ly, lx)`` array in a zero ghost layer."""
    out = np.zeros(tuple(s + 2 for s in interior.shape))
    out[1:-1, 1:-1, 1:-1] = interior
    return out
