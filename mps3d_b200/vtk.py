"""VTK RectilinearGrid output from device buffers (mgridlib/cartwrite.f90),
over the C ABI: mps_write_vtr_dev (Writeserialvtrfile), mps_write_vtr_piece_dev
(Writevtrfile) and mps_write_pvtr (Writepvtrfile).  Fields are ghosted
float64 CUDA tensors of shape (nz+2, ny+2, nx+2); their interiors are
written."""
from __future__ import annotations

import ctypes as C
from typing import Sequence

from . import capi


def _names(names: Sequence[str]):
    arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
    return arr


def _fields(fields):
    return (C.c_void_p * len(fields))(*[C.c_void_p(f.data_ptr()) for f in fields])


def _grid_of(f, llen):
    nz, ny, nx = (s - 2 for s in f.shape)
    return capi.Grid(nx, ny, nz, *[float(v) for v in llen])


def write_vtr(filename: str, fields, names: Sequence[str], llen, off=(0.0, 0.0, 0.0), stream=None):
    """<filename>.vtr of the fields' interiors over a box of lengths llen."""
    o = (C.c_double * 3)(*[float(v) for v in off])
    st = capi.load().mps_write_vtr_dev(filename.encode(), C.byref(_grid_of(fields[0], llen)), o, len(fields),
                                       _names(names), _fields(fields), C.c_void_p(capi.stream_arg(stream)))
    if st != 0:
        raise capi.SolverError(st, "mps_write_vtr_dev")


def write_vtr_piece(dirname: str, rank: int, pind, fields, names: Sequence[str], llen, off=(0.0, 0.0, 0.0),
                    stream=None):
    """<dirname>/file_<rank:08d>.vtr: one rank's piece (pind: 1-based block index)."""
    o = (C.c_double * 3)(*[float(v) for v in off])
    pi = (C.c_int * 3)(*[int(v) for v in pind])
    st = capi.load().mps_write_vtr_piece_dev(dirname.encode(), int(rank), pi, C.byref(_grid_of(fields[0], llen)), o,
                                             len(fields), _names(names), _fields(fields),
                                             C.c_void_p(capi.stream_arg(stream)))
    if st != 0:
        raise capi.SolverError(st, "mps_write_vtr_piece_dev")


def write_pvtr(dirname: str, lxyz, pxyz, names: Sequence[str]):
    """<dirname>.pvtr, the index of the pieces (and the folder dirname)."""
    lx = (C.c_int * 3)(*[int(v) for v in lxyz])
    px = (C.c_int * 3)(*[int(v) for v in pxyz])
    st = capi.load().mps_write_pvtr(dirname.encode(), lx, px, len(names), _names(names))
    if st != 0:
        raise capi.SolverError(st, "mps_write_pvtr")
