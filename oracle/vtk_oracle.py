"""Restatement of the reference's VTK writers (TEST INFRASTRUCTURE ONLY: the
byte-level checker of mps_write_vtr_dev, mps_write_vtr_piece_dev and
mps_write_pvtr).

Follows mgridlib/cartwrite.f90: Writeserialvtrfile (:8-161), Writevtrfile
(:163-317), Writepvtrfile (:319-438).  Fortran details that fix the bytes:
every line is written as trim(str) of a blank-padded CHARACTER(300), so a
line keeps its trailing newline and any blanks before it; integers go
through the (i8) edit descriptor (right-justified in 8 characters) and
keep their leading blanks under trim; the extent string joins the six
fields with single blanks except between ymax and zmin (:78-79); each
appended block is a default-kind INTEGER (INTSIZE = 4, globalvars.f90:10)
byte count followed by the doubles, stream access, little endian.
"""
from __future__ import annotations

import os
import struct

import numpy as np


def i8(v: int) -> str:
    return "%8d" % v


def extent(x0, x1, y0, y1, z0, z1) -> str:
    return i8(x0) + " " + i8(x1) + " " + i8(y0) + " " + i8(y1) + i8(z0) + " " + i8(z1)


def _vtr_bytes(whole, piece, lx, ly, lz, off, length, names, interiors):
    nl = "\n"
    out = []
    put = lambda s: out.append(s.encode())  # noqa: E731
    scalars_size = lx * ly * lz * 8
    put('<?xml version="1.0"?>' + nl)
    put('<VTKFile type="RectilinearGrid" version="0.1" byte_order="LittleEndian">' + nl)
    put('  <RectilinearGrid WholeExtent="' + whole + '">' + nl)
    put('    <Piece Extent="' + piece + '">' + nl)
    put("      <PointData>  </PointData>" + nl)
    put("      <CellData> " + nl)
    b = 0
    for nm in names:
        put('         <DataArray type="Float64" Name="' + nm.rstrip(' ') + '" format="appended" offset="' + i8(b) +
            '"           />' + nl)
        b += 4 + scalars_size
    put("      </CellData>" + nl)
    put("      <Coordinates>" + nl)
    nn = (lx + 1, ly + 1, lz + 1)
    for a, ax in enumerate("XYZ"):
        put('<DataArray type="Float64" Name="' + ax + '"  format="appended" offset="' + i8(b) + '" />' + nl)
        b += 4 + nn[a] * 8
    put("      </Coordinates>" + nl)
    put("    </Piece>" + nl)
    put("  </RectilinearGrid>" + nl)
    put('  <AppendedData encoding="raw">' + nl)
    put("_")
    for f in interiors:  # (lz, ly, lx) C order == Fortran (lx, ly, lz)
        out.append(struct.pack("<i", scalars_size))
        out.append(np.ascontiguousarray(f, dtype="<f8").tobytes())
    for a in range(3):
        d = length[a] / (nn[a] - 1)
        c = np.array([off[a] + i * d for i in range(nn[a])], dtype="<f8")
        out.append(struct.pack("<i", nn[a] * 8))
        out.append(c.tobytes())
    put(nl + "  </AppendedData>" + nl)
    put("</VTKFile>" + nl)
    return b"".join(out)


def serial_vtr(filename, ghosted_fields, names, length, off=(0.0, 0.0, 0.0)):
    """Writeserialvtrfile: <filename>.vtr of the interiors of ghosted
    (nz+2, ny+2, nx+2) fields over a box of the given lengths."""
    nz, ny, nx = (s - 2 for s in ghosted_fields[0].shape)
    e = extent(0, nx, 0, ny, 0, nz)
    data = _vtr_bytes(e, e, nx, ny, nz, off, length, names, [f[1:-1, 1:-1, 1:-1] for f in ghosted_fields])
    with open(filename + ".vtr", "wb") as fh:
        fh.write(data)
    return data


def piece_vtr(dirname, rank, pind, ghosted_fields, names, length, off=(0.0, 0.0, 0.0)):
    """Writevtrfile: <dirname>/file_<rank:08d>.vtr of one rank's piece, pind
    the rank's 1-based (x, y, z) block index."""
    nz, ny, nx = (s - 2 for s in ghosted_fields[0].shape)
    e = extent(nx * (pind[0] - 1), nx * pind[0], ny * (pind[1] - 1), ny * pind[1], nz * (pind[2] - 1), nz * pind[2])
    data = _vtr_bytes(e, e, nx, ny, nz, off, length, names, [f[1:-1, 1:-1, 1:-1] for f in ghosted_fields])
    with open(os.path.join(dirname, "file_%08d.vtr" % rank), "wb") as fh:
        fh.write(data)
    return data


def pvtr(dirname, lxyz, pxyz, names):
    """Writepvtrfile: the bytes of <dirname>.pvtr (pieces in rank order,
    find3dindex: x fastest, globalvars.f90:73-97)."""
    nl = "\n"
    lx, ly, lz = lxyz
    px, py, pz = pxyz
    s = ['<?xml version="1.0"?>' + nl,
         '<VTKFile type="PRectilinearGrid" version="0.1" byte_order="LittleEndian">' + nl,
         '<PRectilinearGrid WholeExtent="' + extent(0, lx * px, 0, ly * py, 0, lz * pz) + '" GhostLevel="0">' + nl,
         "<PPointData>  </PPointData>" + nl, "<PCellData> " + nl]
    s += ['<PDataArray type="Float64" Name="' + nm.rstrip(' ') + '"/>' + nl for nm in names]
    s += ["</PCellData>" + nl, "<PCoordinates>" + nl]
    s += ['<PDataArray type="Float64" Name="' + a + '"/>' + nl for a in "XYZ"]
    s += ["</PCoordinates>" + nl]
    for r in range(px * py * pz):
        i, j, k = r % px + 1, (r // px) % py + 1, r // (px * py) + 1
        s.append('<Piece Extent="' + extent(lx * (i - 1), lx * i, ly * (j - 1), ly * j, lz * (k - 1), lz * k) +
                 '" Source="' + dirname + "/file_%08d.vtr" % r + '"/>' + nl)
    s += ["</PRectilinearGrid>" + nl, "</VTKFile>" + nl]
    return "".join(s).encode()


def read_vtr(path):
    """Minimal reader of the files above: {name: array} of the cell data
    (Fortran order reshaped to (nz, ny, nx)) and the X/Y/Z coordinates,
    located through the DataArray offsets of the header."""
    raw = open(path, "rb").read()
    head, rest = raw.split(b'<AppendedData encoding="raw">\n_', 1)
    import re

    ext = [int(v) for v in re.search(rb'Piece Extent="([^"]*)"', head).group(1).split()]
    nx, ny, nz = ext[1] - ext[0], ext[3] - ext[2], ext[5] - ext[4]
    out = {}
    for m in re.finditer(rb'Name="([^"]+)"\s+format="appended" offset="\s*(\d+)"', head):
        name, off = m.group(1).decode(), int(m.group(2))
        (nbytes,) = struct.unpack("<i", rest[off:off + 4])
        a = np.frombuffer(rest[off + 4:off + 4 + nbytes], dtype="<f8")
        out[name] = a.reshape(nz, ny, nx) if name not in "XYZ" else a
    return out
