"""The .pvtr index writer (host only) against the restatement of the
reference's Writepvtrfile (mgridlib/cartwrite.f90:319-438), byte for byte,
and the restated writers' own consistency (offsets locate every block)."""
import os

import numpy as np

from mps3d_b200 import vtk
from oracle import vtk_oracle as VO


def test_pvtr_bytes_match_reference_writer(tmp_path):
    d = str(tmp_path / "output_0000003")
    names = ["Electrons", "Potential", "Efieldx   "]
    vtk.write_pvtr(d, (16, 8, 12), (2, 3, 2), names)
    assert os.path.isdir(d)
    got = open(d + ".pvtr", "rb").read()
    assert got == VO.pvtr(d, (16, 8, 12), (2, 3, 2), names)
    assert b'WholeExtent="       0       32        0       24       0       24"' in got
    assert got.count(b"<Piece ") == 12


def test_restated_vtr_reads_back(tmp_path):
    rng = np.random.default_rng(91)
    f = [rng.standard_normal((6, 5, 7)), rng.standard_normal((6, 5, 7))]
    VO.serial_vtr(str(tmp_path / "x"), f, ["a", "b"], (0.7, 0.3, 0.4), off=(0.1, 0.0, -0.2))
    back = VO.read_vtr(str(tmp_path / "x.vtr"))
    np.testing.assert_array_equal(back["a"], f[0][1:-1, 1:-1, 1:-1])
    np.testing.assert_array_equal(back["b"], f[1][1:-1, 1:-1, 1:-1])
    np.testing.assert_allclose(back["X"], 0.1 + np.arange(6) * 0.7 / 5, rtol=0, atol=1e-15)
    np.testing.assert_allclose(back["Z"], -0.2 + np.arange(5) * 0.4 / 4, rtol=0, atol=1e-15)
