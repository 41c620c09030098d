"""VTK output from device buffers against the restatement of the reference's
writers (mgridlib/cartwrite.f90): the serial .vtr and the per-rank pieces,
byte for byte, and read back."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mps3d_b200 import vtk  # noqa: E402
from oracle import vtk_oracle as VO  # noqa: E402

pytestmark = pytest.mark.gpu


def _fields(shape, n, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(shape) * 10 ** q for q in range(n)]


@pytest.mark.parametrize("shape", [(5, 4, 3), (19, 18, 17), (67, 67, 67)])
def test_serial_vtr_bytes_match_reference_writer(tmp_path, shape):
    f = _fields(shape, 3, 92)
    names = ["Electrons", "Potential", "Temp  "]
    llen, off = (0.01, 0.02, 0.03), (0.0, 0.5, -1.0)
    vtk.write_vtr(str(tmp_path / "gpu"), [torch.from_numpy(a).cuda() for a in f], names, llen, off)
    ref = VO.serial_vtr(str(tmp_path / "ref"), f, names, llen, off)
    assert open(str(tmp_path / "gpu.vtr"), "rb").read() == ref
    back = VO.read_vtr(str(tmp_path / "gpu.vtr"))
    np.testing.assert_array_equal(back["Potential"], f[1][1:-1, 1:-1, 1:-1])


def test_piece_vtr_bytes_match_reference_writer(tmp_path):
    d = str(tmp_path / "out")
    f = _fields((10, 7, 9), 2, 93)
    names = ["ne", "phi"]
    vtk.write_pvtr(d, (7, 5, 8), (2, 1, 3), names)
    for rank, pind in ((0, (1, 1, 1)), (5, (2, 1, 3))):
        vtk.write_vtr_piece(d, rank, pind, [torch.from_numpy(a).cuda() for a in f], names, (0.5, 0.4, 0.6),
                            off=(0.5 * (pind[0] - 1), 0.0, 0.6 * (pind[2] - 1)))
        got = open(f"{d}/file_{rank:08d}.vtr", "rb").read()
        ref = VO._vtr_bytes(VO.extent(7 * (pind[0] - 1), 7 * pind[0], 0, 5, 8 * (pind[2] - 1), 8 * pind[2]),
                            VO.extent(7 * (pind[0] - 1), 7 * pind[0], 0, 5, 8 * (pind[2] - 1), 8 * pind[2]),
                            7, 5, 8, (0.5 * (pind[0] - 1), 0.0, 0.6 * (pind[2] - 1)), (0.5, 0.4, 0.6), names,
                            [a[1:-1, 1:-1, 1:-1] for a in f])
        assert got == ref
