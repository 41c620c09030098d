"""The C-ABI library loads and exports every function include/*.h declares
(no compute: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from mps3d_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b(mps_[A-Za-z0-9_]+)\s*\(", src, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_parsed():
    names = declared_functions()
    assert "mps_linsolve" in names and "mps_vcycle_once" in names
    assert set(names) == set(capi.EXPORTS)


@pytest.fixture(scope="module")
def lib():
    build.build()
    return ctypes.CDLL(build.LIB)


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(lib, name):
    assert hasattr(lib, name)


def test_default_opts_and_version(lib):
    o = capi.default_opts()
    assert o.tol == 1e-10 and o.nu1 == 2 and o.nu2 == 2 and o.restart == 30
    assert o.hierarchy == capi.HIER_GEOM and o.max_coarse == 125
    assert b"sm_100a" in capi.load().mps_version()


def test_no_cpu_fallback(monkeypatch, tmp_path):
    # a missing library raises instead of silently running something else
    monkeypatch.setattr(capi, "LIBPATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(capi, "_lib", None)
    with pytest.raises(RuntimeError):
        capi.load()


def test_stream_argument_for_the_legacy_default_stream():
    # torch's default stream is the legacy default stream (cuda_stream 0); the
    # library reads NULL as the handle's own stream, so 0 goes out as
    # cudaStreamLegacy and other streams pass through unchanged
    assert capi.stream_arg(0) == capi.CUDA_STREAM_LEGACY == 1
    assert capi.stream_arg(0x7F00AB12) == 0x7F00AB12

    class FakeStream:
        cuda_stream = 0

    assert capi.stream_arg(FakeStream()) == 1
