"""CPU-side checks of the drop-in boundary: the shared library builds for
sm_100a, loads without a GPU and exports every entry point the header
declares; the Python binding covers the same list."""
import os
import re
import ctypes

from ggi_tlm_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "tlm_gpu.h")).read()
    return sorted(set(re.findall(r"^int\s+(tlm_gpu_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(build.build())
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s


def test_binding_covers_header():
    assert sorted(capi.EXPORTS) == header_symbols()
