"""The C-ABI library exports every entry point include/sdpx_b200.h declares
(CPU-only: loads the shared object, makes no device call)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sdpx_b200.h")
LIB = os.path.join(ROOT, "sdpx.jl_b200", "libsdpx_b200.so")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(sdpx_b200_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        import __graft_entry__  # builds in place
        __graft_entry__.build()
    return ctypes.CDLL(LIB)


def test_header_declares_core_entry_points():
    names = declared_symbols()
    for must in ("sdpx_b200_create", "sdpx_b200_schur_build", "sdpx_b200_factorize",
                 "sdpx_b200_solve", "sdpx_b200_refine", "sdpx_b200_line_search"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_without_gpu(lib):
    lib.sdpx_b200_abi_version.restype = ctypes.c_int
    assert lib.sdpx_b200_abi_version() == 1
