"""The C-ABI library exports every entry point that include/*.h declares
(CPU-only: loads the shared object, makes no device call)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))
LIB = os.path.join(ROOT, "sdpx.jl_b200", "libsdpx_b200.so")


def declared_symbols():
    names = set()
    for h in HEADERS:
        names |= set(re.findall(r"\b(sdpx_b200_[a-z0-9_]+)\s*\(", open(h).read()))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        import __graft_entry__  # builds in place
        __graft_entry__.build()
    return ctypes.CDLL(LIB)


def test_header_declares_core_entry_points():
    names = declared_symbols()
    for must in ("sdpx_b200_create", "sdpx_b200_schur_build", "sdpx_b200_factorize",
                 "sdpx_b200_solve", "sdpx_b200_refine", "sdpx_b200_line_search",
                 "sdpx_b200_normal_nt_scaling", "sdpx_b200_normal_factorize",
                 "sdpx_b200_normal_solve", "sdpx_b200_batch_create",
                 "sdpx_b200_batch_optimize", "sdpx_b200_batch_autotune"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_without_gpu(lib):
    lib.sdpx_b200_abi_version.restype = ctypes.c_int
    assert lib.sdpx_b200_abi_version() == 1
