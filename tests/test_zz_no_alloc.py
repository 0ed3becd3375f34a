"""Allocation-free Gram entry point (sdpx_b200_gram_noalloc).

Some callers cannot call cudaMalloc: a runtime that owns all device memory
through its own caching pool (Julia's or Python's GPU allocators), or a serving
loop where an implicit cudaMalloc/cudaFree would synchronise the device.  For
them the library offers S = PᵀP on caller-provided device buffers with the
split-K scratch held in a fixed device array inside the library (m ≤ 2048).

This test calls it through the C ABI and compares it with the regular entry
point (the identity-metric Schur assembly of a handle, which allocates its own
scratch) on two calls in a row, to the 1e-12 relative tolerance of the FP64
Schur parity tests.  It sits in its own file so pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from sdpx_b200 import generators as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend, load_library
    lib = load_library()
    lib.sdpx_b200_gram_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                           ctypes.c_void_p, ctypes.c_void_p]
    lib.sdpx_b200_gram_noalloc.restype = ctypes.c_int
    lib.sdpx_b200_gram_noalloc_error.restype = ctypes.c_char_p
    return torch, lib, CudaBackend


def _reference_gram(CudaBackend, prob):
    with CudaBackend(prob) as be:
        be.schur_build(identity=True)
        return be.schur_matrix()


def _noalloc_gram(torch, lib, prob):
    k, m = prob.k[0], prob.m
    P = torch.from_numpy(np.ascontiguousarray(prob.Av[0])).to("cuda")   # k²×m column-major
    S = torch.full((m, m), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = lib.sdpx_b200_gram_noalloc(P.data_ptr(), k * k, m, S.data_ptr(), stream.cuda_stream)
    assert rc == 0, lib.sdpx_b200_gram_noalloc_error()
    stream.synchronize()
    return S.cpu().numpy().T        # column-major m×m


def test_noalloc_gram_matches_handle_path_twice(env):
    torch, lib, CudaBackend = env
    for seed, (m, k) in ((3, (300, 24)), (4, (130, 40))):
        prob = G.sdpa_dense(m=m, blocks=[k], seed=seed)
        ref = _reference_gram(CudaBackend, prob)
        got = _noalloc_gram(torch, lib, prob)
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err <= 1e-12, err
        assert np.array_equal(got, got.T)


def test_noalloc_gram_rejects_oversized_problem(env):
    torch, lib, _ = env
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.sdpx_b200_gram_noalloc(dummy.data_ptr(), 1, 4096, dummy.data_ptr(), None)
    assert rc != 0
    assert b"2048" in lib.sdpx_b200_gram_noalloc_error()
