"""Allocation-free Gram entry point (sdpx_b200_gram_noalloc).

Some callers cannot call cudaMalloc: a runtime that owns all device memory
through its own caching pool (Julia's or Python's GPU allocators), or a serving
loop where an implicit cudaMalloc/cudaFree would synchronise the device.  For
them the library offers S = PᵀP on caller-provided device buffers with the
split-K scratch held in a fixed device array inside the library (m ≤ 2048,
K ≤ 2^30).

The GPU tests call it through the C ABI and compare it with the regular entry
point (the identity-metric Schur assembly of a handle, which allocates its own
scratch) on two calls in a row, and with NumPy's PᵀP (an independent FP64
product), to the 1e-12 relative tolerance of the FP64 Schur parity tests; the
largest admitted m (2048) is checked the same way and m = 2049 is rejected.
The rejection paths for oversized K and NULL operands return before any device
work, so they run without a GPU.  The file sits on its own so pytest collects
it last.
"""
import ctypes

import numpy as np
import pytest

from sdpx_b200 import generators as G

TOL = 1e-12


def _bind(lib):
    lib.sdpx_b200_gram_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                           ctypes.c_void_p, ctypes.c_void_p]
    lib.sdpx_b200_gram_noalloc.restype = ctypes.c_int
    lib.sdpx_b200_gram_noalloc_error.restype = ctypes.c_char_p
    return lib


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend, load_library
    return torch, _bind(load_library()), CudaBackend


def _reference_gram(CudaBackend, prob):
    with CudaBackend(prob) as be:
        be.schur_build(identity=True)
        return be.schur_matrix()


def _noalloc_gram(torch, lib, P_host):
    """P_host: K×m column-major (Fortran-ordered) FP64 array."""
    K, m = P_host.shape
    P = torch.from_numpy(np.ascontiguousarray(P_host.T)).to("cuda")   # m rows of K = column-major P
    S = torch.full((m, m), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = lib.sdpx_b200_gram_noalloc(P.data_ptr(), K, m, S.data_ptr(), stream.cuda_stream)
    assert rc == 0, lib.sdpx_b200_gram_noalloc_error()
    stream.synchronize()
    return S.cpu().numpy().T        # column-major m×m


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.gpu
def test_noalloc_gram_matches_handle_path_twice(env):
    torch, lib, CudaBackend = env
    for seed, (m, k) in ((3, (300, 24)), (4, (130, 40))):
        prob = G.sdpa_dense(m=m, blocks=[k], seed=seed)
        P = np.asarray(prob.Av[0]).T                    # k²×m (Av rows are vec(A_i))
        ref = _reference_gram(CudaBackend, prob)
        npref = P.T @ P
        for _ in range(2):
            got = _noalloc_gram(torch, lib, P)
            assert _rel(got, ref) <= TOL
            assert _rel(got, npref) <= TOL
            assert np.array_equal(got, got.T)


@pytest.mark.gpu
def test_noalloc_gram_largest_m_against_numpy(env):
    torch, lib, _ = env
    rng = np.random.default_rng(11)
    m, K = 2048, 96
    P = rng.standard_normal((K, m))
    got = _noalloc_gram(torch, lib, P)
    assert _rel(got, P.T @ P) <= TOL


@pytest.mark.gpu
def test_noalloc_gram_rejects_oversized_m(env):
    torch, lib, _ = env
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.sdpx_b200_gram_noalloc(dummy.data_ptr(), 1, 2049, dummy.data_ptr(), None)
    assert rc == -1
    assert b"2048" in lib.sdpx_b200_gram_noalloc_error()


def test_noalloc_gram_rejects_oversized_k_and_null_without_device_work():
    """K > 2^30 and NULL operands are refused by argument checks that run before
    any CUDA call; the non-NULL pointers here are never dereferenced."""
    from sdpx_b200.cuda_backend import load_library
    lib = _bind(load_library())
    fake = ctypes.c_void_p(0x1000)
    rc = lib.sdpx_b200_gram_noalloc(fake, (1 << 30) + 1, 4, fake, None)
    assert rc == -1
    assert b"2^30" in lib.sdpx_b200_gram_noalloc_error()
    rc = lib.sdpx_b200_gram_noalloc(None, 16, 4, fake, None)
    assert rc == -1
    assert b"NULL" in lib.sdpx_b200_gram_noalloc_error()
