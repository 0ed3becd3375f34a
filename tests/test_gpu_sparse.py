"""Sparse Schur engine on the B200 (SDPX's SparseCons path) against the oracle.

* Kernel level, on one interior iterate: the device S built from the flat
  coordinate entries equals the oracle's sparse assembly (and so the dense
  one) to 1e-12 relative; the entry extraction reports the oracle's active
  positions and stored entries.  Cases: 2×2 and 1×1 blocks; a 150-order block
  whose coefficients carry up to 80 stored entries (more than one 64-entry
  round of the per-position product).
* Solve level: with the sparse engine the device solve reaches the oracle's
  status, iterations (±1) and objective (1e-7 relative).
* A block above the kernel's 160 limit is refused with an error.
"""
import numpy as np
import pytest

from sdpx_b200 import SolverOptions, generators as G, solve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend
    return CudaBackend


def _iterate(prob, seed=1):
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for k in prob.k:
        g = rng.standard_normal((k, k))
        X.append(np.eye(k) + 0.2 * g @ g.T / k)
        g = rng.standard_normal((k, k))
        Y.append(np.eye(k) + 0.2 * g @ g.T / k)
    return rng.standard_normal(prob.m) * 0.1, X, Y


CASES = {
    "small_blocks": lambda: G.sdpa_sparse(m=60, blocks=[12, 5, 2], lp=4, seed=3),
    "wide_coefficients": lambda: G.sdpa_sparse(m=90, blocks=[150, 33], lp=0, active=0.7,
                                               pairs=(20, 40), seed=4),
}


@pytest.mark.parametrize("name", list(CASES))
def test_sparse_schur_matches_oracle(cuda, name):
    from oracle.sdpx_oracle import OracleBackend
    from oracle.sparse_oracle import block_coo
    prob = CASES[name]()
    it = _iterate(prob)
    ob = OracleBackend(prob)
    ob.sparse_schur = True
    ob.set_iterate(*it)
    ob.compute_residuals([0.05] * prob.L, False, True)
    ob.schur_build()
    S_ref = ob.schur_matrix()
    active = entries = 0
    for l, k in enumerate(prob.k):
        if k >= 2:
            a, ptr, _, _ = block_coo(prob.Av[l], k)
            active += a.size
            entries += int(ptr[-1])
    with cuda(prob) as be:
        be.set_sparse_schur(True)
        be.set_iterate(*it)
        be.compute_residuals([0.05] * prob.L, False, True)
        be.schur_build()
        S = be.schur_matrix()
        info = be.sparse_schur_info()
        be.schur_build()
        assert np.array_equal(S, be.schur_matrix())        # fixed block order: repeatable
    assert info == dict(active_positions=active, stored_entries=entries)
    assert np.max(np.abs(S - S_ref)) <= 1e-12 * np.max(np.abs(S_ref))
    assert np.array_equal(S, S.T)


def test_sparse_solve_matches_oracle(cuda):
    from oracle.sdpx_oracle import OracleBackend
    from sdpx_b200.driver import solve_with_backend
    prob = G.sdpa_sparse(m=120, blocks=[20, 16, 12, 10], lp=6, active=0.6, seed=3)
    ob = OracleBackend(prob)
    ob.sparse_schur = True
    ref = solve_with_backend(ob, SolverOptions().with_tolerance(1e-8))
    got = solve(prob, tolerance=1e-8, sparse_schur=True)
    dense = solve(prob, tolerance=1e-8)
    assert got.status == ref.status and ref.status.value == "Optimal"
    assert abs(got.iterations - ref.iterations) <= 1
    assert got.pObj == pytest.approx(ref.pObj, rel=1e-7)
    assert got.dObj == pytest.approx(ref.dObj, rel=1e-7)
    assert got.pObj == pytest.approx(dense.pObj, rel=1e-7)


def test_sparse_engine_refuses_large_block(cuda):
    from sdpx_b200.cuda_backend import SDPXB200Error
    prob = G.sdpa_sparse(m=20, blocks=[170], seed=1)
    with cuda(prob) as be:
        with pytest.raises(SDPXB200Error, match="160"):
            be.set_sparse_schur(True)
