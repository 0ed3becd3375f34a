"""The two FP64 Schur engines on the same iterate.

The FP64 Schur assembly (Gram S = P̂ᵀP̂ and block products T = L_X⁻¹·A_i,
P_i = T·L_Y) runs either on the FP64 DMMA tiles or, by default, as exact int8
digit products.  Both must reproduce the oracle's Schur matrix (the reference's
`schur_build!`, src/schur.jl:511-562) to the FP64 parity bound, agree with each
other, and the digit engine must repeat bit for bit (its integer levels carry no
rounding; only the fixed-order FP64 level sums round).
"""
import numpy as np
import pytest

from sdpx_b200 import generators as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend
    return CudaBackend


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1.0, float(np.max(np.abs(b)))))


def interior_iterate(prob, seed=5):
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for k in prob.k:
        G1 = rng.standard_normal((k, k))
        G2 = rng.standard_normal((k, k))
        X.append(np.eye(k) + 0.3 * G1 @ G1.T / k)
        Y.append(np.eye(k) + 0.3 * G2 @ G2.T / k)
    return rng.standard_normal(prob.m) * 0.1, X, Y


@pytest.mark.parametrize("build", [
    lambda: G.sdpa_dense(m=60, blocks=[12, 5, 2], lp=4, seed=11),
    lambda: G.sdpa_dense(m=150, blocks=[70, 33], lp=9, seed=2),
])
def test_fp64_engines_agree_with_oracle(cuda, build):
    from oracle.sdpx_oracle import OracleBackend
    prob = build()
    ob = OracleBackend(prob)
    x, X, Y = interior_iterate(prob)
    ob.set_iterate(x, X, Y)
    ob.compute_residuals([0.05] * prob.L, False, True)
    ob.schur_build()
    S_o = ob.schur_matrix()
    with cuda(prob) as cb:
        cb.set_iterate(x, X, Y)
        cb.compute_residuals([0.05] * prob.L, False, True)
        cb.set_gram_engine("dmma")
        cb.schur_build()
        S_d = cb.schur_matrix()
        cb.set_gram_engine("int8")
        cb.schur_build()
        S_i = cb.schur_matrix()
        cb.schur_build()
        S_i2 = cb.schur_matrix()
    assert rel(S_d, S_o) <= 1e-12
    assert rel(S_i, S_o) <= 1e-12
    assert rel(S_i, S_d) <= 1e-12
    assert np.array_equal(S_i, S_i2)
