"""Mixed-precision path on the GPU.

* The split-BF16 tcgen05 Schur assembly agrees with the FP64 assembly on the
  same iterate to FP32-class accuracy (5e-5 relative to max|S|): three BF16
  planes carry 24 significant bits, products accumulate in FP32, and the
  rounding of the two block products is amplified by |L_X⁻¹||A_i||L_Y|
  relative to |P_i| (measured 1e-6 … 1e-5 on these iterates).
* A full mixed solve reaches the same status as the FP64 device path with
  objectives within 1e-7 relative (the north-star parity criterion).
"""
import numpy as np
import pytest

from sdpx_b200 import SolverOptions, generators as G, solve

pytestmark = pytest.mark.gpu

SPLIT_TOL = 5e-5


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend
    return CudaBackend


def _iterate(prob, seed=5):
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for k in prob.k:
        G1 = rng.standard_normal((k, k))
        G2 = rng.standard_normal((k, k))
        X.append(np.eye(k) + 0.3 * G1 @ G1.T / k)
        Y.append(np.eye(k) + 0.3 * G2 @ G2.T / k)
    return rng.standard_normal(prob.m) * 0.1, X, Y


@pytest.mark.parametrize("m,blocks,lp", [(60, [12, 5, 2], 4), (100, [50], 0), (300, [136, 40], 30)])
def test_split_schur_matches_fp64(cuda, m, blocks, lp):
    prob = G.sdpa_dense(m=m, blocks=blocks, lp=lp, seed=21)
    with cuda(prob) as be:
        x, X, Y = _iterate(prob)
        be.set_iterate(x, X, Y)
        be.compute_residuals([0.1] * prob.L, False, True)
        be.schur_build()
        S64 = be.schur_matrix()
        be._set_mode("mixed")
        be.schur_build()
        Smix = be.schur_matrix()
        be.schur_build()                      # repeatable (planes reused)
        Smix2 = be.schur_matrix()
    scale = np.max(np.abs(S64))
    err = np.max(np.abs(Smix - S64)) / scale
    assert err <= SPLIT_TOL, err
    assert np.array_equal(Smix, Smix2)
    assert np.array_equal(Smix, Smix.T)


def test_mixed_solve_matches_fp64_solve(cuda):
    prob = G.sdpa_dense(m=100, blocks=[50], seed=0)
    r64 = solve(prob, tolerance=1e-8, precision="fp64")
    rmx = solve(prob, tolerance=1e-8, precision="mixed")
    assert rmx.status == r64.status
    assert rmx.pObj == pytest.approx(r64.pObj, rel=1e-7)
    assert rmx.dObj == pytest.approx(r64.dObj, rel=1e-7)
    assert rmx.relative_gap <= 1e-8
    assert "mixed" in rmx.precision_trace


def test_mixed_identity_schur_and_guarded_solve(cuda):
    """The identity-metric S = 𝒜ᵀ𝒜 (KKT cold start) built in mixed mode agrees
    with the FP64 build to the split tolerance, and the guarded solve refined
    against the FP64 operator 𝒜ᵀ𝒜 reaches the FP64 solve's direction."""
    prob = G.sdpa_dense(m=120, blocks=[30, 7, 2], lp=5, seed=8)
    with cuda(prob) as be:
        be.schur_build(identity=True)
        S64 = be.schur_matrix()
        assert be.factorize()["ok"]
        be.set_rhs("cold_dual")
        be.solve_direction()
        dx64 = be.get_direction()[0].copy()
        be._set_mode("mixed")
        be.schur_build(identity=True)
        Smix = be.schur_matrix()
        assert be.factorize()["ok"]
        be.set_rhs("cold_dual")
        be.solve_direction()
        steps, res = be.refine("auto", 0.0, 8, 0)
        dxm = be.get_direction()[0].copy()
        residual, rnorm = be.direction_residual()
        assert be.counters()["operator_applications"] > 0
    scale = np.max(np.abs(S64))
    assert np.max(np.abs(Smix - S64)) / scale <= SPLIT_TOL
    assert residual <= 1e-10 * max(rnorm, 1.0)
    assert np.allclose(dxm, dx64, rtol=1e-9, atol=1e-9 * np.max(np.abs(dx64)))
