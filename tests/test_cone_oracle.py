"""CPU checks of the LP/SOC oracle against the reference's own identities.

* NT scaling roundtrip W⁻¹(W v) = v for Lorentz dimensions 2, 3, 5 with the
  reference's vectors (test/soc_native_algebra.jl:61-87), and the defining
  Nesterov–Todd properties W z = W⁻¹ s = λ and Hs⁻¹ = (WᵀW)⁻¹.
* The signed rank-one (SYRK) form of each cone's metric equals the dense
  Hs⁻¹ assembled column by column as in src/soc_native.jl:1192-1201.
* The LP pack follows src/lp_solver.jl:1892-1915 and the recovered direction
  solves the reduced KKT system.
"""
import math

import numpy as np
import pytest

from oracle import cone_oracle as O


def test_reference_nt_roundtrip():
    ok, w, lam, eta, eta2 = O.nt_scaling([3.0, 0.3, -0.2], [2.5, -0.1, 0.25])
    assert ok
    for dim in (2, 3, 5):
        s = [3.0] + [0.15] * (dim - 1)
        z = [2.0] + [-0.1] * (dim - 1)
        ok, w, lam, eta, _ = O.nt_scaling(s, z)
        assert ok
        src = np.linspace(0.1, 0.1 * dim, dim)
        back = O.apply_winv(w, eta, O.apply_w(w, eta, src))
        assert np.allclose(back, src, atol=1e-11, rtol=1e-11)


@pytest.mark.parametrize("dim", [2, 3, 8, 64])
def test_nt_properties(dim):
    rng = np.random.default_rng(dim)
    u = rng.standard_normal(dim - 1)
    s = np.concatenate([[1.5 * np.linalg.norm(u) + 1.0], u])
    u = rng.standard_normal(dim - 1)
    z = np.concatenate([[1.5 * np.linalg.norm(u) + 1.0], u])
    ok, w, lam, eta, eta2 = O.nt_scaling(s, z)
    assert ok
    assert abs(w[0] ** 2 - np.dot(w[1:], w[1:]) - 1.0) < 1e-12
    Wz = O.apply_w(w, eta, z)
    Winv_s = O.apply_winv(w, eta, s)
    assert np.allclose(Wz, lam, rtol=1e-12, atol=1e-12)
    assert np.allclose(Winv_s, lam, rtol=1e-12, atol=1e-12)
    W = np.column_stack([O.apply_w(w, eta, e) for e in np.eye(dim)])
    assert np.allclose(W, W.T, atol=1e-12)
    Hinv = O.hs_inverse_matrix(w, eta2)
    assert np.allclose(Hinv @ (W.T @ W), np.eye(dim), atol=1e-10)


def test_signed_rank_one_metric_matches_dense():
    rng = np.random.default_rng(3)
    m, q = 20, 9
    A = rng.standard_normal((m, q))
    u = rng.standard_normal(q - 1)
    s = np.concatenate([[1.5 * np.linalg.norm(u) + 1.0], u])
    u = rng.standard_normal(q - 1)
    z = np.concatenate([[1.5 * np.linalg.norm(u) + 1.0], u])
    ok, w, lam, eta, eta2 = O.nt_scaling(s, z)
    dense = A @ O.hs_inverse_matrix(w, eta2) @ A.T
    J = np.diag([1.0] + [-1.0] * (q - 1))
    uvec = A @ (J @ w)
    signed = (2 * np.outer(uvec, uvec) - np.outer(A[:, 0], A[:, 0]) + A[:, 1:] @ A[:, 1:].T) / eta2
    assert np.allclose(signed, dense, rtol=1e-11, atol=1e-11)


def test_lp_pack_and_recovery_solve_reduced_kkt():
    m, n_lp, cones = 30, 50, [4, 6]
    A, xl, zl, sc, zc = O.random_lp_soc(m, n_lp, cones, density=0.4, seed=5)
    weights = zl / xl
    rows = np.arange(n_lp)
    D, Dinv, Dis = O.lp_pack(weights, rows, np.ones(n_lp), 1e-9)
    assert np.allclose(D, weights + 1e-9) and np.allclose(Dis, np.sqrt(1.0 / D))
    scal = []
    for s, z in zip(sc, zc):
        ok, w, lam, eta, eta2 = O.nt_scaling(s, z)
        assert ok
        scal.append((w, eta, eta2))
    M = O.normal_matrix(A, n_lp, cones, Dinv, scal, 1e-9)
    rng = np.random.default_rng(1)
    rx = rng.standard_normal(A.shape[1])
    ry = rng.standard_normal(m)
    dx, dy = O.recover(A, n_lp, cones, Dinv, scal, M - 1e-9 * np.eye(m), rx, ry)
    # [H  -Aᵀ; A  0][dx; dy] = [rx; ry] with H = blockdiag(D, Hs)
    Hdx = np.empty_like(dx)
    Hdx[:n_lp] = D * dx[:n_lp]
    o = n_lp
    for q, (w, eta, eta2) in zip(cones, scal):
        Hs = np.linalg.inv(O.hs_inverse_matrix(w, eta2))
        Hdx[o:o + q] = Hs @ dx[o:o + q]
        o += q
    assert np.allclose(Hdx - A.T @ dy, rx, atol=1e-8)
    assert np.allclose(A @ dx, ry, atol=1e-8)
