"""GPU parity of the LP/SOC reduced normal system against the oracle.

* NT scaling (w, λ, η, η²), the NT maps W, W⁻¹, Hs⁻¹ and the LP pack are
  compared BIT-FOR-BIT with the oracle's sequential IEEE restatement of
  src/soc_lorentz_kernels.jl:21-255 and src/lp_solver.jl:1892-1915 (the device
  code evaluates the same recurrences with FMA contraction off).
* The normal matrix Q = Bᵀ D⁻¹ B + δI is a tensor-core SYRK of the W⁻¹-scaled
  operand, the oracle forms A·M·Aᵀ with the dense per-cone metric as
  src/soc_native.jl:1192-1216 does; the two round differently, so entries are
  compared against the standard forward-error bound
  |ΔQ_ij| ≤ 256·eps·(|B|ᵀ|M||B|)_ij, M = blockdiag(|D⁻¹|, |Hs_k⁻¹|).
* Directions from the Cholesky solve satisfy the reduced KKT system and agree
  with the oracle's to a condition-scaled tolerance.
"""
import numpy as np
import pytest

from oracle import cone_oracle as O

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def N():
    from sdpx_b200 import normal
    return normal


def _interior(rng, q, spread=1.5):
    u = rng.standard_normal(q - 1)
    return np.concatenate([[spread * np.linalg.norm(u) + 1.0], u])


def _cones(dims, seed):
    rng = np.random.default_rng(seed)
    s = np.concatenate([_interior(rng, q) for q in dims])
    z = np.concatenate([_interior(rng, q) for q in dims])
    return s, z


def _oracle_scalings(dims, s, z):
    out, o = [], 0
    for q in dims:
        out.append(O.nt_scaling(list(s[o:o + q]), list(z[o:o + q])))
        o += q
    return out


def _bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


def test_nt_scaling_bit_exact(N):
    dims = [1, 2, 3, 5, 8, 64, 200]
    s, z = _cones(dims, 11)
    # the reference's own roundtrip vectors (test/soc_native_algebra.jl:61-87)
    dims += [3, 2, 3, 5]
    s = np.concatenate([s, [3.0, 0.3, -0.2], [3.0, 0.15], [3.0, 0.15, 0.15], [3.0] + [0.15] * 4])
    z = np.concatenate([z, [2.5, -0.1, 0.25], [2.0, -0.1], [2.0, -0.1, -0.1], [2.0] + [-0.1] * 4])
    B = np.zeros((sum(dims), 1))
    with N.NormalSystem(B, 0, dims) as ns:
        ok, first_bad, out = ns.soc_nt_scaling(s, z)
    assert ok and first_bad == -1
    ref = _oracle_scalings(dims, s, z)
    w = np.concatenate([r[1] for r in ref])
    lam = np.concatenate([r[2] for r in ref])
    assert np.array_equal(_bits(out["w"]), _bits(w))
    assert np.array_equal(_bits(out["lambda"]), _bits(lam))
    assert np.array_equal(_bits(out["eta"]), _bits([r[3] for r in ref]))
    assert np.array_equal(_bits(out["eta_squared"]), _bits([r[4] for r in ref]))


def test_nt_scaling_failures_flagged(N):
    dims = [3, 3, 3, 3, 2]
    s = np.array([2.0, 0.1, 0.1, 1.0, 1.0, 0.0, 2.0, 0.1, 0.1, 2.0, np.nan, 0.0, 1.0, 0.5])
    z = np.array([2.0, 0.1, 0.1, 2.0, 0.1, 0.1, 0.0, 0.0, 0.0, 2.0, 0.1, 0.1, 1.0, -0.5])
    B = np.zeros((sum(dims), 2))
    with N.NormalSystem(B, 0, dims) as ns:
        ok, first_bad, out = ns.soc_nt_scaling(s, z)
        assert not ok and first_bad == 1
        # boundary slack, zero dual, non-finite slack fail; interior ones succeed
        assert out["ok"].tolist() == [True, False, False, False, True]
        ref = _oracle_scalings(dims, s, z)
        assert [r[0] for r in ref] == out["ok"].tolist()
        assert out["eta"][1] == 0.0 and out["eta_squared"][2] == 0.0
        # no valid scaling is held: the assembly refuses
        with pytest.raises(N.SDPXB200Error):
            ns.assemble_reduced_schur(np.zeros(0), 0.0)


def test_nt_maps_bit_exact_and_roundtrip(N):
    dims = [2, 3, 5, 17, 64]
    s, z = _cones(dims, 4)
    v = np.random.default_rng(9).standard_normal(sum(dims))
    with N.NormalSystem(np.zeros((sum(dims), 1)), 0, dims) as ns:
        assert ns.soc_nt_scaling(s, z)[0]
        got = [ns.soc_nt_apply_w(v), ns.soc_nt_apply_winv(v), ns.soc_nt_apply_hs_inverse(v)]
        back = ns.soc_nt_apply_winv(ns.soc_nt_apply_w(v))
    ref = _oracle_scalings(dims, s, z)
    exp = [[], [], []]
    o = 0
    for q, (_, w, _, eta, eta2) in zip(dims, ref):
        seg = v[o:o + q]
        exp[0].append(O.apply_w(w, eta, seg))
        exp[1].append(O.apply_winv(w, eta, seg))
        exp[2].append(O.apply_hs_inverse(w, eta2, seg))
        o += q
    for g, e in zip(got, exp):
        assert np.array_equal(_bits(g), _bits(np.concatenate(e)))
    assert np.allclose(back, v, rtol=1e-11, atol=1e-11)


def test_lp_pack_bit_exact(N):
    rng = np.random.default_rng(2)
    n_lp, nw = 300, 120
    rows = rng.integers(0, nw, n_lp)
    coef = rng.choice([1.0, -1.0, 0.5, 3.0], n_lp)
    weights = rng.uniform(0.01, 100.0, nw)
    B = rng.standard_normal((n_lp, 7))
    with N.NormalSystem(B, n_lp, row_for_variable=rows, diagonal_coefficient=coef,
                        n_weights=nw) as ns:
        D, Di, Ds = ns.lp_standard_pack(weights, 1e-9)
    eD, eDi, eDs = O.lp_pack(weights, rows, coef, 1e-9)
    for a, b in ((D, eD), (Di, eDi), (Ds, eDs)):
        assert np.array_equal(_bits(a), _bits(b))


def _system(m, n_lp, dims, density, seed):
    A, xl, zl, sc, zc = O.random_lp_soc(m, n_lp, dims, density=density, seed=seed)
    s = np.concatenate(sc) if dims else np.zeros(0)
    z = np.concatenate(zc) if dims else np.zeros(0)
    return A.T.copy(), zl / xl, s, z  # B = Aᵀ (variables × equalities)


def _bound(B, n_lp, dims, Dinv, ref):
    """|B|ᵀ M |B| with M = blockdiag(|D⁻¹|, |W_k⁻¹|ᵀ|W_k⁻¹|).  |W⁻¹|ᵀ|W⁻¹| ≥ |Hs⁻¹|
    entrywise, so this bounds the rounding of both the scaled-operand SYRK and
    the oracle's dense-metric product."""
    absB = np.abs(B)
    MB = np.empty_like(absB)
    MB[:n_lp] = np.abs(Dinv)[:, None] * absB[:n_lp]
    o = n_lp
    for q, r in zip(dims, ref):
        Winv = np.abs(np.column_stack([O.apply_winv(r[1], r[3], e) for e in np.eye(q)]))
        MB[o:o + q] = (Winv.T @ Winv) @ absB[o:o + q]
        o += q
    return absB.T @ MB


@pytest.mark.parametrize("m,n_lp,dims,density", [
    (40, 90, [3, 5, 8], 0.4),          # small mixed system
    (130, 0, [64] * 6, 0.3),           # cones only
    (257, 800, [], 0.1),               # LP only, m not a tile multiple
    (600, 4000, [64] * 20, 0.1),       # the 10%-dense LP+SOC shape, reduced
])
def test_normal_matrix_and_solve_match_oracle(N, m, n_lp, dims, density):
    B, weights, s, z = _system(m, n_lp, dims, density, seed=m)
    reg = 1e-9
    with N.NormalSystem(B, n_lp, dims) as ns:
        if dims:
            assert ns.soc_nt_scaling(s, z)[0]
        Q = ns.assemble_reduced_schur(weights, reg)
        ok, att, used = ns.factor_reduced(weights, reg)
        assert ok and att == 1 and used == reg
        L = ns.matrix(1)
        rng = np.random.default_rng(m + 1)
        rhs = rng.standard_normal(B.shape[0] + m)
        sol = ns.solve_factor(rhs)
    ref = _oracle_scalings(dims, s, z)
    _, Dinv, _ = O.lp_pack(weights, np.arange(n_lp), np.ones(n_lp), reg)
    scal = [(r[1], r[3], r[4]) for r in ref]
    Qo = O.normal_matrix(B.T, n_lp, dims, Dinv, scal, reg)
    bound = 256 * EPS * _bound(B, n_lp, dims, Dinv, ref)
    assert np.all(np.abs(Q - Qo) <= bound + 1e-300), float(np.max(np.abs(Q - Qo) / (bound + 1e-300)))
    assert np.allclose(np.tril(L) @ np.tril(L).T, Q, rtol=0, atol=1e-12 * np.abs(Q).max())
    dx_o, dy_o = O.recover(B.T, n_lp, dims, Dinv, scal, Qo, rhs[:B.shape[0]], rhs[B.shape[0]:])
    cond = np.linalg.cond(Qo)
    tol = max(1e-11, 64 * EPS * cond)
    dx, dy = sol[:B.shape[0]], sol[B.shape[0]:]
    assert np.linalg.norm(dy - dy_o) <= tol * np.linalg.norm(dy_o)
    assert np.linalg.norm(dx - dx_o) <= tol * max(np.linalg.norm(dx_o), 1.0)
    # equality rows of the regularized reduced KKT system: Bᵀdx + δ·dy = ry
    assert np.allclose(B.T @ dx + reg * dy, rhs[B.shape[0]:], atol=1e-8 * np.linalg.norm(rhs))


def test_regularization_retries(N):
    # more equalities than variables: BᵀD⁻¹B is rank deficient, so a tiny δ
    # leaves roundoff-sized pivots and the ×10 retry loop has to raise it.
    rng = np.random.default_rng(7)
    n_lp, m = 40, 120
    B = rng.standard_normal((n_lp, m))
    w = rng.uniform(0.5, 2.0, n_lp)
    with N.NormalSystem(B, n_lp) as ns:
        ok, att, used = ns.factor_reduced(w, 1e-16, max_attempts=8)
        assert ok and 2 <= att <= 8
        r = 1e-16
        for _ in range(att - 1):
            r *= 10.0
        assert used == r
        ok, att, used = ns.factor_reduced(w, 1e-40, max_attempts=2)
        assert not ok and att == 2
        with pytest.raises(N.PosDefError):
            ns.solve_factor(np.zeros(n_lp + m))


def test_no_equalities(N):
    dims = [4]
    n_lp = 5
    B = np.zeros((n_lp + 4, 0))
    s, z = _cones(dims, 1)
    w = np.linspace(1.0, 2.0, n_lp)
    with N.NormalSystem(B, n_lp, dims) as ns:
        assert ns.soc_nt_scaling(s, z)[0]
        ok, att, _ = ns.factor_reduced(w, 0.0)
        assert ok and att == 1
        rx = np.arange(1.0, 10.0)
        dx = ns.solve_factor(rx)
        hs = ns.soc_nt_apply_hs_inverse(rx[n_lp:])
    assert np.array_equal(dx[:n_lp], (1.0 / w) * rx[:n_lp])
    assert np.array_equal(dx[n_lp:], hs)
