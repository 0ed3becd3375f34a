"""Sparse Schur oracle (SDPX's SparseCons path) against the dense oracle.

* `block_coo` keeps exactly the stored entries: active variables ascending,
  each coefficient's entries in increasing column-major linear index, and the
  dense coefficients are rebuilt from them.
* On an interior iterate the sparse assembly ⟨Y·A_p·X⁻¹, A_r⟩ over the active
  pairs equals the dense assembly P̂ᵀP̂ (src/schur.jl:511-562) to 1e-13
  relative, 2×2 and 1×1 blocks included.
* A complete solve with the sparse path reaches the dense solve's status,
  iteration count and objective (1e-10 relative).
"""
import numpy as np

from oracle.sdpx_oracle import OracleBackend, oracle_solve
from oracle.sparse_oracle import block_coo
from sdpx_b200 import SolverOptions, generators as G
from sdpx_b200.driver import solve_with_backend


def _iterate(prob, seed=1):
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for k in prob.k:
        g = rng.standard_normal((k, k))
        X.append(np.eye(k) + 0.2 * g @ g.T / k)
        g = rng.standard_normal((k, k))
        Y.append(np.eye(k) + 0.2 * g @ g.T / k)
    return rng.standard_normal(prob.m) * 0.1, X, Y


def test_block_coo_keeps_stored_entries_in_order():
    prob = G.sdpa_sparse(m=40, blocks=[9, 4], seed=2)
    for l, k in enumerate(prob.k):
        active, ptr, lin, val = block_coo(prob.Av[l], k)
        assert np.all(np.diff(active) > 0)
        rebuilt = np.zeros_like(prob.Av[l])
        for p, i in enumerate(active):
            seg = lin[ptr[p]:ptr[p + 1]]
            assert np.all(np.diff(seg) > 0)
            rebuilt[i, seg] = val[ptr[p]:ptr[p + 1]]
        assert np.array_equal(rebuilt, prob.Av[l])


def test_sparse_schur_equals_dense_schur():
    prob = G.sdpa_sparse(m=60, blocks=[12, 5, 2], lp=4, seed=3)
    ob = OracleBackend(prob)
    ob.set_iterate(*_iterate(prob))
    ob.compute_residuals([0.05] * prob.L, False, True)
    dense = ob.schur_build().copy()
    ob.sparse_schur = True
    sparse = ob.schur_build().copy()
    assert np.max(np.abs(sparse - dense)) <= 1e-13 * np.max(np.abs(dense))


def test_sparse_solve_matches_dense_solve():
    prob = G.sdpa_sparse(m=120, blocks=[20, 16, 12, 10], lp=6, active=0.6, seed=3)
    opts = SolverOptions().with_tolerance(1e-8)
    rd = oracle_solve(prob, opts)
    ob = OracleBackend(prob)
    ob.sparse_schur = True
    rs = solve_with_backend(ob, opts)
    assert rd.status.value == "Optimal" and rs.status == rd.status
    assert rs.iterations == rd.iterations
    assert abs(rs.pObj - rd.pObj) <= 1e-10 * max(1.0, abs(rd.pObj))
