"""Adjoint of the solution map on the CPU oracle, pinned by finite differences.

SDPX has no adjoint, so there is no reference gradient: the oracle's adjoint
(`OracleBackend.adjoint`, the implicit-function derivative of the linearised
KKT conditions) is checked against central differences of complete oracle
solves, L(θ + h·δ) − L(θ − h·δ) over 2h with h = 1e-3 and solves to a 1e-10
gap, for every data kind (b, c, C, A_i) and every loss seed (x, y, X, Y).
Tolerance 3% of max(|FD|, |adjoint|, 0.3): the solves stall near a 1e-11 gap,
which puts ≈ 1e-8/h of noise on each difference.
"""
import numpy as np
import pytest

from oracle.sdpx_oracle import OracleBackend, oracle_solve
from sdpx_b200 import SolverOptions, generators as G
from sdpx_b200.problem import SDPProblem

H = 1e-3


def _solve(prob, tol=1e-10):
    return oracle_solve(prob, SolverOptions().with_tolerance(tol))


def _sym(rng, k):
    M = rng.standard_normal((k, k))
    return M + M.T


def _close(a, f):
    return abs(a - f) <= 0.03 * max(abs(f), abs(a), 0.3)


@pytest.mark.parametrize("n_eq", [0, 2])
def test_adjoint_matches_finite_differences(n_eq):
    if n_eq:
        prob = G.sdpa_dense_equalities(m=12, blocks=[5, 3], lp=2, n_eq=n_eq, seed=1)
    else:
        prob = G.sdpa_dense(m=12, blocks=[5, 3], lp=2, seed=1)
    rng = np.random.default_rng(0)
    wx = rng.standard_normal(prob.m)
    wy = rng.standard_normal(prob.n)
    WX = [_sym(rng, k) for k in prob.k]
    WY = [_sym(rng, k) for k in prob.k]

    def loss(r):
        return (wx @ r.x + (wy @ r.y if prob.n else 0.0)
                + sum(float(np.sum(a * b)) for a, b in zip(WX, r.X))
                + sum(float(np.sum(a * b)) for a, b in zip(WY, r.Y)))

    r0 = _solve(prob, 1e-9)
    be = OracleBackend(prob)
    be.set_iterate(r0.x, r0.X, r0.Y, y=r0.y)
    be.compute_residuals([0.0] * prob.L, True, True)
    be.schur_build()
    assert be.factorize()["ok"]
    g = be.adjoint(wx, wy if prob.n else None, WX, WY, A_index=(3,))

    def fd(make):
        return (loss(_solve(make(H))) - loss(_solve(make(-H)))) / (2 * H)

    E = _sym(rng, prob.k[0])
    dc = rng.standard_normal(prob.m)
    checks = [
        (g["grad_c"] @ dc,
         fd(lambda h: SDPProblem(prob.c + h * dc, prob.k, prob.Av, prob.C, prob.B, prob.b))),
        (float(np.sum(g["grad_C"][0] * E)),
         fd(lambda h: SDPProblem(prob.c, prob.k, prob.Av, [prob.C[0] + h * E] + prob.C[1:],
                                 prob.B, prob.b))),
    ]

    def moved_A(h):
        Av = [a.copy() for a in prob.Av]
        Av[0][3] += h * E.reshape(-1)
        return SDPProblem(prob.c, prob.k, Av, prob.C, prob.B, prob.b)

    checks.append((float(np.sum(g["grad_A"][0][0] * E)), fd(moved_A)))
    if prob.n:
        db = rng.standard_normal(prob.n)
        checks.append((g["grad_b"] @ db,
                       fd(lambda h: SDPProblem(prob.c, prob.k, prob.Av, prob.C, prob.B,
                                               prob.b + h * db))))
    for a, f in checks:
        assert _close(a, f), (a, f)


def test_adjoint_a_gradient_identity():
    """∂L/∂A_i = λx_i·Y − x_i·∂L/∂C block by block."""
    prob = G.sdpa_dense(m=10, blocks=[4], lp=1, seed=2)
    r = _solve(prob, 1e-9)
    be = OracleBackend(prob)
    be.set_iterate(r.x, r.X, r.Y)
    be.compute_residuals([0.0] * prob.L, True, True)
    be.schur_build()
    be.factorize()
    g = be.adjoint(wx=np.ones(prob.m), A_index=(0, 5))
    for q, i in enumerate((0, 5)):
        for l in range(prob.L):
            expect = g["lambda_x"][i] * r.Y[l] - r.x[i] * g["grad_C"][l]
            assert np.allclose(g["grad_A"][q][l], expect, rtol=1e-12, atol=1e-14)
