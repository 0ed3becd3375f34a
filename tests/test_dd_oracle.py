"""Double-double (Float64x2) oracle and the adjoint's exact derivative.

* The error-free transformations are exact: TwoSum and TwoProduct against
  rational arithmetic, double-double division to 1e-30.
* The adjoint (`OracleBackend.adjoint`, the implicit-function derivative of the
  HKM-linearised KKT conditions) is the exact derivative of the central-path
  point at fixed μ: on that path X·Y = μI, so dY = −X⁻¹·dX·Y is already
  symmetric.  Central points are computed by Newton steps at fixed μ to a
  scaled residual ≤ 1e-13 for data θ ± h·δ (h = 1e-6); the central difference of
  L = ⟨wx, x⟩ + Σ⟨WX, X⟩ + Σ⟨WY, Y⟩ must match the double-double adjoint
  (`dd_adjoint`) at the unperturbed central point to 1e-6 relative for every
  data kind (c, C, A_i), each loss seed alone and all together; the float64
  oracle adjoint matches the double-double one to 1e-10 there.
"""
from fractions import Fraction

import numpy as np
import pytest

from oracle.dd_oracle import DD, central_point, dd_adjoint, two_prod, two_sum
from oracle.sdpx_oracle import OracleBackend, oracle_solve
from sdpx_b200 import SolverOptions, generators as G
from sdpx_b200.problem import SDPProblem

H = 1e-6
MU = 1e-3
FD_TOL = 1e-6


def test_error_free_transformations_are_exact():
    rng = np.random.default_rng(0)
    a = rng.standard_normal(300) * 10.0 ** rng.uniform(-8, 8, 300)
    b = rng.standard_normal(300) * 10.0 ** rng.uniform(-8, 8, 300)
    p, e = two_prod(a, b)
    s, f = two_sum(a, b)
    for i in range(300):
        A, B = Fraction(float(a[i])), Fraction(float(b[i]))
        assert Fraction(float(p[i])) + Fraction(float(e[i])) == A * B
        assert Fraction(float(s[i])) + Fraction(float(f[i])) == A + B
    q = (DD(a) * DD(b) + DD(a)) / DD(b)
    for i in range(0, 300, 37):
        num = (Fraction(float(a[i])) * Fraction(float(b[i])) + Fraction(float(a[i])))
        exact = num / Fraction(float(b[i]))
        got = Fraction(float(q.hi[i])) + Fraction(float(q.lo[i]))
        assert abs(float((got - exact) / exact)) <= 1e-30


def _sym(rng, k):
    M = rng.standard_normal((k, k))
    return M + M.T


@pytest.fixture(scope="module")
def central():
    prob = G.sdpa_dense(m=12, blocks=[5, 3], lp=2, seed=1)
    r = oracle_solve(prob, SolverOptions().with_tolerance(1e-4))
    x, X, Y, res = central_point(prob, MU, (r.x, r.X, r.Y))
    assert res <= 1e-14
    return prob, (x, X, Y)


@pytest.mark.parametrize("seed_kind", ["x", "X", "Y", "all"])
def test_adjoint_is_the_central_path_derivative(central, seed_kind):
    prob, (x, X, Y) = central
    rng = np.random.default_rng({"x": 1, "X": 2, "Y": 3, "all": 4}[seed_kind])
    wx = rng.standard_normal(prob.m) if seed_kind in ("x", "all") else None
    WX = [_sym(rng, k) for k in prob.k] if seed_kind in ("X", "all") else None
    WY = [_sym(rng, k) for k in prob.k] if seed_kind in ("Y", "all") else None

    def loss(x_, X_, Y_):
        v = 0.0 if wx is None else float(wx @ x_)
        if WX is not None:
            v += sum(float(np.sum(a * b)) for a, b in zip(WX, X_))
        if WY is not None:
            v += sum(float(np.sum(a * b)) for a, b in zip(WY, Y_))
        return v

    gd = dd_adjoint(prob, x, X, Y, wx, WX, WY, A_index=(3,))
    ob = OracleBackend(prob)
    ob.set_iterate(x, X, Y)
    ob.compute_residuals([0.0] * prob.L, True, True)
    ob.schur_build()
    assert ob.factorize()["ok"]
    go = ob.adjoint(wx, None, WX, WY, A_index=(3,))
    scale = max(1.0, float(np.max(np.abs(gd["grad_c"]))))
    assert np.max(np.abs(go["grad_c"] - gd["grad_c"])) <= 1e-10 * scale

    def fd(make):
        vals = []
        for s in (H, -H):
            q = make(s)
            xx, XX, YY, res = central_point(q, MU, (x, X, Y))
            assert res <= 1e-13             # difference noise ≤ 1e-13 / h = 1e-7
            vals.append(loss(xx, XX, YY))
        return (vals[0] - vals[1]) / (2 * H)

    E = _sym(rng, prob.k[0])
    dc = rng.standard_normal(prob.m)

    def moved_A(t):
        Av = [a.copy() for a in prob.Av]
        Av[0][3] += t * E.reshape(-1)
        return SDPProblem(prob.c, prob.k, Av, prob.C, prob.B, prob.b)

    checks = [
        (float(gd["grad_c"] @ dc),
         fd(lambda t: SDPProblem(prob.c + t * dc, prob.k, prob.Av, prob.C, prob.B, prob.b))),
        (float(np.sum(gd["grad_C"][0] * E)),
         fd(lambda t: SDPProblem(prob.c, prob.k, prob.Av, [prob.C[0] + t * E] + prob.C[1:],
                                 prob.B, prob.b))),
        (float(np.sum(gd["grad_A"][0][0] * E)), fd(moved_A)),
    ]
    for ad, f in checks:
        assert abs(ad - f) <= FD_TOL * max(abs(f), 1.0), (seed_kind, ad, f)
