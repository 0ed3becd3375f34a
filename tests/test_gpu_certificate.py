"""GPU certificate (`sdpx_b200_certificate`) against the oracle restatement of
`result_certificate` (src/validation.jl:948-1115) on the same iterate.

Validity and failure sets must agree exactly.  Objectives agree to 1e-12
relative.  Residuals and backward errors are sums of roundoff-sized terms whose
summation order differs between the device passes and the oracle, so they are
compared in absolute terms: within 1e-12 of each other, scaled by the data
(backward errors are already relative).
"""
import math

import numpy as np
import pytest

from oracle.certificate_oracle import result_certificate

pytestmark = pytest.mark.gpu

FIELDS_ABS = ("primal_affine_residual", "dual_affine_residual", "primal_block_backward_error",
              "primal_block_strict_backward_error", "dual_backward_error",
              "dual_strict_backward_error")


def _scale(prob, x):
    amax = max(float(np.max(np.abs(A))) for A in prob.Av)
    cmax = max(float(np.max(np.abs(C))) for C in prob.C)
    return 1.0 + cmax + float(np.max(np.abs(prob.c))) + amax * float(np.sum(np.abs(x)))


def _compare(g, o, scale):
    assert g["valid"] == o["valid"], (g["failures"], o["failures"])
    assert sorted(g["failures"]) == sorted(o["failures"])
    assert g["primal_psd_failing_blocks"] == len(o["primal_psd_failing_blocks"])
    assert g["dual_psd_failing_blocks"] == len(o["dual_psd_failing_blocks"])
    for f in ("primal_objective", "dual_objective", "complementarity"):
        assert math.isclose(g[f], o[f], rel_tol=1e-12, abs_tol=1e-12 * scale), (f, g[f], o[f])
    for f in FIELDS_ABS:
        tol = 1e-12 * (scale if "residual" in f and "backward" not in f else 1.0)
        assert abs(g[f] - o[f]) <= tol, (f, g[f], o[f])
    for f in ("primal_cone_violation", "dual_cone_violation"):
        assert math.isclose(g[f], o[f], rel_tol=1e-9, abs_tol=1e-14), (f, g[f], o[f])


@pytest.fixture(scope="module")
def solved():
    from sdpx_b200 import generators as G, solve
    prob = G.sdpa_dense(m=30, blocks=[8, 4, 3, 2], lp=3, seed=4)
    r = solve(prob, tolerance=1e-8, certificate=True)
    return prob, r


def test_certificate_matches_oracle_at_solution(solved):
    prob, r = solved
    o = result_certificate(prob.Av, prob.C, prob.k, prob.c, r.x, r.X, r.Y, 1e-8, 1e-8, 1e-8)
    assert r.certificate["valid"] and o["valid"]
    _compare(r.certificate, o, _scale(prob, r.x))


@pytest.mark.parametrize("shift", [(0, 5.0), (1, 3.0), (2, 0.75), (3, 2.0), (4, 1.5)])
def test_planted_indefinite_block(solved, shift):
    """Blocks of order 8 (unresolved shift), 4 and 3 (bisection), 2 (closed
    form) and a 1×1 block made indefinite."""
    from sdpx_b200 import certificate
    prob, r = solved
    l, s = shift
    X = [B.copy() for B in r.X]
    X[l] = X[l] - s * np.eye(X[l].shape[0])
    g = certificate(prob, type(r)(**{**r.__dict__, "X": X}), eps_primal=1e-8, eps_dual=1e-8,
                    eps_gap=1e-8)
    o = result_certificate(prob.Av, prob.C, prob.k, prob.c, r.x, X, r.Y, 1e-8, 1e-8, 1e-8)
    assert "primal_psd" in g["failures"]
    _compare(g, o, _scale(prob, r.x))


def test_nonfinite_iterate(solved):
    from sdpx_b200 import certificate
    prob, r = solved
    x = r.x.copy()
    x[3] = np.inf
    g = certificate(prob, type(r)(**{**r.__dict__, "x": x}))
    assert not g["valid"] and "nonfinite" in g["failures"]


def test_readme_moment_on_gpu():
    from sdpx_b200 import generators as G, solve
    r = solve(G.readme_moment(), tolerance=1e-8, certificate=True)
    assert r.status.value == "Optimal"
    assert abs(-r.pObj - (math.sqrt(5.0) - 1.0) / 2.0) < 1e-8
    assert r.certificate["valid"], r.certificate["failures"]


# ---- equality rows (n > 0): src/validation.jl:454-482, 629-644, 666-740 ----

@pytest.fixture(scope="module")
def solved_eq():
    from sdpx_b200 import generators as G, solve
    prob = G.sdpa_dense_equalities(m=30, blocks=[8, 4], lp=3, n_eq=4, seed=5)
    r = solve(prob, tolerance=1e-8, certificate=True)
    return prob, r


def _oracle_eq(prob, r, x=None, y=None):
    return result_certificate(prob.Av, prob.C, prob.k, prob.c, r.x if x is None else x, r.X,
                              r.Y, 1e-8, 1e-8, 1e-8, B=prob.B, b=prob.b,
                              y=r.y if y is None else y)


def test_certificate_with_equality_rows(solved_eq):
    prob, r = solved_eq
    o = _oracle_eq(prob, r)
    assert r.status.value == "Optimal"
    assert r.certificate["valid"] and o["valid"], (r.certificate["failures"], o["failures"])
    _compare(r.certificate, o, _scale(prob, r.x))
    assert abs(r.certificate["equality_backward_error"] - o["equality_backward_error"]) <= 1e-12
    assert math.isclose(r.certificate["dual_objective"], o["dual_objective"], rel_tol=1e-12)


def test_certificate_flags_violated_equality(solved_eq):
    """x moved by 1e-4 along B's first column: the equality backward error
    (and the primal residual) fail, and the failure set equals the oracle's."""
    from sdpx_b200 import certificate
    prob, r = solved_eq
    x = r.x + 1e-4 * prob.B[:, 0] / np.linalg.norm(prob.B[:, 0])
    g = certificate(prob, type(r)(**{**r.__dict__, "x": x}), eps_primal=1e-8, eps_dual=1e-8,
                    eps_gap=1e-8)
    o = _oracle_eq(prob, r, x=x)
    assert "equality_backward_error" in o["failures"]
    assert sorted(g["failures"]) == sorted(o["failures"])
    assert abs(g["equality_backward_error"] - o["equality_backward_error"]) <= 1e-12
