"""CPU checks of the certificate oracle (restatement of `result_certificate`,
src/validation.jl:948-1115) on the reference's own known answers:

* README quick start (README.md:44-75): W2 = (√5 − 1)/2 ≈ 0.618034 and
  `certificate(result).valid == true`;
* the `sdp_closed_form` gate (benchmark/gates.jl:118-140): valid certificate;
* planted defects (an indefinite X block, a non-finite x) make it invalid with
  the reference's failure symbols.
"""
import math

import numpy as np

from oracle.certificate_oracle import block_psd_certificate, result_certificate
from oracle.sdpx_oracle import oracle_solve
from sdpx_b200 import SolverOptions, generators as G


def _cert(prob, r, tol=1e-10):
    return result_certificate(prob.Av, prob.C, prob.k, prob.c, r.x, r.X, r.Y, tol, tol, tol)


def test_readme_moment_known_answer():
    prob = G.readme_moment()
    r = oracle_solve(prob, SolverOptions().with_tolerance(1e-8))
    assert r.status.value == "Optimal"
    assert abs(-r.pObj - (math.sqrt(5.0) - 1.0) / 2.0) < 1e-8
    cert = _cert(prob, r, 1e-8)
    assert cert["valid"], cert["failures"]


def test_closed_form_gate_certificate_valid():
    prob = G.gate_closed_form()
    r = oracle_solve(prob, SolverOptions())
    cert = _cert(prob, r)
    assert cert["valid"], cert["failures"]
    assert abs(cert["primal_objective"] - 2 * math.sqrt(6.0)) < 1e-8


def test_planted_defects():
    prob = G.gate_closed_form()
    r = oracle_solve(prob, SolverOptions())
    X = [B.copy() for B in r.X]
    X[0] = X[0] - 3.0 * np.eye(X[0].shape[0])
    cert = result_certificate(prob.Av, prob.C, prob.k, prob.c, r.x, X, r.Y)
    assert not cert["valid"]
    assert "primal_psd" in cert["failures"] and "primal_residual" in cert["failures"]
    x = r.x.copy()
    x[0] = np.nan
    cert = result_certificate(prob.Av, prob.C, prob.k, prob.c, x, r.X, r.Y)
    assert "nonfinite" in cert["failures"]


def test_block_psd_shift_resolution():
    # order 3: the bisection resolves the required shift to the smallest eigenvalue
    M = np.diag([1.0, 2.0, -0.25])
    d = block_psd_certificate(M, 1e-10)
    assert not d["ok"] and d["resolved"] and abs(d["required"] - 0.25) < 1e-12
    # order 2: closed form
    d = block_psd_certificate(np.array([[1.0, 2.0], [2.0, 1.0]]), 1e-10)
    assert not d["ok"] and abs(d["required"] - 1.0) < 1e-15
    # order 6: unresolved, reported at the allowed shift
    d = block_psd_certificate(np.diag([1.0] * 5 + [-1.0]), 1e-10)
    assert not d["ok"] and not d["resolved"] and d["required"] == d["allowed"]


def test_equality_rows_certificate_t2():
    """T2 (test/correctness.jl:97-122) solved by the oracle: its certificate
    with the equality row is valid; moving x₁ off the row fails it with the
    equality backward error."""
    from oracle.sdpx_oracle import oracle_solve
    from sdpx_b200 import SolverOptions, generators as G
    prob = G.toy_t2()
    r = oracle_solve(prob, SolverOptions().with_tolerance(1e-8))
    c = result_certificate(prob.Av, prob.C, prob.k, prob.c, r.x, r.X, r.Y, 1e-8, 1e-8, 1e-8,
                           B=prob.B, b=prob.b, y=r.y)
    assert c["valid"], c["failures"]
    assert abs(c["dual_objective"] - 5.5) < 1e-7
    x = r.x.copy()
    x[0] += 1e-3
    bad = result_certificate(prob.Av, prob.C, prob.k, prob.c, x, r.X, r.Y, 1e-8, 1e-8, 1e-8,
                             B=prob.B, b=prob.b, y=r.y)
    assert "equality_backward_error" in bad["failures"]
    assert bad["equality_backward_error"] > 1e-5
