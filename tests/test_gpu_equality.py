"""Equality rows (n > 0) on the B200 against the oracle.

The device restates SDPX's n > 0 KKT route (src/kkt.jl:1466-1680 factor,
:2570-2595 solve): B̃ = L_S⁻¹B with unit ∞-norm columns, Q = B̃ᵀB̃ by Cholesky
with the diagonal rank test, the column-pivoted QR of B̃ when that test fails.
Pins: T2 / T3 of test/correctness.jl:97-135 (optimum 11/2, T2's fixed-policy
iteration count 15 ± 2, T3 on the rank-revealing QR with rank 1) and the
README moment SDP with its two equality rows; kernel-level parity of the
directions (dx, dy) with the oracle on full-rank and rank-deficient blocks.
FP64 tolerance: 1e-9 relative on directions, 1e-7 on objectives.
"""
import json
import math
import os

import numpy as np
import pytest

from sdpx_b200 import SolverOptions, generators as G
from sdpx_b200.driver import solve_with_backend

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "gates.json")))


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend
    return CudaBackend


def _fixed():
    return SolverOptions(parameter_policy="fixed", parameter_strategy="fixed", scaling="none")


def _dual_residual(prob, r):
    d = prob.c.copy()
    for l in range(prob.L):
        d -= prob.Av[l] @ r.Y[l].reshape(-1)
    return float(np.max(np.abs(d - prob.B @ r.y)))


def test_t2_fixed_policy(cuda):
    from oracle.sdpx_oracle import oracle_solve
    pin = GOLD["T2_fixed_policy"]
    prob = G.toy_t2()
    with cuda(prob) as be:
        r = solve_with_backend(be, _fixed())
        kind, rank, _ = be.equality_info()
    ro = oracle_solve(prob, _fixed())
    assert r.status.value == "Optimal"
    assert abs(r.iterations - pin["iterations"]) <= pin["iteration_slack"]
    assert abs(r.iterations - ro.iterations) <= 1
    assert abs(r.pObj - pin["objective"]) < pin["objective_abs"]
    assert float(np.max(np.abs(prob.B.T @ r.x - prob.b))) < 1e-6
    assert _dual_residual(prob, r) < 1e-6
    assert kind == "normal_equations" and rank == 1


def test_t3_rank_revealing_qr(cuda):
    pin = GOLD["T3_fixed_policy"]
    prob = G.toy_t3()
    with cuda(prob) as be:
        r = solve_with_backend(be, _fixed())
        kind, rank, _ = be.equality_info()
    assert r.status.value == "Optimal"
    assert abs(r.pObj - pin["objective"]) < pin["objective_abs"]
    assert np.all(np.isfinite(r.x)) and np.all(np.isfinite(r.y))
    assert kind == "rank_revealing_qr" and rank == 1
    assert r.y[1] == 0.0


@pytest.mark.parametrize("build,opt", [
    (G.toy_t2, 5.5), (G.toy_t3, 5.5),
    (G.readme_moment_equalities, -(math.sqrt(5) - 1) / 2),
])
def test_default_options(cuda, build, opt):
    """Cold start, Ruiz scaling of B's rows and the adaptive controller."""
    prob = build()
    with cuda(prob) as be:
        r = solve_with_backend(be, SolverOptions().with_tolerance(1e-8))
    assert r.status.value == "Optimal"
    assert abs(r.pObj - opt) < 1e-6
    assert r.p_res < 1e-6 and r.d_res < 1e-6


def _iterate(prob, seed=4):
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for k in prob.k:
        G1 = rng.standard_normal((k, k))
        G2 = rng.standard_normal((k, k))
        X.append(np.eye(k) + 0.3 * G1 @ G1.T / k)
        Y.append(np.eye(k) + 0.3 * G2 @ G2.T / k)
    return rng.standard_normal(prob.m) * 0.1, X, Y, rng.standard_normal(prob.n)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


@pytest.mark.parametrize("rank,solver", [(None, "auto"), (None, "qr"), (3, "auto")])
def test_directions_match_oracle(cuda, rank, solver):
    """One predictor solve on the same iterate: residuals, equality factor
    kind and rank, (dx, dy), the KKT residual and one refinement pass."""
    from oracle.sdpx_oracle import OracleBackend
    prob = G.sdpa_dense_equalities(m=60, blocks=[10, 5], lp=4, n_eq=5, seed=3, rank=rank)
    x, X, Y, y = _iterate(prob)
    ob = OracleBackend(prob)
    ob.configure_equality(1e-8, solver)
    ob.set_iterate(x, X, Y, y=y)
    po, do, _ = ob.compute_residuals([0.1] * prob.L, False, True)
    ob.schur_build()
    assert ob.factorize()["ok"]
    ob.predictor_rhs()
    ob.solve_direction()
    with cuda(prob) as cb:
        cb.configure_equality(1e-8, solver)
        cb.set_iterate(x, X, Y, y=y)
        pc, dc, ok = cb.compute_residuals([0.1] * prob.L, False, True)
        assert ok
        cb.schur_build()
        assert cb.factorize()["ok"]
        assert cb.equality_info()[:2] == ob.equality_info()[:2]
        cb.predictor_rhs()
        cb.solve_direction()
        dx, _, _ = cb.get_direction()
        dy = cb.get_equality_direction()
        res, rn = cb.direction_residual()
        steps, res2 = cb.refine("auto", 0.0, 8, 1)
    assert abs(pc - po) <= 1e-12 * max(1.0, po) and abs(dc - do) <= 1e-12 * max(1.0, do)
    assert _rel(dx, ob.dx) <= 1e-9
    assert _rel(dy, ob.dy) <= 1e-9
    assert res <= 1e-9 * max(rn, 1.0)
    assert res2 <= res
    if rank is not None:
        assert ob.equality_info()[1] == rank


def test_solve_matches_oracle(cuda):
    """A whole solve with five equality rows: same status, objective to 1e-7,
    iteration counts within one."""
    from oracle.sdpx_oracle import oracle_solve
    prob = G.sdpa_dense_equalities(m=80, blocks=[12, 6], lp=5, n_eq=5, seed=6)
    opts = SolverOptions().with_tolerance(1e-8)
    ro = oracle_solve(prob, opts)
    with cuda(prob) as be:
        r = solve_with_backend(be, opts)
    assert r.status.value == ro.status.value == "Optimal"
    assert abs(r.pObj - ro.pObj) <= 1e-7 * max(1.0, abs(ro.pObj))
    assert abs(r.iterations - ro.iterations) <= 1
    assert r.p_res < 1e-7 and r.d_res < 1e-7


@pytest.mark.parametrize("build,opt", [
    (lambda: G.sdpa_dense_equalities(m=80, blocks=[12, 6], lp=5, n_eq=5, seed=6), None),
    (G.toy_t2, 5.5),
])
def test_mixed_precision_with_equality_rows(cuda, build, opt):
    """Mixed mode (B̃ from the FP32 factor, Q in FP64 with regularisation
    retries, guard against the FP64 KKT operator with the B terms) reaches
    the FP64 path's optimum."""
    prob = build()
    opts = SolverOptions().with_tolerance(1e-8)
    with cuda(prob, precision="fp64") as be:
        r64 = solve_with_backend(be, opts)
    with cuda(prob, precision="mixed") as be:
        rm = solve_with_backend(be, SolverOptions(precision="mixed").with_tolerance(1e-8))
    assert rm.status.value == r64.status.value == "Optimal"
    assert abs(rm.pObj - r64.pObj) <= 1e-7 * max(1.0, abs(r64.pObj))
    assert rm.p_res < 1e-7 and rm.d_res < 1e-7
    if opt is not None:
        assert abs(rm.pObj - opt) < 1e-6
    else:
        assert "mixed" in rm.precision_trace
