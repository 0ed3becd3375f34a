"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

* Kernel level: on the same iterate, every Newton-step product — residual
  norms, the Schur matrix, the KKT direction, the block directions, the
  affine step bounds, the corrector and the step lengths — agrees with the
  oracle.  Tolerance 1e-10 relative (the plain-FP64 parity target; the
  Schur matrix itself is held to 1e-12).
* Solve level: the reference's gate problems reach the recorded status,
  iteration count (±1) and objective (1e-9 relative), and a seeded n=50/m=100
  SDPA-form instance matches the oracle's status, iteration count and
  objectives (1e-7 relative).
"""
import json
import math
import os

import numpy as np
import pytest

from sdpx_b200 import SolverOptions, generators as G, solve
from sdpx_b200.driver import solve_with_backend

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "gates.json")))
REL = 1e-10


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend
    return CudaBackend


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def blocks_rel(A, B):
    return max(rel(a, b) for a, b in zip(A, B))


def interior_iterate(prob, seed=3):
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for k in prob.k:
        G1 = rng.standard_normal((k, k))
        G2 = rng.standard_normal((k, k))
        X.append(np.eye(k) + 0.2 * G1 @ G1.T / k)
        Y.append(np.eye(k) + 0.2 * G2 @ G2.T / k)
    x = rng.standard_normal(prob.m) * 0.1
    return x, X, Y


PROBLEMS = {
    "mixed_blocks": lambda: G.sdpa_dense(m=60, blocks=[12, 5, 2], lp=4, seed=11),
    "single_block": lambda: G.sdpa_dense(m=100, blocks=[50], seed=0),
    "gate_dense": G.gate_dense,
}


@pytest.mark.parametrize("name", list(PROBLEMS))
def test_newton_step_kernels_match_oracle(cuda, name):
    from oracle.sdpx_oracle import OracleBackend
    prob = PROBLEMS[name]()
    ob = OracleBackend(prob)
    with cuda(prob) as cb:
        x, X, Y = interior_iterate(prob)
        for be in (ob, cb):
            be.set_iterate(x, X, Y)
        mu = [0.05] * prob.L
        ro = ob.compute_residuals(mu, False, True)
        rc = cb.compute_residuals(mu, False, True)
        assert ro[2] and rc[2]
        assert abs(ro[0] - rc[0]) <= REL * max(1.0, ro[0])
        assert abs(ro[1] - rc[1]) <= REL * max(1.0, ro[1])
        for be in (ob, cb):
            be.schur_build()
        S_o, S_c = ob.schur_matrix(), cb.schur_matrix()
        assert rel(S_c, S_o) <= 1e-12
        fo, fc = ob.factorize(), cb.factorize()
        assert fo["ok"] == fc["ok"] and fo["reg_attempts"] == fc["reg_attempts"]
        assert abs(fo["quality"] - fc["quality"]) <= 1e-10
        # Directions inherit the conditioning of S: two correct FP64 solves can
        # differ by ~κ(S)·eps.  κ(S) ≥ (max L_ii / min L_ii)² = 1/quality².
        kappa = 1.0 / max(fo["quality"], 1e-300) ** 2
        DIR = max(REL, 64 * 2.2e-16 * kappa)
        for be in (ob, cb):
            be.predictor_rhs()
        assert rel(cb.get_rhs(), ob.get_rhs()) <= REL
        for be in (ob, cb):
            be.solve_direction()
            be.direction_blocks()
        dxo, dXo, dYo = ob.get_direction()
        dxc, dXc, dYc = cb.get_direction()
        assert rel(dxc, dxo) <= DIR
        assert blocks_rel(dXc, dXo) <= DIR and blocks_rel(dYc, dYo) <= DIR
        ao, ac = ob.affine_diagnostics(True), cb.affine_diagnostics(True)
        for key in ("complementarity", "affine_complementarity", "tX", "tY", "mu", "mu_aff"):
            assert abs(ao[key] - ac[key]) <= max(1e-9, 10 * DIR) * max(1.0, abs(ao[key])), key
        assert ao["uniform"] == ac["uniform"]
        assert ob.block_margins() == pytest.approx(cb.block_margins(), rel=1e-12)
        for be in (ob, cb):
            be.mehrotra_corrector_rhs(0.3, ao["mu"], not ao["uniform"])
            be.solve_direction()
        so = ob.refine("auto", 0.0, 8, 1)
        sc = cb.refine("auto", 0.0, 8, 1)
        go, gc = ob.direction_residual(), cb.direction_residual()
        assert gc[0] <= max(1e-12 * max(gc[1], 1.0), 10 * go[0])
        for be in (ob, cb):
            be.direction_blocks()
        dxo, dXo, dYo = ob.get_direction()
        dxc, dXc, dYc = cb.get_direction()
        assert rel(dxc, dxo) <= DIR
        assert blocks_rel(dYc, dYo) <= DIR
        for rule in ("backtrack", "fraction_to_boundary"):
            lo = ob.line_search(rule, 0.95, 0.95, 0.8, 1e-10, math.sqrt(2.2e-16))
            lc = cb.line_search(rule, 0.95, 0.95, 0.8, 1e-10, math.sqrt(2.2e-16))
            assert lo[0] == pytest.approx(lc[0], rel=max(1e-9, 10 * DIR))
            assert lo[1] == pytest.approx(lc[1], rel=max(1e-9, 10 * DIR))
        uo, uc = ob.update(0.7, 0.6), cb.update(0.7, 0.6)
        assert uo[0] == pytest.approx(uc[0], rel=1e-12) and uo[1] == uc[1]
        # The objectives after the update are linear in the directions, which
        # are held to DIR; the Schur matrix itself stays within 1e-12 above.
        assert ob.objectives() == pytest.approx(cb.objectives(), rel=max(1e-12, DIR))


@pytest.mark.parametrize("m,blocks,lp", [
    (40, [9, 3], 5),
    # blocks wider than a warp and not a multiple of 32, two 128-column groups
    # of 1×1 rows, several 16-constraint chunks of the 1×1 row maxima
    (60, [45, 70], 150),
])
def test_equilibration_matches_oracle(cuda, m, blocks, lp):
    from oracle.sdpx_oracle import OracleBackend
    prob = G.sdpa_dense(m=m, blocks=blocks, lp=lp, seed=4)
    ob = OracleBackend(prob)
    with cuda(prob) as cb:
        eo, ec = ob.equilibrate(), cb.equilibrate()
        assert eo.objective_scale == pytest.approx(ec.objective_scale, rel=1e-14)
        assert rel(ec.s, eo.s) <= 1e-14
        for a, b in zip(ec.E, eo.E):
            assert rel(a, b) <= 1e-14
        assert eo.ruiz_passes == ec.ruiz_passes
        # scaled data: compare through the identity Schur matrix Σ⟨A_i, A_j⟩
        for be in (ob, cb):
            be.schur_build(identity=True)
        assert rel(cb.schur_matrix(), ob.schur_matrix()) <= 1e-12


def _gate_measure(r):
    return dict(status=r.status.value, iterations=r.iterations, objective=r.pObj,
                relative_gap=abs(r.pObj - r.dObj) / max(1.0, abs(r.pObj)),
                primal_residual=r.p_res, dual_residual=r.d_res)


# The sdp_dense gate has a singular Schur matrix (m = 180 variables against
# 3·36 = 108 independent symmetric 8×8 coefficients), and from iteration 2 on its
# dual residual sits at the 1e-15 rounding floor, where the adaptive
# controller's `achieved_residual_reduction > 5/4` centring test
# (src/adaptive_parameters.jl:326-330) compares two rounding-noise values: with
# plain sums the iteration count follows the summation order (the CPU oracle
# takes 10 instead of 9 with ⟨A_i, Y⟩ summed pairwise, test_oracle_gates.py).
# The device computes P and d as compensated sums rounded once, independent of
# its summation order, and meets the reference's ±1 rule (benchmark/gates.jl:65).
ITER_SLACK = {"sdp_closed_form": 1, "sdp_dense": 1}


@pytest.mark.parametrize("name,build", [("sdp_closed_form", G.gate_closed_form),
                                        ("sdp_dense", G.gate_dense)])
def test_gate_on_gpu(cuda, name, build):
    r = solve(build(), tolerance=GOLD[name]["tolerance"])
    m = _gate_measure(r)
    base, rules = GOLD[name], GOLD["compare"]
    assert m["status"] == base["status"]
    assert abs(m["iterations"] - base["iterations"]) <= ITER_SLACK[name]
    assert abs(m["objective"] - base["objective"]) / max(1.0, abs(base["objective"])) <= rules["objective_rel"]
    for key in ("relative_gap", "primal_residual", "dual_residual"):
        assert m[key] <= max(rules["residual_factor"] * base[key], rules["absolute_floor"])


def test_t1_fixed_policy_on_gpu(cuda):
    from sdpx_b200.cuda_backend import CudaBackend
    pin = GOLD["T1_fixed_policy"]
    opts = SolverOptions(parameter_policy="fixed", parameter_strategy="fixed", scaling="none")
    prob = G.toy_t1()
    with CudaBackend(prob) as be:
        r = solve_with_backend(be, opts)
    assert r.status.value == "Optimal"
    assert abs(r.iterations - pin["iterations"]) <= pin["iteration_slack"]
    assert abs(r.pObj - 2 * math.sqrt(6)) < pin["objective_abs"]


def test_sdpa_n50_m100_matches_oracle_solve(cuda):
    from oracle.sdpx_oracle import oracle_solve
    prob = G.sdpa_dense(m=100, blocks=[50], seed=0)
    to, tc = [], []
    ro = oracle_solve(prob, SolverOptions().with_tolerance(1e-8), trace=to)
    rc = solve(prob, tolerance=1e-8, trace=tc)
    assert rc.status == ro.status
    assert rc.iterations == ro.iterations
    assert rc.pObj == pytest.approx(ro.pObj, rel=1e-7)
    assert rc.dObj == pytest.approx(ro.dObj, rel=1e-7)
    assert rc.relative_gap <= 1e-8
    # per-iteration objectives track the oracle trajectory
    for a, b in zip(to[:6], tc[:6]):
        assert b["pObj"] == pytest.approx(a["pObj"], rel=1e-8, abs=1e-10)
