"""Parity at the sizes where the large-problem code paths engage.

* m = 600 with PSD blocks 200 + 180 and 100 nonnegatives: the stacked length
  K = 200² + 180² + 100 = 72 500 exceeds one 65 472-row chunk of the exact
  int8 digit Gram (two chunks), the split-BF16 SYRK runs ≈ 18 K chunks, and
  the FP32 Schur factor of the mixed mode takes the tiled path (m > 447).  On
  one interior iterate the Schur matrix of both FP64 engines (int8 digits and
  DMMA tiles) is held to 1e-12 of the oracle's, the FP64 directions to the
  condition-scaled bound of the kernel parity tests, the split Schur matrix
  to the split tolerance (5e-5 relative), and the mixed Newton direction
  (FP32 tiled factor, FP64 refinement against the matrix-free operator) to
  1e-9 of the oracle's.
* The m = 2000 instance of the bench (seed 0) solved on the device in both
  precision modes reaches the CPU oracle's status with objectives within 1e-7
  relative of its complete solve (tests/golden/headline_m2000.json, made by
  tests/golden/make_headline_fixture.py) and a valid original-coordinate
  certificate.
"""
import json
import math
import os

import numpy as np
import pytest

from sdpx_b200 import generators as G, solve

pytestmark = pytest.mark.gpu

HEADLINE = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                       "headline_m2000.json")))
REL = 1e-10
SPLIT_TOL = 5e-5
OBJ_TOL = 1e-7


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


def _iterate(prob, seed=3):
    rng = np.random.default_rng(seed)
    X, Y = [], []
    for k in prob.k:
        G1 = rng.standard_normal((k, k))
        G2 = rng.standard_normal((k, k))
        X.append(np.eye(k) + 0.2 * G1 @ G1.T / k)
        Y.append(np.eye(k) + 0.2 * G2 @ G2.T / k)
    return rng.standard_normal(prob.m) * 0.1, X, Y


@pytest.fixture(scope="module")
def chunked_case():
    """The m = 600 instance, one iterate, and the oracle's Schur matrix and
    predictor direction at it."""
    from oracle.sdpx_oracle import OracleBackend
    prob = G.sdpa_dense(m=600, blocks=[200, 180], lp=100, seed=17)
    assert sum(k * k for k in prob.k) > 65472
    x, X, Y = _iterate(prob)
    ob = OracleBackend(prob)
    ob.set_iterate(x, X, Y)
    ob.compute_residuals([0.05] * prob.L, False, True)
    ob.schur_build()
    S = ob.schur_matrix()
    fo = ob.factorize()
    assert fo["ok"]
    ob.predictor_rhs()
    rhs = ob.get_rhs()
    ob.solve_direction()
    ob.direction_blocks()
    dx, dX, dY = ob.get_direction()
    kappa = 1.0 / max(fo["quality"], 1e-300) ** 2
    return dict(prob=prob, it=(x, X, Y), S=S, rhs=rhs, dx=dx, dX=dX, dY=dY,
                DIR=max(REL, 64 * 2.2e-16 * kappa), quality=fo["quality"],
                reg_attempts=fo["reg_attempts"])


@pytest.mark.parametrize("engine", ["int8", "dmma"])
def test_chunked_fp64_schur_and_direction_match_oracle(cuda, chunked_case, engine):
    c = chunked_case
    prob = c["prob"]
    with cuda(prob) as be:
        be.set_gram_engine(engine)
        be.set_iterate(*c["it"])
        be.compute_residuals([0.05] * prob.L, False, True)
        be.schur_build()
        S = be.schur_matrix()
        assert rel(S, c["S"]) <= 1e-12
        f = be.factorize()  # m = 600: the single-launch cooperative FP64 Cholesky
        assert f["ok"] and f["reg_attempts"] == c["reg_attempts"]
        assert abs(f["quality"] - c["quality"]) <= 1e-10
        be.predictor_rhs()
        assert rel(be.get_rhs(), c["rhs"]) <= REL
        be.solve_direction()
        be.direction_blocks()
        dx, dX, dY = be.get_direction()
    assert rel(dx, c["dx"]) <= c["DIR"]
    assert max(rel(a, b) for a, b in zip(dX, c["dX"])) <= c["DIR"]
    assert max(rel(a, b) for a, b in zip(dY, c["dY"])) <= c["DIR"]


def test_chunked_mixed_schur_and_refined_direction(cuda, chunked_case):
    c = chunked_case
    prob = c["prob"]
    with cuda(prob) as be:
        be._set_mode("mixed")
        be.set_iterate(*c["it"])
        be.compute_residuals([0.05] * prob.L, False, True)
        be.schur_build()
        Smix = be.schur_matrix()
        be.schur_build()
        assert np.array_equal(Smix, be.schur_matrix())
        assert be.factorize()["ok"]          # FP32 factor, tiled path (m = 600 > 447)
        be.predictor_rhs()
        be.solve_direction()
        be.refine("auto", 0.0, 8, 0)
        residual, rnorm = be.direction_residual()
        dx = be.get_direction()[0].copy()
        assert be.counters()["operator_applications"] > 0
    scale = np.max(np.abs(c["S"]))
    assert np.max(np.abs(Smix - c["S"])) / scale <= SPLIT_TOL
    assert np.array_equal(Smix, Smix.T)
    assert residual <= 1e-10 * max(rnorm, 1.0)
    assert rel(dx, c["dx"]) <= max(1e-9, c["DIR"])


@pytest.fixture(scope="module")
def headline_problem():
    sh = HEADLINE["shape"]
    return G.sdpa_dense(m=sh["m"], blocks=sh["blocks"], lp=sh["lp"], seed=sh["seed"])


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_headline_instance_matches_cpu_solve(cuda, headline_problem, precision):
    r = solve(headline_problem, tolerance=HEADLINE["tolerance"], precision=precision,
              certificate=True)
    assert r.status.value == HEADLINE["status"]
    assert math.isclose(r.pObj, HEADLINE["pObj"], rel_tol=OBJ_TOL)
    assert math.isclose(r.dObj, HEADLINE["dObj"], rel_tol=OBJ_TOL)
    assert r.relative_gap <= HEADLINE["tolerance"]
    assert r.certificate["valid"], r.certificate["failures"]
