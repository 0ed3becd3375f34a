"""LP + Lorentz-cone interior-point loop on the B200 (sdpx_b200_normal_optimize)
against its oracle (oracle/cone_ipm_oracle.py).

On the same instance the device loop reaches the oracle's status, its
iteration count within ±1 and its objectives within 1e-7 relative; the device
solution satisfies the KKT conditions to the tolerance; an LP-only instance
matches an independent LP solver (HiGHS through scipy) to 1e-7.  The mixed
form (split-BF16 A·D·Aᵀ on the tensor cores, Δy refined against the FP64
operator) reaches the FP64 form's status and objectives (1e-7) with its
split iterations counted.
"""
import numpy as np
import pytest

from sdpx_b200 import SolverOptions, generators as G

pytestmark = pytest.mark.gpu
TOL = 1e-8


@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.normal import NormalSystem
    return NormalSystem


CASES = [(20, 30, [4, 5], 1, 0.3), (60, 150, [8] * 5, 2, 0.3), (40, 0, [6] * 8, 4, 0.3),
         (300, 2000, [16] * 10, 3, 0.1)]


@pytest.mark.parametrize("m,n_lp,cones,seed,density", CASES)
def test_device_loop_matches_oracle(gpu, m, n_lp, cones, seed, density):
    from oracle.cone_ipm_oracle import cone_ipm_solve
    B, b, c = G.lp_soc_problem(m, n_lp, cones, density=density, seed=seed)
    A = np.ascontiguousarray(B.T)
    ref = cone_ipm_solve(A, b, c, n_lp, cones, SolverOptions().with_tolerance(TOL))
    with gpu(B, n_lp, cones) as ns:
        got = ns.optimize(b, c, tolerance=TOL)
    assert got.status == ref.status == "Optimal", (got.status, got.message)
    assert abs(got.iterations - ref.iterations) <= 1
    assert got.pObj == pytest.approx(ref.pObj, rel=1e-7)
    assert got.dObj == pytest.approx(ref.dObj, rel=1e-7)
    assert np.max(np.abs(A @ got.x - b)) <= TOL * (1 + np.max(np.abs(b)))
    assert np.max(np.abs(A.T @ got.y + got.z - c)) <= TOL * (1 + np.max(np.abs(c)))
    assert float(got.x @ got.z) <= TOL * max(1.0, abs(got.pObj))


def test_device_lp_matches_linprog(gpu):
    from scipy.optimize import linprog
    B, b, c = G.lp_soc_problem(60, 200, [], density=0.4, seed=2)
    A = np.ascontiguousarray(B.T)
    ref = linprog(c, A_eq=A, b_eq=b, bounds=(0, None), method="highs")
    with gpu(B, 200, []) as ns:
        got = ns.optimize(b, c, tolerance=TOL)
    assert got.status == "Optimal" and ref.status == 0
    assert abs(got.pObj - ref.fun) <= 1e-7 * max(1.0, abs(ref.fun))


@pytest.mark.parametrize("m,n_lp,cones,seed,density", [CASES[1], CASES[3]])
def test_mixed_assembly_matches_fp64(gpu, m, n_lp, cones, seed, density):
    B, b, c = G.lp_soc_problem(m, n_lp, cones, density=density, seed=seed)
    A = np.ascontiguousarray(B.T)
    with gpu(B, n_lp, cones) as ns:
        r64 = ns.optimize(b, c, tolerance=TOL)
        rmx = ns.optimize(b, c, tolerance=TOL, precision="mixed")
    assert rmx.status == r64.status == "Optimal", rmx.message
    assert rmx.split_iterations > 0
    assert rmx.split_iterations + rmx.fp64_iterations == rmx.iterations
    assert rmx.pObj == pytest.approx(r64.pObj, rel=1e-7)
    assert rmx.dObj == pytest.approx(r64.dObj, rel=1e-7)
    assert np.max(np.abs(A @ rmx.x - b)) <= TOL * (1 + np.max(np.abs(b)))
    assert np.max(np.abs(A.T @ rmx.y + rmx.z - c)) <= TOL * (1 + np.max(np.abs(c)))
