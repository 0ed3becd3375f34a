"""Oracle of the LP + Lorentz-cone interior-point loop (oracle/cone_ipm_oracle.py).

SDPX has no reduced LP+SOC route to pin against, so the oracle loop is checked
on its outcome: for LP-only instances its optimum equals an independent LP
solver's (HiGHS through scipy.optimize.linprog, 1e-7 relative); for LP+SOC
instances the returned point satisfies the KKT conditions — primal and dual
residuals within the tolerance, x and z in their cones, the duality gap
xᵀz within the tolerance — which makes it optimal to that tolerance.
"""
import numpy as np
import pytest

from oracle.cone_ipm_oracle import cone_ipm_solve
from sdpx_b200 import SolverOptions, generators as G

TOL = 1e-8


def _in_cones(v, n_lp, cones):
    if n_lp and np.min(v[:n_lp]) <= 0:
        return False
    o = n_lp
    for q in cones:
        seg = v[o:o + q]
        if seg[0] <= np.linalg.norm(seg[1:]):
            return False
        o += q
    return True


@pytest.mark.parametrize("m,n_lp,seed", [(20, 50, 1), (60, 200, 2)])
def test_lp_only_matches_linprog(m, n_lp, seed):
    from scipy.optimize import linprog
    B, b, c = G.lp_soc_problem(m, n_lp, [], density=0.4, seed=seed)
    A = np.ascontiguousarray(B.T)
    r = cone_ipm_solve(A, b, c, n_lp, [], SolverOptions().with_tolerance(TOL))
    ref = linprog(c, A_eq=A, b_eq=b, bounds=(0, None), method="highs")
    assert r.status == "Optimal" and ref.status == 0
    assert abs(r.pObj - ref.fun) <= 1e-7 * max(1.0, abs(ref.fun))


@pytest.mark.parametrize("m,n_lp,cones,seed", [(20, 30, [4, 5], 1), (60, 150, [8] * 5, 2),
                                               (40, 0, [6] * 8, 4)])
def test_lp_soc_solution_satisfies_kkt(m, n_lp, cones, seed):
    B, b, c = G.lp_soc_problem(m, n_lp, cones, density=0.3, seed=seed)
    A = np.ascontiguousarray(B.T)
    r = cone_ipm_solve(A, b, c, n_lp, cones, SolverOptions().with_tolerance(TOL))
    assert r.status == "Optimal", r.message
    assert np.max(np.abs(A @ r.x - b)) <= TOL * (1 + np.max(np.abs(b)))
    assert np.max(np.abs(A.T @ r.y + r.z - c)) <= TOL * (1 + np.max(np.abs(c)))
    assert _in_cones(r.x, n_lp, cones) and _in_cones(r.z, n_lp, cones)
    gap = float(r.x @ r.z)
    assert gap <= TOL * max(1.0, (abs(r.pObj) + abs(r.dObj)) / 2)
    assert abs(r.pObj - r.dObj) <= 1e-7 * max(1.0, abs(r.pObj))
