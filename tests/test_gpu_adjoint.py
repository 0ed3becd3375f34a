"""Device adjoint (`sdpx_b200_adjoint`) against the oracle's adjoint on the same
iterate, and against finite differences of complete GPU solves.

The oracle adjoint is pinned by finite differences in test_adjoint_oracle.py;
here the device gradients must match it to 1e-9 relative at a well-conditioned
interior iterate (the formula is the derivative of the Newton map at any
iterate; at a 1e-9 solution the Newton system's conditioning turns the FP64
rounding of the two paths into ≈ 1e-4 differences), and the config-4 shaped case
(SDPA-form loss ⟨W, X_sdpa⟩ + ⟨v, y_sdpa⟩, i.e. seeds on SDPX's Y and x,
gradients for c, C and A_1..A_3) must match central differences of GPU solves
(h = 1e-3) to 3%.
"""
import numpy as np
import pytest

from sdpx_b200 import SolverOptions, generators as G
from sdpx_b200.problem import SDPProblem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend
    return CudaBackend


def _sym(rng, k):
    M = rng.standard_normal((k, k))
    return M + M.T


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


@pytest.mark.parametrize("n_eq", [0, 3])
def test_adjoint_matches_oracle(cuda, n_eq):
    from oracle.sdpx_oracle import OracleBackend
    if n_eq:
        prob = G.sdpa_dense_equalities(m=40, blocks=[9, 4], lp=3, n_eq=n_eq, seed=4)
    else:
        prob = G.sdpa_dense(m=40, blocks=[9, 4], lp=3, seed=4)
    rng = np.random.default_rng(1)

    class It:  # a well-conditioned interior iterate
        x = rng.standard_normal(prob.m) * 0.1
        X = [np.eye(k) + 0.3 * (lambda M: M @ M.T / k)(rng.standard_normal((k, k)))
             for k in prob.k]
        Y = [np.eye(k) + 0.3 * (lambda M: M @ M.T / k)(rng.standard_normal((k, k)))
             for k in prob.k]
        y = rng.standard_normal(prob.n)
    r = It
    seeds = dict(wx=rng.standard_normal(prob.m),
                 wy=rng.standard_normal(prob.n) if prob.n else None,
                 WX=[_sym(rng, k) for k in prob.k], WY=[_sym(rng, k) for k in prob.k])
    idx = (0, 7, 39)
    ob = OracleBackend(prob)
    ob.set_iterate(r.x, r.X, r.Y, y=r.y)
    ob.compute_residuals([0.0] * prob.L, True, True)
    ob.schur_build()
    ob.factorize()
    go = ob.adjoint(A_index=idx, **seeds)
    with cuda(prob) as cb:
        cb.set_iterate(r.x, r.X, r.Y, y=r.y)
        cb.compute_residuals([0.0] * prob.L, True, True)
        cb.schur_build()
        assert cb.factorize()["ok"]
        gd = cb.adjoint(A_index=idx, **seeds)
    assert _rel(gd["grad_c"], go["grad_c"]) <= 1e-9
    if prob.n:
        assert _rel(gd["grad_b"], go["grad_b"]) <= 1e-9
    for l in range(prob.L):
        assert _rel(gd["grad_C"][l], go["grad_C"][l]) <= 1e-9
        for q in range(len(idx)):
            assert _rel(gd["grad_A"][q][l], go["grad_A"][q][l]) <= 1e-9


def test_config4_shaped_gradient_against_finite_differences(cuda):
    """Solve to 1e-9 on the GPU, differentiate L = ⟨W, Y⟩ + ⟨v, x⟩ (SDPA's
    ⟨W, X⟩ + ⟨v, y⟩) through `sdpx_b200.adjoint`, compare one random direction
    of c, C and A_1..A_3 with central differences of GPU solves."""
    from sdpx_b200 import adjoint, solve
    prob = G.sdpa_dense(m=30, blocks=[12], lp=0, seed=9)
    rng = np.random.default_rng(3)
    v = rng.standard_normal(prob.m)
    W = [_sym(rng, prob.k[0])]
    loss = lambda r: float(v @ r.x + np.sum(W[0] * r.Y[0]))
    r = solve(prob, tolerance=1e-9)
    assert r.status.value == "Optimal"
    g = adjoint(prob, r, wx=v, WY=W, A_index=(0, 1, 2))
    h = 1e-3

    def fd(make):
        return (loss(solve(make(h), tolerance=1e-10)) - loss(solve(make(-h), tolerance=1e-10))) / (2 * h)

    E = _sym(rng, prob.k[0])
    dc = rng.standard_normal(prob.m)
    pairs = [(g["grad_c"] @ dc,
              fd(lambda t: SDPProblem(prob.c + t * dc, prob.k, prob.Av, prob.C, prob.B, prob.b))),
             (float(np.sum(g["grad_C"][0] * E)),
              fd(lambda t: SDPProblem(prob.c, prob.k, prob.Av, [prob.C[0] + t * E], prob.B,
                                      prob.b)))]
    for q in range(3):
        def moved(t, q=q):
            Av = [prob.Av[0].copy()]
            Av[0][q] += t * E.reshape(-1)
            return SDPProblem(prob.c, prob.k, Av, prob.C, prob.B, prob.b)
        pairs.append((float(np.sum(g["grad_A"][q][0] * E)), fd(moved)))
    for a, f in pairs:
        assert abs(a - f) <= 0.03 * max(abs(f), abs(a), 0.3), (a, f)
