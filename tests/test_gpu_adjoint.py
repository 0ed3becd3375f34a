"""Device adjoint (`sdpx_b200_adjoint`, `sdpx_b200_adjoint_refined`) against the
oracles.

* At a well-conditioned interior iterate the device gradients match the
  oracle's adjoint to 1e-9 relative (with and without equality rows).
* At a central point (μ = 1e-3) the device adjoint — one FP64 solve, and the
  double-double refined solve — matches the double-double implicit-KKT
  gradient of oracle/dd_oracle.py (1e-9 and 1e-12) and central differences of
  central points at fixed μ (h = 1e-6) to 1e-6 relative for c, C and A_i:
  the adjoint is the exact derivative of the central-path point.
* At a 1e-9 solution the Schur matrix is ill-conditioned (one FP64 solve is
  accurate to ≈ 1e-5 there); the refined device adjoint matches the
  double-double gradient of the same iterate to 1e-6 relative.
* Complete GPU solves of the config-4 shape (SDPA-form loss ⟨W, X_sdpa⟩ +
  ⟨v, y_sdpa⟩, i.e. seeds on SDPX's Y and x) match central differences of
  solves (h = 1e-3) to 3%: those differences carry the solves' own
  termination noise (≈ 1e-10 / h), so this check guards signs and scales of
  the end-to-end gradient, not its digits.
"""
import numpy as np
import pytest

from sdpx_b200 import SolverOptions, generators as G
from sdpx_b200.problem import SDPProblem

FD_TOL = 1e-6

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


def _device_gradients(cb, x, X, Y, seeds, idx):
    cb.set_iterate(x, X, Y)
    cb.compute_residuals([0.0] * len(X), True, True)
    cb.schur_build()
    assert cb.factorize()["ok"]
    g64 = cb.adjoint(A_index=idx, **seeds)
    gref = cb.adjoint_refined(seeds.get("wx"), seeds.get("WX"), seeds.get("WY"), idx, steps=3)
    return g64, gref


def test_device_adjoint_is_the_central_path_derivative(cuda):
    from oracle.dd_oracle import central_point, dd_adjoint
    from oracle.sdpx_oracle import oracle_solve
    prob = G.sdpa_dense(m=30, blocks=[12, 4], lp=3, seed=9)
    r = oracle_solve(prob, SolverOptions().with_tolerance(1e-4))
    mu = 1e-3
    x, X, Y, res = central_point(prob, mu, (r.x, r.X, r.Y))
    assert res <= 1e-13
    rng = np.random.default_rng(5)
    seeds = dict(wx=rng.standard_normal(prob.m), WX=[_sym(rng, k) for k in prob.k],
                 WY=[_sym(rng, k) for k in prob.k])
    idx = (0, 7)
    gd = dd_adjoint(prob, x, X, Y, A_index=idx, **seeds)
    with cuda(prob) as cb:
        g64, gref = _device_gradients(cb, x, X, Y, seeds, idx)
    assert gref["residual"] <= 1e-20
    for g, tol in ((g64, 1e-9), (gref, 1e-12)):
        assert _rel(g["grad_c"], gd["grad_c"]) <= tol
        for l in range(prob.L):
            assert _rel(g["grad_C"][l], gd["grad_C"][l]) <= tol
            for q in range(len(idx)):
                assert _rel(g["grad_A"][q][l], gd["grad_A"][q][l]) <= tol

    def loss(x_, X_, Y_):
        return (float(seeds["wx"] @ x_) + sum(float(np.sum(a * b)) for a, b in zip(seeds["WX"], X_))
                + sum(float(np.sum(a * b)) for a, b in zip(seeds["WY"], Y_)))

    h = 1e-6

    def fd(make):
        vals = []
        for t in (h, -h):
            xx, XX, YY, rr = central_point(make(t), mu, (x, X, Y))
            assert rr <= 1e-13
            vals.append(loss(xx, XX, YY))
        return (vals[0] - vals[1]) / (2 * h)

    E = _sym(rng, prob.k[0])
    dc = rng.standard_normal(prob.m)

    def moved_A(t):
        Av = [a.copy() for a in prob.Av]
        Av[0][7] += t * E.reshape(-1)
        return SDPProblem(prob.c, prob.k, Av, prob.C, prob.B, prob.b)

    checks = [(float(gref["grad_c"] @ dc),
               fd(lambda t: SDPProblem(prob.c + t * dc, prob.k, prob.Av, prob.C, prob.B,
                                       prob.b))),
              (float(np.sum(gref["grad_C"][0] * E)),
               fd(lambda t: SDPProblem(prob.c, prob.k, prob.Av,
                                       [prob.C[0] + t * E] + prob.C[1:], prob.B, prob.b))),
              (float(np.sum(gref["grad_A"][1][0] * E)), fd(moved_A))]
    for ad, f in checks:
        assert abs(ad - f) <= FD_TOL * max(abs(f), 1.0), (ad, f)


def test_refined_adjoint_at_a_solution_matches_double_double(cuda):
    from oracle.dd_oracle import dd_adjoint
    from sdpx_b200 import adjoint, solve
    prob = G.sdpa_dense(m=30, blocks=[12], lp=0, seed=9)
    rng = np.random.default_rng(3)
    v = rng.standard_normal(prob.m)
    W = [_sym(rng, prob.k[0])]
    r = solve(prob, tolerance=1e-9)
    assert r.status.value == "Optimal"
    idx = (0, 1, 2)
    gd = dd_adjoint(prob, r.x, r.X, r.Y, wx=v, WY=W, A_index=idx)
    gr = adjoint(prob, r, wx=v, WY=W, A_index=idx, refine=3)
    assert gr["residual"] <= 1e-15
    assert _rel(gr["grad_c"], gd["grad_c"]) <= FD_TOL
    assert _rel(gr["grad_C"][0], gd["grad_C"][0]) <= FD_TOL
    for q in range(len(idx)):
        assert _rel(gr["grad_A"][q][0], gd["grad_A"][q][0]) <= FD_TOL


def test_refined_adjoint_residual_never_grows(cuda):
    """On the differentiable-SDP shape at 1e-9 solutions the double-double
    conjugate gradients never return a larger residual than the FP64 solve,
    and 32 steps reach double-double accuracy."""
    from sdpx_b200 import SolverOptions
    from sdpx_b200.cuda_backend import CudaBackend
    opts = SolverOptions(scaling="none").with_tolerance(1e-9)
    tested = reached = 0
    for inst in range(8):
        prob = G.sdpa_dense(m=500, blocks=[200], lp=0, seed=1000 + inst)
        rng = np.random.default_rng(inst)
        v = rng.standard_normal(prob.m)
        with CudaBackend(prob) as cb:
            r = cb.optimize(opts)
            cb.set_iterate(r.x, r.X, r.Y)
            if not cb.compute_residuals([0.0] * prob.L, True, True)[2]:
                continue  # the returned slack is not positive definite
            cb.schur_build()
            if not cb.factorize()["ok"]:
                continue
            res = [cb.adjoint_refined(v, None, None, (0,), steps=s)["residual"]
                   for s in (0, 3, 32)]
        tested += 1
        assert all(np.isfinite(res)), res
        assert res[1] <= res[0] and res[2] <= res[0], res
        reached += res[2] <= 1e-20
    assert tested >= 4 and reached >= tested - 1
