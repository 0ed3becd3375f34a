"""The device residuals P = 𝒜x − X − C and d = c − 𝒜ᵀY are compensated sums
rounded once (Dot2), so at the rounding floor they equal the correctly
rounded values, whatever the device's summation order.

The data are built so that both residuals cancel to the rounding floor: C is
the FP64 value of 𝒜x − X and c the FP64 value of 𝒜ᵀY, each with the
coefficients spread over six decades.  The exact residuals come from rational
arithmetic (`fractions.Fraction`) rounded once; the device's max-norms
(`compute_residuals`) must match them to Dot2's error bound
(|err| ≤ eps·|r| + γ²·Σ|terms|, a few units in the last place here), which plain
FP64 sums miss by orders of magnitude on the same data.
"""
from fractions import Fraction

import numpy as np
import pytest

from sdpx_b200.problem import SDPProblem

pytestmark = pytest.mark.gpu

EPS = 2.0 ** -53


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend
    return CudaBackend


def _sym(rng, k, spread):
    G = rng.standard_normal((k, k)) * 10.0 ** rng.uniform(-spread, spread, (k, k))
    return np.triu(G) + np.triu(G, 1).T


def _floor_problem(m, blocks, seed):
    """Problem and iterate whose residuals sit at the rounding floor."""
    rng = np.random.default_rng(seed)
    Av, C, X, Y = [], [], [], []
    x = rng.standard_normal(m) * 10.0 ** rng.uniform(-3, 3, m)
    c = np.zeros(m)
    for k in blocks:
        A = np.stack([_sym(rng, k, 3) for _ in range(m)])        # (m, k, k)
        G1, G2 = rng.standard_normal((k, k)), rng.standard_normal((k, k))
        Xl = np.eye(k) + G1 @ G1.T / k
        Yl = np.eye(k) + G2 @ G2.T / k
        Xl, Yl = (Xl + Xl.T) / 2, (Yl + Yl.T) / 2
        Cl = np.einsum("i,ijk->jk", x, A) - Xl
        Cl = (Cl + Cl.T) / 2
        c += np.einsum("ijk,jk->i", A, Yl)
        Av.append(np.ascontiguousarray(A.reshape(m, k * k)))
        C.append(Cl)
        X.append(Xl)
        Y.append(Yl)
    prob = SDPProblem(c, list(blocks), Av, C, np.zeros((m, 0)), np.zeros(0))
    return prob, x, X, Y


def _exact_residuals(prob, x, X, Y):
    """max|P| and max|d| from rational sums rounded once, and the Σ|terms|."""
    xf = [Fraction(v) for v in x]
    pmax, pscale = 0.0, 0.0
    d = [Fraction(v) for v in prob.c]
    dscale = np.abs(prob.c).copy()
    for l, k in enumerate(prob.k):
        A = prob.Av[l]
        Xv, Cv, Yv = X[l].reshape(-1), prob.C[l].reshape(-1), Y[l].reshape(-1)
        for e in range(k * k):
            s = sum((xf[i] * Fraction(A[i, e]) for i in range(prob.m)), Fraction(0))
            s -= Fraction(Xv[e]) + Fraction(Cv[e])
            pmax = max(pmax, abs(float(s)))
            pscale = max(pscale, float(np.abs(x) @ np.abs(A[:, e])) + abs(Xv[e]) + abs(Cv[e]))
        Yf = [Fraction(v) for v in Yv]
        for i in range(prob.m):
            d[i] -= sum((Fraction(A[i, e]) * Yf[e] for e in range(k * k)), Fraction(0))
        dscale += np.abs(A) @ np.abs(Yv)
    dmax = max(abs(float(v)) for v in d)
    return pmax, float(pscale), dmax, float(np.max(dscale))


def _plain_residuals(prob, x, X, Y):
    p = max(float(np.max(np.abs(x @ prob.Av[l] - X[l].reshape(-1) - prob.C[l].reshape(-1))))
            for l in range(prob.L))
    d = prob.c.copy()
    for l in range(prob.L):
        d -= prob.Av[l] @ Y[l].reshape(-1)
    return p, float(np.max(np.abs(d)))


# The products run over the lower-triangle copy of 𝒜 (Kt = Σ k(k+1)/2 rows):
# odd Kt takes the scalar kernels, even Kt the 128-bit ones.
@pytest.mark.parametrize("m,blocks,seed", [(40, [6, 3], 0),    # Kt = 27
                                           (37, [8, 3], 1)])   # Kt = 42
def test_residuals_are_correctly_rounded(cuda, m, blocks, seed):
    prob, x, X, Y = _floor_problem(m, blocks, seed)
    pmax, pscale, dmax, dscale = _exact_residuals(prob, x, X, Y)
    with cuda(prob) as cb:
        cb.set_iterate(x, X, Y)
        p_dev, d_dev, ok = cb.compute_residuals([0.0] * prob.L, True, False)
    n = max(prob.m, max(k * k for k in prob.k)) + 2
    gamma = n * EPS / (1 - n * EPS)
    assert abs(p_dev - pmax) <= 2 * EPS * pmax + gamma * gamma * pscale + 1e-300
    assert abs(d_dev - dmax) <= 2 * EPS * dmax + gamma * gamma * dscale + 1e-300
    # the data do cancel to the floor: plain FP64 sums are off by far more
    p_pl, d_pl = _plain_residuals(prob, x, X, Y)
    assert pmax < 1e-12 * pscale and dmax < 1e-12 * dscale
    assert abs(p_pl - pmax) > 1e3 * (2 * EPS * pmax + gamma * gamma * pscale) or \
        abs(d_pl - dmax) > 1e3 * (2 * EPS * dmax + gamma * gamma * dscale)
