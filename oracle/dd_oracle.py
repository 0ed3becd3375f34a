"""Double-double (Float64x2) CPU oracle — TEST INFRASTRUCTURE ONLY.

A value is an unevaluated sum hi + lo of two float64 arrays with
|lo| ≤ ulp(hi)/2 (about 106 significant bits).  The arithmetic follows the
published error-free transformations: Knuth's TwoSum, Dekker's FastTwoSum,
Veltkamp's splitting and Dekker's TwoProduct (exact without a fused
multiply-add), and the double-double addition / multiplication / division of
Hida, Li and Bailey's QD library (ARITH-15, 2001).  These are the reference
arithmetic for

* the implicit-KKT gradient of the adjoint (`dd_adjoint`): the same linear
  system the device adjoint solves (sdpx_b200_adjoint), solved to
  double-double accuracy by iterative refinement on a float64 factor with
  double-double residuals, and
* the central-path point at a fixed μ (`central_point`), whose derivative
  with respect to the data the adjoint is, for finite-difference checks.

Nothing here is imported by the product; only tests/ and bench.py's CPU legs.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np
import scipy.linalg as sla

_SPLIT = 134217729.0  # 2^27 + 1


# ------------------------------------------------------------ primitives ---
def two_sum(a, b):
    """s + e = a + b exactly (Knuth)."""
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


def fast_two_sum(a, b):
    """s + e = a + b exactly when |a| ≥ |b| (Dekker)."""
    s = a + b
    return s, b - (s - a)


def split(a):
    """a = hi + lo with 26-bit halves (Veltkamp)."""
    c = _SPLIT * a
    hi = c - (c - a)
    return hi, a - hi


def two_prod(a, b):
    """p + e = a·b exactly (Dekker)."""
    p = a * b
    ah, al = split(a)
    bh, bl = split(b)
    return p, ((ah * bh - p) + ah * bl + al * bh) + al * bl


class DD:
    """Array of double-double numbers."""

    __slots__ = ("hi", "lo")

    def __init__(self, hi, lo=None):
        self.hi = np.asarray(hi, dtype=np.float64)
        self.lo = np.zeros_like(self.hi) if lo is None else np.asarray(lo, dtype=np.float64)

    def __add__(self, o):
        o = _dd(o)
        s, e = two_sum(self.hi, o.hi)
        t, f = two_sum(self.lo, o.lo)
        e = e + t
        s, e = fast_two_sum(s, e)
        e = e + f
        return DD(*fast_two_sum(s, e))

    def __neg__(self):
        return DD(-self.hi, -self.lo)

    def __sub__(self, o):
        return self + (-_dd(o))

    def __mul__(self, o):
        o = _dd(o)
        p, e = two_prod(self.hi, o.hi)
        e = e + (self.hi * o.lo + self.lo * o.hi)
        return DD(*fast_two_sum(p, e))

    def __truediv__(self, o):
        o = _dd(o)
        q1 = self.hi / o.hi
        r = self - o * q1
        q2 = r.hi / o.hi
        r = r - o * q2
        q3 = r.hi / o.hi
        q1, q2 = fast_two_sum(q1, q2)
        return DD(q1, q2) + DD(q3)

    def __getitem__(self, idx):
        return DD(self.hi[idx], self.lo[idx])

    def __setitem__(self, idx, v):
        v = _dd(v)
        self.hi[idx] = v.hi
        self.lo[idx] = v.lo

    @property
    def T(self):
        return DD(self.hi.T, self.lo.T)

    @property
    def shape(self):
        return self.hi.shape

    def reshape(self, *s, order="C"):
        return DD(self.hi.reshape(*s, order=order), self.lo.reshape(*s, order=order))

    def copy(self):
        return DD(self.hi.copy(), self.lo.copy())

    def to_float(self):
        return self.hi + self.lo


def _dd(v):
    return v if isinstance(v, DD) else DD(v)


def dd_sum(a: DD, axis=-1) -> DD:
    """Pairwise double-double sum along `axis`."""
    hi = np.moveaxis(a.hi, axis, -1)
    lo = np.moveaxis(a.lo, axis, -1)
    cur = DD(hi, lo)
    while cur.hi.shape[-1] > 1:
        n = cur.hi.shape[-1]
        if n % 2:
            pad = np.zeros(cur.hi.shape[:-1] + (1,))
            cur = DD(np.concatenate([cur.hi, pad], -1), np.concatenate([cur.lo, pad], -1))
            n += 1
        cur = cur[..., 0:n:2] + cur[..., 1:n:2]
    return cur[..., 0]


def dd_matmul(A: DD, B: DD) -> DD:
    """C = A·B in double-double (one rank-one update per inner index)."""
    A, B = _dd(A), _dd(B)
    m, kk = A.shape
    n = B.shape[1]
    C = DD(np.zeros((m, n)))
    for t in range(kk):
        a_h, a_l = A.hi[:, t:t + 1], A.lo[:, t:t + 1]
        b_h, b_l = B.hi[t:t + 1, :], B.lo[t:t + 1, :]
        p, e = two_prod(a_h, b_h)
        e = e + (a_h * b_l + a_l * b_h)
        C = C + DD(p, e)
    return C


def dd_inverse_spd(X: np.ndarray, steps: int = 3) -> DD:
    """X⁻¹ of a float64 SPD matrix to double-double accuracy: the float64
    inverse refined by Newton–Schulz steps Z ← Z + Z(I − XZ)."""
    k = X.shape[0]
    L = np.linalg.cholesky(X)
    Z0 = sla.cho_solve((L, True), np.eye(k))
    Z = DD(0.5 * (Z0 + Z0.T))
    I = DD(np.eye(k))
    Xd = DD(X)
    for _ in range(steps):
        Rm = I - dd_matmul(Xd, Z)
        Z = Z + dd_matmul(Z, Rm)
        Z = DD(0.5 * (Z.hi + Z.hi.T), 0.5 * (Z.lo + Z.lo.T))
    return Z


def dd_sym(M: DD) -> DD:
    return DD(M.hi, M.lo) * 0.5 + DD(M.hi.T, M.lo.T) * 0.5


# ------------------------------------------------ stacked-data operators ---
def dd_amul(Av: Sequence[np.ndarray], k: Sequence[int], v: DD) -> List[DD]:
    """mat(𝒜v) per block in double-double: Σ_i v_i A_i."""
    out = []
    for l, kl in enumerate(k):
        A = Av[l]                                    # (m, k²), row i = vec(A_i)
        acc = DD(np.zeros(kl * kl))
        for i in range(A.shape[0]):
            p, e = two_prod(A[i], v.hi[i])
            acc = acc + DD(p, e + A[i] * v.lo[i])
        out.append(acc.reshape(kl, kl))
    return out


def dd_atmul(Av: Sequence[np.ndarray], Z: Sequence[DD]) -> DD:
    """⟨A_i, Z⟩ summed over blocks, in double-double."""
    m = Av[0].shape[0]
    tot = DD(np.zeros(m))
    for A, Zl in zip(Av, Z):
        zh, zl = Zl.hi.reshape(-1), Zl.lo.reshape(-1)
        rows = max(1, (1 << 22) // max(1, zh.size))     # ≈ 32 MB per temporary
        part_h, part_l = np.zeros(m), np.zeros(m)
        for r0 in range(0, m, rows):
            Ab = A[r0:r0 + rows]
            p, e = two_prod(Ab, zh[None, :])
            sb = dd_sum(DD(p, e + Ab * zl[None, :]), axis=1)
            part_h[r0:r0 + rows], part_l[r0:r0 + rows] = sb.hi, sb.lo
        tot = tot + DD(part_h, part_l)
    return tot


# ------------------------------------------------ adjoint reference ---
def dd_adjoint(prob, x, X, Y, wx=None, WX=None, WY=None, A_index=(), refine=4):
    """Gradient of L = ⟨wx, x⟩ + Σ⟨WX_l, X_l⟩ + Σ⟨WY_l, Y_l⟩ at the iterate
    (x, X, Y) (no equality rows) by the implicit-function derivative of the
    HKM-linearised KKT conditions — the system sdpx_b200_adjoint solves —
    with every product and the Schur solve in double-double:
    S·λ = wx + 𝒜ᵀ(WX − G), G = X⁻¹·sym(WY)·Y, S·v = 𝒜ᵀ(X⁻¹ mat(𝒜v) Y);
    ∂L/∂c = −λ, ∂L/∂C = sym(X⁻¹ΛY) − sym(WX − G), Λ = mat(𝒜λ),
    ∂L/∂A_i = λ_i·Y − x_i·∂L/∂C.  λ is refined on the float64 Cholesky factor
    of S with double-double residuals.  Returns float64 (rounded) gradients."""
    L, m = len(prob.k), prob.m
    Xi = [dd_inverse_spd(np.asarray(Xl)) for Xl in X]
    Yd = [DD(np.asarray(Yl)) for Yl in Y]
    D = []
    w = DD(np.zeros(m) if wx is None else np.asarray(wx, dtype=np.float64))
    Gs = []
    for l in range(L):
        kl = prob.k[l]
        Dl = DD(np.zeros((kl, kl)))
        if WX is not None:
            Dl = Dl + DD(np.asarray(WX[l], dtype=np.float64))
        if WY is not None:
            Ws = np.asarray(WY[l], dtype=np.float64)
            Ws = DD(0.5 * Ws + 0.5 * Ws.T)
            Gl = dd_matmul(Xi[l], dd_matmul(Ws, Yd[l]))
            Dl = Dl - Gl
        D.append(Dl)
    w = w + dd_atmul(prob.Av, D)

    def S_mul(v: DD) -> DD:
        M = dd_amul(prob.Av, prob.k, v)
        Z = [dd_matmul(Xi[l], dd_matmul(M[l], Yd[l])) for l in range(L)]
        return dd_atmul(prob.Av, Z)

    # float64 Schur factor: S_ij = ⟨A_i, X⁻¹ A_j Y⟩
    S = np.zeros((m, m))
    for l, kl in enumerate(prob.k):
        A3 = prob.Av[l].reshape(m, kl, kl)
        T = np.matmul(np.matmul(Xi[l].to_float(), A3), np.asarray(Y[l]))
        S += prob.Av[l] @ T.reshape(m, -1).T
    S = 0.5 * (S + S.T)
    fac = sla.cho_factor(S, lower=True)
    lam = DD(sla.cho_solve(fac, w.to_float()))
    for _ in range(refine):
        r = w - S_mul(lam)
        lam = lam + DD(sla.cho_solve(fac, r.to_float()))
    Lam = dd_amul(prob.Av, prob.k, lam)
    gC = []
    for l in range(L):
        Zl = dd_matmul(Xi[l], dd_matmul(Lam[l], Yd[l]))
        gC.append(dd_sym(Zl) - dd_sym(D[l]))
    gCf = [g.to_float() for g in gC]
    gA = [[lam.to_float()[i] * np.asarray(Y[l]) - x[i] * gCf[l] for l in range(L)]
          for i in A_index]
    return dict(grad_c=-lam.to_float(), grad_C=gCf, grad_A=gA, lambda_x=lam.to_float())


# ---------------------------------------------- central-path point ---
def central_point(prob, mu: float, start, iterations: int = 40, tol: float = 1e-15):
    """The point of the central path 𝒜x − X = C, 𝒜ᵀY = c, X·Y = μI (every
    block, 1×1 blocks included) reached from `start` = (x, X, Y) by HKM Newton
    steps with target μ on the oracle's kernels (src/step.jl:95-108), each
    step halved until X and Y stay positive definite; full steps near the
    path converge quadratically.  Returns (x, X, Y, scaled residual)."""
    from oracle.sdpx_oracle import OracleBackend, kchol
    be = OracleBackend(prob)
    x, X, Y = start
    be.set_iterate(np.array(x, dtype=np.float64), [np.array(a) for a in X],
                   [np.array(a) for a in Y])
    scale = max(1.0, max(float(np.max(np.abs(Cl))) for Cl in prob.C))
    res = np.inf
    for _ in range(iterations):
        p_res, d_res, ok = be.compute_residuals([mu] * prob.L, False, True)
        if not ok:
            raise RuntimeError("central_point left the interior")
        cres = max(float(np.max(np.abs(R))) for R in be.R)
        res = max(p_res, d_res, cres) / scale
        if res <= tol:
            break
        be.schur_build()
        if not be.factorize()["ok"]:
            raise RuntimeError("central_point: Schur factorisation failed")
        be.predictor_rhs()
        be.solve_direction()
        be.direction_blocks()
        t = 1.0
        while t > 1e-8:
            if all(kchol(Xl + t * dX)[0] and kchol(Yl + t * dY)[0]
                   for Xl, Yl, dX, dY in zip(be.X, be.Y, be.dX, be.dY)):
                break
            t *= 0.5
        be.update(t, t)
    xo, Xo, _, Yo = be.get_iterate()
    return xo, Xo, Yo, res
