"""CPU oracle of the Float64x2 Newton system — TEST INFRASTRUCTURE ONLY.

Only `tests/` may import this module.  It restates, for one-block dense SDPs,
the dense loop with its Newton system formed and solved in double-double while
the iterate stays in FP64 — the arithmetic of the batched engine's Float64x2
mode and of SDPX's extended-precision setting (a target-precision operator and
residuals, src/kernels/mixed_precision_kkt.jl:1475-1586; the Float64x2
provider, ext/SDPXMultiFloatLinearAlgebraExt.jl:743-778):

* residuals P = 𝒜x − X − C, d = c − 𝒜ᵀY, R = −XY (+μI) (src/step.jl:25-72);
* X⁻¹ from the FP64 inverse by three Newton–Schulz steps Z ← sym(Z + Z(I − XZ));
* S_ij = ⟨A_i, X⁻¹A_jY⟩ for i ≥ j, mirrored (src/schur.jl:511-562 in the HKM form);
* Cholesky of S with the regularisation retries of src/kkt.jl:1419-1445;
* right-hand sides, corrector targets, direction blocks (src/step.jl:95-108,
  src/kernels/threaded.jl:574-663, 837-1067), the refinement residual
  ρ = r − S·dx and corrections (src/kkt.jl:3689-3780, 3891-3963).

Everything else (controller, step lengths, update) is the FP64 oracle's
(`OracleBackend`), driven by the shared driver.
"""
from __future__ import annotations

import math

import numpy as np

from . import sdpx_oracle as O
from .dd_oracle import DD, dd_inverse_spd, dd_matmul, dd_sum, two_prod


def _dd(a):
    return a if isinstance(a, DD) else DD(np.asarray(a, dtype=np.float64))


def dd_sqrt(d: DD) -> DD:
    """√d: one Newton correction of the FP64 root."""
    s = np.sqrt(d.hi)
    p, e = two_prod(s, s)
    return DD(s) + DD((d.hi - p - e + d.lo) / (2 * s))


def dd_cholesky(S: DD):
    """Lower Cholesky factor in double-double, None at a pivot that is not > 0."""
    m = S.shape[0]
    L = S.copy()
    for j in range(m):
        d = L[j, j]
        if not d.hi > 0:
            return None
        lj = dd_sqrt(d)
        L[j, j] = lj
        if j + 1 < m:
            col = L[j + 1:, j] / lj
            L[j + 1:, j] = col
            c2 = DD(col.hi[:, None], col.lo[:, None])
            L[j + 1:, j + 1:] = L[j + 1:, j + 1:] - dd_matmul(c2, c2.T)
    return DD(np.tril(L.hi), np.tril(L.lo))


def dd_cholsolve(L: DD, b) -> DD:
    m = L.shape[0]
    y = _dd(b).copy()
    for j in range(m):
        y[j] = y[j] / L[j, j]
        if j + 1 < m:
            y[j + 1:] = y[j + 1:] - L[j + 1:, j] * DD(np.full(m - j - 1, y.hi[j]),
                                                      np.full(m - j - 1, y.lo[j]))
    for j in range(m - 1, -1, -1):
        if j + 1 < m:
            y[j] = y[j] - dd_sum(L[j + 1:, j] * y[j + 1:])
        y[j] = y[j] / L[j, j]
    return y


def _col(v: DD) -> DD:
    return DD(v.hi[:, None], v.lo[:, None])


def _sym(M: DD) -> DD:
    return DD(0.5 * (M.hi + M.hi.T), 0.5 * (M.lo + M.lo.T))


class DDNewtonBackend(O.OracleBackend):
    """The FP64 oracle with the Newton system in double-double (one block)."""

    def __init__(self, prob):
        super().__init__(prob)
        if len(self.k) != 1 or self.n:
            raise ValueError("the Float64x2 Newton oracle takes one block and no equality rows")

    def _amul(self, v) -> DD:          # Σ v_i A_i (k×k)
        k = self.k[0]
        return dd_matmul(DD(self.Av[0].T), _col(_dd(v))).reshape(k, k, order="F")

    def _atmul(self, Z: DD) -> DD:     # ⟨A_i, Z⟩ for every i
        return dd_matmul(DD(self.Av[0]), _col(Z.reshape(-1, order="F"))).reshape(-1)

    def compute_residuals(self, mu, use_affine, factor):
        k = self.k[0]
        P = self._amul(self.x) - DD(self.X[0]) - DD(self.C[0])
        self.Pdd = P
        self.P[0] = P.to_float()
        self.block_norms[0] = float(np.max(np.abs(P.hi)))
        d = DD(self.c) - self._atmul(DD(self.Y[0]))
        self.ddd = d
        self.d = d.to_float()
        R = -dd_matmul(DD(self.X[0]), DD(self.Y[0]))
        if not use_affine:
            R = R + DD(mu[0] * np.eye(k))
        self.Rdd = R
        self.R[0] = R.to_float()
        ok = True
        if factor:
            ok1, self.LX[0] = O.kchol(self.X[0])
            ok2, self.MY[0] = O.kchol(self.Y[0])
            ok = ok1 and ok2
            if ok:
                self.Xi = dd_inverse_spd(self.X[0], steps=3)
        return self.block_norms[0], float(np.max(np.abs(self.d))), ok

    def schur_build(self, identity=False):
        k, m = self.k[0], self.m
        Yd = DD(self.Y[0])
        cols = [dd_matmul(dd_matmul(self.Xi, DD(self.Av[0][j].reshape(k, k, order="F"))), Yd)
                .reshape(-1, order="F") for j in range(m)]
        G = DD(np.stack([g.hi for g in cols], 1), np.stack([g.lo for g in cols], 1))
        full = dd_matmul(DD(self.Av[0]), G)           # S_ij = ⟨A_i, G_j⟩; the lower part
        lo_h, lo_l = np.tril(full.hi), np.tril(full.lo)  # is kept and mirrored
        self.Sdd = DD(lo_h + np.tril(lo_h, -1).T, lo_l + np.tril(lo_l, -1).T)
        self.S = np.tril(self.Sdd.to_float())
        return self.S

    def factorize(self):
        S = self.Sdd
        L = dd_cholesky(S)
        att, reg = 0, 0.0
        while L is None and att < 6:
            att += 1
            reg = O.SQRT_EPS if att == 1 else reg * 10
            Sb = S.copy()
            shift = np.maximum(np.abs(np.diag(S.hi)), 1.0) * reg
            for i in range(S.shape[0]):
                Sb[i, i] = Sb[i, i] + DD(shift[i])
            L = dd_cholesky(Sb)
        self.Ldd = L
        if L is None:
            return dict(ok=False, reg_attempts=att, quality=0.0)
        dg = np.abs(np.diag(L.hi))
        return dict(ok=True, reg_attempts=att, quality=float(np.clip(dg.min() / dg.max(), 0, 1)))

    def solve_direction(self):
        self.dxdd = dd_cholsolve(self.Ldd, self.rdd)
        self.dx = self.dxdd.to_float()

    def direction_residual(self):
        self.rhodd = self.rdd - dd_matmul(self.Sdd, _col(self.dxdd)).reshape(-1)
        self.rho = self.rhodd.to_float()
        return float(np.max(np.abs(self.rho))), float(np.max(np.abs(self.r)))

    def refine(self, policy, tol, cap, fixed_steps):
        if policy == "fixed":
            steps, limit, adaptive = 0, fixed_steps, False
        else:
            if cap <= 0:
                return 0, 0.0
            steps, limit, adaptive = 0, cap, True
        rel = tol if tol > 0 else O.REFINE_DEFAULT_TOL_ULPS * O.EPS
        abstol = rel * max(float(np.max(np.abs(self.r))), 1.0)
        residual, _ = self.direction_residual()
        for _ in range(limit):
            if adaptive and residual <= abstol:
                break
            best = self.dxdd.copy()
            self.dxdd = self.dxdd + dd_cholsolve(self.Ldd, self.rhodd)
            self.dx = self.dxdd.to_float()
            corrected, _ = self.direction_residual()
            if not math.isfinite(corrected) or corrected > residual:
                self.dxdd, self.dx = best, best.to_float()
                self.direction_residual()
                break
            steps += 1
            small = corrected > residual * O.REFINE_MIN_DECREASE
            residual = corrected
            if adaptive and small:
                break
        return steps, residual

    def _rhs_from_R(self):
        Z = dd_matmul(self.Xi, dd_matmul(self.Pdd, DD(self.Y[0])) - self.Rdd)
        self.rdd = -(self.ddd + self._atmul(Z))
        self.r = self.rdd.to_float()

    def direction_blocks(self):
        dX = self._amul(self.dxdd) + self.Pdd
        dY = _sym(dd_matmul(self.Xi, self.Rdd - dd_matmul(dX, DD(self.Y[0]))))
        self.dX[0] = dX.to_float()
        self.dY[0] = dY.to_float()

    def _corrector(self, target):
        k = self.k[0]
        R = -dd_matmul(DD(self.X[0]), DD(self.Y[0])) - dd_matmul(DD(self.dX[0]), DD(self.dY[0]))
        self.Rdd = R + DD(target * np.eye(k))
        self.R[0] = self.Rdd.to_float()
        self._rhs_from_R()

    def mehrotra_corrector_rhs(self, sigma, mu, block_local):
        kl = self.k[0]
        target = sigma * float(np.sum(self.X[0] * self.Y[0])) / kl if block_local else sigma * mu
        self._corrector(target)

    def fixed_corrector_rhs(self, beta, mu):
        kl = self.k[0]
        rl = float(np.sum((self.X[0] + self.dX[0]) * (self.Y[0] + self.dY[0]))) / mu[0] / kl
        self._corrector(max(rl * rl if rl < 1 else rl, beta) * mu[0])

    def solution_residuals(self):
        p, d, _ = self.compute_residuals([0.0], True, False)
        return p, d


def dd_newton_solve(prob, opts):
    """Complete solve with the Float64x2 Newton system (shared driver)."""
    from sdpx_b200.driver import solve_with_backend
    return solve_with_backend(DDNewtonBackend(prob), opts)
