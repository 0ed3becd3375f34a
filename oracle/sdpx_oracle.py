"""CPU oracle for the SDPX dense-SDP Newton step — TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only `tests/`,
`__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` may import it.
It restates, in NumPy/SciPy (LAPACK potrf/trsm through OpenBLAS), the Float64
kernels of the reference's hot path so that

  * the shared host driver (`sdpx_b200.driver`) run on this backend can be
    pinned against SDPX's own golden solves (benchmark/gates.jl,
    benchmark/baselines/gates.json, test/correctness.jl), and
  * the CUDA backend can be compared kernel-by-kernel (Schur matrix, KKT
    direction, residuals, step lengths) on the same iterate.

Parity pins: the gate problems `sdp_closed_form` and `sdp_dense`, the
fixed-policy T1 toy problem and the equality-row problems T2 (15 ± 2
iterations) and T3 (rank-deficient, rank-revealing QR) of
test/correctness.jl; see tests/test_oracle_gates.py.

Every method cites the reference function it follows (paths inside SDPX.jl).
"""
from __future__ import annotations

import math
from typing import List, Optional, Tuple

import numpy as np
import scipy.linalg as sla
from scipy.linalg import lapack

EPS = np.finfo(np.float64).eps
SQRT_EPS = math.sqrt(EPS)
REFINE_DEFAULT_TOL_ULPS = 64
REFINE_MIN_DECREASE = 0.5


# ---------------------------------------------------------------------------
#   Small dense kernels (src/kernels/generic.jl)
# ---------------------------------------------------------------------------

def kchol(A: np.ndarray) -> Tuple[bool, np.ndarray]:
    """No-throw lower Cholesky, src/kernels/generic.jl:133-155 (1×1 and 2×2
    closed forms, LAPACK potrf otherwise). Returns (ok, L) with L lower."""
    k = A.shape[0]
    if k == 1:
        d11 = A[0, 0]
        if not d11 > 0:
            return False, A.copy()
        return True, np.array([[math.sqrt(d11)]])
    if k == 2:
        d11 = A[0, 0]
        if not d11 > 0:
            return False, A.copy()
        l11 = math.sqrt(d11)
        l21 = A[1, 0] / l11
        d22 = A[1, 1] - l21 * l21
        if not d22 > 0:
            return False, A.copy()
        return True, np.array([[l11, 0.0], [l21, math.sqrt(d22)]])
    c, info = lapack.dpotrf(A, lower=1, clean=1)
    return info == 0, c


def kchol_lapack(A: np.ndarray) -> Tuple[bool, np.ndarray]:
    """`LinearAlgebra.cholesky!(Symmetric(A, :L); check=false)` (LAPACK potrf,
    every size) as the standard provider's `la_cholesky_factor!` calls it
    (src/la_backend.jl:686-698)."""
    if A.shape[0] == 0:
        return True, A.copy()
    c, info = lapack.dpotrf(A, lower=1, clean=1)
    return info == 0 and bool(np.all(np.isfinite(np.diag(c)))), c


def kcholsolve(L: np.ndarray, M: np.ndarray) -> np.ndarray:
    """M ← X⁻¹M from the lower factor, src/kernels/generic.jl:218-248."""
    k = L.shape[0]
    if k == 1:
        return M / L[0, 0] / L[0, 0]
    if k == 2:
        l11, l21, l22 = L[0, 0], L[1, 0], L[1, 1]
        y1 = M[0] / l11
        y2 = (M[1] - l21 * y1) / l22
        x2 = y2 / l22
        out = np.empty_like(M)
        out[0] = (y1 - l21 * x2) / l11
        out[1] = x2
        return out
    Y = sla.solve_triangular(L, M, lower=True, check_finite=False)
    return sla.solve_triangular(L, Y, lower=True, trans="T", check_finite=False)


def trial_isposdef(X, t, dX) -> bool:
    """src/kernels/generic.jl:292-309."""
    k = X.shape[0]
    if k == 1:
        return X[0, 0] + t * dX[0, 0] > 0
    if k == 2:
        a = X[0, 0] + t * dX[0, 0]
        if not a > 0:
            return False
        b = X[1, 0] + t * dX[1, 0]
        d = X[1, 1] + t * dX[1, 1]
        return a * d > b * b
    return kchol(X + t * dX)[0]


def trial_has_cholesky_margin(X, t, dX, ratio) -> bool:
    """src/kernels/generic.jl:318-340."""
    if not ratio > 0:
        return trial_isposdef(X, t, dX)
    ok, L = kchol(X + t * dX)
    if not ok:
        return False
    d = np.abs(np.diag(L))
    dmin, dmax = d.min(), d.max()
    return bool(np.isfinite(dmin) and np.isfinite(dmax) and dmax > 0 and dmin > ratio * dmax)


def fraction_to_boundary_bound(X, dX) -> float:
    """Largest step in [0,1] keeping X + t·dX positive definite,
    src/kernels/generic.jl:350-422 (closed forms for k ≤ 2, 64-step bisection)."""
    k = X.shape[0]
    if k == 1:
        d = dX[0, 0]
        return min(1.0, -X[0, 0] / d) if d < 0 else 1.0
    if k == 2:
        a, b, d = X[0, 0], X[0, 1], X[1, 1]
        da = dX[0, 0]
        db = (dX[0, 1] + dX[1, 0]) / 2.0
        dd = dX[1, 1]
        a1, b1, d1 = a + da, b + db, d + dd
        if a1 > 0 and a1 * d1 > b1 * b1:
            return 1.0
        c0 = a * d - b * b
        c1 = da * d + a * dd - 2.0 * b * db
        c2 = da * dd - db * db
        root, found = 1.0, False
        if c2 == 0:
            if c1 < 0:
                cand = -c0 / c1
                if 0 < cand <= 1:
                    root, found = cand, True
        else:
            disc = c1 * c1 - 4.0 * c2 * c0
            if disc >= 0:
                sd = math.sqrt(disc)
                den = 2.0 * c2
                cand1 = (-c1 - sd) / den
                cand2 = (-c1 + sd) / den
                if 0 < cand1 <= root:
                    root, found = cand1, True
                if 0 < cand2 <= root:
                    root, found = cand2, True
        if found:
            return root
    elif trial_isposdef(X, 1.0, dX):
        return 1.0
    lo, hi = 0.0, 1.0
    for _ in range(64):
        mid = (lo + hi) / 2.0
        if trial_isposdef(X, mid, dX):
            lo = mid
        else:
            hi = mid
    return lo


def symmetrize(M):
    """src/kernels/generic.jl:425-433."""
    return (M + M.T) / 2.0


def gershgorin_lower(M) -> float:
    """`_cold_start_psd_lower_bound` (src/cold_start.jl:152-186), lower triangle authoritative."""
    k = M.shape[0]
    if k == 1:
        return M[0, 0]
    if k == 2:
        c = (M[0, 0] + M[1, 1]) / 2
        r = math.hypot((M[0, 0] - M[1, 1]) / 2, M[1, 0])
        return c - r
    Lw = np.tril(M)
    S = Lw + np.tril(Lw, -1).T
    off = np.abs(S).sum(axis=1) - np.abs(np.diag(S))
    return float(np.min(np.diag(S) - off))


# ---------------------------------------------------------------------------
#   Ruiz equilibration (src/ingest.jl:1431-1519)
# ---------------------------------------------------------------------------

def equilibrate_problem(Av: List[np.ndarray], C: List[np.ndarray], c: np.ndarray, k: List[int]):
    """Dense `equilibrate`: per-block adaptive Ruiz congruence (2..8 passes,
    log tolerance 1/20), then per-variable scale s_i = max_l ‖A_i^(l)‖∞ and a
    single objective scale. Returns scaled copies and (E, s, objective_scale)."""
    Av2 = [a.copy() for a in Av]
    C2 = [x.copy() for x in C]
    E = [np.ones(kl) for kl in k]
    passes = []
    m = c.shape[0]
    for l, kl in enumerate(k):
        A3 = Av2[l].reshape(m, kl, kl)
        used = 0
        for it in range(1, 9):
            used = it
            rn = np.abs(C2[l]).max(axis=1)
            rn = np.maximum(rn, np.abs(A3).max(axis=(0, 2)))
            pos = rn[rn > 0]
            converged = it >= 2 and (np.all(np.isfinite(pos)) and
                                     (pos.size == 0 or np.max(np.abs(np.log(pos))) <= 1.0 / 20.0))
            e = np.where(rn > 0, 1.0 / np.sqrt(np.where(rn > 0, rn, 1.0)), 1.0)
            C2[l] *= np.outer(e, e)
            A3 *= np.outer(e, e)[None, :, :]
            E[l] *= e
            if converged:
                break
        passes.append(used)
    maxima = np.zeros(m)
    for l in range(len(k)):
        maxima = np.maximum(maxima, np.abs(Av2[l]).max(axis=1))
    s = np.where(maxima > 0, maxima, 1.0)
    cc = c / s
    objective_scale = float(np.max(np.abs(cc))) if cc.size else 0.0
    if not (objective_scale > 0 and math.isfinite(objective_scale)):
        objective_scale = 1.0
    cc = cc / objective_scale
    for l in range(len(k)):
        Av2[l] /= s[:, None]
    return Av2, C2, cc, E, s, objective_scale, passes


# ---------------------------------------------------------------------------
#   Equality block of the KKT system (src/kkt.jl)
# ---------------------------------------------------------------------------

QR_MAX_COLUMNS = 2048          # `_equality_qr_allowed`, Float64 (src/kkt.jl:553-576)
QR_MAX_ELEMENTS = 50_000_000   # `_equality_qr_maximum_elements`, Float64 (src/kkt.jl:540-551)


def equality_rank_tau(rows: int, cols: int, requested: float) -> float:
    """`_equality_cholesky_rank_tau`, Float64 branch (src/kkt.jl:76-112):
    max(max(rows, cols)·eps, min(√eps, requested accuracy))."""
    if not requested > 0:
        requested = SQRT_EPS
    requested = min(SQRT_EPS, requested)
    return max(float(max(rows, cols)) * EPS, min(SQRT_EPS, requested))


def normalize_equality_columns(Bt: np.ndarray):
    """`_normalize_equality_panel_columns!` (src/kkt.jl:281-304): column j is
    multiplied by 1/‖B̃[:, j]‖∞ (zero columns, and reciprocals that overflow,
    keep scale one).  Returns (B̂, scale)."""
    n = Bt.shape[1]
    scale = np.ones(n)
    out = Bt.copy()
    for j in range(n):
        norm = float(np.max(np.abs(Bt[:, j]))) if Bt.shape[0] else 0.0
        s = 1.0 if norm == 0.0 else 1.0 / norm
        if not math.isfinite(s):
            s = 1.0
        scale[j] = s
        if s != 1.0:
            out[:, j] = Bt[:, j] * s
    return out, scale


def has_exact_duplicate_columns(M: np.ndarray) -> bool:
    """`_has_exact_duplicate_columns` (src/kkt.jl:411-440): two columns equal
    entry by entry (signed zeros equal, NaN never equal)."""
    n = M.shape[1]
    for i in range(n - 1):
        for j in range(i + 1, n):
            if np.array_equal(M[:, i], M[:, j]):
                return True
    return False


def cholesky_has_numerical_rank(Lq: np.ndarray, Bt: np.ndarray, tau: float) -> bool:
    """`_cholesky_has_numerical_rank` (src/kkt.jl:114-178) on the factor's
    diagonal: min|L_jj| > τ·max|L_jj|, and in the suspicious band
    min ≤ √τ·max no two columns of B̂ may be exactly equal."""
    if Lq.shape[0] == 0:
        return True
    d = np.abs(np.diag(Lq))
    if not np.all(np.isfinite(d)):
        return False
    lo, hi = float(d.min()), float(d.max())
    if not hi > 0:
        return False
    if not lo > tau * hi:
        return False
    if lo <= math.sqrt(tau) * hi and has_exact_duplicate_columns(Bt):
        return False
    return True


def equality_qr_allowed(rows: int, cols: int) -> bool:
    """Dimension gates of `_equality_qr_allowed` (src/kkt.jl:553-576)."""
    return 0 < cols <= QR_MAX_COLUMNS and rows * cols <= QR_MAX_ELEMENTS


def equality_qr(Bt: np.ndarray, tau: float):
    """`la_qr_factor!(…; pivoted=true)` (src/la_backend.jl:823-850: LAPACK
    geqp3, column-norm pivoting) and `_equality_qr_factor_handle`
    (src/la_backend.jl:956-1024): rank = leading count of |R_jj| > τ·max|R_jj|,
    quality = min/max over those diagonals.  Returns (R, perm, rank, quality)."""
    R, perm = sla.qr(Bt, mode="r", pivoting=True, check_finite=False)
    d = np.abs(np.diag(R))
    largest = float(d.max()) if d.size else 0.0
    threshold = tau * largest
    rank, smallest = 0, largest
    for v in d:
        if not v > threshold:
            break
        rank += 1
        smallest = min(smallest, float(v))
    quality = min(max(smallest / largest, 0.0), 1.0) if rank > 0 and largest > 0 else 0.0
    return R, np.asarray(perm, dtype=np.int64), rank, quality


def equality_qr_solve(R: np.ndarray, perm: np.ndarray, rank: int, rhs: np.ndarray) -> np.ndarray:
    """`la_factor_solve!(::EqualityQRFactor)` (src/la_backend.jl:1425-1455):
    RᵀR z = rhs[perm] on the leading rank×rank block, dependent directions
    zero, scattered back through the permutation."""
    z = np.array(rhs[perm[:rank]], dtype=np.float64)
    for row in range(rank):
        v = z[row]
        for col in range(row):
            v -= R[col, row] * z[col]
        z[row] = v / R[row, row]
    for row in range(rank - 1, -1, -1):
        v = z[row]
        for col in range(row + 1, rank):
            v -= R[row, col] * z[col]
        z[row] = v / R[row, row]
    out = np.zeros(rhs.shape[0])
    out[perm[:rank]] = z
    return out


# ---------------------------------------------------------------------------
#   Backend: the driver seam (see sdpx_b200.driver)
# ---------------------------------------------------------------------------

class OracleBackend:
    """NumPy restatement of the reference's dense Float64 kernels behind the
    same method set as the CUDA backend."""

    def __init__(self, prob):
        self.prob0 = prob
        self.k = list(prob.k)
        self.m = prob.m
        self.n = prob.n
        self.Av = [a.copy() for a in prob.Av]
        self.C = [x.copy() for x in prob.C]
        self.c = prob.c.copy()
        self.B = np.array(prob.B, dtype=np.float64).reshape(self.m, self.n)
        self.b = np.array(prob.b, dtype=np.float64).reshape(self.n)
        L = len(self.k)
        self.x = np.zeros(self.m)
        self.y = np.zeros(self.n)
        self.p = np.zeros(self.n)          # b − Bᵀx
        self.dy = np.zeros(self.n)
        self.rho_p = np.zeros(self.n)      # p − Bᵀdx
        self.eq = None                     # current equality factor
        self.eq_qr_sticky = False
        self.requested_accuracy = SQRT_EPS
        self.equality_solver = "auto"
        self.X = [np.eye(kl) for kl in self.k]
        self.Y = [np.eye(kl) for kl in self.k]
        self.P = [None] * L
        self.R = [None] * L
        self.LX = [None] * L
        self.MY = [None] * L
        self.dX = [None] * L
        self.dY = [None] * L
        self.block_norms = np.zeros(L)
        self.d = np.zeros(self.m)
        self.r = np.zeros(self.m)
        self.dx = np.zeros(self.m)
        self.rho = np.zeros(self.m)
        self.S = None
        self.Sfac = None
        self.kept = {}
        self.best = None
        self.eq_applied = False
        self.sparse_schur = False      # `sparse = :on`: the SparseCons Schur path

    # -- helpers -----------------------------------------------------------
    def _mat(self, l, vec):
        kl = self.k[l]
        return vec.reshape(kl, kl)

    def _buildP(self, l, x):          # src/schur.jl:36-39
        return self._mat(l, x @ self.Av[l])

    def _accumulate(self, l, M):      # src/schur.jl:41-44 (⟨A_i, M⟩ for all i)
        return self.Av[l] @ M.reshape(-1)

    def configure_equality(self, requested_accuracy, solver):
        """Options the equality factor reads: `_requested_accuracy`
        (src/kkt.jl:518-521) and `equality_solver` (src/types/workspaces.jl:181)."""
        if solver not in ("auto", "qr"):
            raise NotImplementedError(f"equality_solver={solver!r}")
        self.requested_accuracy = float(requested_accuracy)
        self.equality_solver = solver

    def precision_label(self):
        return "fp64"

    def precision_history(self):
        return []

    def begin_iteration(self, info):
        pass

    def fallback_to_fp64(self, reason):
        return False

    # -- problem-level ------------------------------------------------------
    def equilibrate(self):
        from sdpx_b200.problem import Equilibration
        Av2, C2, cc, E, s, objscale, passes = equilibrate_problem(self.Av, self.C, self.c, self.k)
        self.Av, self.C, self.c = Av2, C2, cc
        self.B = self.B / s[:, None]       # `_scale_equality_rows!` (src/ingest.jl:1176-1184)
        self.eq_applied = True
        return Equilibration(E, s, objscale, passes)

    def data_norms(self):
        maxC = max((float(np.max(np.abs(Cl))) for Cl in self.C), default=0.0)
        bn = float(np.max(np.abs(self.b))) if self.n else 0.0
        return maxC, float(np.max(np.abs(self.c))) if self.m else 0.0, bn

    def fixed_start(self, omega_p, omega_d):
        self.x = np.zeros(self.m)
        self.y = np.zeros(self.n)
        self.X = [omega_p * np.eye(kl) for kl in self.k]
        self.Y = [omega_d * np.eye(kl) for kl in self.k]

    # -- residuals (src/kernels/threaded.jl:423-506, src/step.jl:25-93) ------
    def compute_residuals(self, mu, use_affine, factor):
        d = self.c.copy()
        for l in range(len(self.k)):
            P = self._buildP(l, self.x) - self.X[l] - self.C[l]
            self.P[l] = P
            self.block_norms[l] = np.max(np.abs(P)) if P.size else 0.0
            d -= self._accumulate(l, self.Y[l])
        if self.n:
            d -= self.B @ self.y                      # src/step.jl:41
            self.p = self.b - self.B.T @ self.x       # src/step.jl:43-45
        self.d = d
        p_res = float(np.max(self.block_norms)) if len(self.k) else 0.0
        if self.n:
            p_res = max(p_res, float(np.max(np.abs(self.p))))   # src/step.jl:51
        d_res = float(np.max(np.abs(d))) if d.size else 0.0
        ok = True
        for l in range(len(self.k)):
            R = -(self.X[l] @ self.Y[l])
            if not use_affine:
                R = R + mu[l] * np.eye(self.k[l])
            self.R[l] = R
            if factor:
                ok1, self.LX[l] = kchol(self.X[l])
                ok2, self.MY[l] = kchol(self.Y[l])
                ok = ok and ok1 and ok2
        return p_res, d_res, ok

    def block_primal_residual(self):
        return float(np.max(self.block_norms)) if len(self.k) else 0.0

    # -- Schur (src/schur.jl:511-562) -----------------------------------------
    def schur_build(self, identity=False):
        m = self.m
        if self.sparse_schur and not identity:
            # SparseCons path (src/schur.jl:936-1032, 1173-1197)
            from oracle.sparse_oracle import sparse_schur_build
            self.S = sparse_schur_build(self.Av, self.k, self.LX, self.Y, m)
            return self.S
        S = np.zeros((m, m))
        for l, kl in enumerate(self.k):
            A3 = self.Av[l].reshape(m, kl, kl)
            if identity:
                Phat = self.Av[l]
            else:
                # Ppanel = L_X⁻¹ [A_1 … A_m] (batched trsm), then block·M_Y
                panel = np.transpose(A3, (1, 0, 2)).reshape(kl, m * kl)   # [A_1 A_2 …]
                T = sla.solve_triangular(self.LX[l], panel, lower=True, check_finite=False)
                T3 = T.reshape(kl, m, kl).transpose(1, 0, 2)               # T_i
                P3 = T3 @ self.MY[l]
                Phat = P3.transpose(0, 2, 1).reshape(m, kl * kl)             # vec (column-major)
            S += Phat @ Phat.T
        self.S = np.tril(S)
        return self.S

    def schur_matrix(self):
        return np.tril(self.S) + np.tril(self.S, -1).T

    # -- KKT (src/kkt.jl:1404-1445, 2570-2595, 3634-3963) ----------------------
    def factorize(self):
        Sfull = self.schur_matrix()
        ok, Lf = kchol(Sfull)
        attempts, reg = 0, 0.0
        while not ok and attempts < 6:
            attempts += 1
            reg = SQRT_EPS if attempts == 1 else reg * 10
            Sb = Sfull.copy()
            Sb[np.diag_indices_from(Sb)] += reg * np.maximum(np.abs(np.diag(Sfull)), 1.0)
            ok, Lf = kchol(Sb)
        self.Sfac = Lf if ok else None
        if not ok:
            return dict(ok=False, reg_attempts=attempts, quality=0.0)
        dg = np.abs(np.diag(Lf))
        q = float(np.clip(dg.min() / dg.max(), 0, 1)) if dg.max() > 0 and np.isfinite(dg.max()) else 0.0
        rank_deficient = False
        if self.n:
            ok_eq, rank_deficient = self._factor_equality()
            if not ok_eq:
                return dict(ok=False, reg_attempts=attempts, quality=0.0)
            if self.eq[0] == "qr":
                q = min(q, self.eq[4])       # `_kkt_factorization_quality` (src/step.jl:338-345)
        if rank_deficient:
            q = 0.0                          # src/step.jl:797-801
        return dict(ok=True, reg_attempts=attempts, quality=q)

    def _factor_equality(self):
        """Equality part of `_factor_dense_kkt_native!` (src/kkt.jl:1466-1680)
        for the standard Float64 provider: B̃ = L_S⁻¹B with unit-∞-norm columns,
        then Q = B̃ᵀB̃ by Cholesky with the rank test, or the column-pivoted QR
        of B̃ when that test fails (`:standard_compatibility`) or QR was
        already in use.  Returns (ok, rank_deficient)."""
        Bt = sla.solve_triangular(self.Sfac, self.B, lower=True, check_finite=False)
        Bt, scale = normalize_equality_columns(Bt)
        tau = equality_rank_tau(Bt.shape[0], Bt.shape[1], self.requested_accuracy)
        direct_qr = self.equality_solver == "qr" or self.eq_qr_sticky
        self.eq = None
        if not direct_qr:
            Q = Bt.T @ Bt
            ok, Lq = kchol_lapack(Q)
            if ok and cholesky_has_numerical_rank(Lq, Bt, tau):
                self.eq = ("chol", Bt, scale, Lq)
                return True, False
            if not equality_qr_allowed(*Bt.shape):
                return False, False
        R, perm, rank, quality = equality_qr(Bt, tau)
        self.eq = ("qr", Bt, scale, (R, perm, rank), quality)
        self.eq_qr_sticky = True
        return True, rank < self.n

    def _solve_Q(self, rhs):
        """`_solve_Q!` (src/kkt.jl:2407-2486) for the current equality factor."""
        if self.eq[0] == "chol":
            Lq = self.eq[3]
            z = sla.solve_triangular(Lq, rhs, lower=True, check_finite=False)
            return sla.solve_triangular(Lq, z, lower=True, trans="T", check_finite=False)
        R, perm, rank = self.eq[3]
        return equality_qr_solve(R, perm, rank, rhs)

    def _solve(self, rhs, prhs=None):
        """`_solve_dense_kkt_owned!` (src/kkt.jl:2570-2595).  Returns (dx, dy)."""
        rt = sla.solve_triangular(self.Sfac, rhs, lower=True, check_finite=False)
        if not self.n:
            return sla.solve_triangular(self.Sfac, rt, lower=True, trans="T",
                                        check_finite=False), np.zeros(0)
        _, Bt, scale = self.eq[:3]
        q = scale * prhs - Bt.T @ rt                 # `_form_scaled_equality_rhs!`
        dyh = self._solve_Q(q)
        dx = sla.solve_triangular(self.Sfac, rt + Bt @ dyh, lower=True, trans="T",
                                  check_finite=False)
        return dx, dyh * scale                       # `_recover_original_equality_multiplier!`

    def solve_direction(self):
        self.dx, self.dy = self._solve(self.r, self.p if self.n else None)

    def _schur_mul(self, v):
        return self.schur_matrix() @ v

    def direction_residual(self):
        """`_kkt_direction_residual!` (src/kkt.jl:3689-3708): ρ = r − S·dx + B·dy,
        ρ_p = p − Bᵀdx.  Returns (max(‖ρ‖∞, ‖ρ_p‖∞), max(‖r‖∞, ‖p‖∞)); the second
        value is the scale of the acceptance and cold-start gates
        (src/kkt.jl:3670-3687, src/solver/interior_point.jl:785-789)."""
        self.rho = self.r - self._schur_mul(self.dx)
        res = float(np.max(np.abs(self.rho)))
        rn = float(np.max(np.abs(self.r)))
        if self.n:
            self.rho = self.rho + self.B @ self.dy
            self.rho_p = self.p - self.B.T @ self.dx
            res = max(float(np.max(np.abs(self.rho))), float(np.max(np.abs(self.rho_p))))
            rn = max(rn, float(np.max(np.abs(self.p))))
        return res, rn

    def _correct(self):
        """`_apply_kkt_correction!` (src/kkt.jl:3762-3780)."""
        ddx, ddy = self._solve(self.rho, self.rho_p if self.n else None)
        self.dx = self.dx + ddx
        if self.n:
            self.dy = self.dy + ddy

    def refine(self, policy, tol, cap, fixed_steps):
        """`_refine_native_direction!` (src/kkt.jl:3891-3963)."""
        if policy == "fixed":
            steps = 0
            residual, _ = self.direction_residual()
            for _ in range(fixed_steps):
                best = (self.dx.copy(), self.dy.copy())
                self._correct()
                corrected, _ = self.direction_residual()
                if not math.isfinite(corrected) or corrected > residual:
                    self.dx, self.dy = best
                    break
                steps += 1
                residual = corrected
            return steps, residual
        if cap <= 0:
            return 0, 0.0
        rel = tol if tol > 0 else REFINE_DEFAULT_TOL_ULPS * EPS
        abstol = rel * max(float(np.max(np.abs(self.r))), 1.0)
        steps = 0
        residual, _ = self.direction_residual()
        for _ in range(cap):
            if residual <= abstol:
                break
            best = (self.dx.copy(), self.dy.copy())
            self._correct()
            corrected, _ = self.direction_residual()
            if not math.isfinite(corrected) or corrected > residual:
                self.dx, self.dy = best
                break
            steps += 1
            small = corrected > residual * REFINE_MIN_DECREASE
            residual = corrected
            if small:
                break
        return steps, residual

    # -- RHS and directions (src/step.jl:95-108, src/kernels/threaded.jl:542-1067)
    def _rhs_from_R(self):
        v = np.zeros(self.m)
        for l in range(len(self.k)):
            Z = self.P[l] @ self.Y[l] - self.R[l]
            Z = kcholsolve(self.LX[l], Z)
            v += self._accumulate(l, Z)
        self.r = -(self.d + v)

    def predictor_rhs(self):
        self._rhs_from_R()

    def direction_blocks(self):
        for l in range(len(self.k)):
            dX = self._buildP(l, self.dx) + self.P[l]
            dY = self.R[l] - dX @ self.Y[l]
            dY = kcholsolve(self.LX[l], dY)
            self.dX[l] = dX
            self.dY[l] = symmetrize(dY)

    def affine_diagnostics(self, adaptive):
        """`_affine_predictor_diagnostics!` / `_legacy_predictor_diagnostics!`
        (src/step.jl:546-619)."""
        L = len(self.k)
        if adaptive:
            bX = min((fraction_to_boundary_bound(self.X[l], self.dX[l]) for l in range(L)), default=1.0)
            bY = min((fraction_to_boundary_bound(self.Y[l], self.dY[l]) for l in range(L)), default=1.0)
            tX = bX if bX < 1 else 1.0
            tY = bY if bY < 1 else 1.0
        else:
            tX = tY = 1.0
        compl = 0.0
        aff = 0.0
        uniform = adaptive
        ref = None
        for l in range(L):
            val = float(np.sum(self.X[l] * self.Y[l]))
            compl += val
            kl = self.k[l]
            if adaptive and kl > 0:
                if not math.isfinite(val):
                    uniform = False
                elif ref is None:
                    ref = (val, kl)
                elif not ((kl == ref[1] and val == ref[0]) or
                          (kl != ref[1] and val / kl == ref[0] / ref[1])):
                    uniform = False
            aff += float(np.sum((self.X[l] + tX * self.dX[l]) * (self.Y[l] + tY * self.dY[l])))
        den = float(max(sum(self.k), 1))
        mu = compl / den
        mu_aff = max(0.0, aff / den)
        if adaptive:
            quality = min(max(mu_aff / mu, 0.0), 2.0) if mu > 0 else 1.0
        else:
            quality = min(max(aff / compl, 0.0), 2.0) if compl > 0 else 1.0
        return dict(complementarity=compl, affine_complementarity=aff, mu=mu, mu_aff=mu_aff,
                    quality=quality, tX=tX, tY=tY, uniform=uniform)

    def block_margins(self):
        """`_block_factorization_margins` (src/step.jl:273-281)."""
        def q(Lm):
            d = np.abs(np.diag(Lm))
            if d.size == 0:
                return 1.0
            return float(np.clip(d.min() / d.max(), 0, 1)) if d.max() > 0 and np.isfinite(d.max()) else 0.0
        p = min((q(Lm) for Lm in self.LX), default=1.0)
        dd = min((q(Lm) for Lm in self.MY), default=1.0)
        return min(1.0, p), min(1.0, dd)

    def mehrotra_corrector_rhs(self, sigma, mu, block_local):
        """src/kernels/threaded.jl:916-1067."""
        for l, kl in enumerate(self.k):
            if block_local:
                target = sigma * float(np.sum(self.X[l] * self.Y[l])) / kl
            else:
                target = sigma * mu
            R = -(self.X[l] @ self.Y[l]) - self.dX[l] @ self.dY[l]
            R[np.diag_indices(kl)] += target
            self.R[l] = R
        self._rhs_from_R()

    def fixed_corrector_rhs(self, beta, mu):
        """src/kernels/threaded.jl:837-901."""
        for l, kl in enumerate(self.k):
            rl = float(np.sum((self.X[l] + self.dX[l]) * (self.Y[l] + self.dY[l]))) / mu[l] / kl
            gl = max(rl * rl if rl < 1 else rl, beta)
            R = -(self.X[l] @ self.Y[l]) - self.dX[l] @ self.dY[l]
            R[np.diag_indices(kl)] += gl * mu[l]
            self.R[l] = R
        self._rhs_from_R()

    # -- step length (src/kernels/threaded.jl:1602-1818) ---------------------
    def line_search(self, rule, fp, fd, gamma, min_step, margin):
        L = len(self.k)
        if rule == "fraction_to_boundary":
            bX = min((fraction_to_boundary_bound(self.X[l], self.dX[l]) for l in range(L)), default=1.0)
            bY = min((fraction_to_boundary_bound(self.Y[l], self.dY[l]) for l in range(L)), default=1.0)
            return (fp * bX if bX < 1 else 1.0), (fd * bY if bY < 1 else 1.0)
        tX = 1.0
        while True:
            ok = all(trial_has_cholesky_margin(self.X[l], tX, self.dX[l], margin) for l in range(L))
            if ok or tX < min_step:
                break
            tX *= gamma
        tY = 1.0
        while True:
            ok = all(trial_has_cholesky_margin(self.Y[l], tY, self.dY[l], margin) for l in range(L))
            if ok or tY < min_step:
                break
            tY *= gamma
        return tX, tY

    # -- update (src/kernels/threaded.jl:665-835, interior_point.jl:1287-1321)
    def update(self, tX, tY):
        dots = []
        finite = True
        for l in range(len(self.k)):
            self.X[l] = self.X[l] + tX * self.dX[l]
            self.Y[l] = self.Y[l] + tY * self.dY[l]
            dots.append(float(np.sum(self.X[l] * self.Y[l])))
            finite = finite and bool(np.all(np.isfinite(self.X[l])) and np.all(np.isfinite(self.Y[l])))
        self.x = self.x + tX * self.dx
        finite = finite and bool(np.all(np.isfinite(self.x)))
        if self.n:                       # src/solver/interior_point.jl:2228-2229
            self.y = self.y + tY * self.dy
            finite = finite and bool(np.all(np.isfinite(self.y)))
        return float(sum(dots)), finite, dots

    def accepted_trial_residuals(self, block_primal_residual, tX, tY):
        p_after = abs(1.0 - tX) * block_primal_residual
        if self.n:                       # p+ = (1 − tX)p + tX·ρ_p
            self.p = (1.0 - tX) * self.p + tX * self.rho_p
            p_after = max(p_after, float(np.max(np.abs(self.p))))
        self.d = (1.0 - tY) * self.d - tY * self.rho
        return p_after, float(np.max(np.abs(self.d))) if self.d.size else 0.0

    def objectives(self):
        pObj = float(self.c @ self.x)
        dObj = float(sum(np.sum(Cl * Yl) for Cl, Yl in zip(self.C, self.Y)))
        if self.n:                       # src/kernels/threaded.jl:833
            dObj += float(self.b @ self.y)
        return pObj, dObj

    def solution_residuals(self):
        """`solution_residuals` (src/validation.jl:15-60) on the working problem."""
        p = 0.0
        d = self.c.copy()
        for l in range(len(self.k)):
            P = self._buildP(l, self.x) - self.X[l] - self.C[l]
            p = max(p, float(np.max(np.abs(P))))
            d -= self._accumulate(l, self.Y[l])
        if self.n:
            d -= self.B @ self.y
            p = max(p, float(np.max(np.abs(self.b - self.B.T @ self.x))))
        return p, float(np.max(np.abs(d))) if d.size else 0.0

    # -- cold start helpers ----------------------------------------------------
    def set_rhs(self, which):
        if which == "cold_primal":
            r = np.zeros(self.m)
            for l in range(len(self.k)):
                r += self._accumulate(l, self.C[l])
            self.r = r
            self.p = self.b.copy()       # src/solver/interior_point.jl:820
        elif which == "cold_dual":
            self.r = self.c.copy()
            self.p = np.zeros(self.n)    # src/solver/interior_point.jl:860-861
        else:
            raise ValueError(which)

    def keep_direction_as(self, name):
        self.kept[name] = self.dx.copy()

    def cold_start_iterate(self):
        x = self.kept["x"]
        v = self.dx
        self.x = x.copy()
        self.X = [self._buildP(l, x) - self.C[l] for l in range(len(self.k))]
        self.Y = [self._buildP(l, v) for l in range(len(self.k))]
        self.y = -self.dy                # src/solver/interior_point.jl:920-923

    def _psd_stats(self, M):
        low = np.tril(M)
        if not np.all(np.isfinite(low)):
            return False, 0.0, 0.0
        return True, float(np.max(np.abs(low))), gershgorin_lower(M)

    def _psd_shift_block(self, M):
        """`_cold_start_psd_shift!` (src/cold_start.jl:287-308)."""
        finite, scale, margin = self._psd_stats(M)
        if not finite:
            return False
        safety = SQRT_EPS * max(1.0, scale)
        slack = 8.0 * EPS * max(1.0, scale)
        if margin > safety:
            return True
        for _ in range(16):
            shift = safety - margin + slack
            if not math.isfinite(shift):
                return False
            M[np.diag_indices_from(M)] += shift
            finite, scale, margin = self._psd_stats(M)
            if not finite:
                return False
            safety = SQRT_EPS * max(1.0, scale)
            if margin > safety:
                return True
        return False

    def psd_shift(self, which):
        mats = self.X if which == "X" else self.Y
        ok = True
        for M in mats:
            ok = self._psd_shift_block(M) and ok
        return ok

    def add_identity(self, which, shift):
        for M in (self.X if which == "X" else self.Y):
            M[np.diag_indices_from(M)] += shift

    def block_dots(self):
        dots = [float(np.sum(X * Y)) for X, Y in zip(self.X, self.Y)]
        return dots, [float(np.trace(X)) for X in self.X], [float(np.trace(Y)) for Y in self.Y]

    def scale_iterate(self, which, factor):
        if which == "X":
            self.X = [factor * X for X in self.X]
        else:
            self.Y = [factor * Y for Y in self.Y]

    def store_best(self):
        self.best = (self.x.copy(), [X.copy() for X in self.X], [Y.copy() for Y in self.Y],
                     self.y.copy())

    def restore_best(self):
        if self.best is not None:
            self.x, self.X, self.Y = self.best[0].copy(), [X.copy() for X in self.best[1]], \
                [Y.copy() for Y in self.best[2]]
            self.y = self.best[3].copy()

    def set_iterate(self, x, X, Y, y=None):
        self.x = np.array(x, dtype=np.float64)
        self.y = np.zeros(self.n) if y is None else np.array(y, dtype=np.float64).reshape(self.n)
        self.X = [np.array(M, dtype=np.float64) for M in X]
        self.Y = [np.array(M, dtype=np.float64) for M in Y]

    def get_direction(self):
        return self.dx.copy(), [M.copy() for M in self.dX], [M.copy() for M in self.dY]

    def get_equality_direction(self):
        return self.dy.copy()

    def adjoint(self, wx=None, wy=None, WX=None, WY=None, A_index=()):
        """Gradient of L = ⟨wx, x⟩ + ⟨wy, y⟩ + Σ_l ⟨WX_l, X_l⟩ + Σ_l ⟨WY_l, Y_l⟩
        at the current iterate with respect to c, b, C_l and the selected A_i,
        through the Newton system the solver factors (the reference has no
        adjoint; this restates the implicit-function derivative of the
        linearised KKT conditions and is pinned by finite differences).

        The HKM-linearised KKT map from data residuals (P, d, p) to (dx, dy) is
        dX = 𝒜dx + P, dY = −sym(X⁻¹dX·Y), S·dx − B·dy = r with
        r = −d − 𝒜ᵀ(X⁻¹PY), Bᵀdx = p.  With G = X⁻¹·sym(WY)·Y the seed on dx is
        w = wx + 𝒜ᵀWX − 𝒜ᵀG, one KKT solve with right-hand side (w, −wy) gives
        λx = dx and λy = −dy, and with Λ = mat(𝒜λx):
            ∂L/∂c = −λx,  ∂L/∂b = λy,
            ∂L/∂C_l = sym(X⁻¹ΛY) − sym(WX − G),
            ∂L/∂A_i = λx_i·Y − x_i·∂L/∂C  (per block)."""
        L = len(self.k)
        w = np.zeros(self.m) if wx is None else np.array(wx, dtype=np.float64)
        D = []
        for l in range(L):
            kl = self.k[l]
            Dl = np.zeros((kl, kl))
            if WX is not None:
                Dl = Dl + WX[l]
                w = w + self._accumulate(l, WX[l])
            if WY is not None:
                Ws = symmetrize(np.asarray(WY[l], dtype=np.float64))
                Gl = kcholsolve(self.LX[l], Ws @ self.Y[l])
                Dl = Dl - Gl
                w = w - self._accumulate(l, Gl)
            D.append(Dl)
        pr = None
        if self.n:
            pr = -(np.zeros(self.n) if wy is None else np.asarray(wy, dtype=np.float64))
        lx, mdy = self._solve(w, pr)
        ly = -mdy if self.n else np.zeros(0)
        gC = []
        for l in range(L):
            Lam = self._buildP(l, lx)
            Z = kcholsolve(self.LX[l], Lam @ self.Y[l])
            gC.append(symmetrize(Z) - symmetrize(D[l]))
        gA = [[lx[i] * self.Y[l] - self.x[i] * gC[l] for l in range(L)] for i in A_index]
        return dict(grad_c=-lx, grad_b=ly, grad_C=gC, grad_A=gA, lambda_x=lx, lambda_y=ly)

    def equality_info(self):
        """(kind, rank, quality) of the current equality factor."""
        if self.eq is None:
            return "none", 0, 0.0
        if self.eq[0] == "chol":
            return "normal_equations", self.n, 1.0
        return "rank_revealing_qr", int(self.eq[3][2]), float(self.eq[4])

    def get_rhs(self):
        return self.r.copy()

    def get_iterate(self):
        return self.x.copy(), [X.copy() for X in self.X], self.y.copy(), [Y.copy() for Y in self.Y]

    # -- original coordinates -------------------------------------------------
    def restore_original(self):
        pass

    def original_c(self):
        return self.prob0.c

    def original_C(self):
        return self.prob0.C

    def original_b(self):
        return self.prob0.b

    def rebuild_slack(self, x):
        p = self.prob0
        return [(x @ p.Av[l]).reshape(p.k[l], p.k[l]) - p.C[l] for l in range(p.L)]

    def original_residuals(self, x, X, y, Y):
        p = self.prob0
        pr = 0.0
        d = p.c.copy()
        for l in range(p.L):
            P = (x @ p.Av[l]).reshape(p.k[l], p.k[l]) - X[l] - p.C[l]
            pr = max(pr, float(np.max(np.abs(P))))
            d -= p.Av[l] @ Y[l].reshape(-1)
        if p.n:
            B = np.asarray(p.B, dtype=np.float64).reshape(p.m, p.n)
            d -= B @ np.asarray(y, dtype=np.float64)
            pr = max(pr, float(np.max(np.abs(np.asarray(p.b) - B.T @ np.asarray(x)))))
        return pr, float(np.max(np.abs(d))) if d.size else 0.0


def oracle_solve(prob, opts=None, trace=None):
    """Full CPU solve: the shared driver on the NumPy kernels."""
    from sdpx_b200.controller import SolverOptions
    from sdpx_b200.driver import solve_with_backend
    if opts is None:
        opts = SolverOptions().with_tolerance(1e-8)
    return solve_with_backend(OracleBackend(prob), opts, trace=trace)
