"""CPU oracle of SDPX's cold-path result certificate — TEST INFRASTRUCTURE ONLY.

Only `tests/` may import this module.  It restates `result_certificate`
(src/validation.jl:948-1115) for the optimality kind of a dense SDP, with
equality rows Bᵀx = b when they are given, and its helpers:

* `solution_residuals` (src/validation.jl:15-56),
* `_primal_block_backward_errors` (:526-600, dense branch),
* `_dual_backward_errors` (:666-740, dense branch) with the equality terms of
  `_accumulate_equality_dual_scales!` (:629-644),
* `_equality_backward_errors` (:454-482, dense B),
* `_componentwise_backward_errors` / `_componentwise_ratio` (:418-431, :506-513),
* `_block_psd_certificate`, `_blocks_psd_certificate`, `_psd_violation`
  (:765-932),
* `dual_objective` (src/solver/interior_point.jl:7-14).

Problem layout: `Av[l]` is (m, k_l²) with row i = vec(A_i^(l)) column-major,
`C[l]` is k_l × k_l, `c` is (m,).  Sums run in the reference's loop order.
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

from .sdpx_oracle import kchol

EPS = np.finfo(np.float64).eps


def _ratio(residual, scale):
    if scale == 0.0:
        return 0.0 if residual == 0.0 else math.inf
    return abs(residual) / scale


def _cw(residual, nominal, realized):
    return _ratio(residual, nominal + realized), _ratio(residual, realized)


def _knrm_inf(a):
    a = np.asarray(a)
    return 0.0 if a.size == 0 else float(np.max(np.abs(a)))


def _buildP(Av_l, k, x):
    return (x @ Av_l).reshape(k, k, order="F")


def primal_block_backward_errors(Av, C, k, x, X):
    mixed = strict = 0.0
    for l, kl in enumerate(k):
        R = _buildP(Av[l], kl, x) - X[l] - C[l]
        nominal = np.abs(C[l]).reshape(-1, order="F").copy()
        realized = (np.abs(X[l]) + np.abs(C[l])).reshape(-1, order="F").copy()
        absA = np.abs(Av[l])
        nominal = nominal + absA.sum(axis=0)
        realized = realized + np.abs(x) @ absA
        r = R.reshape(-1, order="F")
        for idx in range(r.size):
            a, b = _cw(r[idx], nominal[idx], realized[idx])
            mixed, strict = max(mixed, a), max(strict, b)
    return mixed, strict


def dual_backward_errors(Av, k, c, Y, B=None, y=None):
    res = c.copy()
    nominal = np.abs(c).copy()
    realized = np.abs(c).copy()
    for l, kl in enumerate(k):
        yv = Y[l].reshape(-1, order="F")
        res = res - Av[l] @ yv
        absA = np.abs(Av[l])
        nominal = nominal + absA.sum(axis=1)
        realized = realized + absA @ np.abs(yv)
    if B is not None and B.shape[1]:
        res = res - B @ y
        nominal = nominal + np.abs(B).sum(axis=1)
        realized = realized + np.abs(B) @ np.abs(y)
    mixed = strict = 0.0
    for i in range(res.size):
        a, b = _cw(res[i], nominal[i], realized[i])
        mixed, strict = max(mixed, a), max(strict, b)
    return mixed, strict, res


def equality_backward_errors(B, b, x):
    """`_equality_backward_errors` (src/validation.jl:454-482), row order."""
    mixed = strict = 0.0
    for j in range(B.shape[1]):
        lhs, nominal, realized = 0.0, abs(b[j]), abs(b[j])
        for i in range(B.shape[0]):
            lhs += B[i, j] * x[i]
            nominal += abs(B[i, j])
            realized += abs(B[i, j]) * abs(x[i])
        a, s = _cw(abs(lhs - b[j]), nominal, realized)
        mixed, strict = max(mixed, a), max(strict, s)
    return mixed, strict


def solution_residuals(Av, C, k, c, x, X, Y, B=None, b=None, y=None):
    p = 0.0
    for l, kl in enumerate(k):
        p = max(p, _knrm_inf(_buildP(Av[l], kl, x) - X[l] - C[l]))
    if B is not None and B.shape[1]:
        p = max(p, _knrm_inf(b - B.T @ x))
    d = c.copy()
    for l in range(len(k)):
        d = d - Av[l] @ Y[l].reshape(-1, order="F")
    if B is not None and B.shape[1]:
        d = d - B @ y
    return p, _knrm_inf(d)


def _shifted_chol(M, shift):
    S = (M + M.T) / 2.0
    S = S + shift * np.eye(M.shape[0])
    return kchol(S)[0]


def block_psd_certificate(M, tol):
    """`_block_psd_certificate` (src/validation.jl:765-904)."""
    k = M.shape[0]
    finite = bool(np.all(np.isfinite(M)))
    scale = max(_knrm_inf(M), 1.0)
    allowed = max(tol, 128 * EPS) * scale
    sym = 0.0
    for col in range(k):
        for row in range(col):
            sym = max(sym, abs(M[row, col] - M[col, row]))
    if not finite:
        return dict(ok=False, finite=False, symmetry=sym, allowed=allowed, required=allowed,
                    resolved=False)
    if k == 1:
        req = max(0.0, -M[0, 0])
        return dict(ok=req <= allowed, finite=True, symmetry=0.0, allowed=allowed, required=req,
                    resolved=True)
    if k == 2:
        off = (M[0, 1] + M[1, 0]) / 2.0
        center = (M[0, 0] + M[1, 1]) / 2.0
        radius = math.hypot((M[0, 0] - M[1, 1]) / 2.0, off)
        req = max(0.0, -(center - radius))
        return dict(ok=req <= allowed and sym <= allowed, finite=True, symmetry=sym,
                    allowed=allowed, required=req, resolved=True)
    if _shifted_chol(M, 0.0):
        return dict(ok=sym <= allowed, finite=True, symmetry=sym, allowed=allowed, required=0.0,
                    resolved=True)
    allowed_ok = _shifted_chol(M, allowed)
    if k > 4:
        return dict(ok=allowed_ok and sym <= allowed, finite=True, symmetry=sym, allowed=allowed,
                    required=allowed, resolved=False)
    lower, upper, resolved = 0.0, allowed, allowed_ok
    if not resolved:
        lower = upper
        for _ in range(64):
            cand = upper + upper
            if not math.isfinite(cand):
                break
            upper = cand
            if _shifted_chol(M, upper):
                resolved = True
                break
            lower = upper
    if resolved:
        for _ in range(48):
            mid = (lower + upper) / 2.0
            if _shifted_chol(M, mid):
                upper = mid
            else:
                lower = mid
    return dict(ok=allowed_ok and sym <= allowed, finite=True, symmetry=sym, allowed=allowed,
                required=upper, resolved=resolved)


def psd_violation(details):
    """`_psd_violation` (src/validation.jl:919-932)."""
    v = 0.0
    for d in details:
        if d["ok"]:
            continue
        if not d["finite"]:
            return math.inf
        excess = max(0.0, d["symmetry"] - d["allowed"])
        shift = d["required"] if d["resolved"] else d["allowed"]
        v = max(v, excess, shift)
    return v


def result_certificate(Av: List[np.ndarray], C: List[np.ndarray], k: List[int], c: np.ndarray,
                       x, X, Y, eps_primal=1e-10, eps_dual=1e-10, eps_gap=1e-10,
                       legacy=False, B=None, b=None, y=None) -> dict:
    """`result_certificate` for the optimality kind (equality rows B, b with
    multipliers y when n > 0)."""
    x = np.asarray(x, dtype=np.float64)
    neq = 0 if B is None else np.asarray(B).reshape(x.size, -1).shape[1]
    if neq:
        B = np.asarray(B, dtype=np.float64).reshape(x.size, neq)
        b = np.asarray(b, dtype=np.float64)
        y = np.asarray(y, dtype=np.float64)
    p_obj = float(c @ x)
    d_obj = 0.0
    for l in range(len(k)):
        d_obj += float(np.sum(C[l] * Y[l]))
    if neq:
        d_obj += float(b @ y)
    p_aff, d_aff = solution_residuals(Av, C, k, c, x, X, Y, B if neq else None, b, y)
    gap = p_obj - d_obj
    oscale = max(1.0, (abs(p_obj) + abs(d_obj)) / 2.0)
    gap_rel = abs(gap) / oscale
    compl = 0.0
    for l in range(len(k)):
        compl += float(np.sum(X[l] * Y[l]))
    pd = [block_psd_certificate(X[l], max(eps_primal, eps_gap)) for l in range(len(k))]
    dd = [block_psd_certificate(Y[l], max(eps_dual, eps_gap)) for l in range(len(k))]
    pviol, dviol = psd_violation(pd), psd_violation(dd)
    p_res, d_res = max(p_aff, pviol), max(d_aff, dviol)
    pscale = 1.0 + max(max((_knrm_inf(Cl) for Cl in C), default=0.0),
                       _knrm_inf(b) if neq else 0.0)
    dscale = 1.0 + _knrm_inf(c)
    pb_mixed, pb_strict = primal_block_backward_errors(Av, C, k, x, X)
    db_mixed, db_strict, _ = dual_backward_errors(Av, k, c, Y, B if neq else None, y)
    eq_mixed, eq_strict = equality_backward_errors(B, b, x) if neq else (0.0, 0.0)
    failures = []
    primal_finite = (math.isfinite(p_obj) and math.isfinite(p_res) and
                     bool(np.all(np.isfinite(x))) and all(np.all(np.isfinite(M)) for M in X))
    dual_finite = (math.isfinite(d_obj) and math.isfinite(d_res) and
                   all(np.all(np.isfinite(M)) for M in Y) and
                   (not neq or bool(np.all(np.isfinite(y)))))
    finite = primal_finite and dual_finite and math.isfinite(gap_rel) and math.isfinite(compl)
    gap_ok = (0.0 <= gap <= eps_gap) if legacy else (gap_rel <= eps_gap)
    if not finite:
        failures.append("nonfinite")
    if not p_res / pscale <= eps_primal:
        failures.append("primal_residual")
    if not eq_mixed <= eps_primal:
        failures.append("equality_backward_error")
    if not pb_mixed <= eps_primal:
        failures.append("primal_block_backward_error")
    if not d_res / dscale <= eps_dual:
        failures.append("dual_residual")
    if not db_mixed <= eps_dual:
        failures.append("dual_backward_error")
    if not gap_ok:
        failures.append("duality_gap")
    if not all(d["ok"] for d in pd):
        failures.append("primal_psd")
    if not all(d["ok"] for d in dd):
        failures.append("dual_psd")
    return dict(valid=not failures, failures=failures, primal_objective=p_obj,
                dual_objective=d_obj, gap=gap, gap_relative=gap_rel, primal_residual=p_res,
                dual_residual=d_res, primal_affine_residual=p_aff, dual_affine_residual=d_aff,
                primal_cone_violation=pviol, dual_cone_violation=dviol,
                primal_residual_scaled=p_res / pscale, dual_residual_scaled=d_res / dscale,
                equality_backward_error=eq_mixed, equality_strict_backward_error=eq_strict,
                primal_block_backward_error=pb_mixed,
                primal_block_strict_backward_error=pb_strict,
                dual_backward_error=db_mixed, dual_strict_backward_error=db_strict,
                complementarity=compl, complementarity_relative=abs(compl) / oscale,
                primal_psd_failing_blocks=[l for l, d in enumerate(pd) if not d["ok"]],
                dual_psd_failing_blocks=[l for l, d in enumerate(dd) if not d["ok"]])
