"""CPU oracle of the LP + Lorentz-cone interior-point loop — TEST INFRASTRUCTURE ONLY.

Restates, in NumPy, the loop of `sdpx_b200_normal_optimize`: SDPX's LP loop
`solve_lp!` (src/lp_solver.jl:3651-4400 — residuals, best snapshot,
termination on scaled residuals and relative gap, regularised reduced factor
with ×10 retries decaying to √(eps·√eps) (`_lp_regularization_floor`
:3435-3444), Mehrotra predictor-corrector under the adaptive controller
(src/adaptive_parameters.jl), `_fraction_to_boundary` (:3197-3205) steps and
the regularisation-aware direction gate (`_lp_direction_accuracy_gate!`
:3029-3195)) for the standard form

    min cᵀx  s.t.  Ax = b,  x ∈ R₊^{n_lp} × L^{q_1} × …,

with the Lorentz cones entering through the reference's Nesterov–Todd scaling
(oracle/cone_oracle.py) of the pair (z, x): λ = W·x = W⁻¹·z, the primal block
of the reduced system is W² and `apply_hs_inverse` gives its inverse W⁻²; the
cones' Δz comes from the dual equation Δz = rd − AᵀΔy.  SDPX has no such reduced LP+SOC
route (its route classifier sends LP+SOC models elsewhere), so this loop pins
the device loop rather than a reference solve; the cone arithmetic under it
is pinned bit-exactly to the reference's recurrences.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.linalg as sla

from oracle import cone_oracle as O

EPS = np.finfo(np.float64).eps


@dataclass
class ConeResult:
    status: str
    iterations: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    pObj: float
    dObj: float
    p_res: float
    d_res: float
    message: str


def _jordan(u, v):
    out = np.empty_like(u)
    out[0] = float(u @ v)
    out[1:] = u[0] * v[1:] + v[0] * u[1:]
    return out


def _jordan_div(lam, t):
    det = lam[0] * lam[0] - float(lam[1:] @ lam[1:])
    q0 = (lam[0] * t[0] - float(lam[1:] @ t[1:])) / det
    q = np.empty_like(t)
    q[1:] = (t[1:] - q0 * lam[1:]) / lam[0]
    q[0] = q0
    return q


def _soc_boundary_step(v, d):
    aa = d[0] * d[0] - float(d[1:] @ d[1:])
    bb = v[0] * d[0] - float(v[1:] @ d[1:])
    cc = v[0] * v[0] - float(v[1:] @ v[1:])
    best = math.inf
    if d[0] < 0:
        best = -v[0] / d[0]
    if len(v) == 1:
        return best
    if aa == 0.0:
        if bb < 0:
            best = min(best, -cc / (2 * bb))
        return best
    disc = bb * bb - aa * cc
    if disc < 0:
        return best
    sq = math.sqrt(disc)
    qq = -(bb + (sq if bb >= 0 else -sq))
    r1 = qq / aa
    r2 = cc / qq if qq != 0 else math.inf
    for r in (r1, r2):
        if r > 0:
            best = min(best, r)
    return best


class _Cones:
    def __init__(self, n_lp, dims):
        self.n_lp = n_lp
        self.dims = list(dims)
        self.offs = list(np.cumsum([0] + self.dims)[:-1] + n_lp)

    def segs(self):
        return [(o, q) for o, q in zip(self.offs, self.dims)]


def cone_ipm_solve(A, b, c, n_lp, dims, opts, trace=None) -> ConeResult:
    from sdpx_b200.controller import AdaptiveIPMController, IterationDiagnostics, at_precision_floor
    m, n = A.shape
    K = _Cones(n_lp, dims)
    x = np.zeros(n)
    z = np.zeros(n)
    x[:n_lp] = 1.0
    z[:n_lp] = 1.0
    for o, q in K.segs():
        x[o] = 1.0
        z[o] = 1.0
    y = np.zeros(m)
    nu = float(n_lp + len(dims))
    reg_floor = max(math.sqrt(EPS * math.sqrt(EPS)), 1e-60)
    reg = reg_floor
    tau = max(math.sqrt(EPS), opts.eps_primal, opts.eps_dual)
    pscale = 1.0 + (float(np.max(np.abs(b))) if m else 0.0)
    dscale = 1.0 + float(np.max(np.abs(c)))
    ctl = AdaptiveIPMController(opts)
    absB_rows = np.sum(np.abs(A), axis=0)      # per variable
    absB_cols = np.sum(np.abs(A), axis=1)      # per equality
    best = None
    best_gap = math.inf
    best_feas = math.inf
    iters = 0
    status, message = "", ""
    p_res = d_res = math.inf
    while True:
        rp = b - A @ x
        rd = c - A.T @ y - z
        p_res = float(np.max(np.abs(rp))) if m else 0.0
        d_res = float(np.max(np.abs(rd)))
        pobj, dobj = float(c @ x), float(b @ y)
        gap = float(x @ z)
        gap_rel = gap / max(1.0, (abs(pobj) + abs(dobj)) / 2)
        feas = max(p_res / pscale, d_res / dscale)
        gtie = max(1e-12, abs(best_gap) * 1e-6)
        ftie = max(1e-12, abs(best_feas) * 1e-6)
        if (best is None or gap_rel < best_gap - gtie or
                (abs(gap_rel - best_gap) <= gtie and feas < best_feas - ftie)):
            best = (x.copy(), y.copy(), z.copy())
            best_gap, best_feas = gap_rel, feas
        if p_res / pscale <= opts.eps_primal and d_res / dscale <= opts.eps_dual and \
                gap_rel <= opts.eps_gap:
            status, message = "Optimal", "Optimal"
            break
        if iters >= opts.iter_max:
            status, message = "IterLimit", "iteration limit"
            break
        w_lp = z[:n_lp] / x[:n_lp]
        scal = []
        ok = True
        for o, q in K.segs():
            good, w, lam, eta, eta2 = O.nt_scaling(list(z[o:o + q]), list(x[o:o + q]))
            if not good:
                ok = False
                break
            scal.append((np.array(w), np.array(lam), eta, eta2))
        if not ok:
            status, message = "NumericalBreakdown", "NT scaling failed"
            break
        reg = max(reg_floor, reg / 10)
        attempt = reg
        fac = None
        for _ in range(8):
            D = w_lp + attempt
            Dinv = 1.0 / D
            M = O.normal_matrix(A, n_lp, dims, Dinv, [(s[0], s[2], s[3]) for s in scal], attempt)
            try:
                fac = sla.cho_factor(M, lower=True, check_finite=False)
                if not np.all(np.isfinite(fac[0])):
                    raise np.linalg.LinAlgError
                reg = attempt
                break
            except (np.linalg.LinAlgError, ValueError):
                fac = None
                attempt *= 10
        if fac is None:
            status, message = "NumericalBreakdown", "reduced system singular"
            break

        def winv(k, v):
            w, _, eta, _ = scal[k]
            return O.apply_winv(w, eta, v)

        def wmap(k, v):
            w, _, eta, _ = scal[k]
            return O.apply_w(w, eta, v)

        def target(dxa=None, dza=None, sigma_mu=0.0):
            t = np.empty(n)
            rc = np.empty(n)
            qb = {}
            xl, zl = x[:n_lp], z[:n_lp]
            if dxa is None:
                t[:n_lp] = -(xl * zl)
            else:
                t[:n_lp] = sigma_mu - xl * zl - dxa[:n_lp] * dza[:n_lp]
            rc[:n_lp] = t[:n_lp] / xl
            for k, (o, q) in enumerate(K.segs()):
                lam = scal[k][1]
                tc = -_jordan(lam, lam)
                if dxa is not None:
                    tc = tc - _jordan(wmap(k, dxa[o:o + q]), winv(k, dza[o:o + q]))
                    tc[0] += sigma_mu
                t[o:o + q] = tc
                qk = _jordan_div(lam, tc)
                qb[k] = qk
                rc[o:o + q] = wmap(k, qk)
            return t, rc, qb

        def direction(t, rc, qb):
            rx = rc - rd
            dxv, dyv = O.recover(A, n_lp, dims, Dinv, [(s[0], s[2], s[3]) for s in scal],
                                 M, rx, rp)
            # LP: Δz from the complementarity row (`_lp_complete_direction!`);
            # cones: from the dual equation, Δz = rd − AᵀΔy, exactly dual
            # feasible (W(q − WΔx) cancels catastrophically as W² becomes
            # ill-conditioned near the boundary)
            dzv = rd - A.T @ dyv
            dzv[:n_lp] = (t[:n_lp] - z[:n_lp] * dxv[:n_lp]) / x[:n_lp]
            return dxv, dyv, dzv, rx

        def knorm():
            kk = 0.0
            for j in range(n_lp):
                kk = max(kk, abs(w_lp[j]) + absB_rows[j])
            for k, (o, q) in enumerate(K.segs()):
                for i in range(q):
                    e = np.zeros(q)
                    e[i] = 1.0
                    col = wmap(k, wmap(k, e))
                    kk = max(kk, float(np.sum(np.abs(col))) + absB_rows[o + i])
            for e_ in range(m):
                kk = max(kk, absB_cols[e_])
            return kk

        def gate(dxv, dyv, rx, kn):
            Ddx = np.empty(n)
            Ddx[:n_lp] = D * dxv[:n_lp]
            for k, (o, q) in enumerate(K.segs()):
                Ddx[o:o + q] = wmap(k, wmap(k, dxv[o:o + q]))
            rho_x = rx - (Ddx - A.T @ dyv)
            rho_y = rp - A @ dxv - attempt * dyv if m else np.zeros(0)
            eta_f = max(float(np.max(np.abs(rho_x))), float(np.max(np.abs(rho_y))) if m else 0.0)
            scale = max(float(np.max(np.abs(rx))), float(np.max(np.abs(rp))) if m else 0.0) + \
                (kn + attempt) * max(float(np.max(np.abs(dxv))),
                                     float(np.max(np.abs(dyv))) if m else 0.0)
            return math.isfinite(eta_f) and eta_f <= tau * scale

        def ftb(v, d, frac):
            st = 1.0
            for j in range(n_lp):
                if d[j] < 0:
                    st = min(st, -frac * v[j] / d[j])
            for o, q in K.segs():
                st = min(st, frac * _soc_boundary_step(v[o:o + q], d[o:o + q]))
            return max(st, 0.0)

        kn = knorm()
        t, rc, qb = target()
        dxa, dya, dza, rx = direction(t, rc, qb)
        if not gate(dxa, dya, rx, kn):
            status, message = "NumericalBreakdown", "affine direction gate"
            break
        apa, ada = ftb(x, dxa, 1.0), ftb(z, dza, 1.0)
        mu = gap / nu
        mu_aff = float((x + apa * dxa) @ (z + ada * dza)) / nu
        quality = min(max(mu_aff / mu, 0.0), 1.0)
        h = ctl.history
        diag = IterationDiagnostics(
            iteration=iters + 1, primal_residual=p_res / pscale, dual_residual=d_res / dscale,
            relative_gap=gap_rel, mu=mu, mu_aff=mu_aff, affine_primal_step=apa,
            affine_dual_step=ada,
            previous_primal_step=h[-1]["primal_step"] if h else 1.0,
            previous_dual_step=h[-1]["dual_step"] if h else 1.0,
            backtracking_count=0, regularization=attempt, refinement_count=0,
            factorization_quality=1.0 if attempt <= reg_floor else reg_floor / attempt,
            achieved_residual_reduction=h[-1]["achieved_residual_reduction"] if h else 1.0,
            primal_psd_margin=float(np.min(x)) / max(float(np.max(x)), 1.0),
            dual_psd_margin=float(np.min(z)) / max(float(np.max(z)), 1.0),
            precision_floor=at_precision_floor(p_res, d_res, gap_rel, pscale, dscale))
        params = ctl.select(diag)
        t, rc, qb = target(dxa, dza, params.sigma * mu)
        dx, dy, dz, rx = direction(t, rc, qb)
        if not gate(dx, dy, rx, kn):
            status, message = "NumericalBreakdown", "corrector direction gate"
            break
        ap = ftb(x, dx, params.primal_fraction_to_boundary)
        ad = ftb(z, dz, params.dual_fraction_to_boundary)
        x = x + ap * dx
        z = z + ad * dz
        y = y + ad * dy
        iters += 1
        ctl.record(iteration=iters, predictor_quality=quality, complementarity_before=gap,
                   complementarity_after=float(x @ z), primal_residual=p_res,
                   dual_residual=d_res, primal_step=ap, dual_step=ad,
                   primal_residual_after=abs(1 - ap) * p_res,
                   dual_residual_after=abs(1 - ad) * d_res, backtracking_count=0,
                   affine_primal_step=apa, affine_dual_step=ada, mu_before=mu,
                   mu_affine=mu_aff, relative_gap=gap_rel, regularization=attempt,
                   refinement_count=0, refinement_residual=0.0, factorization_quality=1.0,
                   primal_psd_margin=diag.primal_psd_margin,
                   dual_psd_margin=diag.dual_psd_margin, precision_floor=diag.precision_floor,
                   selected=params)
        if trace is not None:
            trace.append(dict(iteration=iters, gap=gap_rel, p_res=p_res, d_res=d_res, tX=ap, tY=ad,
                              sigma=params.sigma))
        if not (np.all(np.isfinite(x)) and np.all(np.isfinite(z)) and np.all(np.isfinite(y))):
            status, message = "NumericalBreakdown", "non-finite iterate"
            break
    if status != "Optimal" and best is not None:
        x, y, z = best
    return ConeResult(status, iters, x, y, z, float(c @ x), float(b @ y), p_res, d_res, message)
