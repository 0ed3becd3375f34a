"""CPU oracle for the LP/SOC normal-matrix rows — TEST INFRASTRUCTURE ONLY.

Only `tests/`, `__graft_entry__.smoke()` and the CPU-baseline leg of
`bench.py` may import this module.  It restates, in scalar Python/NumPy with
the reference's operation order:

* the Lorentz Nesterov–Todd scaling `_soc_nt_scaling!` and the maps W, W⁻¹,
  Hs⁻¹ = (WᵀW)⁻¹ (src/soc_lorentz_kernels.jl:21-255);
* the LP standard-form pack `_lp_standard_pack_range!`
  (src/lp_solver.jl:1892-1915): D_j = w_row(j)·g_j² + δ, D⁻¹, D^{-1/2};
* the normal matrix of a standard-form LP+SOC system, M = A·diag(D⁻¹, Hs_k⁻¹)·Aᵀ + δI
  (`_lp_assemble_reduced_schur!`, src/lp_solver.jl:1998-2040, generalised to
  Lorentz blocks through the per-cone metric of `_native_soc_add_metric!`,
  src/soc_native.jl:1119-1218), and the direction recovery of
  `_lp_solve_factor!` (src/lp_solver.jl:2177-2213).

The combined LP+SOC normal matrix has no reference route (SDPX classifies LP+SOC
models fail-closed); its parity is pinned on the sub-steps above and on the
reference's own NT-scaling identities (test/soc_native_algebra.jl:61-87).
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np


def tail_norm(v) -> float:
    """`_soc_tail_norm` (src/soc_lorentz_kernels.jl:21-34)."""
    scale = 0.0
    for x in v[1:]:
        scale = max(scale, abs(x))
    if scale == 0.0:
        return scale
    ss = 0.0
    for x in v[1:]:
        y = x / scale
        ss += y * y
    return scale * math.sqrt(ss)


def sqrt_determinant(v) -> Tuple[bool, float]:
    """`_soc_sqrt_determinant` (src/soc_lorentz_kernels.jl:42-62)."""
    scale = 0.0
    for x in v:
        if not math.isfinite(x):
            return False, 0.0
        scale = max(scale, abs(x))
    if scale == 0.0:
        return False, 0.0
    head = v[0]
    tail = tail_norm(v)
    margin = head - tail
    if not margin > 0:
        return False, 0.0
    residual = (margin / scale) * (head / scale + tail / scale)
    if not residual > 0:
        return False, 0.0
    result = scale * math.sqrt(residual)
    return (math.isfinite(result) and result > 0), result


def nt_scaling(s, z):
    """`_soc_nt_scaling!` (src/soc_lorentz_kernels.jl:72-185) → (ok, w, lam, eta, eta²)."""
    n = len(s)
    sok, ss = sqrt_determinant(s)
    zok, zs = sqrt_determinant(z)
    fail = (False, None, None, 0.0, 0.0)
    if not (sok and zok):
        return fail
    eta = math.sqrt(ss) / math.sqrt(zs)
    eta2 = eta * eta
    if not (math.isfinite(eta2) and eta2 > 0):
        return fail
    a = [s[0] / ss] + [s[i] / ss for i in range(1, n)]
    b = [z[0] / zs] + [z[i] / zs for i in range(1, n)]
    raw = [a[0] + b[0]] + [a[i] - b[i] for i in range(1, n)]
    if not all(math.isfinite(x) for x in a + b + raw):
        return fail
    mscale = 1.0
    for i in range(n):
        mscale = max(mscale, abs(a[i]), abs(b[i]))
    inv_m = 1.0 / mscale
    cross = (a[0] * inv_m) * (b[0] * inv_m)
    for i in range(1, n):
        cross += (a[i] * inv_m) * (b[i] * inv_m)
    radicand = inv_m * inv_m + cross
    if not (math.isfinite(radicand) and radicand > 0):
        return fail
    wscale = math.sqrt(2.0) * mscale * math.sqrt(radicand)
    if not (math.isfinite(wscale) and wscale > 0):
        return fail
    nts = 1.0
    for i in range(1, n):
        nts = max(nts, abs(raw[i] / wscale))
    inv_t = 1.0 / nts
    hacc = inv_t * inv_t
    for i in range(1, n):
        val = (raw[i] / wscale) / nts
        hacc += val * val
    nhead = nts * math.sqrt(hacc)
    if not (math.isfinite(nhead) and nhead > 0):
        return fail
    gamma = wscale / 2.0
    lscale = max(1.0, abs(a[0]), abs(b[0]), abs(gamma))
    for i in range(1, n):
        lscale = max(lscale, abs(a[i]), abs(b[i]))
    inv_l = 1.0 / lscale
    aa_h = a[0] * inv_l
    bb_h = b[0] * inv_l
    gg = gamma * inv_l
    den = aa_h + bb_h + 2.0 * gg
    if not (math.isfinite(den) and den > 0):
        return fail
    geo = math.sqrt(ss) * math.sqrt(zs)
    lam_head = geo * gamma
    if not math.isfinite(lam_head):
        return fail
    lam = [lam_head]
    for i in range(1, n):
        aa = a[i] * inv_l
        bb = b[i] * inv_l
        scaled = (gg + bb_h) * aa + (gg + aa_h) * bb
        val = geo * (scaled / den) * lscale
        if not math.isfinite(val):
            return fail
        lam.append(val)
    w = [nhead] + [raw[i] / wscale for i in range(1, n)]
    return True, np.array(w), np.array(lam), eta, eta2


def apply_w(w, eta, v):
    """`_soc_nt_apply_w!` (src/soc_lorentz_kernels.jl:187-206)."""
    head = v[0]
    dt = 0.0
    for i in range(1, len(v)):
        dt += w[i] * v[i]
    corr = head + dt / (1.0 + w[0])
    out = np.empty(len(v))
    out[0] = eta * (w[0] * head + dt)
    for i in range(1, len(v)):
        out[i] = eta * (v[i] + corr * w[i])
    return out


def apply_winv(w, eta, v):
    """`_soc_nt_apply_winv!` (src/soc_lorentz_kernels.jl:208-227)."""
    head = v[0]
    dt = 0.0
    for i in range(1, len(v)):
        dt += w[i] * v[i]
    corr = -head + dt / (1.0 + w[0])
    out = np.empty(len(v))
    out[0] = (w[0] * head - dt) / eta
    for i in range(1, len(v)):
        out[i] = (v[i] + corr * w[i]) / eta
    return out


def apply_hs_inverse(w, eta2, v):
    """`_soc_nt_apply_hs_inverse!` (src/soc_lorentz_kernels.jl:229-255)."""
    head = v[0]
    ld = w[0] * head
    for i in range(1, len(v)):
        ld -= w[i] * v[i]
    out = np.empty(len(v))
    out[0] = (2.0 * w[0] * ld - head) / eta2
    for i in range(1, len(v)):
        out[i] = (-2.0 * w[i] * ld + v[i]) / eta2
    return out


def lp_pack(weights, row_for_variable, coefficient, regularization):
    """`_lp_standard_pack_range!` (src/lp_solver.jl:1892-1915) → (D, D⁻¹, D^{-1/2})."""
    n = len(coefficient)
    D = np.empty(n)
    Dinv = np.empty(n)
    Dis = np.empty(n)
    for j in range(n):
        c = coefficient[j]
        d = weights[row_for_variable[j]] * c * c + regularization
        D[j] = d
        Dinv[j] = 1.0 / d
        Dis[j] = math.sqrt(Dinv[j])
    return D, Dinv, Dis


def hs_inverse_matrix(w, eta2):
    """Dense Hs⁻¹ of one cone, column by column through `apply_hs_inverse`
    (the reference's metric assembly, src/soc_native.jl:1192-1201)."""
    q = len(w)
    M = np.empty((q, q))
    e = np.zeros(q)
    for c in range(q):
        e[c] = 1.0
        M[:, c] = apply_hs_inverse(w, eta2, e)
        e[c] = 0.0
    return M


def normal_matrix(A, n_lp, cone_dims, Dinv, scalings, regularization):
    """M = A_LP diag(D⁻¹) A_LPᵀ + Σ_k A_k Hs_k⁻¹ A_kᵀ + δI for A (m × n), variables
    ordered [LP | cone 1 | cone 2 | …]."""
    m = A.shape[0]
    ALP = A[:, :n_lp]
    M = (ALP * Dinv[None, :]) @ ALP.T
    o = n_lp
    for q, (w, eta, eta2) in zip(cone_dims, scalings):
        Ak = A[:, o:o + q]
        M += Ak @ hs_inverse_matrix(w, eta2) @ Ak.T
        o += q
    M[np.diag_indices(m)] += regularization
    return M


def recover(A, n_lp, cone_dims, Dinv, scalings, M, rx, ry):
    """`_lp_solve_factor!` generalised to Lorentz blocks:
    t = D⁻¹ rx; dy = M⁻¹ (ry − A t); dx = t + D⁻¹ Aᵀ dy."""
    def apply_dinv(v):
        out = np.empty_like(v)
        out[:n_lp] = Dinv * v[:n_lp]
        o = n_lp
        for q, (w, eta, eta2) in zip(cone_dims, scalings):
            out[o:o + q] = apply_hs_inverse(w, eta2, v[o:o + q])
            o += q
        return out
    t = apply_dinv(rx)
    red = ry - A @ t
    Lc = np.linalg.cholesky(M)
    dy = np.linalg.solve(Lc.T, np.linalg.solve(Lc, red))
    dx = t + apply_dinv(A.T @ dy)
    return dx, dy


def random_lp_soc(m, n_lp, cone_dims, density=0.1, seed=0):
    """Interior LP+SOC data: A with N(0,1) entries under a Bernoulli(density)
    mask, LP slacks/duals ~ U(0.5,1.5), cone points (t, u), u ~ N(0,1), t = 1.5‖u‖+1."""
    rng = np.random.default_rng(seed)
    n = n_lp + sum(cone_dims)
    A = rng.standard_normal((m, n)) * (rng.random((m, n)) < density)
    xl = rng.uniform(0.5, 1.5, n_lp)
    zl = rng.uniform(0.5, 1.5, n_lp)
    s_cones, z_cones = [], []
    for q in cone_dims:
        u = rng.standard_normal(q - 1)
        s_cones.append(np.concatenate([[1.5 * np.linalg.norm(u) + 1.0], u]))
        u = rng.standard_normal(q - 1)
        z_cones.append(np.concatenate([[1.5 * np.linalg.norm(u) + 1.0], u]))
    return A, xl, zl, s_cones, z_cones
