"""Seeded synthetic SDP instances.

* `gate_closed_form`, `gate_dense`: the reference's deterministic gate problems
  (benchmark/gates.jl:96-199), rebuilt from the same written-out 64-bit LCG so
  they are bit-identical to the ones SDPX records baselines for.
* `toy_t1`: the 2×2 toy problem of test/correctness.jl:65-80 (optimum 2√6).
* `sdpa_sparse`: the same construction with structurally sparse coefficients
  (a few stored entries per A_i and block), the regime of SDPX's SparseCons path.
* `sdpa_dense`: strictly feasible dense SDPs in SDPA primal-dual form, mapped to
  SDPX's core form.  With `blocks=[50], lp=0, m=100` this is the n=50/m=100
  workload; with `blocks=[400, 200], lp=500, m=2000` it is the two-block plus
  500-nonnegatives workload at m=2000.

SDPA form:  max bᵀy  s.t.  Z = C − Σ yᵢAᵢ ⪰ 0  (dual of min ⟨C,X⟩, ⟨Aᵢ,X⟩ = bᵢ).
SDPX form:  min cᵀx  s.t.  X = Σ xᵢÂᵢ − Ĉ ⪰ 0  with x ≡ y, Âᵢ = −Aᵢ, Ĉ = −C,
c = −b (src/ir/lower_sdp.jl objective sign at :497-501).  SDPX's slack X is
SDPA's Z and SDPX's dual Y is SDPA's X; objectives change sign.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np

from .problem import SDPProblem, ingest

_MASK64 = (1 << 64) - 1


class GateStream:
    """The reference's reproducible LCG (benchmark/gates.jl:96-113)."""

    def __init__(self, seed: int):
        self.state = seed & _MASK64

    def uniform(self) -> float:
        self.state = (0x5851F42D4C957F2D * self.state + 0x14057B7EF767814F) & _MASK64
        return float(self.state >> 11) / float(1 << 53)

    def signed(self) -> float:
        return 2.0 * self.uniform() - 1.0


def gate_closed_form() -> SDPProblem:
    """`closed_form_sdp` (benchmark/gates.jl:118-140); optimum 2√6."""
    A = np.zeros((2, 2, 2))
    A[0, 0, 0] = 1.0
    A[1, 1, 1] = 1.0
    return ingest([2.0, 3.0], [A], [np.array([[0.0, 1.0], [1.0, 0.0]])])


def toy_t1() -> SDPProblem:
    """T1 of test/correctness.jl:65-80: min 2x₁+3x₂ s.t. [[x₁,−1],[−1,x₂]] ⪰ 0."""
    A = np.zeros((2, 2, 2))
    A[0, 0, 0] = 1.0
    A[1, 1, 1] = 1.0
    C = np.array([[0.0, 1.0], [1.0, 0.0]])
    return ingest([2.0, 3.0], [A], [C])


def toy_t2() -> SDPProblem:
    """T2 of test/correctness.jl:97-106: T1 plus the equality x₁ = 2
    (B = [1; 0], b = [2]); optimum x₂ = 1/2, p* = 11/2."""
    t1 = toy_t1()
    return ingest(t1.c, [t1.Av[0].reshape(2, 2, 2)], t1.C, np.array([[1.0], [0.0]]), [2.0])


def toy_t3() -> SDPProblem:
    """T3 of test/correctness.jl:124-135: the T2 equality row duplicated
    (B = [1 1; 0 0], b = [2, 2]: n = 2, rank 1)."""
    t1 = toy_t1()
    return ingest(t1.c, [t1.Av[0].reshape(2, 2, 2)], t1.C, np.array([[1.0, 1.0], [0.0, 0.0]]),
                  [2.0, 2.0])


def readme_moment_equalities() -> SDPProblem:
    """The README quick-start moment SDP (README.md:44-75) with its two
    equality rows kept: variables (W0, W2, W4), maximize W2, i.e.
    min −W2 s.t. W0 = 1, W0 − W2 − W4 = 0 and [[W0, W2], [W2, W4]] ⪰ 0
    (C = 0).  Optimum W2 = (√5 − 1)/2."""
    A = np.zeros((3, 2, 2))
    A[0, 0, 0] = 1.0
    A[1, 0, 1] = A[1, 1, 0] = 1.0
    A[2, 1, 1] = 1.0
    B = np.array([[1.0, 1.0], [0.0, -1.0], [0.0, -1.0]])
    return ingest([0.0, -1.0, 0.0], [A], [np.zeros((2, 2))], B, [1.0, 0.0])


def readme_moment() -> SDPProblem:
    """The quick-start moment SDP of the reference's README (README.md:44-75):
    maximize W2 s.t. W0 = 1, W0 − W2 − W4 = 0, [[W0, W2], [W2, W4]] ⪰ 0.
    The two equality rows eliminate W0 = 1 and W4 = 1 − W2, leaving the core
    form min −W2 s.t. W2·[[0,1],[1,−1]] − [[−1,0],[0,−1]] ⪰ 0; the optimum is
    W2 = (√5 − 1)/2 (objective −0.618034…)."""
    A = np.array([[0.0, 1.0], [1.0, -1.0]])
    C = np.array([[-1.0, 0.0], [0.0, -1.0]])
    return _assemble(np.array([-1.0]), [A.reshape(1, 2, 2)], [C], [2], 0)


def gate_dense(variables: int = 180, side: int = 8, blocks: int = 3, seed: int = 5) -> SDPProblem:
    """`dense_sdp` (benchmark/gates.jl:151-199).  Julia comprehensions fill
    column-major, so the side×side draw is filled column by column."""
    s = GateStream(seed)
    coef = [np.zeros((variables, side, side)) for _ in range(blocks)]
    for blk in range(blocks):
        for var in range(variables):
            entry = np.empty((side, side))
            for col in range(side):
                for row in range(side):
                    entry[row, col] = s.signed()
            coef[blk][var] = entry + entry.T
    interior = np.array([s.signed() for _ in range(variables)])
    constants = []
    objective = np.zeros(variables)
    for blk in range(blocks):
        combination = np.zeros((side, side))
        for var in range(variables):
            combination += interior[var] * coef[blk][var]
        constants.append(combination - np.eye(side))
        factor = np.empty((side, side))
        for col in range(side):
            for row in range(side):
                factor[row, col] = s.signed()
        dual = factor @ factor.T + side * np.eye(side)
        for var in range(variables):
            objective[var] += float(np.sum(coef[blk][var] * dual))
    return ingest(objective, coef, constants)


def sdpa_dense(m: int, blocks: Sequence[int], lp: int = 0, seed: int = 0,
               dtype=np.float64) -> SDPProblem:
    """Strictly feasible dense SDP in SDPX core form (construction below)."""
    return _sdpa_dense(m, blocks, lp, seed)[0]


def sdpa_dense_equalities(m: int, blocks: Sequence[int], lp: int = 0, n_eq: int = 1,
                          seed: int = 0, rank: Optional[int] = None) -> SDPProblem:
    """`sdpa_dense` plus `n_eq` equality rows Bᵀx = b that keep its strictly
    feasible point: B (m×n_eq, N(0,1) from `default_rng(seed + 1)`), b = Bᵀy0
    with y0 the dual point of the generator (x = y0 gives X = Z0 ≻ 0).  With
    `rank` < n_eq the columns past `rank` are combinations of the first ones
    (the first of them an exact copy), a rank-deficient equality block."""
    prob, y0 = _sdpa_dense(m, blocks, lp, seed)
    rng = np.random.default_rng(seed + 1)
    r = n_eq if rank is None else rank
    B = np.zeros((m, n_eq))
    B[:, :r] = rng.standard_normal((m, r))
    for j in range(r, n_eq):
        B[:, j] = B[:, 0] if j == r else B[:, :r] @ rng.standard_normal(r)
    return SDPProblem(prob.c, prob.k, prob.Av, prob.C, B, B.T @ y0)


def _sdpa_dense(m, blocks, lp, seed):
    """Strictly feasible dense SDP (SDPA primal-dual form) in SDPX core form.

    Draw order from `numpy.random.default_rng(seed)`, per PSD block of order n:
    G (m×n×n, N(0,1)) with Aᵢ = (G+Gᵀ)/2, then W (n×n, N(0,1)) with
    X0 = I + 0.1·WWᵀ/n; for the LP block (`lp` nonnegatives): aᵢ (m×lp,
    N(0,1)) then x0 ~ U(0.5,1.5).  Then y0 ~ N(0,1)^m; then per PSD block
    V (n×n) with Z0 = I + 0.1·VVᵀ/n; then the LP slack s0 ~ U(0.5,1.5).
    b_i = Σ_l ⟨A_i^l, X0_l⟩ + a_iᵀx0,  C_l = Σ y0_i A_i^l + Z0_l,
    c_lp = Σ y0_i a_i + s0.  The LP block becomes `lp` 1×1 PSD blocks.
    """
    rng = np.random.default_rng(seed)
    As: List[np.ndarray] = []
    X0s: List[np.ndarray] = []
    for n in blocks:
        G = rng.standard_normal((m, n, n))
        A = G + np.transpose(G, (0, 2, 1))
        A *= 0.5
        del G
        W = rng.standard_normal((n, n))
        As.append(A)
        X0s.append(np.eye(n) + 0.1 * (W @ W.T) / n)
    if lp > 0:
        a_lp = rng.standard_normal((m, lp))
        x0_lp = rng.uniform(0.5, 1.5, lp)
    b = np.zeros(m)
    for A, X0 in zip(As, X0s):
        b += A.reshape(m, -1) @ X0.reshape(-1)
    if lp > 0:
        b += a_lp @ x0_lp
    y0 = rng.standard_normal(m)
    Cs = []
    for A, n in zip(As, blocks):
        V = rng.standard_normal((n, n))
        Z0 = np.eye(n) + 0.1 * (V @ V.T) / n
        Cs.append((y0 @ A.reshape(m, -1)).reshape(n, n) + Z0)
    if lp > 0:
        s0 = rng.uniform(0.5, 1.5, lp)
        c_lp = y0 @ a_lp + s0
    # Map to SDPX: Âᵢ = −Aᵢ, Ĉ = −C, c = −b.
    A_sdpx = [-A for A in As]
    C_sdpx = [-C for C in Cs]
    if lp > 0:
        A_sdpx.append(-a_lp.reshape(m, lp, 1, 1))
        C_sdpx.append(-c_lp)
    return _assemble(-b, A_sdpx, C_sdpx, list(blocks), lp), y0


def sdpa_sparse(m: int, blocks: Sequence[int], lp: int = 0, active: float = 0.5,
                pairs: Sequence[int] = (1, 3), seed: int = 0) -> SDPProblem:
    """Strictly feasible SDP with structurally sparse coefficients (the regime
    of SDPX's `SparseCons` path: every A_i touches a few entries of a block).

    Draw order from `numpy.random.default_rng(seed)`, per PSD block of order n:
    the activity mask (m draws U(0,1) < `active`), the pair counts
    q_i ~ U{pairs[0]..pairs[1]} (m draws), then for the Σq_i pairs their rows,
    columns (U{0..n−1}) and values (N(0,1)); pair (r, c, v) adds v at (r, c)
    and (c, r) of A_i (once when r = c), so an active A_i stores 1–2·q_i
    entries.  A variable active in no block is then made active in block
    i mod L with one diagonal pair of value 1.  Then, as `sdpa_dense`, per
    block X0 = I + 0.1·WWᵀ/n, the LP block (aᵢ ~ N(0,1), x0 ~ U(0.5,1.5)),
    y0 ~ N(0,1)^m, per block Z0 = I + 0.1·VVᵀ/n, LP slack s0 ~ U(0.5,1.5);
    b_i = Σ⟨A_i, X0⟩ + a_iᵀx0, C = Σ y0_i A_i + Z0, mapped to SDPX's form."""
    rng = np.random.default_rng(seed)
    As: List[np.ndarray] = []
    acts = []
    for n in blocks:
        A = np.zeros((m, n, n))
        act = rng.random(m) < active
        q = rng.integers(pairs[0], pairs[1] + 1, size=m)
        q = np.where(act, q, 0)
        tot = int(q.sum())
        var = np.repeat(np.arange(m), q)
        r = rng.integers(0, n, size=tot)
        c = rng.integers(0, n, size=tot)
        v = rng.standard_normal(tot)
        np.add.at(A, (var, r, c), v)
        off = r != c
        np.add.at(A, (var[off], c[off], r[off]), v[off])
        As.append(A)
        acts.append(act)
    if blocks:
        anyact = np.logical_or.reduce(acts)
        for i in np.nonzero(~anyact)[0]:
            l = int(i) % len(blocks)
            As[l][i, 0, 0] = 1.0
    X0s = []
    for n in blocks:
        W = rng.standard_normal((n, n))
        X0s.append(np.eye(n) + 0.1 * (W @ W.T) / n)
    if lp > 0:
        a_lp = rng.standard_normal((m, lp))
        x0_lp = rng.uniform(0.5, 1.5, lp)
    b = np.zeros(m)
    for A, X0 in zip(As, X0s):
        b += A.reshape(m, -1) @ X0.reshape(-1)
    if lp > 0:
        b += a_lp @ x0_lp
    y0 = rng.standard_normal(m)
    Cs = []
    for A, n in zip(As, blocks):
        V = rng.standard_normal((n, n))
        Cs.append((y0 @ A.reshape(m, -1)).reshape(n, n) + np.eye(n) + 0.1 * (V @ V.T) / n)
    A_sdpx = [-A for A in As]
    C_sdpx = [-C for C in Cs]
    if lp > 0:
        s0 = rng.uniform(0.5, 1.5, lp)
        A_sdpx.append(-a_lp.reshape(m, lp, 1, 1))
        C_sdpx.append(-(y0 @ a_lp + s0))
    return _assemble(-b, A_sdpx, C_sdpx, list(blocks), lp)


def _assemble(c, A_sdpx, C_sdpx, blocks, lp) -> SDPProblem:
    """Build the container without the O(m k²) symmetry re-checks of `ingest`
    (the generator symmetrises by construction)."""
    m = c.shape[0]
    ks, Av, Cs = [], [], []
    for A, C, n in zip(A_sdpx[:len(blocks)], C_sdpx[:len(blocks)], blocks):
        ks.append(n)
        Av.append(np.ascontiguousarray(A.reshape(m, n * n)))
        Cs.append(np.ascontiguousarray(C))
    if lp > 0:
        a = A_sdpx[-1].reshape(m, lp)
        cvec = C_sdpx[-1]
        for j in range(lp):
            ks.append(1)
            Av.append(np.ascontiguousarray(a[:, j:j + 1]))
            Cs.append(np.array([[cvec[j]]]))
    return SDPProblem(np.ascontiguousarray(c), ks, Av, Cs, np.zeros((m, 0)), np.zeros(0))


def lp_soc_standard(m: int, n_lp: int, cones: Sequence[int], density: float = 0.1,
                    seed: int = 0):
    """Interior point of a standard-form LP + Lorentz-cone system.

    Draw order (numpy default_rng(seed)): A (m × n, n = n_lp + Σq) as N(0,1)
    entries under a Bernoulli(density) mask (normals first, then the mask);
    LP slacks x, duals s ~ U(0.5, 1.5); per cone a slack point (t, u) and then
    a dual point, u ~ N(0,1)^{q−1}, t = 1.5‖u‖ + 1 (strictly inside the cone).

    Returns (B, weights, s, z): B = Aᵀ (n × m, the reduced system's
    variable-major layout), LP weights s/x, and the cone slack and dual points
    (Σq each)."""
    rng = np.random.default_rng(seed)
    n = n_lp + int(sum(cones))
    A = rng.standard_normal((m, n)) * (rng.random((m, n)) < density)
    x = rng.uniform(0.5, 1.5, n_lp)
    s_lp = rng.uniform(0.5, 1.5, n_lp)
    sc, zc = [], []
    for q in cones:
        for dst in (sc, zc):
            u = rng.standard_normal(q - 1)
            dst.append(np.concatenate([[1.5 * np.linalg.norm(u) + 1.0], u]))
    cat = (lambda v: np.concatenate(v)) if cones else (lambda v: np.zeros(0))
    return np.asfortranarray(A.T), s_lp / x, cat(sc), cat(zc)


def lp_soc_problem(m: int, n_lp: int, cones: Sequence[int], density: float = 0.1,
                   seed: int = 0):
    """Standard-form LP + Lorentz-cone problem  min cᵀx s.t. Ax = b, x ∈ K
    with a strictly feasible primal-dual pair: the draws of `lp_soc_standard`
    (A, the LP primal and dual points, the cone primal and dual points) and
    then y0 ~ N(0,1)^m; b = A x0, c = Aᵀy0 + z0.  Returns (B = Aᵀ, b, c)."""
    B, w, sc, zc = lp_soc_standard(m, n_lp, cones, density, seed)
    # lp_soc_standard returns the LP weights s/x; redraw the same LP points
    rng = np.random.default_rng(seed)
    n = n_lp + int(sum(cones))
    rng.standard_normal((m, n))
    rng.random((m, n))
    x_lp = rng.uniform(0.5, 1.5, n_lp)
    z_lp = rng.uniform(0.5, 1.5, n_lp)
    x0 = np.concatenate([x_lp, sc])
    z0 = np.concatenate([z_lp, zc])
    y0 = np.random.default_rng(seed + 1).standard_normal(m)
    b = B.T @ x0
    c = B @ y0 + z0
    return B, b, c
