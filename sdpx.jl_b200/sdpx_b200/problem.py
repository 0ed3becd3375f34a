"""Host-side SDP problem container in SDPX's core form.

SDPX solves the geometric form (src/types/problems.jl:1-11, src/step.jl:25-72)

    min  cᵀx   s.t.  X_l = Σ_i x_i A_i^(l) − C_l ⪰ 0   (l = 1..L),   Bᵀx = b

with dual (y, Y_l ⪰ 0).  `ingest` mirrors `SDPX.ingest(c, A, C, B, b)`
(src/ingest.jl:620,797) for dense coefficients: `A[l]` is an array of shape
(m, k_l, k_l) whose slice `A[l][i]` is the symmetric coefficient A_i^(l).

Storage follows SDPX's `DenseCons` (src/types/constraints.jl:12-27): for every
block the coefficients are one k_l² × m column-major matrix `Av[l]` whose column
i is vec(A_i^(l)).  Because every A_i is symmetric, that memory is identical to
a C-ordered (m, k_l, k_l) array, which is how it is held here (`Av[l]` has shape
(m, k_l*k_l), row i = vec(A_i)).  This is also the layout uploaded to HBM.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np


@dataclass
class SDPProblem:
    """Dense SDP in SDPX core form; all arrays float64, C-contiguous."""

    c: np.ndarray                 # (m,)
    k: List[int]                  # block orders
    Av: List[np.ndarray]          # per block (m, k*k); row i = vec(A_i)
    C: List[np.ndarray]           # per block (k, k)
    B: np.ndarray                 # (m, n)
    b: np.ndarray                 # (n,)

    @property
    def m(self) -> int:
        return int(self.c.shape[0])

    @property
    def n(self) -> int:
        return int(self.b.shape[0])

    @property
    def L(self) -> int:
        return len(self.k)

    def copy(self) -> "SDPProblem":
        return SDPProblem(self.c.copy(), list(self.k), [a.copy() for a in self.Av],
                          [c.copy() for c in self.C], self.B.copy(), self.b.copy())


def ingest(c: Sequence[float], A: Sequence[np.ndarray], C: Sequence[np.ndarray],
           B: Optional[np.ndarray] = None, b: Optional[Sequence[float]] = None) -> SDPProblem:
    """Build an `SDPProblem` from SDPX-style dense data.

    Mirrors the dense branch of `SDPX.ingest` (src/ingest.jl:675 `_ingest_dense`):
    `A[l]` is (m, k, k), `C[l]` is (k, k), `B` is (m, n), `b` is (n,).
    Coefficients must be symmetric; a non-symmetric coefficient raises.
    Equality rows (n > 0) are accepted by the container but the B200 core
    handles n == 0 only and rejects n > 0 at solve time.
    """
    c = np.ascontiguousarray(np.asarray(c, dtype=np.float64).reshape(-1))
    m = c.shape[0]
    if len(A) != len(C):
        raise ValueError("A and C must have one entry per block")
    ks: List[int] = []
    Av: List[np.ndarray] = []
    Cs: List[np.ndarray] = []
    for l, (Al, Cl) in enumerate(zip(A, C)):
        Al = np.asarray(Al, dtype=np.float64)
        if Al.ndim != 3 or Al.shape[0] != m or Al.shape[1] != Al.shape[2]:
            raise ValueError(f"A[{l}] must have shape (m, k, k) with m={m}")
        k = Al.shape[1]
        Cl = np.asarray(Cl, dtype=np.float64).reshape(k, k)
        if not np.array_equal(Al, np.transpose(Al, (0, 2, 1))):
            raise ValueError(f"A[{l}] coefficients must be symmetric")
        if not np.array_equal(Cl, Cl.T):
            raise ValueError(f"C[{l}] must be symmetric")
        ks.append(k)
        Av.append(np.ascontiguousarray(Al.reshape(m, k * k)))
        Cs.append(np.ascontiguousarray(Cl))
    if B is None:
        B = np.zeros((m, 0))
    B = np.ascontiguousarray(np.asarray(B, dtype=np.float64).reshape(m, -1))
    b = np.ascontiguousarray(np.asarray([] if b is None else b, dtype=np.float64).reshape(-1))
    if B.shape[1] != b.shape[0]:
        raise ValueError("B and b disagree on the equality count")
    return SDPProblem(c, ks, Av, Cs, B, b)


@dataclass
class Equilibration:
    """Scaling record of SDPX's `equilibrate` (src/ingest.jl:1431-1519)."""

    E: List[np.ndarray]          # per block diagonal congruence factors
    s: np.ndarray                # per-variable scales
    objective_scale: float
    ruiz_passes: List[int] = field(default_factory=list)


def unequilibrate(eq: Equilibration, x, X, y, Y):
    """Inverse map of `equilibrate`; restates src/ingest.jl:1522-1549."""
    x = np.asarray(x) / eq.s
    Xo, Yo = [], []
    for l, (Xl, Yl) in enumerate(zip(X, Y)):
        e = eq.E[l]
        outer = np.outer(e, e)
        Xo.append(np.asarray(Xl) / outer)
        Yo.append(np.asarray(Yl) * outer)
    y = np.asarray(y, dtype=np.float64)
    if eq.objective_scale != 1.0:
        y = y * eq.objective_scale
        Yo = [Yl * eq.objective_scale for Yl in Yo]
    return x, Xo, y, Yo
