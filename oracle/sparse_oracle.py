"""CPU oracle for the sparse Schur path — TEST INFRASTRUCTURE ONLY.

Restates SDPX's `SparseCons` Schur assembly in NumPy so that the device's
sparse engine (`sdpx_b200_set_sparse_schur`) can be checked against it and
against the dense assembly of the same iterate:

* `block_coo`           — `build_block_coo` (src/types/constraints.jl:79-101):
  the stored entries of every structurally active coefficient, in the block's
  `schur_order` (ascending variable index), each coefficient's entries in
  increasing column-major linear index (`lin`).
* `sparse_schur_block`  — `sparse_schur_block!` (src/schur.jl:936-1032), COO
  branch: W2 = X⁻¹ from the block factor (`kcholsolve!` on the identity),
  W1 = Y·A_p·X⁻¹ by `_two_sided_coo_product!` (:601-656: one rank-one term
  per stored entry, coefficient applied to the right factor's row), then
  ⟨W1, A_r⟩ for r ≥ p by `_dot_dense_coo` (:566-579).  The 2×2 packed branch
  of the reference computes the same quantity from three scalars.
* `sparse_schur_build`  — the lower-triangle scatter of every block's pairs in
  block order (`_reduce_sparse_schur_serial!`, :1173-1197, `schur_lower_only`).
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp


def block_coo(Av_l: np.ndarray, k: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(active, ptr, lin, val) of one block; Av_l is (m, k²), row i = vec(A_i)."""
    nz = Av_l != 0.0
    active = np.nonzero(nz.any(axis=1))[0]
    ptr = [0]
    lin, val = [], []
    for i in active:
        q = np.nonzero(nz[i])[0]
        lin.append(q)
        val.append(Av_l[i, q])
        ptr.append(ptr[-1] + q.size)
    lin_a = np.concatenate(lin) if lin else np.zeros(0, dtype=np.int64)
    val_a = np.concatenate(val) if val else np.zeros(0)
    return active, np.asarray(ptr, dtype=np.int64), lin_a.astype(np.int64), val_a


def x_inverse(LX: np.ndarray) -> np.ndarray:
    """X⁻¹ from the lower factor: `kcholsolve!(LX, I)` (src/kernels/generic.jl:218-248)."""
    k = LX.shape[0]
    Z = sla.solve_triangular(LX, np.eye(k), lower=True, check_finite=False)
    return sla.solve_triangular(LX.T, Z, lower=False, check_finite=False)


def sparse_schur_block(Y: np.ndarray, Xinv: np.ndarray, k: int, ptr, lin, val) -> np.ndarray:
    """Packed pairs of one block: out[p, r] = ⟨Y·A_p·X⁻¹, A_r⟩ for r ≥ p (zero below)."""
    na = len(ptr) - 1
    out = np.zeros((na, na))
    if na == 0:
        return out
    rows, cols = lin % k, lin // k
    G = sp.csr_matrix((val, lin, ptr), shape=(na, k * k))
    for p in range(na):
        W1 = np.zeros((k, k))
        for t in range(ptr[p], ptr[p + 1]):
            # dest += left[:, row] * (coefficient * right[column, :])
            W1 += np.outer(Y[:, rows[t]], val[t] * Xinv[cols[t], :])
        w = W1.reshape(-1, order="F")
        out[p, p:] = G[p:] @ w
    return out


def sparse_schur_build(Av: List[np.ndarray], k: List[int], LX: List[np.ndarray],
                       Y: List[np.ndarray], m: int) -> np.ndarray:
    """Lower triangle of S = Σ_l Σ_{pairs} ⟨Y_l A_p X_l⁻¹, A_r⟩, blocks in order."""
    S = np.zeros((m, m))
    for l, kl in enumerate(k):
        active, ptr, lin, val = block_coo(Av[l], kl)
        if active.size == 0:
            continue
        pairs = sparse_schur_block(Y[l], x_inverse(LX[l]), kl, ptr, lin, val)
        iu, ju = np.triu_indices(active.size)
        # pair (p, r), r ≥ p, lands in S[ids[r], ids[p]] (lower: ids ascending)
        np.add.at(S, (active[ju], active[iu]), pairs[iu, ju])
    return np.tril(S)
