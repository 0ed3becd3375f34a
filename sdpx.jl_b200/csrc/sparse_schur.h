// Sparse Schur assembly for structurally sparse constraint matrices (SDPX's
// `SparseCons` path, src/schur.jl:549-1300 and src/types/constraints.jl:26-101).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace sdpx {

// Largest block order the per-position kernel keeps in shared memory
// (k² doubles ≤ 200 KB).
constexpr int kSparseSchurMaxK = 160;

// nnz[i] = number of nonzero entries of column i of the k²-row slab of 𝒜
// starting at row `off` (one CTA per column).
void coo_count(const double* A, long long K, int m, long long off, int kk, int* nnz,
               cudaStream_t st);

// Flat coordinate entries of the active columns ids[0..na) of the slab, in
// increasing linear (column-major) index: lin[ptr[p] .. ptr[p+1]) and val[…]
// (one warp per active column; ptr is the global entry offset array).
void coo_fill(const double* A, long long K, long long off, int kk, const int* ids,
              const long long* ptr, int na, int* lin, double* val, cudaStream_t st);

// One block's Schur contribution, added into the lower triangle of S
// (column-major, leading dimension lds):
//   S[ids[r], ids[p]] += ⟨Y·A_p·X⁻¹, A_r⟩  for every active pair r ≥ p,
// with Y and Xinv the block's k×k matrices (column-major) and the COO entries
// of positions [0, na) at ptr/lin/val.  One CTA per position p builds
// W = Y·A_p·X⁻¹ in shared memory from the entries of A_p (a sum of nnz_p
// rank-one terms, `_two_sided_coo_product!`) and gathers ⟨W, A_r⟩ for r ≥ p
// (`_dot_dense_coo`).  Pairs of one launch write distinct entries of S.
void sparse_schur_block(const double* Y, const double* Xinv, int k, const long long* ptr,
                        const int* lin, const double* val, const int* ids, int na, double* S,
                        long long lds, cudaStream_t st);

}  // namespace sdpx
