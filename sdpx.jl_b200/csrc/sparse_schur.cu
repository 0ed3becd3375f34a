// Sparse Schur assembly (SDPX's SparseCons path).
//
// Coefficients of a PSD block are held, per structurally active variable, as
// flat coordinate entries in increasing column-major linear index — the
// `SparseBlockCOO` of src/types/constraints.jl:60-101 — extracted on the device
// from the block's k²-row slab of the stacked constraint matrix 𝒜.  The Schur
// contribution of a block is S_pr = ⟨Y·A_p·X⁻¹, A_r⟩ over the active pairs
// r ≥ p (`sparse_schur_block!`, src/schur.jl:936-1032): W = Y·A_p·X⁻¹ as a sum
// of nnz_p rank-one terms (`_two_sided_coo_product!`, :601-656), then one
// gather per stored entry of A_r (`_dot_dense_coo`, :566-579).  Work per block
// is Σ_p nnz_p·k² + Σ_{p≤r} nnz_r instead of the dense path's 2k³m + m²k².
#include "sparse_schur.h"

#include "common.cuh"

namespace sdpx {

namespace {

constexpr int kFillWarps = 8;
constexpr int kSchurThreads = 256;
constexpr int kEntryCache = 64;  // entries of A_p staged in shared memory per round

__global__ void k_coo_count(const double* __restrict__ A, long long K, long long off, int kk,
                            int* __restrict__ nnz) {
  __shared__ int red[32];
  const int i = blockIdx.x;
  const double* col = A + off + (long long)i * K;
  int c = 0;
  for (int q = threadIdx.x; q < kk; q += blockDim.x) c += col[q] != 0.0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = c;
  __syncthreads();
  if (w == 0) {
    c = lane < (int)(blockDim.x >> 5) ? red[lane] : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) nnz[i] = c;
  }
}

// One warp per active column: stream the slab in 32-row chunks, compact the
// nonzero rows with a ballot so the entries keep increasing linear index.
__global__ void k_coo_fill(const double* __restrict__ A, long long K, long long off, int kk,
                           const int* __restrict__ ids, const long long* __restrict__ ptr, int na,
                           int* __restrict__ lin, double* __restrict__ val) {
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * kFillWarps + (threadIdx.x >> 5);
  if (p >= na) return;
  const double* col = A + off + (long long)ids[p] * K;
  long long cursor = ptr[p];
  const long long end = ptr[p + 1];
  for (int q0 = 0; q0 < kk; q0 += 32) {
    const int q = q0 + lane;
    const double v = q < kk ? col[q] : 0.0;
    const bool nz = v != 0.0;
    const unsigned mask = __ballot_sync(0xffffffffu, nz);
    const long long at = cursor + __popc(mask & ((1u << lane) - 1u));
    if (nz && at < end) {
      lin[at] = q;
      val[at] = v;
    }
    cursor += __popc(mask);
  }
}

__global__ void __launch_bounds__(kSchurThreads)
    k_sparse_schur_block(const double* __restrict__ Y, const double* __restrict__ Xi, int k,
                         const long long* __restrict__ ptr, const int* __restrict__ lin,
                         const double* __restrict__ val, const int* __restrict__ ids, int na,
                         double* S, long long lds) {
  extern __shared__ __align__(16) double W[];  // k×k, column-major
  __shared__ int er[kEntryCache], ec[kEntryCache];
  __shared__ double ea[kEntryCache];
  const int p = blockIdx.x;
  const int kk = k * k;
  const long long t0 = ptr[p], t1 = ptr[p + 1];
  // W = Y·A_p·X⁻¹ = Σ_t a_t · Y[:, r_t] · X⁻¹[c_t, :]  (entries in increasing
  // linear index; each output element accumulates them in that order)
  for (int e = threadIdx.x; e < kk; e += kSchurThreads) W[e] = 0.0;
  for (long long tb = t0; tb < t1; tb += kEntryCache) {
    const int cnt = (int)min((long long)kEntryCache, t1 - tb);
    __syncthreads();
    if (threadIdx.x < cnt) {
      const int q = lin[tb + threadIdx.x];
      er[threadIdx.x] = q % k;
      ec[threadIdx.x] = q / k;
      ea[threadIdx.x] = val[tb + threadIdx.x];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kk; e += kSchurThreads) {
      const int i = e % k, j = e / k;
      double s = W[e];
      for (int t = 0; t < cnt; ++t) s += Y[i + er[t] * k] * (ea[t] * Xi[ec[t] + j * k]);
      W[e] = s;
    }
  }
  __syncthreads();
  // S[ids[r], ids[p]] += ⟨W, A_r⟩ for r ≥ p; column ids[p] belongs to this CTA.
  double* Scol = S + (long long)ids[p] * lds;
  for (int r = p + threadIdx.x; r < na; r += kSchurThreads) {
    double v = 0.0;
    for (long long t = ptr[r]; t < ptr[r + 1]; ++t) v += W[lin[t]] * val[t];
    Scol[ids[r]] += v;
  }
}

}  // namespace

void coo_count(const double* A, long long K, int m, long long off, int kk, int* nnz,
               cudaStream_t st) {
  if (m == 0) return;
  k_coo_count<<<m, 256, 0, st>>>(A, K, off, kk, nnz);
  SDPX_LAUNCH_CHECK();
}

void coo_fill(const double* A, long long K, long long off, int kk, const int* ids,
              const long long* ptr, int na, int* lin, double* val, cudaStream_t st) {
  if (na == 0) return;
  k_coo_fill<<<ceil_div(na, kFillWarps), 32 * kFillWarps, 0, st>>>(A, K, off, kk, ids, ptr, na,
                                                                    lin, val);
  SDPX_LAUNCH_CHECK();
}

void sparse_schur_block(const double* Y, const double* Xinv, int k, const long long* ptr,
                        const int* lin, const double* val, const int* ids, int na, double* S,
                        long long lds, cudaStream_t st) {
  if (na == 0) return;
  if (k < 1 || k > kSparseSchurMaxK)
    throw std::invalid_argument("sparse Schur: block order outside [1, 160]");
  const size_t smem = sizeof(double) * (size_t)k * k;
  smem_attr_ensure(reinterpret_cast<const void*>(k_sparse_schur_block), smem);
  k_sparse_schur_block<<<na, kSchurThreads, smem, st>>>(Y, Xinv, k, ptr, lin, val, ids, na, S,
                                                        lds);
  SDPX_LAUNCH_CHECK();
}

}  // namespace sdpx
