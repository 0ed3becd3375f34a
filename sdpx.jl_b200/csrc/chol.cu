// Cholesky (lower, right-looking, panel width NB).  Orders whose NB-wide
// panel fits in shared memory (the line-search trials and block factors) take
// one launch per panel that factors the whole panel in place; larger orders
// factor the diagonal tile once (one CTA per matrix), solve the rows below it
// with one thread per row, and update the trailing lower tiles.  A matrix whose
// pivot is not positive (or NaN) records `info = pivot index + 1` and every
// later CTA of that matrix returns at once — the no-throw contract of SDPX's
// `kchol!` (src/kernels/generic.jl:133-155).
//
// Inside a panel the columns are processed in blocks of 8: l_cc = sqrt(a_cc),
// l_rc = a_rc · (1/l_cc) (the reciprocal scaling of LAPACK's dpotf2),
// a_rq -= l_rc · l_qc, every element updated in increasing column order.
#include "chol.h"
#include "blas_f64.h"

namespace sdpx {

// Right-looking factor of the leading w columns of the rows×w panel P (shared,
// column-major, leading dimension ld; rows ≥ w).  Returns the failing column
// or -1.  All threads of the CTA take part.
//
// Blocked by 8 columns: every thread factors the 8×8 diagonal block in its
// registers (l_cc = sqrt(a_cc), column below scaled by 1/l_cc, as LAPACK's
// unblocked dpotf2 does) — the same arithmetic in every thread, so the factor
// needs no publication and no barrier of its own; each row below the block is
// solved in registers (x = a · L_bb^{-T}); after one barrier the trailing
// columns of the panel receive the rank-8 update (the block's rows read as
// warp broadcasts) while thread 0 writes the factored block back.  Two
// barriers per 8 columns.  Every element sees its updates in increasing column
// order.
template <class T>
__device__ int factor_panel_smem(T* P, int ld, int rows, int w) {
  __syncthreads();
  for (int kb = 0; kb < w; kb += 8) {
    const int kw = min(8, w - kb);
    T D[8][8], inv[8];
#pragma unroll
    for (int c = 0; c < 8; ++c)
#pragma unroll
      for (int r = 0; r < 8; ++r)
        D[c][r] = (c < kw && r < kw && r >= c) ? P[(kb + c) * ld + kb + r] : T(0);
    int fail = -1;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      inv[c] = T(0);
      if (c < kw && fail < 0) {
        const T piv = D[c][c];
        if (!(piv > T(0))) {
          fail = c;
        } else {
          const T lc = sqrt(piv);
          inv[c] = T(1) / lc;
          D[c][c] = lc;
#pragma unroll
          for (int r = c + 1; r < 8; ++r) D[c][r] *= inv[c];
#pragma unroll
          for (int q = c + 1; q < 8; ++q)
#pragma unroll
            for (int r = q; r < 8; ++r) D[q][r] -= D[c][r] * D[c][q];
        }
      }
    }
    if (fail >= 0) return kb + fail;  // the same in every thread
    // rows below the block: x = a · L_bb^{-T}
    for (int r = kb + kw + threadIdx.x; r < rows; r += blockDim.x) {
      T x[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) x[c] = (c < kw) ? P[(kb + c) * ld + r] : T(0);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < kw) {
          x[c] *= inv[c];
#pragma unroll
          for (int q = c + 1; q < 8; ++q) x[q] -= x[c] * D[c][q];
        }
      }
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c < kw) P[(kb + c) * ld + r] = x[c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int c = 0; c < 8; ++c)
#pragma unroll
        for (int r = 0; r < 8; ++r)
          if (c < kw && r < kw && r >= c) P[(kb + c) * ld + kb + r] = D[c][r];
    }
    // trailing panel columns q ∈ [kb+kw, w), rows r ≥ q.  With fewer rows
    // than threads (the diagonal tiles, the short last panels) several threads
    // share a row and take every `slices`-th column of it; each element gets
    // the same sum in the same order either way.
    {
      const int r0 = kb + kw, nrow = rows - r0;
      const int slices = nrow > 0 ? max(1, (int)blockDim.x / nrow) : 1;
      for (int idx = threadIdx.x; idx < nrow * slices; idx += blockDim.x) {
        const int r = r0 + idx % nrow, sl = idx / nrow;
        T x[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) x[c] = (c < kw) ? P[(kb + c) * ld + r] : T(0);
        const int qe = min(w, r + 1);
        for (int q = r0 + sl; q < qe; q += slices) {
          T a = P[q * ld + r];
#pragma unroll
          for (int c = 0; c < 8; ++c)
            if (c < kw) a -= x[c] * P[(kb + c) * ld + q];
          P[q * ld + r] = a;
        }
      }
    }
    __syncthreads();
  }
  return -1;
}

template <class T>
__device__ void note_pivots(const T* P, int ld, int w, T* dmin, T* dmax, int b) {
  if (threadIdx.x != 0) return;
  T lo = dmin[b], hi = dmax[b];
  for (int c = 0; c < w; ++c) {
    T v = fabs(P[c * ld + c]);
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  dmin[b] = lo;
  dmax[b] = hi;
}

// The lower part of the w×w diagonal tile at (c0, c0) into shared D (column
// c at D[c·LD + …], zeros above the diagonal and outside w).  NT threads; each
// issues all of its NB·NB/NT loads before any shared store, so the tile costs
// one memory round trip.
template <class T, int NB, int NT>
__device__ __forceinline__ void load_diag_tile(T* D, int LD, const MatDesc<T>& M, int c0, int w) {
  constexpr int PER = NB * NB / NT;
  static_assert(NB * NB % NT == 0, "tile split");
  T v[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = threadIdx.x + k * NT, r = e % NB, c = e / NB;
    v[k] = (r < w && c < w && r >= c) ? M.a[(size_t)(c0 + c) * M.ld + (c0 + r)] : T(0);
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = threadIdx.x + k * NT, r = e % NB, c = e / NB;
    if (r < w && c < w) D[c * LD + r] = v[k];
  }
}

// Tiled path, step 1: factor the diagonal tile of panel j (one CTA per matrix).
template <class T, int NB>
__global__ void __launch_bounds__(256) k_potrf_diag(const MatDesc<T>* mats, int j, int* info, T* dmin, T* dmax) {
  __shared__ T D[NB * (NB + 1)];
  constexpr int LD = NB + 1;
  const int b = blockIdx.x;
  const MatDesc<T> M = mats[b];
  const int c0 = j * NB;
  if (c0 >= M.n || info[b] != 0) return;
  const int w = min(NB, M.n - c0);
  load_diag_tile<T, NB, 256>(D, LD, M, c0, w);
  const int fail = factor_panel_smem<T>(D, LD, w, w);
  if (fail >= 0) {
    if (threadIdx.x == 0) info[b] = c0 + fail + 1;
    return;
  }
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int r = e % NB, c = e / NB;
    if (r < w && c < w && r >= c) M.a[(size_t)(c0 + c) * M.ld + (c0 + r)] = D[c * LD + r];
  }
  note_pivots(D, LD, w, dmin, dmax, b);
}

// Tiled path, step 2: rows below the diagonal tile, X = B · L_jj^{-T}, one
// thread per row with the row held in registers (forward substitution in the
// column order of the right-looking panel factor, scaling by the reciprocal
// pivots).
template <class T, int NB>
__global__ void __launch_bounds__(128) k_potrf_trsm_rows(const MatDesc<T>* mats, int j,
                                                         const int* info) {
  __shared__ T D[NB * (NB + 1)];
  constexpr int LD = NB + 1;
  const int b = blockIdx.y;
  const MatDesc<T> M = mats[b];
  const int c0 = j * NB;
  if (c0 >= M.n || info[b] != 0) return;
  const int w = min(NB, M.n - c0);
  const int first = c0 + w + blockIdx.x * blockDim.x;
  if (first >= M.n) return;
  load_diag_tile<T, NB, 128>(D, LD, M, c0, w);
  __shared__ T inv[NB];
  __syncthreads();  // the diagonal tile is loaded
  for (int c = threadIdx.x; c < w; c += blockDim.x) inv[c] = T(1) / D[c * LD + c];
  __syncthreads();
  const int r = first + threadIdx.x;
  if (r >= M.n) return;
  T x[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) x[c] = (c < w) ? M.a[(size_t)(c0 + c) * M.ld + r] : T(0);
#pragma unroll
  for (int c = 0; c < NB; ++c) {
    if (c < w) {
      x[c] *= inv[c];
#pragma unroll
      for (int q = c + 1; q < NB; ++q) x[q] -= x[c] * D[c * LD + q];
    }
  }
#pragma unroll
  for (int c = 0; c < NB; ++c)
    if (c < w) M.a[(size_t)(c0 + c) * M.ld + r] = x[c];
}

// Whole panel in shared memory (orders n with n·NB elements ≤ 224 KB): one CTA
// per matrix loads rows [c0, n) of panel j, factors it in place and writes it
// back; the trailing tiles are then updated by k_potrf_update.
template <class T, int NB>
__global__ void __launch_bounds__(512) k_potrf_panel_smem(const MatDesc<T>* mats, int j, int* info, T* dmin, T* dmax) {
  extern __shared__ __align__(16) unsigned char raw[];
  T* Pn = reinterpret_cast<T*>(raw);  // rows × NB, column-major with ld = rows | 1
  const MatDesc<T> M = mats[blockIdx.x];
  const int b = blockIdx.x;
  const int c0 = j * NB;
  if (c0 >= M.n || info[b] != 0) return;
  const int w = min(NB, M.n - c0);
  const int rows = M.n - c0;
  const int ld = rows | 1;  // odd stride: conflict-free column walks
  // A warp per column, lanes along the rows; each lane issues its PU loads of
  // a batch before storing any, so a column costs one memory round trip per
  // 32·PU rows instead of one per element.
  constexpr int PU = 8;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int c = warp; c < w; c += nwarp) {
    const T* src = M.a + (size_t)(c0 + c) * M.ld + c0;
    for (int rb = 0; rb < rows; rb += 32 * PU) {
      T v[PU];
#pragma unroll
      for (int u = 0; u < PU; ++u) {
        const int r = rb + lane + 32 * u;
        v[u] = (r < rows && r >= c) ? src[r] : T(0);
      }
#pragma unroll
      for (int u = 0; u < PU; ++u) {
        const int r = rb + lane + 32 * u;
        if (r < rows) Pn[c * ld + r] = v[u];
      }
    }
  }
  const int fail = factor_panel_smem<T>(Pn, ld, rows, w);
  if (fail >= 0) {
    if (threadIdx.x == 0) info[b] = c0 + fail + 1;
    return;
  }
  for (int c = warp; c < w; c += nwarp) {
    T* dst = M.a + (size_t)(c0 + c) * M.ld + c0;
    for (int r = lane; r < rows; r += 32) dst[r] = (r >= c) ? Pn[c * ld + r] : T(0);
  }
  note_pivots(Pn, ld, w, dmin, dmax, b);
}

// Trailing update A[i,q] -= L[i,j] L[q,j]^T for j < q <= i (lower tiles).
template <class T, int NB>
__global__ void k_potrf_update(const MatDesc<T>* mats, int j, const int* info) {
  extern __shared__ __align__(16) unsigned char raw[];
  T* La = reinterpret_cast<T*>(raw);  // NB × (NB+1): rows of tile i, panel j
  T* Lb = La + NB * (NB + 1);          // rows of tile q
  constexpr int LD = NB + 1;
  const MatDesc<T> M = mats[blockIdx.y];
  if (info[blockIdx.y] != 0) return;
  const int nt = (M.n + NB - 1) / NB;
  if (j >= nt) return;
  const int rem = nt - j - 1;
  const int u = blockIdx.x;
  if (rem <= 0 || u >= rem * (rem + 1) / 2) return;
  int a = (int)((sqrt(8.0 * u + 1.0) - 1.0) * 0.5);
  while ((a + 1) * (a + 2) / 2 <= u) ++a;
  while (a * (a + 1) / 2 > u) --a;
  const int bq = u - a * (a + 1) / 2;
  const int i = j + 1 + a, q = j + 1 + bq;
  const int c0 = j * NB, r0 = i * NB, q0 = q * NB;
  const int w = min(NB, M.n - c0), h = min(NB, M.n - r0), hq = min(NB, M.n - q0);
  // Each thread owns an RB×RB block of outputs, RB = NB/16: 256 threads for
  // NB = 64 (4×4), 48 (3×3) and 32 (2×2).  Its outputs are read together with
  // the two operand tiles (each output tile belongs to this CTA alone), so the
  // read-modify-write at the end waits for no memory.
  constexpr int RB = NB / 16;
  constexpr int TPR = NB / RB;
  const int tr = threadIdx.x % TPR, tc = threadIdx.x / TPR;
  T cur[RB][RB];
#pragma unroll
  for (int x = 0; x < RB; ++x)
#pragma unroll
    for (int y = 0; y < RB; ++y) {
      const int r = tr + x * TPR, c = tc + y * TPR;
      cur[x][y] = (tc < TPR && r < h && c < hq) ? M.a[(size_t)(q0 + c) * M.ld + (r0 + r)] : T(0);
    }
  {
    // All loads of the two tiles are issued before the shared stores (one
    // memory round trip per tile instead of one per loop trip).
    constexpr int PER = NB * NB / 256;
    static_assert(NB * NB % 256 == 0, "tile load split");
    T va[PER], vb[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int e = threadIdx.x + k * 256, r = e % NB, c = e / NB;
      va[k] = (r < h && c < w) ? M.a[(size_t)(c0 + c) * M.ld + (r0 + r)] : T(0);
      vb[k] = (r < hq && c < w) ? M.a[(size_t)(c0 + c) * M.ld + (q0 + r)] : T(0);
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int e = threadIdx.x + k * 256, r = e % NB, c = e / NB;
      La[c * LD + r] = va[k];
      Lb[c * LD + r] = vb[k];
    }
  }
  __syncthreads();
  if (tc < TPR) {
    T acc[RB][RB] = {};
    for (int p = 0; p < w; ++p) {
      T av[RB], bv[RB];
#pragma unroll
      for (int x = 0; x < RB; ++x) av[x] = La[p * LD + tr + x * TPR];
#pragma unroll
      for (int y = 0; y < RB; ++y) bv[y] = Lb[p * LD + tc + y * TPR];
#pragma unroll
      for (int x = 0; x < RB; ++x)
#pragma unroll
        for (int y = 0; y < RB; ++y) acc[x][y] += av[x] * bv[y];
    }
#pragma unroll
    for (int x = 0; x < RB; ++x)
#pragma unroll
      for (int y = 0; y < RB; ++y) {
        int r = tr + x * TPR, c = tc + y * TPR;
        if (r < h && c < hq) M.a[(size_t)(q0 + c) * M.ld + (r0 + r)] = cur[x][y] - acc[x][y];
      }
  }
}

// Strict upper triangle set to zero: a warp per column (rows 0 … c-1).
template <class T>
__global__ void k_zero_upper(const MatDesc<T>* mats) {
  const MatDesc<T> M = mats[blockIdx.y];
  const int lane = threadIdx.x & 31;
  for (int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < M.n;
       c += gridDim.x * (blockDim.x >> 5)) {
    T* col = M.a + (size_t)c * M.ld;
    for (int r = lane; r < c; r += 32) col[r] = T(0);
  }
}

template <class T>
__global__ void k_init_stats(int n, int* info, T* dmin, T* dmax) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n) {
    info[b] = 0;
    dmin[b] = T(1.0 / 0.0);
    dmax[b] = T(0);
  }
}

template <class T, int NB>
void potrf_batched(const MatDesc<T>* d_mats, int nmat, int nmax, int* info, T* dmin, T* dmax,
                   cudaStream_t st, bool zero_upper) {
  if (nmat == 0 || nmax == 0) return;
  const size_t smem = 2 * sizeof(T) * NB * (NB + 1);
  ensure_smem(k_potrf_update<T, NB>, smem);
  k_init_stats<T><<<ceil_div(nmat, 128), 128, 0, st>>>(nmat, info, dmin, dmax);
  const int nt = ceil_div(nmax, NB);
  const int rows_pad = nmax | 1;
  const size_t panel_smem = sizeof(T) * (size_t)rows_pad * NB;
  const bool whole_panel = panel_smem <= 224 * 1024;
  if (whole_panel) ensure_smem(k_potrf_panel_smem<T, NB>, panel_smem);
  int launches = 1;  // k_init_stats
  for (int j = 0; j < nt; ++j) {
    int rem = nt - j - 1;
    if (whole_panel) {
      k_potrf_panel_smem<T, NB><<<nmat, 512, panel_smem, st>>>(d_mats, j, info, dmin, dmax);
      ++launches;
    } else {
      k_potrf_diag<T, NB><<<nmat, 256, 0, st>>>(d_mats, j, info, dmin, dmax);
      ++launches;
      const int below = nmax - (j + 1) * NB;
      if (below > 0) {
        dim3 gt(ceil_div(below, 128), nmat);
        k_potrf_trsm_rows<T, NB><<<gt, 128, 0, st>>>(d_mats, j, info);
        ++launches;
      }
    }
    if (rem > 0) {
      dim3 g2(rem * (rem + 1) / 2, nmat);
      k_potrf_update<T, NB><<<g2, 256, smem, st>>>(d_mats, j, info);
      ++launches;
    }
  }
  if (zero_upper) {
    dim3 gz(std::max(1, ceil_div(nmax, 8)), nmat);
    k_zero_upper<T><<<gz, 256, 0, st>>>(d_mats);
    ++launches;
  }
  SDPX_LAUNCH_CHECK_N(launches);
}

// ---------------------------------------------------------------------------
// One large matrix (the Schur factor): the whole right-looking factorization
// in one cooperative launch of at most one CTA per SM, panels separated by
// grid barriers instead of kernel boundaries.  Per panel j:
//   A  every CTA loads the factored diagonal tile and solves its contiguous
//      share of the rows below (X = B·L_jj⁻ᵀ in the operation order of
//      k_potrf_trsm_rows, 16 threads per row);
//   B  after a barrier, CTA 0 updates the next diagonal tile and factors it
//      in shared memory at once (look-ahead: the factor's latency chain runs
//      while the other CTAs update the remaining trailing lower tiles), with
//      the arithmetic of k_potrf_diag, so the factor is bit-identical to the
//      batched path's; tile updates are FP64 on DMMA m8n8k4 fragments, FP32
//      on 4×4 register tiles;
//   and a barrier before the next panel.  Matrix loads bypass L1 (__ldcg):
//   other SMs wrote the data since this SM may last have cached it.  A pivot
//   failure is published in the barrier state before the barrier, so every
//   CTA reads it at the same panel and all leave together.
//   Barrier waits are bounded (about a second); on a timeout the kernel sets
//   info = −1 and every CTA returns.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned coop_ld(const unsigned* p) {
  return *reinterpret_cast<const volatile unsigned*>(p);
}

__device__ bool coop_barrier(CoopBar* bar, unsigned nblocks, int* info) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g = coop_ld(&bar->gen);
    __threadfence();
    if (atomicAdd(&bar->count, 1u) == nblocks - 1) {
      atomicExch(&bar->count, 0u);
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      unsigned long long spins = 0;
      while (coop_ld(&bar->gen) == g) {
        if (coop_ld(&bar->err) != 0u || ++spins > (1ull << 24)) {
          atomicExch(&bar->err, 1u);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (!ok || coop_ld(&bar->err) != 0u) {
      ok = 0;
      atomicExch(info, -1);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Lower part of the h×w tile at (r0, c0) into shared T (column c at
// T[c·LD + …]), zeros elsewhere up to NB×NB; `lower` masks r < c.
template <class T, int NB>
__device__ __forceinline__ void coop_load_tile(T* Ts, const T* a, int ld, int r0, int c0, int h, int w,
                                               bool lower) {
  constexpr int LD = NB + 1, PER = NB * NB / 256;
  T v[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = threadIdx.x + k * 256, r = e % NB, c = e / NB;
    v[k] = (r < h && c < w && (!lower || r >= c)) ? __ldcg(a + (size_t)(c0 + c) * ld + (r0 + r)) : T(0);
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = threadIdx.x + k * 256, r = e % NB, c = e / NB;
    Ts[c * LD + r] = v[k];
  }
}

// Trailing tile (i, q) of panel j, FP32: 4×4 register tiles (k_potrf_update's
// arithmetic).
template <int NB>
__device__ __forceinline__ void coop_update_tile(float* a, int ld, int n, int c0, int r0, int q0,
                                                 bool diag, float* La, float* Lb) {
  constexpr int LD = NB + 1, RB = NB / 16, TPR = NB / RB;
  const int w = min(NB, n - c0), h = min(NB, n - r0), hq = min(NB, n - q0);
  const int tr = threadIdx.x % TPR, tc = threadIdx.x / TPR;
  float cur[RB][RB];
#pragma unroll
  for (int x = 0; x < RB; ++x)
#pragma unroll
    for (int y = 0; y < RB; ++y) {
      const int r = tr + x * TPR, c = tc + y * TPR;
      cur[x][y] = (r < h && c < hq) ? __ldcg(a + (size_t)(q0 + c) * ld + (r0 + r)) : 0.f;
    }
  __syncthreads();  // the previous tile's reads of La/Lb are done
  coop_load_tile<float, NB>(La, a, ld, r0, c0, h, w, false);
  coop_load_tile<float, NB>(Lb, a, ld, q0, c0, hq, w, false);
  __syncthreads();
  float acc[RB][RB] = {};
  for (int p = 0; p < w; ++p) {
    float av[RB], bv[RB];
#pragma unroll
    for (int x = 0; x < RB; ++x) av[x] = La[p * LD + tr + x * TPR];
#pragma unroll
    for (int y = 0; y < RB; ++y) bv[y] = Lb[p * LD + tc + y * TPR];
#pragma unroll
    for (int x = 0; x < RB; ++x)
#pragma unroll
      for (int y = 0; y < RB; ++y) acc[x][y] += av[x] * bv[y];
  }
#pragma unroll
  for (int x = 0; x < RB; ++x)
#pragma unroll
    for (int y = 0; y < RB; ++y) {
      const int r = tr + x * TPR, c = tc + y * TPR;
      if (r < h && c < hq && (!diag || r >= c))
        a[(size_t)(q0 + c) * ld + (r0 + r)] = cur[x][y] - acc[x][y];
    }
}

// FP64: warp wp owns rows 8·wp … 8·wp+7 of the tile and all eight 8-column
// fragments; K runs over the panel's columns in steps of 4 (zero-padded).
template <int NB>
__device__ __forceinline__ void coop_update_tile(double* a, int ld, int n, int c0, int r0, int q0,
                                                 bool diag, double* La, double* Lb) {
  static_assert(NB == 64, "the DMMA tile update covers 64×64 tiles with 8 warps");
  constexpr int LD = NB + 1;
  const int w = min(NB, n - c0), h = min(NB, n - r0), hq = min(NB, n - q0);
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int r = wp * 8 + g;
  double cur[8][2];
#pragma unroll
  for (int fc = 0; fc < 8; ++fc)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int c = fc * 8 + 2 * t + e;
      cur[fc][e] = (r < h && c < hq) ? __ldcg(a + (size_t)(q0 + c) * ld + (r0 + r)) : 0.0;
    }
  __syncthreads();
  coop_load_tile<double, NB>(La, a, ld, r0, c0, h, w, false);
  coop_load_tile<double, NB>(Lb, a, ld, q0, c0, hq, w, false);
  __syncthreads();
  double acc[8][2] = {};
  for (int kk = 0; kk < w; kk += 4) {
    const double av = La[(kk + t) * LD + r];
#pragma unroll
    for (int fc = 0; fc < 8; ++fc) dmma_8x8x4(acc[fc][0], acc[fc][1], av, Lb[(kk + t) * LD + fc * 8 + g]);
  }
#pragma unroll
  for (int fc = 0; fc < 8; ++fc)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int c = fc * 8 + 2 * t + e;
      if (r < h && c < hq && (!diag || r >= c))
        a[(size_t)(q0 + c) * ld + (r0 + r)] = cur[fc][e] - acc[fc][e];
    }
}

// The NB×NB diagonal tile (shared, ld LD, order w) factored by one CTA with
// the arithmetic of factor_panel_smem — 8×8 block in registers (l_cc =
// sqrt(a_cc), 1/l_cc scaling), rows below solved against it, rank-8 update of
// the trailing columns, every element in increasing column order — so the
// factor is bit-identical to the batched path's.  Only warp 0 runs the 8×8
// block factor (every thread of factor_panel_smem repeats it, which saturates
// the FP64 pipe); its result and the reciprocal pivots go to shared memory.
// The trailing update takes two columns per step for two independent chains.
template <class T, int NB>
__device__ int factor_diag_tile(T* D, int LD, int w, T* sinv, int* sfail) {
  __syncthreads();
  for (int kb = 0; kb < w; kb += 8) {
    const int kw = min(8, w - kb);
    if (threadIdx.x < 32) {
      T B[8][8], inv[8];
#pragma unroll
      for (int c = 0; c < 8; ++c)
#pragma unroll
        for (int r = 0; r < 8; ++r)
          B[c][r] = (c < kw && r < kw && r >= c) ? D[(kb + c) * LD + kb + r] : T(0);
      int fail = -1;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        inv[c] = T(0);
        if (c < kw && fail < 0) {
          const T piv = B[c][c];
          if (!(piv > T(0))) {
            fail = c;
          } else {
            const T lc = sqrt(piv);
            inv[c] = T(1) / lc;
            B[c][c] = lc;
#pragma unroll
            for (int r = c + 1; r < 8; ++r) B[c][r] *= inv[c];
#pragma unroll
            for (int q = c + 1; q < 8; ++q)
#pragma unroll
              for (int r = q; r < 8; ++r) B[q][r] -= B[c][r] * B[c][q];
          }
        }
      }
      __syncwarp();
      if (threadIdx.x == 0) {
        *sfail = fail;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          sinv[c] = inv[c];
#pragma unroll
          for (int r = 0; r < 8; ++r)
            if (c < kw && r < kw && r >= c) D[(kb + c) * LD + kb + r] = B[c][r];
        }
      }
    }
    __syncthreads();
    if (*sfail >= 0) return kb + *sfail;  // the same in every thread
    // rows below the block: x = a · L_bb^{-T}
    for (int r = kb + kw + threadIdx.x; r < w; r += blockDim.x) {
      T x[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) x[c] = (c < kw) ? D[(kb + c) * LD + r] : T(0);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < kw) {
          x[c] *= sinv[c];
#pragma unroll
          for (int q = c + 1; q < 8; ++q) x[q] -= x[c] * D[(kb + c) * LD + kb + q];
        }
      }
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c < kw) D[(kb + c) * LD + r] = x[c];
    }
    __syncthreads();
    {
      const int r0 = kb + kw, nrow = w - r0;
      const int slices = nrow > 0 ? max(1, (int)blockDim.x / nrow) : 1;
      for (int idx = threadIdx.x; idx < nrow * slices; idx += blockDim.x) {
        const int r = r0 + idx % nrow, sl = idx / nrow;
        T x[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) x[c] = (c < kw) ? D[(kb + c) * LD + r] : T(0);
        const int qe = min(w, r + 1);
        int q = r0 + sl;
        for (; q + slices < qe; q += 2 * slices) {
          const int q2 = q + slices;
          T a1 = D[q * LD + r], a2 = D[q2 * LD + r];
#pragma unroll
          for (int c = 0; c < 8; ++c)
            if (c < kw) {
              a1 -= x[c] * D[(kb + c) * LD + q];
              a2 -= x[c] * D[(kb + c) * LD + q2];
            }
          D[q * LD + r] = a1;
          D[q2 * LD + r] = a2;
        }
        if (q < qe) {
          T a1 = D[q * LD + r];
#pragma unroll
          for (int c = 0; c < 8; ++c)
            if (c < kw) a1 -= x[c] * D[(kb + c) * LD + q];
          D[q * LD + r] = a1;
        }
      }
    }
    __syncthreads();
  }
  return -1;
}

// Rows [r0, r1) of panel c0 solved against the factored diagonal tile D:
// X = B·L⁻ᵀ with 16 threads per row, thread s owning columns s, s+16, s+32,
// s+48; column c's value is finished by its owner (x_c ← x_c·(1/l_cc)) and
// shuffled to the row's other threads, which subtract x_c·l_qc from their
// columns q > c — the operation order of k_potrf_trsm_rows.
template <class T, int NB>
__device__ void coop_trsm_rows(T* a, int ld, int c0, int w, int r0, int r1, const T* D, int LD,
                               const T* inv) {
  static_assert(NB == 64, "16 threads × 4 columns per row");
  const int s = threadIdx.x & 15, grp = threadIdx.x >> 4, ngrp = blockDim.x >> 4;
  const unsigned gmask = 0xffffu << (threadIdx.x & 16);
  for (int rb = r0; rb < r1; rb += ngrp) {  // uniform trip count within each warp
    const int r = rb + grp;
    const bool live = r < r1;
    T x[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int c = s + 16 * u;
      x[u] = (live && c < w) ? __ldcg(a + (size_t)(c0 + c) * ld + r) : T(0);
    }
    for (int c = 0; c < w; ++c) {
      const int owner = c & 15, uc = c >> 4;
      T xc = T(0);
      if (s == owner) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (u == uc) {
            x[u] *= inv[c];
            xc = x[u];
          }
      }
      xc = __shfl_sync(gmask, xc, owner, 16);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = s + 16 * u;
        if (q > c && q < w) x[u] -= xc * D[c * LD + q];
      }
    }
    if (live)
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int c = s + 16 * u;
        if (c < w) a[(size_t)(c0 + c) * ld + r] = x[u];
      }
  }
}

// CTA 0: the diagonal tile at (c0, c0) (already updated) factored in its
// shared memory D and written back; the failing pivot (1-based) goes to
// bar->fail, the pivot range to lo/hi (thread 0).
template <class T, int NB>
__device__ void coop_factor_diag(T* a, int n, int ld, int c0, T* D, T* sinv8, int* sfail, CoopBar* bar,
                                 T& lo, T& hi) {
  constexpr int LD = NB + 1;
  const int w = min(NB, n - c0);
  __syncthreads();
  coop_load_tile<T, NB>(D, a, ld, c0, c0, w, w, true);
  const int fail = factor_diag_tile<T, NB>(D, LD, w, sinv8, sfail);
  if (fail >= 0) {
    if (threadIdx.x == 0) atomicExch(&bar->fail, (unsigned)(c0 + fail + 1));
    return;
  }
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int r = e % NB, c = e / NB;
    if (r < w && c < w && r >= c) a[(size_t)(c0 + c) * ld + (c0 + r)] = D[c * LD + r];
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < w; ++c) {
      const T v = fabs(D[c * LD + c]);
      lo = fmin(lo, v);
      hi = fmax(hi, v);
    }
}

template <class T, int NB>
__global__ void __launch_bounds__(256) k_potrf_coop(T* a, int n, int ld, int* info, T* dmin, T* dmax,
                                                   CoopBar* bar, int zero_upper) {
  extern __shared__ __align__(16) unsigned char raw[];
  constexpr int LD = NB + 1;
  T* D = reinterpret_cast<T*>(raw);  // the diagonal tile; in updates, operand La
  T* Lb = D + NB * LD;
  __shared__ T inv[NB];
  __shared__ T sinv8[8];
  __shared__ int sfail;
  const int nt = (n + NB - 1) / NB;
  const unsigned G = gridDim.x;
  T lo = T(INFINITY), hi = T(0);
  if (blockIdx.x == 0) coop_factor_diag<T, NB>(a, n, ld, 0, D, sinv8, &sfail, bar, lo, hi);
  if (nt > 1 && !coop_barrier(bar, G, info)) return;
  for (int j = 0; j < nt; ++j) {
    const int c0 = j * NB, w = min(NB, n - c0);
    __syncthreads();  // CTA 0's own flag write is visible to all of its threads
    const unsigned failed = coop_ld(&bar->fail);  // read after a barrier: the same in every CTA
    if (failed != 0u) {
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        info[0] = (int)failed;
        dmin[0] = lo;
        dmax[0] = hi;
      }
      return;
    }
    if (j == nt - 1) break;
    // A: the rows below against the factored diagonal tile
    __syncthreads();
    coop_load_tile<T, NB>(D, a, ld, c0, c0, w, w, true);
    __syncthreads();
    for (int c = threadIdx.x; c < w; c += blockDim.x) inv[c] = T(1) / D[c * LD + c];
    __syncthreads();
    const int rfirst = c0 + w, nrow = n - rfirst;
    const int per = (nrow + (int)G - 1) / (int)G;
    const int r0 = min(n, rfirst + (int)blockIdx.x * per), r1 = min(n, r0 + per);
    coop_trsm_rows<T, NB>(a, ld, c0, w, r0, r1, D, LD, inv);
    if (!coop_barrier(bar, G, info)) return;
    // B: CTA 0 updates the next diagonal tile and factors it at once (the
    // look-ahead), the other CTAs take the remaining trailing tiles
    const int rem = nt - j - 1, ntile = rem * (rem + 1) / 2;
    if (blockIdx.x == 0) {
      coop_update_tile<NB>(a, ld, n, c0, (j + 1) * NB, (j + 1) * NB, true, D, Lb);
      coop_factor_diag<T, NB>(a, n, ld, (j + 1) * NB, D, sinv8, &sfail, bar, lo, hi);
    }
    const int first = G > 1 ? (int)blockIdx.x - 1 : 1;
    const int step = G > 1 ? (int)G - 1 : 1;
    if (G == 1 || blockIdx.x > 0)
      for (int u = 1 + (G > 1 ? first : 0); u < ntile; u += step) {
        int ti = (int)((sqrt(8.0 * u + 1.0) - 1.0) * 0.5);
        while ((ti + 1) * (ti + 2) / 2 <= u) ++ti;
        while (ti * (ti + 1) / 2 > u) --ti;
        const int tq = u - ti * (ti + 1) / 2;
        const int i = j + 1 + ti, q = j + 1 + tq;
        coop_update_tile<NB>(a, ld, n, c0, i * NB, q * NB, i == q, D, Lb);
      }
    if (!coop_barrier(bar, G, info)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    dmin[0] = lo;
    dmax[0] = hi;
  }
  if (zero_upper) {  // strict upper triangle: a warp per column
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int c = blockIdx.x * nw + (threadIdx.x >> 5); c < n; c += G * nw)
      for (int r = lane; r < c; r += 32) a[(size_t)c * ld + r] = T(0);
  }
}

template <class T, int NB>
void potrf_single(T* a, int n, int ld, int* info, T* dmin, T* dmax, CoopBar* bar, bool zero_upper,
                  cudaStream_t st) {
  if (n <= 0) return;
  const size_t smem = 2 * sizeof(T) * NB * (NB + 1);
  ensure_smem(k_potrf_coop<T, NB>, smem);
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  SDPX_CUDA(cudaGetDevice(&dev));
  SDPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  SDPX_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  SDPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_potrf_coop<T, NB>, 256, smem));
  if (!coop || per_sm < 1) throw CudaError("potrf_single: cooperative launch unavailable");
  const int nt = ceil_div(n, NB);
  const int grid = std::max(1, std::min(sms, nt * (nt - 1) / 2));
  SDPX_CUDA(cudaMemsetAsync(bar, 0, sizeof(CoopBar), st));
  SDPX_CUDA(cudaMemsetAsync(info, 0, sizeof(int), st));
  int zu = zero_upper ? 1 : 0;
  void* args[] = {&a, &n, &ld, &info, &dmin, &dmax, &bar, &zu};
  SDPX_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_potrf_coop<T, NB>), dim3(grid),
                                        dim3(256), args, smem, st));
}
template void potrf_single<double, 64>(double*, int, int, int*, double*, double*, CoopBar*, bool,
                                       cudaStream_t);
template void potrf_single<float, 64>(float*, int, int, int*, float*, float*, CoopBar*, bool,
                                      cudaStream_t);

template void potrf_batched<double, 32>(const MatDesc<double>*, int, int, int*, double*, double*,
                                        cudaStream_t, bool);
template void potrf_batched<double, 48>(const MatDesc<double>*, int, int, int*, double*, double*,
                                        cudaStream_t, bool);
template void potrf_batched<double, 64>(const MatDesc<double>*, int, int, int*, double*, double*,
                                        cudaStream_t, bool);
template void potrf_batched<float, 64>(const MatDesc<float>*, int, int, int*, float*, float*,
                                       cudaStream_t, bool);

// ---------------------------------------------------------------------------
// Triangular inverse W = L^{-1} (lower), blocked by NB.  Step 0 inverts every
// diagonal tile; step i fills block row i:  W[i,j] = -W[i,i] Σ_{p=j}^{i-1} L[i,p] W[p,j].
// W must be zero-initialised (its strict upper triangle stays zero).
// ---------------------------------------------------------------------------
template <class T, int NB>
__global__ void k_trinv_diag(const MatDesc<T>* Ls, const MatDesc<T>* Ws) {
  __shared__ T Lt[NB][NB + 1];
  __shared__ T Wt[NB][NB + 1];
  const MatDesc<T> L = Ls[blockIdx.y], W = Ws[blockIdx.y];
  const int s0 = blockIdx.x * NB;
  if (s0 >= L.n) return;
  const int w = min(NB, L.n - s0);
  for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
    int r = e % w, c = e / w;
    Lt[c][r] = L.a[(size_t)(s0 + c) * L.ld + s0 + r];
  }
  __syncthreads();
  for (int c = threadIdx.x; c < w; c += blockDim.x) {
    Wt[c][c] = T(1) / Lt[c][c];
    for (int r = c + 1; r < w; ++r) {
      T s = T(0);
      for (int p = c; p < r; ++p) s += Lt[p][r] * Wt[c][p];
      Wt[c][r] = -s / Lt[r][r];
    }
    for (int r = 0; r < c; ++r) Wt[c][r] = T(0);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
    int r = e % w, c = e / w;
    W.a[(size_t)(s0 + c) * W.ld + s0 + r] = Wt[c][r];
  }
}

template <class T, int NB>
__global__ void k_trinv_row(const MatDesc<T>* Ls, const MatDesc<T>* Ws, int i) {
  __shared__ T Acc[NB][NB + 1];
  __shared__ T Lt[NB][NB + 1];
  __shared__ T Wt[NB][NB + 1];
  const MatDesc<T> L = Ls[blockIdx.y], W = Ws[blockIdx.y];
  const int nt = (L.n + NB - 1) / NB;
  if (i >= nt) return;
  const int j = blockIdx.x;
  if (j >= i) return;
  const int r0 = i * NB, h = min(NB, L.n - r0);
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) Acc[e / NB][e % NB] = T(0);
  for (int p = j; p < i; ++p) {
    const int p0 = p * NB;
    __syncthreads();
    for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
      int r = e % NB, c = e / NB;
      Lt[c][r] = (r < h) ? L.a[(size_t)(p0 + c) * L.ld + r0 + r] : T(0);       // L[i,p]
      Wt[c][r] = W.a[(size_t)(j * NB + c) * W.ld + p0 + r];                     // W[p,j]
    }
    __syncthreads();
    for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
      int r = e % NB, c = e / NB;
      T s = T(0);
#pragma unroll 8
      for (int q = 0; q < NB; ++q) s += Lt[q][r] * Wt[c][q];
      Acc[c][r] += s;
    }
  }
  __syncthreads();
  // W[i,j] = -W[i,i] · Acc
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    int r = e % NB, c = e / NB;
    Wt[c][r] = (r < h && c < h) ? W.a[(size_t)(r0 + c) * W.ld + r0 + r] : T(0);  // W[i,i]
  }
  __syncthreads();
  for (int e = threadIdx.x; e < h * NB; e += blockDim.x) {
    int r = e % h, c = e / h;
    T s = T(0);
    for (int q = 0; q < h; ++q) s += Wt[q][r] * Acc[c][q];
    W.a[(size_t)(j * NB + c) * W.ld + r0 + r] = -s;
  }
}

template <class T, int NB>
void trinv_batched(const MatDesc<T>* d_L, const MatDesc<T>* d_W, int nmat, int nmax,
                   cudaStream_t st) {
  if (nmat == 0 || nmax == 0) return;
  const int nt = ceil_div(nmax, NB);
  k_trinv_diag<T, NB><<<dim3(nt, nmat), 128, 0, st>>>(d_L, d_W);
  for (int i = 1; i < nt; ++i) k_trinv_row<T, NB><<<dim3(i, nmat), 256, 0, st>>>(d_L, d_W, i);
  SDPX_LAUNCH_CHECK_N(nt);
}
template void trinv_batched<double, 32>(const MatDesc<double>*, const MatDesc<double>*, int, int,
                                        cudaStream_t);

// Inverses of the NB×NB diagonal tiles of a lower factor (for blocked TRSV).
template <class T, int NB>
__global__ void k_diag_tile_inverse(const T* L, long long ld, int n, T* Dinv) {
  extern __shared__ __align__(16) unsigned char raw[];
  T(*Lt)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(raw);
  T(*Wt)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(raw + sizeof(T) * NB * (NB + 1));
  const int s = blockIdx.x, s0 = s * NB;
  const int w = min(NB, n - s0);
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    int r = e % NB, c = e / NB;
    Lt[c][r] = (r < w && c < w) ? L[(size_t)(s0 + c) * ld + s0 + r] : T(r == c ? 1 : 0);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < NB; c += blockDim.x) {
    Wt[c][c] = T(1) / Lt[c][c];
    for (int r = c + 1; r < NB; ++r) {
      T acc = T(0);
      for (int p = c; p < r; ++p) acc += Lt[p][r] * Wt[c][p];
      Wt[c][r] = -acc / Lt[r][r];
    }
    for (int r = 0; r < c; ++r) Wt[c][r] = T(0);
  }
  __syncthreads();
  T* out = Dinv + (size_t)s * NB * NB;
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) out[e] = Wt[e / NB][e % NB];
}

// Forward step s of L y = r:  y_s = Dinv_s r_s ;  r[rows below] -= L[rows, s] y_s.
// CTA 0 writes y_s; CTAs ≥ 1 each update ROWS rows below block s.  r and y are
// distinct buffers so no CTA reads a value written in the same launch.
template <class T, int NB, int ROWS>
__global__ void k_trsv_fwd_step(const T* L, long long ld, int n, const T* Dinv, int s, T* r, T* y) {
  __shared__ T ys[NB];
  const int s0 = s * NB, w = min(NB, n - s0);
  const T* Di = Dinv + (size_t)s * NB * NB;
  for (int t = threadIdx.x; t < NB; t += blockDim.x) {
    T acc = T(0);
    if (t < w)
      for (int p = 0; p < w; ++p) acc += Di[t + p * NB] * r[s0 + p];
    ys[t] = acc;
  }
  __syncthreads();
  if (blockIdx.x == 0) {
    for (int t = threadIdx.x; t < w; t += blockDim.x) y[s0 + t] = ys[t];
    return;
  }
  const int base = s0 + w + (blockIdx.x - 1) * ROWS;
  for (int row = base + threadIdx.x; row < min(n, base + ROWS); row += blockDim.x) {
    T acc = T(0);
    for (int p = 0; p < w; ++p) acc += L[(size_t)(s0 + p) * ld + row] * ys[p];
    r[row] -= acc;
  }
}

// Backward step s of Lᵀ x = y: x_s = Dinv_sᵀ y_s ; y[rows above] -= L[s-block, rows]ᵀ x_s.
template <class T, int NB, int ROWS>
__global__ void k_trsv_bwd_step(const T* L, long long ld, int n, const T* Dinv, int s, T* yv, T* x) {
  __shared__ T xs[NB];
  const int s0 = s * NB, w = min(NB, n - s0);
  const T* Di = Dinv + (size_t)s * NB * NB;
  for (int t = threadIdx.x; t < NB; t += blockDim.x) {
    T acc = T(0);
    if (t < w)
      for (int p = 0; p < w; ++p) acc += Di[p + t * NB] * yv[s0 + p];
    xs[t] = acc;
  }
  __syncthreads();
  if (blockIdx.x == 0) {
    for (int t = threadIdx.x; t < w; t += blockDim.x) x[s0 + t] = xs[t];
    return;
  }
  const int base = (blockIdx.x - 1) * ROWS;
  const int end = min(s0, base + ROWS);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int row = base + warp; row < end; row += nw) {
    T acc = T(0);
    for (int p = lane; p < w; p += 32) acc += L[(size_t)row * ld + s0 + p] * xs[p];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) yv[row] -= acc;
  }
}

template <class T, int NB>
void factor_diag_inverses(const T* L, long long ld, int n, T* Dinv, cudaStream_t st) {
  const size_t smem = 2 * sizeof(T) * NB * (NB + 1);
  ensure_smem(k_diag_tile_inverse<T, NB>, smem);
  k_diag_tile_inverse<T, NB><<<ceil_div(n, NB), 64, smem, st>>>(L, ld, n, Dinv);
  SDPX_LAUNCH_CHECK();
}

template <class T, int NB>
void cholesky_solve(const T* L, long long ld, int n, const T* Dinv, T* rhs, T* work,
                    cudaStream_t st) {
  // rhs ← (L Lᵀ)^{-1} rhs.  `work` (n) receives the intermediate y.
  constexpr int ROWS = 256;
  const int nt = ceil_div(n, NB);
  for (int s = 0; s < nt; ++s) {
    int below = n - std::min(n, (s + 1) * NB);
    int grid = 1 + ceil_div(below, ROWS);
    k_trsv_fwd_step<T, NB, ROWS><<<grid, 256, 0, st>>>(L, ld, n, Dinv, s, rhs, work);
  }
  for (int s = nt - 1; s >= 0; --s) {
    int above = s * NB;
    int grid = 1 + ceil_div(above, ROWS);
    k_trsv_bwd_step<T, NB, ROWS><<<grid, 256, 0, st>>>(L, ld, n, Dinv, s, work, rhs);
  }
  SDPX_LAUNCH_CHECK_N(2 * nt);
}

template void factor_diag_inverses<double, 64>(const double*, long long, int, double*, cudaStream_t);

// ---------------------------------------------------------------------------
// Explicit inverse of a lower-triangular factor by recursive doubling:
//   inv([A 0; B C]) = [A⁻¹ 0; −C⁻¹ B A⁻¹  C⁻¹],
// leaves are the 64×64 diagonal tiles (inverted in shared memory); every
// combination is two DMMA GEMMs with triangular K ranges.
// ---------------------------------------------------------------------------
__global__ void k_diag_tiles_to_matrix(const double* Dinv, int n, double* Linv) {
  const int s = blockIdx.x, s0 = s * 64;
  const int w = min(64, n - s0);
  const double* D = Dinv + (size_t)s * 64 * 64;
  for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
    int r = e % w, c = e / w;
    Linv[(size_t)(s0 + c) * n + s0 + r] = D[r + c * 64];
  }
}

void trinv_recursive_f64(const double* L, int n, double* Linv, double* Dinv, double* tmp,
                         cudaStream_t st) {
  SDPX_CUDA(cudaMemsetAsync(Linv, 0, sizeof(double) * (size_t)n * n, st));
  factor_diag_inverses<double, 64>(L, n, n, Dinv, st);
  const int nt = ceil_div(n, 64);
  k_diag_tiles_to_matrix<<<nt, 256, 0, st>>>(Dinv, n, Linv);
  SDPX_LAUNCH_CHECK();
  auto sub = [&](const double* base, int r0, int c0, int rows, int cols, bool kcontig) {
    Opnd o;
    o.base = base + r0 + (size_t)c0 * n;
    o.inner = 1 << 30;
    o.outer_stride = 0;
    if (kcontig) {  // operand as B: (kk = row, nn = col)
      o.kstride = 1;
      o.inner_stride = n;
      o.mn_extent = cols;
      o.k_extent = rows;
    } else {  // operand as A: (mm = row, kk = col)
      o.kstride = n;
      o.inner_stride = 1;
      o.mn_extent = rows;
      o.k_extent = cols;
    }
    return o;
  };
  auto out = [&](double* base, int r0, int c0, int rows, int cols) {
    OutDesc d;
    d.base = base + r0 + (size_t)c0 * n;
    d.row_inner_stride = 1;
    d.row_outer_stride = 0;
    d.row_inner = 1 << 30;
    d.col_inner_stride = n;
    d.col_outer_stride = 0;
    d.col_inner = 1 << 30;
    d.rows = rows;
    d.cols = cols;
    return d;
  };
  // The pairs of one doubling level are independent: their first products
  // go out as grouped launches, then their second products.
  for (int g = 1; g < nt; g *= 2) {
    GemmGroups first, second;
    auto flush = [&]() {
      gemm_f64_grouped(first, false, true, st);
      gemm_f64_grouped(second, false, true, st);
      first.n = second.n = 0;
    };
    for (int i0 = 0; i0 < nt; i0 += 2 * g) {
      const int a0 = i0 * 64, a1 = std::min(n, (i0 + g) * 64);
      const int c0 = a1, c1 = std::min(n, (i0 + 2 * g) * 64);
      if (c0 >= n) continue;
      const int ra = a1 - a0, rc = c1 - c0;
      if (first.n == kGemmGroups) flush();
      // T = B · A⁻¹   (B = L[c0:c1, a0:a1], A⁻¹ lower: k ≥ col)
      const int q = first.n++;
      first.A[q] = sub(L, c0, a0, rc, ra, false);
      first.B[q] = sub(Linv, a0, a0, ra, ra, true);
      first.C[q] = out(tmp, c0, a0, rc, ra);
      first.alpha[q] = 1.0;
      first.beta[q] = 0.0;
      first.mode[q] = KR_B_LOWER;
      // Linv[c0:c1, a0:a1] = −C⁻¹ · T   (C⁻¹ lower: k ≤ row)
      second.n++;
      second.A[q] = sub(Linv, c0, c0, rc, rc, false);
      second.B[q] = sub(tmp, c0, a0, rc, ra, true);
      second.C[q] = out(Linv, c0, a0, rc, ra);
      second.alpha[q] = -1.0;
      second.beta[q] = 0.0;
      second.mode[q] = KR_A_LOWER;
    }
    flush();
  }
}
template void cholesky_solve<double, 64>(const double*, long long, int, const double*, double*,
                                         double*, cudaStream_t);
template void factor_diag_inverses<float, 64>(const float*, long long, int, float*, cudaStream_t);
template void cholesky_solve<float, 64>(const float*, long long, int, const float*, float*, float*,
                                        cudaStream_t);

}  // namespace sdpx
