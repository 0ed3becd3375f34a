// FP64 tensor-core tile engine (DMMA m8n8k4) with cp.async multi-stage staging.
//
// One CTA computes a BM×BN tile of  A(M×K)·B(K×N)  over a K range.  Operands
// are described by `Opnd` (two-level addressing, see common.cuh).  Each operand
// is staged in shared memory either K-contiguous ([mn][k], ld = BK+4) or
// MN-contiguous ([k][mn], ld = BM+4 / BN+4); both paddings are ≡ 4 (mod 16)
// doubles, which makes the fragment reads of a half-warp (4 rows × 4 k)
// conflict-free.
#pragma once
#include "common.cuh"

namespace sdpx {

template <int BM_, int BN_, int WARPS_M_, int WARPS_N_, bool A_KCONTIG_, bool B_KCONTIG_>
struct F64Cfg {
  static constexpr int BM = BM_, BN = BN_, BK = 16, STAGES = 3;
  static constexpr int WARPS_M = WARPS_M_, WARPS_N = WARPS_N_;
  static constexpr int NT = WARPS_M * WARPS_N * 32;
  static constexpr bool A_KCONTIG = A_KCONTIG_, B_KCONTIG = B_KCONTIG_;
  static constexpr int WTM = BM / WARPS_M, WTN = BN / WARPS_N;
  static constexpr int FM = WTM / 8, FN = WTN / 8;
  static constexpr int LDA = A_KCONTIG ? (BK + 4) : (BM + 4);
  static constexpr int LDB = B_KCONTIG ? (BK + 4) : (BN + 4);
  static constexpr int A_STAGE = A_KCONTIG ? BM * LDA : BK * LDA;
  static constexpr int B_STAGE = B_KCONTIG ? BN * LDB : BK * LDB;
  static constexpr int A_PER_T = BM * BK / NT;
  static constexpr int B_PER_T = BN * BK / NT;
  static constexpr size_t SMEM_BYTES = sizeof(double) * STAGES * (A_STAGE + B_STAGE);
  static_assert(BM * BK % NT == 0 && BN * BK % NT == 0, "tile/thread mismatch");
  static_assert(WTM % 8 == 0 && WTN % 8 == 0, "warp tile must be a multiple of 8");
};

// Per-thread staging plan for one operand: which (mn, kk) elements this thread
// copies into each stage, with the mn offsets precomputed once per CTA tile.
template <int PER_T>
struct StagePlan {
  long long off[PER_T];  // global offset of (mn, 0); -1 when mn is out of range
  int kk[PER_T];
  int sidx[PER_T];       // shared-memory index inside a stage
};

template <int TILE_MN, int PER_T, int NT, int LD, bool KCONTIG>
__device__ __forceinline__ void make_plan(StagePlan<PER_T>& p, const Opnd& o, int mn0) {
  constexpr int BK = 16;
#pragma unroll
  for (int j = 0; j < PER_T; ++j) {
    int idx = threadIdx.x + j * NT;
    int mm, kk;
    if (KCONTIG) {
      mm = idx / BK;
      kk = idx % BK;
      p.sidx[j] = mm * LD + kk;
    } else {
      mm = idx % TILE_MN;
      kk = idx / TILE_MN;
      p.sidx[j] = kk * LD + mm;
    }
    int g = mn0 + mm;
    p.kk[j] = kk;
    p.off[j] = (g < o.mn_extent) ? two_level(g, o.inner, o.inner_stride, o.outer_stride) : -1;
  }
}

template <int PER_T>
__device__ __forceinline__ void issue_stage(double* s, const StagePlan<PER_T>& p, const Opnd& o,
                                            int k0, int k_end) {
#pragma unroll
  for (int j = 0; j < PER_T; ++j) {
    int k = k0 + p.kk[j];
    bool ok = (p.off[j] >= 0) && (k < k_end);
    const double* src = ok ? (o.base + p.off[j] + (long long)k * o.kstride) : o.base;
    cp_async8(s + p.sidx[j], src, ok);
  }
}

// Accumulates A[m0:m0+BM, kb:ke] · B[kb:ke, n0:n0+BN] into acc.
template <class Cfg>
__device__ void f64_tile_mainloop(double (&acc)[Cfg::FM][Cfg::FN][2], const Opnd& A, const Opnd& B,
                                  int m0, int n0, int kb, int ke, double* smem) {
  constexpr int BK = Cfg::BK, ST = Cfg::STAGES;
  double* sA = smem;
  double* sB = smem + ST * Cfg::A_STAGE;
  StagePlan<Cfg::A_PER_T> pa;
  StagePlan<Cfg::B_PER_T> pb;
  make_plan<Cfg::BM, Cfg::A_PER_T, Cfg::NT, Cfg::LDA, Cfg::A_KCONTIG>(pa, A, m0);
  make_plan<Cfg::BN, Cfg::B_PER_T, Cfg::NT, Cfg::LDB, Cfg::B_KCONTIG>(pb, B, n0);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp / Cfg::WARPS_N, wn = warp % Cfg::WARPS_N;
  const int ntiles = (ke > kb) ? (ke - kb + BK - 1) / BK : 0;

#pragma unroll
  for (int s = 0; s < ST - 1; ++s) {
    if (s < ntiles) {
      issue_stage(sA + s * Cfg::A_STAGE, pa, A, kb + s * BK, ke);
      issue_stage(sB + s * Cfg::B_STAGE, pb, B, kb + s * BK, ke);
    }
    cp_async_commit();
  }
  for (int tIdx = 0; tIdx < ntiles; ++tIdx) {
    int pre = tIdx + ST - 1;
    if (pre < ntiles) {
      int s = pre % ST;
      issue_stage(sA + s * Cfg::A_STAGE, pa, A, kb + pre * BK, ke);
      issue_stage(sB + s * Cfg::B_STAGE, pb, B, kb + pre * BK, ke);
    }
    cp_async_commit();
    cp_async_wait<ST - 1>();
    __syncthreads();
    const double* a_s = sA + (tIdx % ST) * Cfg::A_STAGE;
    const double* b_s = sB + (tIdx % ST) * Cfg::B_STAGE;
#pragma unroll
    for (int ks = 0; ks < BK / 4; ++ks) {
      double af[Cfg::FM], bf[Cfg::FN];
      const int kk = ks * 4 + t;
#pragma unroll
      for (int fm = 0; fm < Cfg::FM; ++fm) {
        int mm = wm * Cfg::WTM + fm * 8 + g;
        af[fm] = Cfg::A_KCONTIG ? a_s[mm * Cfg::LDA + kk] : a_s[kk * Cfg::LDA + mm];
      }
#pragma unroll
      for (int fn = 0; fn < Cfg::FN; ++fn) {
        int nn = wn * Cfg::WTN + fn * 8 + g;
        bf[fn] = Cfg::B_KCONTIG ? b_s[nn * Cfg::LDB + kk] : b_s[kk * Cfg::LDB + nn];
      }
#pragma unroll
      for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
        for (int fn = 0; fn < Cfg::FN; ++fn) dmma_8x8x4(acc[fm][fn][0], acc[fm][fn][1], af[fm], bf[fn]);
    }
    __syncthreads();
  }
  cp_async_wait<0>();
}

template <class Cfg>
__device__ __forceinline__ void zero_acc(double (&acc)[Cfg::FM][Cfg::FN][2]) {
#pragma unroll
  for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
}

// Visit every accumulator element with its tile-local (row, col).
template <class Cfg, class F>
__device__ __forceinline__ void for_each_acc(double (&acc)[Cfg::FM][Cfg::FN][2], F&& f) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp / Cfg::WARPS_N, wn = warp % Cfg::WARPS_N;
#pragma unroll
  for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
    for (int fn = 0; fn < Cfg::FN; ++fn)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        int r = wm * Cfg::WTM + fm * 8 + g;
        int col = wn * Cfg::WTN + fn * 8 + 2 * t + c;
        f(r, col, acc[fm][fn][c]);
      }
}

// Write alpha·acc (+ beta·C when beta ≠ 0) through C's two-level addressing:
// the column offsets of this thread's fragments are formed once, the row
// offset once per fragment row (instead of two index divisions per element).
template <class Cfg>
__device__ __forceinline__ void store_acc(double (&acc)[Cfg::FM][Cfg::FN][2], const OutDesc& C,
                                          int m0, int n0, double alpha, double beta) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp / Cfg::WARPS_N, wn = warp % Cfg::WARPS_N;
  long long co[Cfg::FN][2];
#pragma unroll
  for (int fn = 0; fn < Cfg::FN; ++fn)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int col = n0 + wn * Cfg::WTN + fn * 8 + 2 * t + c;
      co[fn][c] = col < C.cols
                      ? two_level(col, C.col_inner, C.col_inner_stride, C.col_outer_stride)
                      : -1;
    }
#pragma unroll
  for (int fm = 0; fm < Cfg::FM; ++fm) {
    const int row = m0 + wm * Cfg::WTM + fm * 8 + g;
    if (row >= C.rows) continue;
    double* rp = C.base + two_level(row, C.row_inner, C.row_inner_stride, C.row_outer_stride);
#pragma unroll
    for (int fn = 0; fn < Cfg::FN; ++fn)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        if (co[fn][c] < 0) continue;
        double* q = rp + co[fn][c];
        *q = (beta == 0.0) ? alpha * acc[fm][fn][c] : alpha * acc[fm][fn][c] + beta * (*q);
      }
  }
}

__device__ __forceinline__ void k_limits(int mode, int K, int m0, int n0, int BM, int BN, int& kb,
                                         int& ke) {
  kb = 0;
  ke = K;
  if (mode == KR_A_LOWER) ke = min(K, m0 + BM);
  else if (mode == KR_A_UPPER) kb = m0;
  else if (mode == KR_B_LOWER) kb = n0;
  else if (mode == KR_B_UPPER) ke = min(K, n0 + BN);
  // A/B triangular restrictions on "row"/"col" above assume the triangular
  // operand is square in its (mn, k) pair, which holds for every use here.
  kb = (kb / 16) * 16;
}

}  // namespace sdpx
