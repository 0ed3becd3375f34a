// FP64 Gram matrix S = PᵀP on the int8 tensor cores (tcgen05.mma.kind::i8)
// by exact integer digit products.
//
// Every column i of P is scaled by a power of two 2^-e_i (|P_ki| 2^-e_i < 1)
// and written as OZ_DIGITS signed int8 digits,
//   v = 2^-6 (d_0 + 2^-7 d_1 + 2^-14 d_2 + …),  d_0, d_t ∈ [-64, 64],
// (d_0 = rint(64 v), then each remainder times 128 rounded), exactly, with the
// remainder below 2^-(6+7·(OZ_DIGITS-1)) = 2^-55 of the column's largest entry.
// Then
//   S_ij = 2^(e_i+e_j-12) Σ_ℓ 2^(-7ℓ) I_ℓ[i,j],   I_ℓ = Σ_{t+u=ℓ} Σ_k d_t[k,i] d_u[k,j],
// keeping the levels ℓ ≤ OZ_DIGITS-1.  Each I_ℓ accumulates exactly in an
// int32 TMEM accumulator (|d_t d_u| ≤ 4096, at most OZ_DIGITS products per
// level, K chunks ≤ 65 472, so |I_ℓ| < 2^31), so the result carries no
// accumulation error at all: only the truncation of the digits and the final
// FP64 sum of the levels round.  Chunks are summed in FP64 in a fixed order.
//
// Tiles: 128 rows of P columns (A) × 64 (B); the eight level accumulators take
// all 8·64 = 512 TMEM columns.  128 threads per CTA, one CTA per SM: thread 0
// issues the TMA boxes (digit pairs (t, t+4): 64 bytes per box row = 32 K
// positions of two digits, 64-byte swizzle, four 48 KB stages), thread 32 issues the 12 MMAs of a stage (M = 128, N ≤ 256, K = 32,
// all 36 digit products) and commits them to the stage's "empty" barrier, all
// four warps convert the int32 levels to FP64 in the epilogue.  Bounded waits with a device error flag;
// the producer drains its own copies before the CTA exits.  No cluster, no
// multicast.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "ozaki.h"
#include "umma.cuh"

namespace sdpx {
namespace {

constexpr int OM = 128, ON = 64, OK = 32;        // tile rows (A), cols (B), K bytes per stage
constexpr int ONT = 128;                          // threads
constexpr int ONST = 4;                           // stages
// Digit planes are stored in pairs: pair p = t mod 4 holds digits p and p + 4
// of every value, interleaved in 32-byte chunks along K, so one 64-byte TMA
// box row carries two digits (half the box rows of one plane per box: the TMA
// unit issues one request per box row).
constexpr int OPAIRS = OZ_DIGITS / 2;
constexpr int OA_BYTES = OM * 2 * OK;             // 8 KB per digit-pair tile of A
constexpr int OB_BYTES = ON * 2 * OK;             // 4 KB per digit-pair tile of B
constexpr int OSTAGE = OPAIRS * (OA_BYTES + OB_BYTES);  // 48 KB
static_assert(OZ_DIGITS == 8, "digit pairs (t, t + 4)");
constexpr size_t OSMEM = ONST * OSTAGE + 1024 + 256;
constexpr int OLEVELS = OZ_DIGITS;                // levels 0 … OZ_DIGITS-1
constexpr int NAN_EXP = INT_MIN;                  // column holds a non-finite value

// Exact helpers on the FP64 pipe (the conversion pipe is the slow one here).
// (double)x for an int32 x: the double 2^52 + (x + 2^31) has x + 2^31 in its
// low mantissa bits; subtracting 2^52 + 2^31 is exact.
__device__ __forceinline__ double i32_to_f64(int x) {
  return __hiloint2double(0x43300000, x ^ (int)0x80000000) - 4503601774854144.0;
}
// v·2^e, identical to ldexp(v, e) (one rounding of the exact product); the
// power of two is built from its exponent field when it is a normal double.
__device__ __forceinline__ double scale2(double v, int e) {
  return (e >= -1022 && e <= 1023) ? v * __longlong_as_double((long long)(e + 1023) << 52)
                                   : ldexp(v, e);
}
// 2^(-7·lv), the weight of digit level lv.
__device__ __forceinline__ double level_scale(int lv) {
  return __longlong_as_double((long long)(1023 - 7 * lv) << 52);
}
// Nearest integer (ties to even, as rint) of |x| < 2^51 by adding and
// subtracting 1.5·2^52; the low word of the sum is the integer itself.
constexpr double kRound = 6755399441055744.0;
__device__ __forceinline__ double round_digit(double x, int& di) {
  const double t = x + kRound;
  di = __double2loint(t);
  return t - kRound;
}

// ---------------------------------------------------------------- digits --
// One CTA per column: largest magnitude → exponent, then the digit planes.
// Digit t of column i, row k, sits in pair plane t mod 4 (2·m·Kp bytes each) at
// i·2·Kp + 64·(k div 32) + 32·(t div 4) + (k mod 32); zero for k ≥ K.
// When dense_hi is given, the rows [0, tail_off) were written by a producer
// that recorded the largest high word of |P_ki| per column (dense_hi[i]); only
// the tail rows are scanned here and the exponent follows from the combined
// high word (the exponent field of the largest magnitude: the same e as frexp
// for a normal maximum).
__global__ void k_oz_digits(const double* __restrict__ P, long long K, long long Kp, int m,
                            int8_t* __restrict__ digits, int* __restrict__ exps,
                            const unsigned* __restrict__ dense_hi, long long tail_off) {
  __shared__ double red[32];
  __shared__ int s_exp;
  const int i = blockIdx.x;
  const double* col = P + (long long)i * K;
  double mx = 0.0;
  bool finite = true;
  for (long long k = (dense_hi ? tail_off : 0) + threadIdx.x; k < K; k += blockDim.x) {
    const double a = fabs(col[k]);
    if (!isfinite(a)) finite = false;
    mx = fmax(mx, a);
  }
  const int all_finite = __syncthreads_and(finite ? 1 : 0);
  mx = block_max(mx, red);
  if (threadIdx.x == 0) {
    int e = 0;
    if (dense_hi) {
      const unsigned hw = max(dense_hi[i], (unsigned)__double2hiint(mx) & 0x7fffffffu);
      if (!all_finite || hw >= 0x7ff00000u) e = NAN_EXP;
      else if (hw >= 0x00100000u) e = (int)(hw >> 20) - 1022;
      else e = -1021;  // subnormal or zero maximum: 2^-e still bounds the column
    } else {
      if (all_finite && mx > 0.0) frexp(mx, &e);  // mx = f·2^e, f ∈ [0.5, 1)
      if (!all_finite) e = NAN_EXP;
    }
    s_exp = e;
    exps[i] = e;
  }
  __syncthreads();
  const int e = s_exp;
  const size_t plane = (size_t)m * Kp;        // bytes per digit; a pair plane is 2·plane
  int8_t* dst = digits + (size_t)i * 2 * Kp;  // row i of every pair plane
  // Four consecutive rows per thread: one char4 store per digit (Kp is a
  // multiple of 64).
  for (long long k0 = 4 * (long long)threadIdx.x; k0 < Kp; k0 += 4 * blockDim.x) {
    double r[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long k = k0 + q;
      r[q] = (k < K && e != NAN_EXP) ? scale2(col[k], 6 - e) : 0.0;  // 64·v, |v| < 1
    }
#pragma unroll
    for (int t = 0; t < OZ_DIGITS; ++t) {
      int d0, d1, d2, d3;
      const double a0 = round_digit(r[0], d0), a1 = round_digit(r[1], d1);
      const double a2 = round_digit(r[2], d2), a3 = round_digit(r[3], d3);
      *reinterpret_cast<char4*>(dst + (size_t)(t & 3) * 2 * plane + (k0 >> 5) * 64 + (t >> 2) * 32 +
                                (k0 & 31)) =
          make_char4((signed char)d0, (signed char)d1, (signed char)d2, (signed char)d3);
      r[0] = (r[0] - a0) * 128.0;
      r[1] = (r[1] - a1) * 128.0;
      r[2] = (r[2] - a2) * 128.0;
      r[3] = (r[3] - a3) * 128.0;
    }
  }
}

// ------------------------------------------------------------------ SYRK --
struct OzMaps {
  CUtensorMap a[OPAIRS], b[OPAIRS];
};

struct OzShared {
  uint64_t full[ONST], empty[ONST], done;
  uint32_t tmem;
};

// Instruction descriptor, kind::i8: D = S32 (bits 4-5 = 2), A = B = signed 8-bit
// (bits 7-9, 10-12 = 1), both K-major, N>>3 at bits 17-22, M>>4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_s8_s32(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_s8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// The MMAs of one stage.  Level ℓ = t + u sits in TMEM columns [64ℓ, 64ℓ+64).
// In shared memory the four pair tiles of B follow each other with uniform
// 512-byte swizzle atoms (64-byte rows), digit u at pair u mod 4 and byte
// offset 32·(u div 4) of each row.  So for a fixed digit t of A, the products
// with the digits u = 0 … min(3, 7-t) are ONE operand of N = 64·(count) rows
// (pairs 0 …, offset 0) writing the contiguous columns [64t, …), and those with
// u = 4 … 7-t another (offset 32) writing [64(t+4), …): 12 MMAs of N ≤ 256 for
// all 36 digit products, each A tile read from shared memory once per MMA.
// The first stage of a tile writes every level through t = 0 (no accumulate).
__device__ __forceinline__ void oz_mma_stage(uint32_t tmem, uint32_t base, bool first) {
  const uint32_t bbase = base + OPAIRS * OA_BYTES;
#pragma unroll
  for (int ta = 0; ta < OZ_DIGITS; ++ta) {
    const uint64_t ad = umma::smem_desc_sw64(base + (ta & 3) * OA_BYTES + (ta >> 2) * 32);
    const uint32_t acc = (first && ta == 0) ? 0u : 1u;
    const int lo = (OZ_DIGITS - ta) < 4 ? (OZ_DIGITS - ta) : 4;  // u = 0 … lo-1
    mma_s8(tmem + (uint32_t)(ta * ON), ad, umma::smem_desc_sw64(bbase), idesc_s8_s32(OM, lo * ON),
           acc);
    if (OZ_DIGITS - ta > 4)  // u = 4 … 7-ta
      mma_s8(tmem + (uint32_t)((ta + 4) * ON), ad, umma::smem_desc_sw64(bbase + 32),
             idesc_s8_s32(OM, (OZ_DIGITS - ta - 4) * ON), acc);
  }
}

__global__ void __launch_bounds__(ONT, 1)
    k_oz_syrk(const __grid_constant__ OzMaps maps, const int2* __restrict__ pairs, int npairs,
              int kchunk, long long Kp, const int* __restrict__ exps, int m,
              double* __restrict__ partial, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  OzShared* sh = reinterpret_cast<OzShared*>(smem + ONST * OSTAGE);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ONST; ++s) {
      umma::mbar_init(&sh->full[s], 1);
      umma::mbar_init(&sh->empty[s], 1);
    }
    umma::mbar_init(&sh->done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == 0) umma::tmem_alloc(&sh->tmem, 512);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = sh->tmem;

  const int u = blockIdx.x;
  const int chunk = u / npairs, pr = u % npairs;
  const int2 tile = pairs[pr];
  const int ra = tile.x * OM, rb = tile.y * ON;
  const long long kb = (long long)chunk * kchunk;
  const long long ke = min(Kp, kb + kchunk);
  const int ntiles = ke > kb ? (int)((ke - kb + OK - 1) / OK) : 0;

  if (threadIdx.x == 0) {
    int issued = 0;
    for (int t = 0; t < ntiles; ++t) {
      const int s = t % ONST;
      if (t >= ONST && !umma::mbar_wait_bounded(&sh->empty[s], ((t / ONST) - 1) & 1, err)) break;
      umma::mbar_expect_tx(&sh->full[s], OSTAGE);
      const uint32_t base = umma::smem_u32(smem + s * OSTAGE);
      const int k = (int)(kb + (long long)t * OK);
#pragma unroll
      for (int d = 0; d < OPAIRS; ++d) {
        umma::tma_load_2d(base + d * OA_BYTES, &maps.a[d], 2 * k, ra, &sh->full[s]);
        umma::tma_load_2d(base + OPAIRS * OA_BYTES + d * OB_BYTES, &maps.b[d], 2 * k, rb,
                          &sh->full[s]);
      }
      ++issued;
    }
    for (int t = max(0, issued - ONST); t < issued; ++t)
      umma::mbar_wait_bounded(&sh->full[t % ONST], (t / ONST) & 1, err);
  } else if (threadIdx.x == 32) {
    for (int t = 0; t < ntiles; ++t) {
      const int s = t % ONST;
      if (!umma::mbar_wait_bounded(&sh->full[s], (t / ONST) & 1, err)) break;
      umma::fence_after_sync();
      const uint32_t base = umma::smem_u32(smem + s * OSTAGE);
      oz_mma_stage(tmem, base, t == 0);
      umma::commit(&sh->empty[s]);
    }
    umma::commit(&sh->done);
  }
  __syncwarp();
  const bool ok = umma::mbar_wait_bounded(&sh->done, 0, err);
  umma::fence_after_sync();
  const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;

  // Epilogue: thread = one A row (TMEM lane), 64 B columns; levels summed from
  // the smallest upward in FP64, then scaled by 2^(e_i + e_j − 12).
  const int row = warp * 32 + lane;
  double* dst = partial + (size_t)u * OM * ON + (size_t)row * ON;
  if (all_ok && ntiles > 0) {
    const int gi = ra + row;
    const int ei = gi < m ? exps[gi] : 0;
    for (int cb = 0; cb < ON; cb += 32) {
      double acc[32];
#pragma unroll
      for (int q = 0; q < 32; ++q) acc[q] = 0.0;
      for (int lv = OLEVELS - 1; lv >= 0; --lv) {
        float raw[32];
        umma::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(lv * ON + cb), raw);
#pragma unroll
        for (int q = 0; q < 32; ++q)
          acc[q] = fma(i32_to_f64(__float_as_int(raw[q])), level_scale(lv), acc[q]);
      }
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const int gj = rb + cb + q;
        const int ej = gj < m ? exps[gj] : 0;
        double v;
        if (ei == NAN_EXP || ej == NAN_EXP)
          v = __longlong_as_double(0x7ff8000000000000ll);
        else
          v = scale2(acc[q], ei + ej - 12);
        dst[cb + q] = v;
      }
    }
  } else {
    for (int q = 0; q < ON; ++q) dst[q] = 0.0;
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
}

// S tile = Σ_chunks of the partial tiles, in chunk order, lower part only.
// Four CTAs per tile, 32 rows each: coalesced reads of the row-major partials
// (a thread's eight loads of a chunk in flight together), the 32 × 64 block
// transposed through shared memory, each warp writing 32 consecutive rows of
// one column of the column-major S.
__global__ void __launch_bounds__(256) k_oz_reduce(const double* __restrict__ partial,
                                                   const int2* __restrict__ pairs, int npairs,
                                                   int nchunk, int m, double* __restrict__ S) {
  __shared__ double blk[ON][33];
  const int pr = blockIdx.x >> 2, r0 = (blockIdx.x & 3) * 32;
  const int2 tile = pairs[pr];
  constexpr int PER = 32 * ON / 256;
  double acc[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) acc[k] = 0.0;
  const size_t tsz = (size_t)OM * ON;
  const double* base = partial + (size_t)pr * tsz + (size_t)r0 * ON;
  for (int ch = 0; ch < nchunk; ++ch) {
    const double* src = base + (size_t)ch * npairs * tsz;
    double v[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) v[k] = src[threadIdx.x + k * 256];
#pragma unroll
    for (int k = 0; k < PER; ++k) acc[k] += v[k];
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = threadIdx.x + k * 256, r = e / ON, c = e % ON;
    blk[c][r] = acc[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = threadIdx.x + k * 256, r = e & 31, c = e >> 5;
    const int gi = tile.x * OM + r0 + r, gj = tile.y * ON + c;
    if (gi < m && gj < m && gi >= gj) S[gi + (size_t)gj * m] = blk[c][r];
  }
}

// ------------------------------------------------------------ row digits --
// One warp per row vector: largest magnitude over the kept elements, then the
// digit planes, four consecutive elements per lane (char4 stores).
struct OzRowsDev {
  const double* base;
  long long rows, is, os, es;
  int inner, len, tri;
};

__global__ void k_oz_digits_rows(const OzRowsDev r, long long Kp, long long plane,
                                 int8_t* __restrict__ digits, int* __restrict__ exps) {
  const int lane = threadIdx.x & 31;
  const long long n = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (n >= r.rows) return;
  const double* v = r.base + (n / r.inner) * r.os + (n % r.inner) * r.is;
  int jlo = 0, jhi = r.len;
  if (r.tri == 1) jhi = (int)(n + 1 < (long long)r.len ? n + 1 : (long long)r.len);
  if (r.tri == 2) jlo = (int)(n < (long long)r.len ? n : (long long)r.len);
  double mx = 0.0;
  bool finite = true;
  for (int j = jlo + lane; j < jhi; j += 32) {
    const double a = fabs(v[(long long)j * r.es]);
    finite = finite && isfinite(a);
    mx = fmax(mx, a);
  }
  const bool all_finite = __all_sync(0xffffffffu, finite);
  mx = warp_max(mx);
  int e = 0;
  if (all_finite && mx > 0.0) frexp(mx, &e);
  if (!all_finite) e = NAN_EXP;
  if (lane == 0) exps[n] = e;
  int8_t* dst = digits + n * 2 * Kp;  // row n of every pair plane (2·plane bytes apart)
  for (long long j0 = 4 * lane; j0 < Kp; j0 += 128) {
    double x[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long j = j0 + q;
      x[q] = (j >= jlo && j < jhi && e != NAN_EXP) ? scale2(v[j * r.es], 6 - e) : 0.0;
    }
#pragma unroll
    for (int t = 0; t < OZ_DIGITS; ++t) {
      char4 c;
      double d;
      int di;
      d = round_digit(x[0], di); c.x = (signed char)di; x[0] = (x[0] - d) * 128.0;
      d = round_digit(x[1], di); c.y = (signed char)di; x[1] = (x[1] - d) * 128.0;
      d = round_digit(x[2], di); c.z = (signed char)di; x[2] = (x[2] - d) * 128.0;
      d = round_digit(x[3], di); c.w = (signed char)di; x[3] = (x[3] - d) * 128.0;
      *reinterpret_cast<char4*>(dst + (t & 3) * 2 * plane + (j0 >> 5) * 64 + (t >> 2) * 32 +
                                (j0 & 31)) = c;
    }
  }
}

// ---------------------------------------------------------------- GEMM ----
// Persistent CTAs over the (128-row X tile, 64-row Y tile) tasks, Y tiles
// fastest (rotated per X tile, see oz_tile) so that concurrent tasks share X
// tiles in L2.  Warp 16 (one thread)
// streams the digit boxes through the four stages and runs ahead into the
// next task; warp 17 (one thread) issues the 12 MMAs of a stage and, at the
// end of a task, commits the eight level accumulators to `tfull`; warps 0-15
// (TMEM lane quarter w % 4, 16-column group w / 4) read the levels, hand the
// accumulator back through `tempty` and then scale and store while the next
// task's MMAs run.  Sixteen epilogue warps keep every scheduler busy: the
// level sums are chains of dependent FP64 operations.
constexpr int GEPI = 16;              // epilogue warps: 4 TMEM lane quarters × 4 column groups
constexpr int GNT = (GEPI + 2) * 32;  // + the TMA warp and the MMA warp

struct OzGemmDev {
  const int* ea;
  const int* eb;
  double* out;
  unsigned* colmax;  // optional: largest high word of |out| per group a / a_inner
  long long ntask, a_is, a_os, b_stride;
  int rows_a, rows_b, kext, kmode, ntile_b, a_inner;
};

struct OzGemmShared {
  uint64_t full[ONST], empty[ONST], tfull, tempty, mdone;
  uint32_t tmem;
  int abort;
};

// Bounded wait that also gives up as soon as another role of the CTA has.
__device__ __forceinline__ bool oz_wait(uint64_t* mbar, uint32_t parity, int* err,
                                        volatile int* abort) {
  const long long t0 = clock64();
  while (!umma::mbar_test(mbar, parity)) {
    if (*abort) return false;
    if (clock64() - t0 > (1LL << 32)) {
      atomicExch(err, 1);
      *abort = 1;
      return false;
    }
    __nanosleep(32);
  }
  return true;
}

// Task u → (X tile mt, Y tile nt).  The Y tiles of one X tile are consecutive
// tasks (they share the X tile in L2), rotated by mt: a persistent CTA takes
// every gridDim-th task, and without the rotation a grid that is a multiple
// of ntile_b would give each CTA one fixed Y tile — one fixed K length under
// the triangular ranges, so some CTAs would run several times longer.
__device__ __forceinline__ void oz_tile(const OzGemmDev& g, long long u, int& mt, int& nt) {
  mt = (int)(u / g.ntile_b);
  nt = (int)((u % g.ntile_b + mt) % g.ntile_b);
}

__device__ __forceinline__ void oz_task(const OzGemmDev& g, long long u, int& mt, int& nt, int& kb,
                                        int& nk) {
  oz_tile(g, u, mt, nt);
  kb = 0;
  int ke = g.kext;
  const int n0 = nt * ON;
  if (g.kmode == 1) ke = min(g.kext, n0 + ON);
  if (g.kmode == 2) kb = min(g.kext, n0) / OK * OK;
  nk = ke > kb ? (ke - kb + OK - 1) / OK : 0;
}

__global__ void __launch_bounds__(GNT, 1)
    k_oz_gemm(const __grid_constant__ OzMaps maps, const OzGemmDev g, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  OzGemmShared* sh = reinterpret_cast<OzGemmShared*>(smem + ONST * OSTAGE);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ONST; ++s) {
      umma::mbar_init(&sh->full[s], 1);
      umma::mbar_init(&sh->empty[s], 1);
    }
    umma::mbar_init(&sh->tfull, 1);
    umma::mbar_init(&sh->tempty, GEPI);
    umma::mbar_init(&sh->mdone, 1);
    sh->abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == 0) umma::tmem_alloc(&sh->tmem, 512);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = sh->tmem;
  volatile int* abort = &sh->abort;

  if (warp == GEPI) {
    if (lane == 0) {
      uint32_t it = 0;
      for (long long u = blockIdx.x; u < g.ntask && !*abort; u += gridDim.x) {
        int mt, nt, kb, nk;
        oz_task(g, u, mt, nt, kb, nk);
        bool ok = true;
        for (int t = 0; t < nk; ++t, ++it) {
          const int s = it % ONST;
          if (it >= ONST && !oz_wait(&sh->empty[s], ((it / ONST) - 1) & 1, err, abort)) {
            ok = false;
            break;
          }
          umma::mbar_expect_tx(&sh->full[s], OSTAGE);
          const uint32_t base = umma::smem_u32(smem + s * OSTAGE);
          const int k = kb + t * OK;
#pragma unroll
          for (int d = 0; d < OPAIRS; ++d) {
            umma::tma_load_2d(base + d * OA_BYTES, &maps.a[d], 2 * k, mt * OM, &sh->full[s]);
            umma::tma_load_2d(base + OPAIRS * OA_BYTES + d * OB_BYTES, &maps.b[d], 2 * k, nt * ON,
                              &sh->full[s]);
          }
        }
        if (!ok) break;
      }
      // Drain this thread's copies in flight before the CTA may exit.
      for (uint32_t t = it > (uint32_t)ONST ? it - ONST : 0; t < it; ++t)
        umma::mbar_wait_bounded(&sh->full[t % ONST], (t / ONST) & 1, err);
    }
  } else if (warp == GEPI + 1) {
    if (lane == 0) {
        uint32_t it = 0, j = 0;
      bool ok = true;
      for (long long u = blockIdx.x; u < g.ntask && ok; u += gridDim.x, ++j) {
        int mt, nt, kb, nk;
        oz_task(g, u, mt, nt, kb, nk);
        if (j > 0 && !oz_wait(&sh->tempty, (j - 1) & 1, err, abort)) break;
        umma::fence_after_sync();
        for (int t = 0; t < nk; ++t, ++it) {
          const int s = it % ONST;
          if (!oz_wait(&sh->full[s], (it / ONST) & 1, err, abort)) {
            ok = false;
            break;
          }
          umma::fence_after_sync();
          const uint32_t base = umma::smem_u32(smem + s * OSTAGE);
          oz_mma_stage(tmem, base, t == 0);
          umma::commit(&sh->empty[s]);
        }
        if (ok) umma::commit(&sh->tfull);
      }
      // Every MMA of this thread completes before the accumulator is freed.
      umma::commit(&sh->mdone);
      umma::mbar_wait_bounded(&sh->mdone, 0, err);
    }
  } else {
    // Epilogue: warp w reads TMEM lanes 32·(w % 4) … (one X row per thread) and
    // the 16 Y columns of group w / 4.
    const int quarter = warp & 3, cgrp = warp >> 2;
    uint32_t j = 0;
    for (long long u = blockIdx.x; u < g.ntask; u += gridDim.x, ++j) {
      if (!oz_wait(&sh->tfull, j & 1, err, abort)) break;
      umma::fence_after_sync();
      int mt, nt;
      oz_tile(g, u, mt, nt);
      // Levels in two batches of four loads in flight, summed smallest first;
      // the accumulator goes back to the MMA warp as soon as the second batch
      // is in registers, before its conversion.
      static_assert(OLEVELS == 8, "two batches of four levels");
      const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(cgrp * 16);
      double acc[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) acc[q] = 0.0;
      {
        uint32_t raw[4][16];
#pragma unroll
        for (int b = 0; b < 4; ++b) umma::tmem_ld16_async(tbase + (uint32_t)((7 - b) * ON), raw[b]);
        umma::tmem_wait_ld();
#pragma unroll
        for (int b = 0; b < 4; ++b) umma::tmem_regs_ready(raw[b]);
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
          for (int q = 0; q < 16; ++q)
            acc[q] = fma(i32_to_f64((int)raw[b][q]), level_scale(7 - b), acc[q]);
      }
      uint32_t raw[4][16];
#pragma unroll
      for (int b = 0; b < 4; ++b) umma::tmem_ld16_async(tbase + (uint32_t)((3 - b) * ON), raw[b]);
      umma::tmem_wait_ld();
#pragma unroll
      for (int b = 0; b < 4; ++b) umma::tmem_regs_ready(raw[b]);
      umma::fence_before_sync();
      __syncwarp();
      if (lane == 0) umma::mbar_arrive(&sh->tempty);
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int q = 0; q < 16; ++q)
          acc[q] = fma(i32_to_f64((int)raw[b][q]), level_scale(3 - b), acc[q]);
      const int ga = mt * OM + quarter * 32 + lane;
      unsigned hw = 0;
      if (ga < g.rows_a) {
        const int ea = g.ea[ga];
        double* row = g.out + (long long)(ga / g.a_inner) * g.a_os + (long long)(ga % g.a_inner) * g.a_is;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int gb = nt * ON + cgrp * 16 + q;
          if (gb < g.rows_b) {
            const int eb = g.eb[gb];
            const double v = (ea == NAN_EXP || eb == NAN_EXP)
                                 ? __longlong_as_double(0x7ff8000000000000ll)
                                 : scale2(acc[q], ea + eb - 12);
            row[(long long)gb * g.b_stride] = v;
            hw = max(hw, (unsigned)__double2hiint(v) & 0x7fffffffu);
          }
        }
      }
      if (g.colmax) {  // one atomic per group of lanes that share a / a_inner
        const int grp = ga < g.rows_a ? ga / g.a_inner : -1;
        const unsigned same = __match_any_sync(0xffffffffu, grp);
        const unsigned mx = __reduce_max_sync(same, hw);
        if (grp >= 0 && lane == __ffs(same) - 1) atomicMax(&g.colmax[grp], mx);
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
}

PFN_cuTensorMapEncodeTiled_v12000 oz_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) throw CudaError("cuTensorMapEncodeTiled is not available");
  return fn;
}

// TMA map of one digit-pair plane: rows × 2·Kp bytes (row-major), boxes of
// 64 bytes (32 K positions of two digits) × box_rows, 64-byte swizzle.
void encode_digit_map(CUtensorMap* map, const int8_t* pair_plane, int rows, long long Kp,
                      int box_rows) {
  if ((reinterpret_cast<uintptr_t>(pair_plane) & 15) != 0 || Kp % 32 != 0)
    throw std::invalid_argument("ozaki: digit plane not 16-byte aligned or Kp not a multiple of 32");
  cuuint64_t dims[2] = {(cuuint64_t)(2 * Kp), (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(2 * Kp)};
  cuuint32_t box[2] = {(cuuint32_t)(2 * OK), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = oz_encoder()(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(pair_plane),
                            dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

// Lower tile pairs (A tile of 128 rows, B tile of 64 rows) that hold an entry
// with i ≥ j.
std::vector<int2> oz_pairs(int m) {
  std::vector<int2> v;
  const int tr = ceil_div(m, OM), tc = ceil_div(m, ON);
  for (int a = 0; a < tr; ++a)
    for (int b = 0; b < tc && b * ON <= a * OM + OM - 1; ++b) v.push_back(make_int2(a, b));
  return v;
}

}  // namespace

OzakiPlan plan_ozaki_syrk(int m, long long K, int sm_count) {
  OzakiPlan p;
  p.m = m;
  p.K = K;
  p.Kp = std::max<long long>(64, (K + 63) / 64 * 64);
  p.ntile_r = ceil_div(m, OM);
  p.ntile_c = ceil_div(m, ON);
  p.ntri = (int)oz_pairs(m).size();
  // Chunks of at most 65 472 K (exact int32 levels: 65 472 · 8 · 4096 < 2^31),
  // enough of them to give about four waves of one CTA per SM.
  const long long maxc = 65472;
  int nc = (int)std::max<long long>(1, (p.Kp + maxc - 1) / maxc);
  while ((long long)p.ntri * nc < 4LL * sm_count && (p.Kp / (nc + 1)) >= 2048) ++nc;
  long long kc = (p.Kp + nc - 1) / nc;
  kc = (kc + OK - 1) / OK * OK;
  p.kchunk = (int)kc;
  p.nchunk = (int)((p.Kp + kc - 1) / kc);
  p.digit_bytes = (size_t)OZ_DIGITS * m * p.Kp;
  p.partial_doubles = (size_t)p.nchunk * p.ntri * OM * ON;
  p.partial_alloc_doubles = p.partial_doubles + (size_t)p.ntri;  // + int2 tile pairs
  return p;
}

void ozaki_syrk(const double* P, const OzakiPlan& plan, int8_t* digits, int* exps, double* partial,
                double* S, int* err, cudaStream_t st, cudaEvent_t ev_begin, cudaEvent_t ev_end,
                const unsigned* dense_hi, long long tail_off) {
  const int m = plan.m;
  if (m <= 0) return;
  k_oz_digits<<<m, 256, 0, st>>>(P, plan.K, plan.Kp, m, digits, exps, dense_hi, tail_off);
  SDPX_LAUNCH_CHECK();
  // The tile-pair table follows the partial tiles in the same buffer
  // (plan.partial_alloc_doubles).  A copy from pageable memory returns once the
  // host data is staged, so the local table may go out of scope afterwards.
  const std::vector<int2> host_pairs = oz_pairs(m);
  int2* d_pairs = reinterpret_cast<int2*>(partial + plan.partial_doubles);
  SDPX_CUDA(cudaMemcpyAsync(d_pairs, host_pairs.data(), sizeof(int2) * host_pairs.size(),
                            cudaMemcpyHostToDevice, st));
  OzMaps maps;
  const size_t plane = (size_t)m * plan.Kp;
  for (int d = 0; d < OPAIRS; ++d) {
    encode_digit_map(&maps.a[d], digits + d * 2 * plane, m, plan.Kp, OM);
    encode_digit_map(&maps.b[d], digits + d * 2 * plane, m, plan.Kp, ON);
  }
  ensure_smem(k_oz_syrk, OSMEM);
  const int units = plan.ntri * plan.nchunk;
  if (ev_begin) SDPX_CUDA(cudaEventRecord(ev_begin, st));
  k_oz_syrk<<<units, ONT, OSMEM, st>>>(maps, d_pairs, plan.ntri, plan.kchunk, plan.Kp, exps, m,
                                       partial, err);
  if (ev_end) SDPX_CUDA(cudaEventRecord(ev_end, st));
  k_oz_reduce<<<plan.ntri * 4, 256, 0, st>>>(partial, d_pairs, plan.ntri, plan.nchunk, m, S);
  SDPX_LAUNCH_CHECK_N(2);
}

long long oz_kpad(int len) { return std::max<long long>(32, (len + 31LL) / 32 * 32); }

void ozaki_digits_rows(const OzRows& r, long long Kp, long long plane, int8_t* digits, int* exps,
                       cudaStream_t st) {
  if (r.rows <= 0) return;
  if (Kp % 32 != 0 || Kp < r.len || plane < r.rows * Kp)
    throw std::invalid_argument("ozaki: digit rows do not fit the planes");
  OzRowsDev d{r.base, r.rows, r.is, r.os, r.es, r.inner, r.len, r.tri};
  constexpr int WARPS = 8;
  const long long blocks = (r.rows + WARPS - 1) / WARPS;
  k_oz_digits_rows<<<(unsigned)blocks, WARPS * 32, 0, st>>>(d, Kp, plane, digits, exps);
  SDPX_LAUNCH_CHECK();
}

void ozaki_gemm(const OzGemm& g, int sm_count, int* err, cudaStream_t st) {
  if (g.rows_a <= 0 || g.rows_b <= 0) return;
  if (g.Kp % 32 != 0 || g.Kp < OK) throw std::invalid_argument("ozaki: contraction width");
  OzMaps maps;
  for (int d = 0; d < OPAIRS; ++d) {
    encode_digit_map(&maps.a[d], g.xd + d * 2 * g.x_plane, g.rows_a, g.Kp, OM);
    encode_digit_map(&maps.b[d], g.yd + d * 2 * g.y_plane, g.rows_b, g.Kp, ON);
  }
  OzGemmDev dv;
  dv.ea = g.ea;
  dv.eb = g.eb;
  dv.out = g.out;
  dv.colmax = g.colmax;
  dv.rows_a = g.rows_a;
  dv.rows_b = g.rows_b;
  dv.kext = (int)g.Kp;
  dv.kmode = g.kmode;
  dv.ntile_b = ceil_div(g.rows_b, ON);
  dv.ntask = (long long)ceil_div(g.rows_a, OM) * dv.ntile_b;
  dv.a_inner = g.a_inner;
  dv.a_is = g.a_is;
  dv.a_os = g.a_os;
  dv.b_stride = g.b_stride;
  ensure_smem(k_oz_gemm, OSMEM);
  const long long grid = std::min<long long>(dv.ntask, std::max(1, sm_count));
  k_oz_gemm<<<(unsigned)grid, GNT, OSMEM, st>>>(maps, dv, err);
  SDPX_LAUNCH_CHECK();
}

}  // namespace sdpx
