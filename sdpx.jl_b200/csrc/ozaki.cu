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
// issues the TMA boxes (K = 32 bytes per row, 32-byte swizzle, four 48 KB
// stages), thread 32 issues the 36 MMAs of a stage (M = 128, N = 64, K = 32)
// and commits them to the stage's "empty" barrier, all four warps convert the
// int32 levels to FP64 in the epilogue.  Bounded waits with a device error flag;
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
constexpr int OA_BYTES = OM * OK;                 // 4 KB per digit tile of A
constexpr int OB_BYTES = ON * OK;                 // 2 KB per digit tile of B
constexpr int OSTAGE = OZ_DIGITS * (OA_BYTES + OB_BYTES);  // 48 KB
constexpr size_t OSMEM = ONST * OSTAGE + 1024 + 256;
constexpr int OLEVELS = OZ_DIGITS;                // levels 0 … OZ_DIGITS-1
constexpr int NAN_EXP = INT_MIN;                  // column holds a non-finite value

// ---------------------------------------------------------------- digits --
// One CTA per column: largest magnitude → exponent, then the digit planes
// (digit t of column i at digits[t·m·Kp + i·Kp + k], zero for k ≥ K).
__global__ void k_oz_digits(const double* __restrict__ P, long long K, long long Kp, int m,
                            int8_t* __restrict__ digits, int* __restrict__ exps) {
  __shared__ double red[32];
  __shared__ int s_exp;
  const int i = blockIdx.x;
  const double* col = P + (long long)i * K;
  double mx = 0.0;
  bool finite = true;
  for (long long k = threadIdx.x; k < K; k += blockDim.x) {
    const double a = fabs(col[k]);
    if (!isfinite(a)) finite = false;
    mx = fmax(mx, a);
  }
  const int all_finite = __syncthreads_and(finite ? 1 : 0);
  mx = block_max(mx, red);
  if (threadIdx.x == 0) {
    int e = 0;
    if (all_finite && mx > 0.0) frexp(mx, &e);  // mx = f·2^e, f ∈ [0.5, 1)
    s_exp = all_finite ? e : NAN_EXP;
    exps[i] = s_exp;
  }
  __syncthreads();
  const int e = s_exp;
  const size_t plane = (size_t)m * Kp;
  int8_t* dst = digits + (size_t)i * Kp;
  for (long long k = threadIdx.x; k < Kp; k += blockDim.x) {
    double r = (k < K && e != NAN_EXP) ? ldexp(col[k], 6 - e) : 0.0;  // 64·v, |v| < 1
#pragma unroll
    for (int t = 0; t < OZ_DIGITS; ++t) {
      const double d = rint(r);
      dst[(size_t)t * plane + k] = (int8_t)d;
      r = (r - d) * 128.0;
    }
  }
}

// ------------------------------------------------------------------ SYRK --
struct OzMaps {
  CUtensorMap a[OZ_DIGITS], b[OZ_DIGITS];
};

struct OzShared {
  uint64_t full[ONST], empty[ONST], done;
  uint32_t tmem;
};

// Shared-memory descriptor, K-major 32-byte swizzle (rows of 32 bytes, 8-row
// atoms of 256 bytes: SBO 256, LBO field 1, layout type 6).
__device__ __forceinline__ uint64_t smem_desc_sw32(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(256 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)6 << 61;
  return d;
}

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
      for (int d = 0; d < OZ_DIGITS; ++d) {
        umma::tma_load_2d(base + d * OA_BYTES, &maps.a[d], k, ra, &sh->full[s]);
        umma::tma_load_2d(base + OZ_DIGITS * OA_BYTES + d * OB_BYTES, &maps.b[d], k, rb,
                          &sh->full[s]);
      }
      ++issued;
    }
    for (int t = max(0, issued - ONST); t < issued; ++t)
      umma::mbar_wait_bounded(&sh->full[t % ONST], (t / ONST) & 1, err);
  } else if (threadIdx.x == 32) {
    constexpr uint32_t IDESC = idesc_s8_s32(OM, ON);
    for (int t = 0; t < ntiles; ++t) {
      const int s = t % ONST;
      if (!umma::mbar_wait_bounded(&sh->full[s], (t / ONST) & 1, err)) break;
      umma::fence_after_sync();
      const uint32_t base = umma::smem_u32(smem + s * OSTAGE);
#pragma unroll
      for (int ta = 0; ta < OZ_DIGITS; ++ta)
#pragma unroll
        for (int tb = 0; tb < OZ_DIGITS - ta; ++tb) {
          const uint64_t ad = smem_desc_sw32(base + ta * OA_BYTES);
          const uint64_t bd = smem_desc_sw32(base + OZ_DIGITS * OA_BYTES + tb * OB_BYTES);
          // level ta+tb; its first product (ta = 0) of the first tile starts it
          const uint32_t acc = (t > 0 || ta > 0) ? 1u : 0u;
          mma_s8(tmem + (uint32_t)((ta + tb) * ON), ad, bd, IDESC, acc);
        }
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
          acc[q] += ldexp((double)__float_as_int(raw[q]), -7 * lv);
      }
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const int gj = rb + cb + q;
        const int ej = gj < m ? exps[gj] : 0;
        double v;
        if (ei == NAN_EXP || ej == NAN_EXP)
          v = __longlong_as_double(0x7ff8000000000000ll);
        else
          v = ldexp(acc[q], ei + ej - 12);
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

__global__ void k_oz_reduce(const double* __restrict__ partial, const int2* __restrict__ pairs,
                            int npairs, int nchunk, int m, double* __restrict__ S) {
  const int pr = blockIdx.x;
  const int2 tile = pairs[pr];
  for (int e = threadIdx.x; e < OM * ON; e += blockDim.x) {
    const int r = e / ON, c = e % ON;
    const int gi = tile.x * OM + r, gj = tile.y * ON + c;
    if (gi >= m || gj >= m || gi < gj) continue;
    double s = 0.0;
    for (int ch = 0; ch < nchunk; ++ch) s += partial[((size_t)ch * npairs + pr) * OM * ON + e];
    S[gi + (size_t)gj * m] = s;
  }
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

void encode_digit_map(CUtensorMap* map, const int8_t* plane, int rows, long long Kp, int box_rows) {
  if ((reinterpret_cast<uintptr_t>(plane) & 15) != 0 || Kp % 16 != 0)
    throw std::invalid_argument("ozaki: digit plane not 16-byte aligned");
  cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)Kp};
  cuuint32_t box[2] = {(cuuint32_t)OK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = oz_encoder()(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(plane),
                            dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
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
                double* S, int* err, cudaStream_t st, cudaEvent_t ev_begin, cudaEvent_t ev_end) {
  const int m = plan.m;
  if (m <= 0) return;
  k_oz_digits<<<m, 256, 0, st>>>(P, plan.K, plan.Kp, m, digits, exps);
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
  for (int d = 0; d < OZ_DIGITS; ++d) {
    encode_digit_map(&maps.a[d], digits + d * plane, m, plan.Kp, OM);
    encode_digit_map(&maps.b[d], digits + d * plane, m, plan.Kp, ON);
  }
  ensure_smem(k_oz_syrk, OSMEM);
  const int units = plan.ntri * plan.nchunk;
  if (ev_begin) SDPX_CUDA(cudaEventRecord(ev_begin, st));
  k_oz_syrk<<<units, ONT, OSMEM, st>>>(maps, d_pairs, plan.ntri, plan.kchunk, plan.Kp, exps, m,
                                       partial, err);
  if (ev_end) SDPX_CUDA(cudaEventRecord(ev_end, st));
  k_oz_reduce<<<plan.ntri, 256, 0, st>>>(partial, d_pairs, plan.ntri, plan.nchunk, m, S);
  SDPX_LAUNCH_CHECK_N(2);
}

}  // namespace sdpx
