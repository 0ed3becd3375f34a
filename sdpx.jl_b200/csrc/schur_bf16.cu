// Split-BF16 Schur assembly on the 5th-generation tensor cores (tcgen05).
//
// Every FP64 (or FP32) operand value v is carried as three BF16 "planes"
// v ≈ v0 + v1 + v2 (v0 = bf16(v), v1 = bf16(v − v0), v2 = bf16(v − v0 − v1),
// 24 significant bits).  A product Σ_k a_k b_k is formed as the six plane
// products with i + j ≤ 2, all accumulated in one FP32 TMEM accumulator
// (the dropped terms are below 2^-24 relative).  Long contractions are cut
// into K chunks whose FP32 tiles are summed in FP64, so the accumulation error
// does not grow with K.
//
// One engine serves the three products of the Schur assembly
//   T_i = L_X⁻¹ A_i         (A operand: rows of W = L_X⁻¹; B operand: columns of A_i)
//   P_i = T_i · L_Y         (A operand: rows of T_i;       B operand: columns of L_Y)
//   S   = P̂ᵀ P̂ (lower)     (A, B: variables' stacked P̂ columns, split K)
// CTA tile 128×128, K tile 64, two smem stages of 6 operand tiles (96 KB each),
// MMA M=128 N=128 K=16 issued by one thread, completion tracked by mbarriers.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "schur_bf16.h"
#include "umma.cuh"

namespace sdpx {

namespace {

constexpr int TM = 128, TN = 128, TK = 64;
constexpr int NTHREADS = 128;
constexpr int TILE_BYTES = TM * TK * 2;        // 16 KB per operand plane tile
constexpr int STAGE_BYTES = 6 * TILE_BYTES;    // A0 A1 A2 B0 B1 B2
constexpr int NSTAGE = 2;
constexpr uint32_t LBO = 128;                  // core matrices adjacent along K
constexpr uint32_t SBO = (TK / 8) * 128;       // 8-row groups
constexpr size_t SMEM_BYTES = NSTAGE * STAGE_BYTES + 256;

__device__ __forceinline__ uint32_t tile_off(int row, int k) {
  return (uint32_t)((row >> 3) * SBO + (k >> 3) * LBO + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ long long row_off(const RowMap& r, int row) {
  return r.base + (long long)(row / r.inner) * r.os + (long long)(row % r.inner) * r.is;
}

// Stage loader: rows [r0, r0+128) of A, [c0, c0+128) of B, K slice [k0, k0+64).
struct Loader {
  long long a_off[8], b_off[8];  // per owned row (-1 = out of range)
  __device__ void init(const PlaneOpnd& A, const PlaneOpnd& B, int r0, int c0) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      int row = tid / 8 + 16 * j;
      int ga = r0 + row, gb = c0 + row;
      a_off[j] = ga < A.rows.extent ? row_off(A.rows, ga) : -1;
      b_off[j] = gb < B.rows.extent ? row_off(B.rows, gb) : -1;
    }
  }
  __device__ void issue(unsigned char* stage, const PlaneOpnd& A, const PlaneOpnd& B, int k0) const {
    const int tid = threadIdx.x;
    const int kc = (tid & 7) * 8;  // element offset of this thread's 16-byte chunk
    const int k = k0 + kc;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      int row = tid / 8 + 16 * j;
      uint32_t so = tile_off(row, kc);
      bool va = a_off[j] >= 0 && k < A.kvalid;
      bool vb = b_off[j] >= 0 && k < B.kvalid;
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        const __nv_bfloat16* ga = va ? A.plane[p] + a_off[j] + k : A.plane[p];
        const __nv_bfloat16* gb = vb ? B.plane[p] + b_off[j] + k : B.plane[p];
        umma::cp_async16(stage + p * TILE_BYTES + so, ga, va);
        umma::cp_async16(stage + (3 + p) * TILE_BYTES + so, gb, vb);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  }
};

__device__ __forceinline__ void split3(float v, __nv_bfloat16& h0, __nv_bfloat16& h1,
                                       __nv_bfloat16& h2) {
  h0 = __float2bfloat16_rn(v);
  float r = v - __bfloat162float(h0);
  h1 = __float2bfloat16_rn(r);
  h2 = __float2bfloat16_rn(r - __bfloat162float(h1));
}

// Accumulate the six plane products over K range [kb, ke) into TMEM.
// Returns false when a bounded wait gave up.
__device__ bool mainloop(const PlaneOpnd& A, const PlaneOpnd& B, int r0, int c0, int kb, int ke,
                         unsigned char* smem, uint64_t* mbar, uint32_t* phase, uint32_t tmem,
                         int* err) {
  const int ntiles = (ke > kb) ? (ke - kb + TK - 1) / TK : 0;
  Loader ld;
  ld.init(A, B, r0, c0);
  constexpr uint32_t IDESC = umma::idesc_bf16_f32(TM, TN);
  bool ok = true;
  if (ntiles == 0) return true;
  ld.issue(smem, A, B, kb);
  for (int t = 0; t < ntiles; ++t) {
    const int s = t & 1;
    if (t + 1 < ntiles) {
      const int s2 = (t + 1) & 1;
      if (t + 1 >= NSTAGE) {
        // stage s2 was read by the MMAs of tile t-1: wait for their commit
        if (!umma::mbar_wait_bounded(&mbar[s2], phase[s2], err)) ok = false;
        phase[s2] ^= 1u;
      }
      ld.issue(smem + s2 * STAGE_BYTES, A, B, kb + (t + 1) * TK);
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    umma::fence_proxy_async_smem();
    // uniform decision: every thread leaves the loop together
    if (!__syncthreads_and(ok ? 1 : 0)) {
      ok = false;
      break;
    }
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
      const uint32_t base = umma::smem_u32(smem + s * STAGE_BYTES);
#pragma unroll
      for (int ks = 0; ks < TK / 16; ++ks) {
        const uint32_t koff = ks * 2 * LBO;
        // (a, b) plane pairs with a + b ≤ 2
        const int pa[6] = {0, 0, 1, 0, 1, 2};
        const int pb[6] = {0, 1, 0, 2, 1, 0};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          uint64_t ad = umma::smem_desc(base + pa[q] * TILE_BYTES + koff, LBO, SBO);
          uint64_t bd = umma::smem_desc(base + (3 + pb[q]) * TILE_BYTES + koff, LBO, SBO);
          umma::mma_bf16(tmem, ad, bd, IDESC, (t > 0 || ks > 0 || q > 0) ? 1u : 0u);
        }
      }
      umma::commit(&mbar[s]);
    }
    __syncthreads();
  }
  // wait for the last committed stage (covers all earlier MMAs of this thread)
  if (ok && ntiles > 0) {
    const int s = (ntiles - 1) & 1;
    if (!umma::mbar_wait_bounded(&mbar[s], phase[s], err)) ok = false;
    phase[s] ^= 1u;
    if (ntiles >= 2) {
      // the other stage's last commit completed earlier (MMAs complete in order);
      // consume its pending phase so both barriers agree with `phase`.
      const int o = s ^ 1;
      if (!umma::mbar_wait_bounded(&mbar[o], phase[o], err)) ok = false;
      phase[o] ^= 1u;
    }
  }
  ok = __syncthreads_and(ok ? 1 : 0) != 0;
  umma::fence_after_sync();
  return ok;
}

__device__ inline void tri_index(int tri, int& ti, int& tj) {
  int a = (int)((sqrt(8.0 * tri + 1.0) - 1.0) * 0.5);
  while ((a + 1) * (a + 2) / 2 <= tri) ++a;
  while (a * (a + 1) / 2 > tri) --a;
  ti = a;
  tj = tri - a * (a + 1) / 2;
}

struct KernelShared {
  uint64_t mbar[2];
  uint32_t tmem;
};

template <int MODE>
__global__ void __launch_bounds__(NTHREADS, 1)
    k_split_gemm(PlaneOpnd A, PlaneOpnd B, OutMap out, int kmode, int Ktot, int ntri, int kchunk,
                 float* partial, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = smem_raw;
  KernelShared* ks = reinterpret_cast<KernelShared*>(smem_raw + NSTAGE * STAGE_BYTES);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    umma::mbar_init(&ks->mbar[0], 1);
    umma::mbar_init(&ks->mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == 0) umma::tmem_alloc(&ks->tmem, 128);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = ks->tmem;
  uint32_t phase[2] = {0u, 0u};

  int r0, c0, kb, ke;
  if (MODE == 0) {  // SYRK: unit = chunk-major (chunk, lower tile)
    const int u = blockIdx.x;
    const int chunk = u / ntri, tri = u % ntri;
    int ti, tj;
    tri_index(tri, ti, tj);
    r0 = ti * TM;
    c0 = tj * TN;
    kb = chunk * kchunk;
    ke = min(Ktot, kb + kchunk);
  } else {
    r0 = blockIdx.y * TM;
    c0 = blockIdx.x * TN;
    kb = 0;
    ke = Ktot;
    if (kmode == 1) ke = min(Ktot, ((r0 + TM + TK - 1) / TK) * TK);  // A lower triangular
    if (kmode == 2) kb = (c0 / TK) * TK;                                // B lower triangular
  }
  bool ok = mainloop(A, B, r0, c0, kb, ke, smem, ks->mbar, phase, tmem, err);

  // Epilogue: warp w owns accumulator rows [32w, 32w+32) (TMEM lanes).
  const int row = warp * 32 + lane;
  if (ok) {
    for (int cb = 0; cb < TN; cb += 32) {
      float v[32];
      umma::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, v);
      if (MODE == 0) {
        float* dst = partial + (size_t)blockIdx.x * TM * TN + (size_t)row * TN + cb;
#pragma unroll
        for (int q = 0; q < 32; q += 4)
          *reinterpret_cast<float4*>(dst + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
      } else {
        const int grow = r0 + row;
        if (grow < out.rows.extent) {
          const long long ro = row_off(out.rows, grow);
#pragma unroll
          for (int q = 0; q < 32; q += 8) {
            const int gcol = c0 + cb + q;
            if (gcol >= out.col_extent) continue;
            const long long co = (long long)(gcol / out.col_inner) * out.col_os +
                                 (long long)(gcol % out.col_inner);
            __align__(16) __nv_bfloat16 h[3][8];
#pragma unroll
            for (int e = 0; e < 8; ++e) split3(v[q + e], h[0][e], h[1][e], h[2][e]);
#pragma unroll
            for (int p = 0; p < 3; ++p)
              *reinterpret_cast<uint4*>(out.plane[p] + ro + co) = *reinterpret_cast<uint4*>(h[p]);
          }
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

// ---------------------------------------------------------------------------
// Lower SYRK S = P̂ᵀP̂ fed by TMA.  One CTA per (K chunk, lower 128×128 tile),
// 128 threads: thread 0 produces (24 TMA boxes of 128 rows × 32 BF16 per stage:
// three planes of the A rows and of the B rows, 64-byte swizzle), thread 32
// issues the 12 MMAs of a stage (2 K steps × the 6 plane products) and commits
// them to the stage's "empty" barrier, all four warps then drain the FP32 TMEM
// tile.  Four 48 KB stages.  Rows beyond m and K beyond Kp arrive as zeros
// (TMA out-of-bounds fill).  Every wait is bounded and records a device error
// instead of spinning; the producer waits for all of its own copies before the
// CTA leaves.
// ---------------------------------------------------------------------------
constexpr int SK = 32;                          // K per stage
constexpr int SNST = 4;                         // stages
constexpr int SPLANE_BYTES = TM * SK * 2;       // 8 KB: 128 rows × 64 B
constexpr int SSTAGE_BYTES = 6 * SPLANE_BYTES;  // 48 KB
constexpr size_t SSMEM_BYTES = SNST * SSTAGE_BYTES + 1024 + 256;

struct SyrkMaps {
  CUtensorMap plane[3];
};

struct SyrkShared {
  uint64_t full[SNST], empty[SNST], done;
  uint32_t tmem;
};

__global__ void __launch_bounds__(NTHREADS, 1)
    k_split_syrk_tma(const __grid_constant__ SyrkMaps maps, int ntri, int kchunk, int Ktot,
                     float* partial, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  SyrkShared* sh = reinterpret_cast<SyrkShared*>(smem + SNST * SSTAGE_BYTES);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < SNST; ++s) {
      umma::mbar_init(&sh->full[s], 1);
      umma::mbar_init(&sh->empty[s], 1);
    }
    umma::mbar_init(&sh->done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == 0) umma::tmem_alloc(&sh->tmem, 128);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = sh->tmem;

  const int u = blockIdx.x;
  const int chunk = u / ntri, tri = u % ntri;
  int ti, tj;
  tri_index(tri, ti, tj);
  const int r0 = ti * TM, c0 = tj * TN;
  const int kb = chunk * kchunk;
  const int ke = min(Ktot, kb + kchunk);
  const int ntiles = ke > kb ? (ke - kb + SK - 1) / SK : 0;

  if (threadIdx.x == 0) {
    // producer
    int issued = 0;
    for (int t = 0; t < ntiles; ++t) {
      const int s = t % SNST;
      if (t >= SNST && !umma::mbar_wait_bounded(&sh->empty[s], ((t / SNST) - 1) & 1, err)) break;
      umma::mbar_expect_tx(&sh->full[s], SSTAGE_BYTES);
      const uint32_t base = umma::smem_u32(smem + s * SSTAGE_BYTES);
      const int k = kb + t * SK;
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        umma::tma_load_2d(base + p * SPLANE_BYTES, &maps.plane[p], k, r0, &sh->full[s]);
        umma::tma_load_2d(base + (3 + p) * SPLANE_BYTES, &maps.plane[p], k, c0, &sh->full[s]);
      }
      ++issued;
    }
    // drain: every issued stage has landed before the CTA may leave
    for (int t = max(0, issued - SNST); t < issued; ++t)
      umma::mbar_wait_bounded(&sh->full[t % SNST], (t / SNST) & 1, err);
  } else if (threadIdx.x == 32) {
    // MMA issuer
    constexpr uint32_t IDESC = umma::idesc_bf16_f32(TM, TN);
    const int pa[6] = {0, 0, 1, 0, 1, 2};
    const int pb[6] = {0, 1, 0, 2, 1, 0};
    for (int t = 0; t < ntiles; ++t) {
      const int s = t % SNST;
      if (!umma::mbar_wait_bounded(&sh->full[s], (t / SNST) & 1, err)) break;
      umma::fence_after_sync();
      const uint32_t base = umma::smem_u32(smem + s * SSTAGE_BYTES);
#pragma unroll
      for (int ks = 0; ks < SK / 16; ++ks) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const uint64_t ad = umma::smem_desc_sw64(base + pa[q] * SPLANE_BYTES + ks * 32);
          const uint64_t bd = umma::smem_desc_sw64(base + (3 + pb[q]) * SPLANE_BYTES + ks * 32);
          umma::mma_bf16(tmem, ad, bd, IDESC, (t > 0 || ks > 0 || q > 0) ? 1u : 0u);
        }
      }
      umma::commit(&sh->empty[s]);
    }
    umma::commit(&sh->done);  // arrives once every MMA issued above has completed
  }
  __syncwarp();
  const bool ok = umma::mbar_wait_bounded(&sh->done, 0, err);
  umma::fence_after_sync();
  const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;

  // Epilogue: warp w owns accumulator rows [32w, 32w+32) (TMEM lanes).
  if (all_ok && ntiles > 0) {
    const int row = warp * 32 + lane;
    for (int cb = 0; cb < TN; cb += 32) {
      float v[32];
      umma::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, v);
      float* dst = partial + (size_t)blockIdx.x * TM * TN + (size_t)row * TN + cb;
#pragma unroll
      for (int q = 0; q < 32; q += 4)
        *reinterpret_cast<float4*>(dst + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
    }
  } else if (ntiles == 0) {
    const int row = warp * 32 + lane;
    float* dst = partial + (size_t)blockIdx.x * TM * TN + (size_t)row * TN;
    for (int q = 0; q < TN; q += 4) *reinterpret_cast<float4*>(dst + q) = make_float4(0, 0, 0, 0);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

__global__ void k_reduce_partials(const float* partial, int ntri, int nchunk, int m, double* S) {
  const int tri = blockIdx.x;
  int ti, tj;
  tri_index(tri, ti, tj);
  for (int e = threadIdx.x; e < TM * TN; e += blockDim.x) {
    const int r = e / TN, c = e % TN;
    const int gi = ti * TM + r, gj = tj * TN + c;
    if (gi >= m || gj >= m) continue;
    double s = 0.0;
    for (int ch = 0; ch < nchunk; ++ch) s += (double)partial[((size_t)ch * ntri + tri) * TM * TN + e];
    S[gi + (size_t)gj * m] = s;
  }
}

// FP64 source → three BF16 planes, generic gather: dst[p][dst_index(t)] from src[src_index(t)].
__device__ __forceinline__ void split3d(double v, __nv_bfloat16& h0, __nv_bfloat16& h1,
                                        __nv_bfloat16& h2) {
  h0 = __double2bfloat16(v);
  double r = v - (double)__bfloat162float(h0);
  h1 = __double2bfloat16(r);
  h2 = __double2bfloat16(r - (double)__bfloat162float(h1));
}

// Dense block of 𝒜 (rows off + p + c·k of every column i) → planes[i][o + c·kp + p].
__global__ void k_split_A_dense(const double* A, long long K, int m, long long off, int k, int kp,
                                __nv_bfloat16* P0, __nv_bfloat16* P1, __nv_bfloat16* P2,
                                long long Kp, long long o) {
  const long long kk = (long long)k * k;
  const long long tot = kk * m;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / kk, q = t % kk;
    const int p = (int)(q % k), c = (int)(q / k);
    const long long d = i * Kp + o + (long long)c * kp + p;
    split3d(A[i * K + off + q], P0[d], P1[d], P2[d]);
  }
}

// 1×1 group rows: planes[i][o + j] from A[od + j, i] · scale[j] (scale null → 1).
__global__ void k_split_diag_rows(const double* A, long long K, int m, long long od, int nd,
                                  const double* LX, const double* MY, __nv_bfloat16* P0,
                                  __nv_bfloat16* P1, __nv_bfloat16* P2, long long Kp, long long o) {
  const long long tot = (long long)nd * m;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t % nd);
    const long long i = t / nd;
    double v = A[od + j + i * K];
    if (LX) v = (v / LX[od + j]) * MY[od + j];
    const long long d = i * Kp + o + j;
    split3d(v, P0[d], P1[d], P2[d]);
  }
}

// k×k FP64 matrix M (column-major, at M) → planes with row-major (transpose = 1,
// element (r,p) at r·kp + p) or column-major (transpose = 0, (p,c) at c·kp + p) padding.
__global__ void k_split_small(const double* M, int k, int kp, int row_major, __nv_bfloat16* P0,
                              __nv_bfloat16* P1, __nv_bfloat16* P2) {
  const int tot = k * k;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
    const int r = t % k, c = t / k;
    const long long d = row_major ? (long long)r * kp + c : (long long)c * kp + r;
    split3d(M[t], P0[d], P1[d], P2[d]);
  }
}

}  // namespace

size_t split_gemm_smem_bytes() { return SMEM_BYTES; }

void split_gemm_planes(const PlaneOpnd& A, const PlaneOpnd& B, const OutMap& out, int kmode,
                       int Ktot, int* err, cudaStream_t st) {
  ensure_smem(k_split_gemm<1>, SMEM_BYTES);
  dim3 grid(ceil_div(out.col_extent, TN), ceil_div(out.rows.extent, TM));
  if (grid.x == 0 || grid.y == 0) return;
  k_split_gemm<1><<<grid, NTHREADS, SMEM_BYTES, st>>>(A, B, out, kmode, Ktot, 0, 0, nullptr, err);
  SDPX_LAUNCH_CHECK();
}

SplitSyrkPlan plan_split_syrk(int m, long long Kp, int sm_count) {
  SplitSyrkPlan p;
  const int nt = ceil_div(m, TM);
  p.ntri = nt * (nt + 1) / 2;
  // K chunks of 2048-4096 (the FP32 accumulation length) rounded so that the
  // units fill whole waves of one CTA per SM where possible.
  long long target = 4096;
  int base_c = (int)std::max<long long>(1, (Kp + target - 1) / target);
  int best_c = base_c;
  double best = -1;
  for (int c = base_c; c <= 2 * base_c + 8; ++c) {
    long long units = (long long)p.ntri * c;
    double waves = (double)units / sm_count;
    double eff = waves / std::ceil(waves);
    if (eff > best + 1e-9) best = eff, best_c = c;
  }
  long long kc = (Kp + best_c - 1) / best_c;
  kc = ((kc + TK - 1) / TK) * TK;
  p.kchunk = (int)kc;
  p.nchunk = (int)((Kp + kc - 1) / kc);
  p.partial_floats = (size_t)p.nchunk * p.ntri * TM * TN;
  return p;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
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

// Tensor map of one plane: rows × Kp BF16, row-major; box 32 × 128, 64-byte swizzle.
static void encode_plane_map(CUtensorMap* map, const __nv_bfloat16* plane, int rows, long long Kp) {
  if ((reinterpret_cast<uintptr_t>(plane) & 15) != 0 || (Kp * 2) % 16 != 0)
    throw std::invalid_argument("split SYRK: plane base or row pitch not 16-byte aligned");
  cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)Kp * 2};
  cuuint32_t box[2] = {(cuuint32_t)SK, (cuuint32_t)TM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = tensor_map_encoder()(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                                    const_cast<__nv_bfloat16*>(plane), dims, strides, box, estr,
                                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

void split_syrk(const PlaneOpnd& P, int m, int Kp, const SplitSyrkPlan& plan, float* partial,
                double* S, int* err, cudaStream_t st) {
  if (P.rows.is != Kp || P.rows.base != 0 || Kp % SK != 0 || plan.kchunk % SK != 0)
    throw std::invalid_argument("split SYRK: planes must be m × Kp row-major, Kp and chunks ≡ 0 mod 32");
  SyrkMaps maps;
  for (int p = 0; p < 3; ++p) encode_plane_map(&maps.plane[p], P.plane[p], m, Kp);
  ensure_smem(k_split_syrk_tma, SSMEM_BYTES);
  const int units = plan.ntri * plan.nchunk;
  k_split_syrk_tma<<<units, NTHREADS, SSMEM_BYTES, st>>>(maps, plan.ntri, plan.kchunk, Kp, partial,
                                                        err);
  k_reduce_partials<<<plan.ntri, 256, 0, st>>>(partial, plan.ntri, plan.nchunk, m, S);
  SDPX_LAUNCH_CHECK_N(2);
}

void split_A_dense(const double* A, long long K, int m, long long off, int k, int kp,
                   __nv_bfloat16* const* planes, long long Kp, long long o, cudaStream_t st) {
  long long tot = (long long)k * k * m;
  k_split_A_dense<<<std::min<long long>(8192, ceil_div(tot, 256)), 256, 0, st>>>(
      A, K, m, off, k, kp, planes[0], planes[1], planes[2], Kp, o);
  SDPX_LAUNCH_CHECK();
}

void split_diag_rows(const double* A, long long K, int m, long long od, int nd, const double* LX,
                     const double* MY, __nv_bfloat16* const* planes, long long Kp, long long o,
                     cudaStream_t st) {
  if (nd == 0) return;
  long long tot = (long long)nd * m;
  k_split_diag_rows<<<std::min<long long>(4096, ceil_div(tot, 256)), 256, 0, st>>>(
      A, K, m, od, nd, LX, MY, planes[0], planes[1], planes[2], Kp, o);
  SDPX_LAUNCH_CHECK();
}

void split_small(const double* M, int k, int kp, bool row_major, __nv_bfloat16* const* planes,
                 cudaStream_t st) {
  k_split_small<<<std::max(1, std::min(1024, ceil_div(k * k, 256))), 256, 0, st>>>(
      M, k, kp, row_major ? 1 : 0, planes[0], planes[1], planes[2]);
  SDPX_LAUNCH_CHECK();
}

}  // namespace sdpx
