// Split-BF16 Schur assembly on the 5th-generation tensor cores (tcgen05).
//
// Every FP64 (or FP32) operand value v is carried as three BF16 "planes"
// v ≈ v0 + v1 + v2 (v0 = bf16(v), v1 = bf16(v − v0), v2 = bf16(v − v0 − v1),
// 24 significant bits).  A product Σ_k a_k b_k is formed as the six plane
// products with i + j ≤ 2 (the dropped terms are below 2^-24 relative) in two
// FP32 TMEM accumulators: the leading product a0·b0 in one, the five
// lower-order products (≈ 2^-8 of it) in the other, so each MMA instruction
// rounds at the magnitude of what it adds; the two are added once in the
// epilogue.  Long contractions are cut into K chunks whose FP32 tiles are
// summed in FP64, so the accumulation error does not grow with K.
//
// One TMA-fed engine serves the three products of the Schur assembly
//   T_i = L_X⁻¹ A_i         (A operand: rows of W = L_X⁻¹; B operand: columns of A_i)
//   P_i = T_i · L_Y         (A operand: rows of T_i;       B operand: columns of L_Y)
//   S   = P̂ᵀ P̂ (lower)     (A, B: variables' stacked P̂ columns, split K)
// Every operand plane is a row-major 2D BF16 tensor (rows × K, row pitch a
// multiple of 8 elements) described by a TMA tensor map.  CTA tile 128×128,
// 128 threads: thread 0 produces (6 TMA boxes of 128 rows × 32 BF16 per stage,
// 64-byte swizzle, four 48 KB stages), thread 32 issues the 12 MMAs of a stage
// (M=128 N=128 K=16, 2 K steps × 6 plane products) and commits them to the
// stage's "empty" barrier; all four warps then drain the FP32 TMEM tile.  Rows
// and K beyond a tensor's extent arrive as zeros (TMA out-of-bounds fill).
// Every wait is bounded and records a device error instead of spinning; the
// producer waits for all of its own copies before the CTA leaves.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "schur_bf16.h"
#include "umma.cuh"

namespace sdpx {

namespace {

constexpr int TM = 128, TN = 128;
constexpr int NTHREADS = 128;
constexpr int SK = 32;                          // K per stage
constexpr int SNST = 4;                         // stages
constexpr int SPLANE_BYTES = TM * SK * 2;       // 8 KB: 128 rows × 64 B
constexpr int SSTAGE_BYTES = 6 * SPLANE_BYTES;  // 48 KB
constexpr size_t SSMEM_BYTES = SNST * SSTAGE_BYTES + 1024 + 256;

__device__ __forceinline__ long long row_off(const RowMap& r, int row) {
  return r.base + (long long)(row / r.inner) * r.os + (long long)(row % r.inner) * r.is;
}

__device__ __forceinline__ void split3(float v, __nv_bfloat16& h0, __nv_bfloat16& h1,
                                       __nv_bfloat16& h2) {
  h0 = __float2bfloat16_rn(v);
  float r = v - __bfloat162float(h0);
  h1 = __float2bfloat16_rn(r);
  h2 = __float2bfloat16_rn(r - __bfloat162float(h1));
}

__device__ inline void tri_index(int tri, int& ti, int& tj) {
  int a = (int)((sqrt(8.0 * tri + 1.0) - 1.0) * 0.5);
  while ((a + 1) * (a + 2) / 2 <= tri) ++a;
  while (a * (a + 1) / 2 > tri) --a;
  ti = a;
  tj = tri - a * (a + 1) / 2;
}

struct TmaMaps {
  CUtensorMap a[3], b[3];
};

struct PipeShared {
  uint64_t full[SNST], empty[SNST], done;
  uint32_t tmem;
};

__device__ __forceinline__ unsigned char* aligned_smem(unsigned char* raw) {
  return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(raw) + 1023) &
                                          ~uintptr_t(1023));
}

// Barrier set-up and the TMEM accumulators (all threads): columns [0, 128)
// hold the leading product a0·b0, columns [128, 256) the lower-order products.
__device__ __forceinline__ uint32_t pipe_init(PipeShared* sh) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < SNST; ++s) {
      umma::mbar_init(&sh->full[s], 1);
      umma::mbar_init(&sh->empty[s], 1);
    }
    umma::mbar_init(&sh->done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if ((threadIdx.x >> 5) == 0) umma::tmem_alloc(&sh->tmem, 256);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  return sh->tmem;
}

// Accumulate A[ra:ra+128, k]·B[rb:rb+128, k]ᵀ over `ntiles` K tiles starting
// at kb into TMEM.  Returns true on every thread when all waits succeeded.
__device__ bool pipe_mainloop(const TmaMaps& maps, int ra, int rb, int kb, int ntiles,
                              unsigned char* smem, PipeShared* sh, uint32_t tmem, int* err) {
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
        umma::tma_load_2d(base + p * SPLANE_BYTES, &maps.a[p], k, ra, &sh->full[s]);
        umma::tma_load_2d(base + (3 + p) * SPLANE_BYTES, &maps.b[p], k, rb, &sh->full[s]);
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
          // q = 0 → leading accumulator; q ≥ 1 → lower-order accumulator (first write at q = 1)
          const uint32_t acc = (t > 0 || ks > 0 || q > 1) ? 1u : 0u;
          umma::mma_bf16(q == 0 ? tmem : tmem + 128, ad, bd, IDESC, acc);
        }
      }
      umma::commit(&sh->empty[s]);
    }
    umma::commit(&sh->done);  // arrives once every MMA issued above has completed
  }
  __syncwarp();
  const bool ok = umma::mbar_wait_bounded(&sh->done, 0, err);
  umma::fence_after_sync();
  return __syncthreads_and(ok ? 1 : 0) != 0;
}

// 32 columns [cb, cb+32) of this warp's 32 accumulator rows: leading plus
// lower-order accumulator (one FP32 addition).
__device__ __forceinline__ void tile_ld32(uint32_t tmem, int warp, int cb, float (&v)[32]) {
  float lo[32];
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  umma::tmem_ld32(tmem + lane_base + (uint32_t)cb, v);
  umma::tmem_ld32(tmem + lane_base + 128u + (uint32_t)cb, lo);
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] += lo[q];
}

__device__ __forceinline__ void pipe_release(uint32_t tmem) {
  umma::fence_before_sync();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) umma::tmem_dealloc(tmem, 256);
}

// Lower SYRK S = P̂ᵀP̂: one CTA per (K chunk, lower 128×128 tile); the FP32
// tile goes to `partial` (summed over chunks in FP64 by k_reduce_partials).
__global__ void __launch_bounds__(NTHREADS, 1)
    k_split_syrk_tma(const __grid_constant__ TmaMaps maps, int ntri, int kchunk, int Ktot,
                     float* partial, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = aligned_smem(smem_raw);
  PipeShared* sh = reinterpret_cast<PipeShared*>(smem + SNST * SSTAGE_BYTES);
  const uint32_t tmem = pipe_init(sh);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x;
  const int chunk = u / ntri, tri = u % ntri;
  int ti, tj;
  tri_index(tri, ti, tj);
  const int kb = chunk * kchunk;
  const int ke = min(Ktot, kb + kchunk);
  const int ntiles = ke > kb ? (ke - kb + SK - 1) / SK : 0;
  const bool ok = pipe_mainloop(maps, ti * TM, tj * TN, kb, ntiles, smem, sh, tmem, err);
  const int row = warp * 32 + lane;
  float* dst0 = partial + (size_t)blockIdx.x * TM * TN + (size_t)row * TN;
  if (ok && ntiles > 0) {
    for (int cb = 0; cb < TN; cb += 32) {
      float v[32];
      tile_ld32(tmem, warp, cb, v);
#pragma unroll
      for (int q = 0; q < 32; q += 4)
        *reinterpret_cast<float4*>(dst0 + cb + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
    }
  } else if (ntiles == 0) {
    for (int q = 0; q < TN; q += 4) *reinterpret_cast<float4*>(dst0 + q) = make_float4(0, 0, 0, 0);
  }
  pipe_release(tmem);
}

// Block products, persistent and warp-specialised.  With K at most
// ceil(k/32) stages per output tile, a CTA per tile spends much of its time
// filling the pipeline and draining the accumulator.  Here one CTA per SM walks
// its tiles: warp 4 (one thread) streams the six plane boxes of each stage and
// runs ahead into the next tile, warp 5 (one thread) issues the MMAs into one
// of two TMEM accumulator buffers (columns [256·b, 256·b + 256): leading
// product at +0, lower-order products at +128) and commits the tile to
// tfull[b]; warps 0-3 drain buffer b, hand it back through tempty[b], and split
// and store while the MMAs of the next tile run into the other buffer.  Tiles
// run the operand with fewer tiles fastest (they share the other operand's
// tile in L2), rotated by the slow index so each CTA sees every K length of the
// triangular ranges.  out = A·Bᵀ split into three BF16 output planes; kmode 0
// contracts the full K, 1 stops at the end of the A tile (A lower-triangular,
// rows of L_X⁻¹), 2 starts at the B tile (B rows are columns of L_Y, zero
// above the diagonal).
constexpr int PG_THREADS = 6 * 32;
// Epilogue staging: per warp one plane's 32 rows × 32 columns (64 B a row,
// padded to 80 B) after the barrier block.
constexpr int EPI_ROW_BYTES = 80;
constexpr int EPI_WARP_BYTES = 32 * EPI_ROW_BYTES;
constexpr size_t PG_SMEM_BYTES = SNST * SSTAGE_BYTES + 1024 + 256 + 4 * EPI_WARP_BYTES;

struct PGemmShared {
  uint64_t full[SNST], empty[SNST], tfull[2], tempty[2], mdone;
  uint32_t tmem;
  int abort;
};

struct PGemmTiles {
  long long ntask;
  int ta, tb, a_fast, kmode, Ktot;
};

__device__ __forceinline__ bool pg_wait(uint64_t* mbar, uint32_t parity, int* err,
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

__device__ __forceinline__ void pg_task(const PGemmTiles& g, long long u, int& r0, int& c0, int& kb,
                                        int& nk) {
  if (g.a_fast) {
    const int slow = (int)(u / g.ta);
    r0 = (int)((u % g.ta + slow) % g.ta) * TM;
    c0 = slow * TN;
  } else {
    const int slow = (int)(u / g.tb);
    c0 = (int)((u % g.tb + slow) % g.tb) * TN;
    r0 = slow * TM;
  }
  kb = 0;
  int ke = g.Ktot;
  if (g.kmode == 1) ke = min(g.Ktot, r0 + TM);
  if (g.kmode == 2) kb = (c0 / SK) * SK;
  nk = ke > kb ? (ke - kb + SK - 1) / SK : 0;
}

__global__ void __launch_bounds__(PG_THREADS, 1)
    k_split_gemm_persistent(const __grid_constant__ TmaMaps maps, OutMap out, PGemmTiles g,
                            int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = aligned_smem(smem_raw);
  PGemmShared* sh = reinterpret_cast<PGemmShared*>(smem + SNST * SSTAGE_BYTES);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < SNST; ++s) {
      umma::mbar_init(&sh->full[s], 1);
      umma::mbar_init(&sh->empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      umma::mbar_init(&sh->tfull[b], 1);
      umma::mbar_init(&sh->tempty[b], 4);
    }
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

  if (warp == 4) {
    if (lane == 0) {
      uint32_t it = 0;
      for (long long u = blockIdx.x; u < g.ntask && !*abort; u += gridDim.x) {
        int r0, c0, kb, nk;
        pg_task(g, u, r0, c0, kb, nk);
        bool ok = true;
        for (int t = 0; t < nk; ++t, ++it) {
          const int s = it % SNST;
          if (it >= SNST && !pg_wait(&sh->empty[s], ((it / SNST) - 1) & 1, err, abort)) {
            ok = false;
            break;
          }
          umma::mbar_expect_tx(&sh->full[s], SSTAGE_BYTES);
          const uint32_t base = umma::smem_u32(smem + s * SSTAGE_BYTES);
          const int k = kb + t * SK;
#pragma unroll
          for (int p = 0; p < 3; ++p) {
            umma::tma_load_2d(base + p * SPLANE_BYTES, &maps.a[p], k, r0, &sh->full[s]);
            umma::tma_load_2d(base + (3 + p) * SPLANE_BYTES, &maps.b[p], k, c0, &sh->full[s]);
          }
        }
        if (!ok) break;
      }
      // every issued stage lands before the CTA may leave
      for (uint32_t t = it > (uint32_t)SNST ? it - SNST : 0; t < it; ++t)
        umma::mbar_wait_bounded(&sh->full[t % SNST], (t / SNST) & 1, err);
    }
  } else if (warp == 5) {
    if (lane == 0) {
      constexpr uint32_t IDESC = umma::idesc_bf16_f32(TM, TN);
      const int pa[6] = {0, 0, 1, 0, 1, 2};
      const int pb[6] = {0, 1, 0, 2, 1, 0};
      uint32_t it = 0, j = 0;
      bool ok = true;
      for (long long u = blockIdx.x; u < g.ntask && ok; u += gridDim.x, ++j) {
        int r0, c0, kb, nk;
        pg_task(g, u, r0, c0, kb, nk);
        const int b = j & 1;
        if (j >= 2 && !pg_wait(&sh->tempty[b], ((j >> 1) - 1) & 1, err, abort)) break;
        umma::fence_after_sync();
        const uint32_t acc0 = tmem + (uint32_t)(b * 256);
        for (int t = 0; t < nk; ++t, ++it) {
          const int s = it % SNST;
          if (!pg_wait(&sh->full[s], (it / SNST) & 1, err, abort)) {
            ok = false;
            break;
          }
          umma::fence_after_sync();
          const uint32_t base = umma::smem_u32(smem + s * SSTAGE_BYTES);
#pragma unroll
          for (int ks = 0; ks < SK / 16; ++ks) {
#pragma unroll
            for (int q = 0; q < 6; ++q) {
              const uint64_t ad = umma::smem_desc_sw64(base + pa[q] * SPLANE_BYTES + ks * 32);
              const uint64_t bd = umma::smem_desc_sw64(base + (3 + pb[q]) * SPLANE_BYTES + ks * 32);
              const uint32_t acc = (t > 0 || ks > 0 || q > 1) ? 1u : 0u;
              umma::mma_bf16(q == 0 ? acc0 : acc0 + 128, ad, bd, IDESC, acc);
            }
          }
          umma::commit(&sh->empty[s]);
        }
        if (ok) umma::commit(&sh->tfull[b]);
      }
      umma::commit(&sh->mdone);  // every MMA completes before the accumulators are freed
      umma::mbar_wait_bounded(&sh->mdone, 0, err);
    }
  } else {
    // Epilogue: warps 0-3, TMEM lane quarter = warp, one accumulator row per
    // thread.  Each 32-column slice is split into the three planes; a plane's
    // 32 × 32 BF16 block goes through this warp's staging rows so that every
    // store instruction writes eight whole 64-byte row segments (a quarter of
    // the L2 write requests of one 16-byte store per row).
    unsigned char* stage = smem + SNST * SSTAGE_BYTES + 256 + warp * EPI_WARP_BYTES;
    uint32_t j = 0;
    for (long long u = blockIdx.x; u < g.ntask; u += gridDim.x, ++j) {
      int r0, c0, kb, nk;
      pg_task(g, u, r0, c0, kb, nk);
      const int b = j & 1;
      if (!pg_wait(&sh->tfull[b], (j >> 1) & 1, err, abort)) break;
      umma::fence_after_sync();
      long long ro[4];
      bool live[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int grow = r0 + warp * 32 + k * 8 + (lane >> 2);
        live[k] = grow < out.rows.extent;
        ro[k] = live[k] ? row_off(out.rows, grow) : 0;
      }
      const uint32_t acc0 = tmem + (uint32_t)(b * 256);
      for (int cb = 0; cb < TN; cb += 32) {
        float v[32];
        if (nk > 0) {
          tile_ld32(acc0, warp, cb, v);
        } else {
#pragma unroll
          for (int q = 0; q < 32; ++q) v[q] = 0.f;
        }
        if (cb + 32 == TN) {  // every read of buffer b is complete: hand it back
          umma::fence_before_sync();
          __syncwarp();
          if (lane == 0) umma::mbar_arrive(&sh->tempty[b]);
        }
        uint32_t pk[3][16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          __nv_bfloat16 x[3], y[3];
          split3(v[2 * e], x[0], x[1], x[2]);
          split3(v[2 * e + 1], y[0], y[1], y[2]);
#pragma unroll
          for (int p = 0; p < 3; ++p) {
            __nv_bfloat162 t = __halves2bfloat162(x[p], y[p]);
            pk[p][e] = *reinterpret_cast<uint32_t*>(&t);
          }
        }
        const int gcol = c0 + cb + (lane & 3) * 8;
        const bool col_ok = gcol < out.col_extent;
        const long long co = (long long)(gcol / out.col_inner) * out.col_os +
                             (long long)(gcol % out.col_inner);
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          __syncwarp();  // the previous plane's reads of the staging rows are done
          uint4* mine = reinterpret_cast<uint4*>(stage + lane * EPI_ROW_BYTES);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            mine[q] = make_uint4(pk[p][4 * q], pk[p][4 * q + 1], pk[p][4 * q + 2], pk[p][4 * q + 3]);
          __syncwarp();
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int rr = k * 8 + (lane >> 2);
            if (live[k] && col_ok)
              *reinterpret_cast<uint4*>(out.plane[p] + ro[k] + co) =
                  *reinterpret_cast<const uint4*>(stage + rr * EPI_ROW_BYTES + (lane & 3) * 16);
          }
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
}

// S tile (ti, tj) = Σ_chunks of the FP32 partial tiles, in FP64 and in chunk
// order.  Four CTAs per tile, 32 rows each: every thread sums 16 elements of
// the row-major partials (coalesced reads, the 16 loads of a chunk in flight
// together), the 32 × 128 block is transposed through shared memory, and each
// warp writes 32 consecutive rows of one column of the column-major S.
__global__ void __launch_bounds__(256) k_reduce_partials(const float* partial, int ntri, int nchunk,
                                                         int m, double* S) {
  __shared__ double blk[TN][33];
  const int tri = blockIdx.x >> 2, r0 = (blockIdx.x & 3) * 32;
  int ti, tj;
  tri_index(tri, ti, tj);
  constexpr int PER = 32 * TN / 256;
  double acc[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) acc[k] = 0.0;
  const size_t tile = (size_t)TM * TN;
  const float* base = partial + (size_t)tri * tile + (size_t)r0 * TN;
  for (int ch = 0; ch < nchunk; ++ch) {
    const float* src = base + (size_t)ch * ntri * tile;
    float v[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) v[k] = src[threadIdx.x + k * 256];
#pragma unroll
    for (int k = 0; k < PER; ++k) acc[k] += (double)v[k];
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = threadIdx.x + k * 256, r = e / TN, c = e % TN;
    blk[c][r] = acc[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = threadIdx.x + k * 256, r = e & 31, c = e >> 5;
    const int gi = ti * TM + r0 + r, gj = tj * TN + c;
    if (gi < m && gj < m) S[gi + (size_t)gj * m] = blk[c][r];
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

// Rows of a column-major FP64 matrix (row r = column r of src, K entries,
// leading dimension ld) → planes[p][r·Kp + k], zeros for K ≤ k < Kp.
__global__ void k_split_rows(const double* __restrict__ src, long long ld, int rows, long long K,
                             long long Kp, __nv_bfloat16* P0, __nv_bfloat16* P1,
                             __nv_bfloat16* P2) {
  const long long tot = (long long)rows * Kp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / Kp, k = t - r * Kp;
    const double v = k < K ? src[r * ld + k] : 0.0;
    split3d(v, P0[t], P1[t], P2[t]);
  }
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
  kc = ((kc + 63) / 64) * 64;
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

// Tensor map of one plane: rows × kext BF16, row-major with a pitch of `pitch`
// elements; box 32 (K) × 128 (rows), 64-byte swizzle, zeros out of bounds.
static void encode_plane_map(CUtensorMap* map, const __nv_bfloat16* plane, long long rows,
                             long long kext, long long pitch) {
  if ((reinterpret_cast<uintptr_t>(plane) & 15) != 0 || (pitch * 2) % 16 != 0 || kext > pitch ||
      rows <= 0 || kext <= 0)
    throw std::invalid_argument("split GEMM: plane base or pitch not 16-byte aligned");
  cuuint64_t dims[2] = {(cuuint64_t)kext, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)pitch * 2};
  cuuint32_t box[2] = {(cuuint32_t)SK, (cuuint32_t)TM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = tensor_map_encoder()(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                                    const_cast<__nv_bfloat16*>(plane), dims, strides, box, estr,
                                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

void split_gemm_planes(const Plane2D& A, const Plane2D& B, int Ktot, const OutMap& out, int kmode,
                       int* err, cudaStream_t st) {
  if (out.rows.extent <= 0 || out.col_extent <= 0 || Ktot <= 0) return;
  TmaMaps maps;
  for (int p = 0; p < 3; ++p) {
    encode_plane_map(&maps.a[p], A.plane[p], A.rows, Ktot, A.pitch);
    encode_plane_map(&maps.b[p], B.plane[p], B.rows, Ktot, B.pitch);
  }
  ensure_smem(k_split_gemm_persistent, PG_SMEM_BYTES);
  PGemmTiles g;
  g.ta = ceil_div(out.rows.extent, TM);
  g.tb = ceil_div(out.col_extent, TN);
  g.a_fast = g.ta < g.tb ? 1 : 0;
  g.kmode = kmode;
  g.Ktot = Ktot;
  g.ntask = (long long)g.ta * g.tb;
  int dev = 0, sms = 148;
  SDPX_CUDA(cudaGetDevice(&dev));
  SDPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const long long grid = std::min<long long>(g.ntask, sms);
  k_split_gemm_persistent<<<(unsigned)grid, PG_THREADS, PG_SMEM_BYTES, st>>>(maps, out, g, err);
  SDPX_LAUNCH_CHECK();
}

void split_syrk(const Plane2D& P, int m, int Kp, const SplitSyrkPlan& plan, float* partial,
                double* S, int* err, cudaStream_t st, cudaEvent_t ev_begin, cudaEvent_t ev_end) {
  if (P.pitch != Kp || Kp % SK != 0 || plan.kchunk % SK != 0)
    throw std::invalid_argument("split SYRK: planes must be m × Kp row-major, Kp and chunks ≡ 0 mod 32");
  TmaMaps maps;
  for (int p = 0; p < 3; ++p) {
    encode_plane_map(&maps.a[p], P.plane[p], m, Kp, Kp);
    maps.b[p] = maps.a[p];
  }
  ensure_smem(k_split_syrk_tma, SSMEM_BYTES);
  const int units = plan.ntri * plan.nchunk;
  if (ev_begin) SDPX_CUDA(cudaEventRecord(ev_begin, st));
  k_split_syrk_tma<<<units, NTHREADS, SSMEM_BYTES, st>>>(maps, plan.ntri, plan.kchunk, Kp, partial,
                                                        err);
  if (ev_end) SDPX_CUDA(cudaEventRecord(ev_end, st));
  k_reduce_partials<<<plan.ntri * 4, 256, 0, st>>>(partial, plan.ntri, plan.nchunk, m, S);
  SDPX_LAUNCH_CHECK_N(2);
}

void split_rows_f64(const double* src, long long ld, int rows, long long K, long long Kp,
                    __nv_bfloat16* const* planes, cudaStream_t st) {
  const long long tot = (long long)rows * Kp;
  if (tot == 0) return;
  k_split_rows<<<(int)std::min<long long>(ceil_div(tot, 256), 148LL * 32), 256, 0, st>>>(
      src, ld, rows, K, Kp, planes[0], planes[1], planes[2]);
  SDPX_LAUNCH_CHECK();
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
