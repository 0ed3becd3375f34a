// FP64 dense kernels on the DMMA tile engine: general GEMM with triangular
// K ranges, in-place right multiplication by a lower-triangular factor, and
// the split-K lower SYRK that assembles the Schur complement S = P̂ᵀP̂.
#include "blas_f64.h"
#include "gemm_f64.cuh"

#include <atomic>
#include <mutex>
#include <stdexcept>

namespace sdpx {

// Tile configurations.  128×128 / 8 warps for the large Schur products,
// 64×64 / 4 warps for per-block k×k products.
using CfgBigKT = F64Cfg<128, 128, 2, 4, true, true>;    // SYRK: both operands K-contiguous
using CfgBigMK = F64Cfg<128, 128, 2, 4, false, true>;   // A MN-contiguous, B K-contiguous
using CfgSmMK = F64Cfg<64, 64, 2, 2, false, true>;
using CfgSmKK = F64Cfg<64, 64, 2, 2, true, true>;
using CfgSmMM = F64Cfg<64, 64, 2, 2, false, false>;
using CfgSmKM = F64Cfg<64, 64, 2, 2, true, false>;
// 32×32 / 4 warps when the 64×64 grid would not fill the GPU (the k×k block
// products of the Newton step: 400×400 is 49 tiles of 64 but 169 of 32).
using CfgTnMK = F64Cfg<32, 32, 2, 2, false, true>;
using CfgTnKK = F64Cfg<32, 32, 2, 2, true, true>;
using CfgTnMM = F64Cfg<32, 32, 2, 2, false, false>;
using CfgTnKM = F64Cfg<32, 32, 2, 2, true, false>;

// Grid: the fast index runs over the dimension with fewer tiles (rows_fast: x
// over row tiles), so CTAs sharing a tile of the larger operand run together.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) k_gemm(Opnd A, Opnd B, OutDesc C, double alpha,
                                                  double beta, int mode, int rows_fast) {
  extern __shared__ __align__(16) double smem[];
  const int n0 = (rows_fast ? blockIdx.y : blockIdx.x) * Cfg::BN;
  const int m0 = (rows_fast ? blockIdx.x : blockIdx.y) * Cfg::BM;
  int kb, ke;
  k_limits(mode, A.k_extent, m0, n0, Cfg::BM, Cfg::BN, kb, ke);
  double acc[Cfg::FM][Cfg::FN][2];
  zero_acc<Cfg>(acc);
  f64_tile_mainloop<Cfg>(acc, A, B, m0, n0, kb, ke, smem);
  store_acc<Cfg>(acc, C, m0, n0, alpha, beta);
}

// Grouped products: CTA b belongs to the group whose tile range holds it
// (first[g] ≤ b < first[g+1]); within a group the row tiles run fastest.
struct GemmGroupsDev {
  GemmGroups g;
  int first[kGemmGroups + 1], tr[kGemmGroups];
};
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) k_gemm_grouped(const __grid_constant__ GemmGroupsDev d) {
  extern __shared__ __align__(16) double smem[];
  int q = 0;
  while (q + 1 < d.g.n && (int)blockIdx.x >= d.first[q + 1]) ++q;
  const int t = (int)blockIdx.x - d.first[q];
  const int m0 = (t % d.tr[q]) * Cfg::BM, n0 = (t / d.tr[q]) * Cfg::BN;
  const Opnd A = d.g.A[q], B = d.g.B[q];
  int kb, ke;
  k_limits(d.g.mode[q], A.k_extent, m0, n0, Cfg::BM, Cfg::BN, kb, ke);
  double acc[Cfg::FM][Cfg::FN][2];
  zero_acc<Cfg>(acc);
  f64_tile_mainloop<Cfg>(acc, A, B, m0, n0, kb, ke, smem);
  store_acc<Cfg>(acc, d.g.C[q], m0, n0, d.g.alpha[q], d.g.beta[q]);
}

// In-place  T ← T · L  for a lower-triangular L (k×k, explicit zeros above the
// diagonal).  One CTA owns BM consecutive rows of T and sweeps the output
// column tiles left to right; output tile [n0, n0+BN) reads only columns ≥ n0,
// which this CTA has not yet overwritten, so the update is race free.
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) k_trmm_right_lower_inplace(Opnd T, Opnd L, OutDesc C) {
  extern __shared__ __align__(16) double smem[];
  const int m0 = blockIdx.x * Cfg::BM;
  const int K = L.k_extent;
  for (int n0 = 0; n0 < C.cols; n0 += Cfg::BN) {
    double acc[Cfg::FM][Cfg::FN][2];
    zero_acc<Cfg>(acc);
    f64_tile_mainloop<Cfg>(acc, T, L, m0, n0, n0, K, smem);
    __syncthreads();
    store_acc<Cfg>(acc, C, m0, n0, 1.0, 0.0);
    __syncthreads();
  }
}

// Split-K lower SYRK.  Work unit u = chunk * ntri + tri (chunk-major, so CTAs
// resident at the same time share one K slab of the panel in L2).  Each unit
// writes its BM×BN partial tile to `partial` (column-major inside the tile);
// `k_syrk_reduce` sums the chunks in a fixed order (bitwise reproducible).
template <class Cfg>
__global__ void __launch_bounds__(Cfg::NT) k_syrk_splitk(Opnd P, int ntri, int kchunk,
                                                          double* partial) {
  extern __shared__ __align__(16) double smem[];
  const int u = blockIdx.x;
  const int chunk = u / ntri, tri = u % ntri;
  int ti = (int)((sqrt(8.0 * tri + 1.0) - 1.0) * 0.5);
  while ((ti + 1) * (ti + 2) / 2 <= tri) ++ti;
  while (ti * (ti + 1) / 2 > tri) --ti;
  const int tj = tri - ti * (ti + 1) / 2;
  const int kb = chunk * kchunk;
  const int ke = min(P.k_extent, kb + kchunk);
  double acc[Cfg::FM][Cfg::FN][2];
  zero_acc<Cfg>(acc);
  f64_tile_mainloop<Cfg>(acc, P, P, ti * Cfg::BM, tj * Cfg::BN, kb, ke, smem);
  double* out = partial + (size_t)u * Cfg::BM * Cfg::BN;
  for_each_acc<Cfg>(acc, [&](int r, int c, double v) { out[c * Cfg::BM + r] = v; });
}

template <int BM, int BN>
__global__ void k_syrk_reduce(const double* partial, int ntri, int nchunk, int m, double* S,
                              long long lds, double beta) {
  const int tri = blockIdx.x;
  int ti = (int)((sqrt(8.0 * tri + 1.0) - 1.0) * 0.5);
  while ((ti + 1) * (ti + 2) / 2 <= tri) ++ti;
  while (ti * (ti + 1) / 2 > tri) --ti;
  const int tj = tri - ti * (ti + 1) / 2;
  for (int e = threadIdx.x; e < BM * BN; e += blockDim.x) {
    int r = e % BM, c = e / BM;
    int gi = ti * BM + r, gj = tj * BN + c;
    if (gi >= m || gj >= m) continue;
    double s = 0.0;
    for (int ch = 0; ch < nchunk; ++ch) s += partial[((size_t)ch * ntri + tri) * BM * BN + e];
    double* p = S + gi + (long long)gj * lds;
    *p = (beta == 0.0) ? s : s + beta * (*p);
  }
}

// SM count of the current device (cached per device).
static int gemm_sm_count() {
  static std::atomic<int> cached[64];
  int dev = 0;
  SDPX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return 148;
  int v = cached[dev].load(std::memory_order_relaxed);
  if (v == 0) {
    SDPX_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    if (v <= 0) v = 148;
    cached[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

template <class Cfg>
static void launch_gemm_cfg(const Opnd& A, const Opnd& B, const OutDesc& C, double alpha,
                            double beta, int mode, cudaStream_t st) {
  ensure_smem(k_gemm<Cfg>, Cfg::SMEM_BYTES);
  const int tr = ceil_div(C.rows, Cfg::BM), tc = ceil_div(C.cols, Cfg::BN);
  if (tr == 0 || tc == 0) return;
  const int rows_fast = (tr < tc && tc <= 65535) ? 1 : 0;  // grid.y is limited to 65535
  if (!rows_fast && tr > 65535) throw std::invalid_argument("gemm_f64: too many row tiles");
  dim3 grid(rows_fast ? tr : tc, rows_fast ? tc : tr);
  k_gemm<Cfg><<<grid, Cfg::NT, Cfg::SMEM_BYTES, st>>>(A, B, C, alpha, beta, mode, rows_fast);
  SDPX_LAUNCH_CHECK();
}

template <class Cfg>
static void launch_gemm_grouped(const GemmGroups& g, cudaStream_t st) {
  ensure_smem(k_gemm_grouped<Cfg>, Cfg::SMEM_BYTES);
  GemmGroupsDev d;
  d.g = g;
  int total = 0;
  for (int q = 0; q < g.n; ++q) {
    d.first[q] = total;
    d.tr[q] = ceil_div(g.C[q].rows, Cfg::BM);
    total += d.tr[q] * ceil_div(g.C[q].cols, Cfg::BN);
  }
  d.first[g.n] = total;
  if (total == 0) return;
  k_gemm_grouped<Cfg><<<total, Cfg::NT, Cfg::SMEM_BYTES, st>>>(d);
  SDPX_LAUNCH_CHECK();
}

void gemm_f64_grouped(const GemmGroups& g, bool a_kcontig, bool b_kcontig, cudaStream_t st) {
  if (g.n <= 0) return;
  if (g.n > kGemmGroups) throw std::invalid_argument("gemm_f64_grouped: too many groups");
  // the rule gemm_f64 applies to one product, applied to each of them: 32×32
  // tiles when every product alone would take them
  bool tiny = true;
  for (int q = 0; q < g.n; ++q)
    tiny = tiny && (long long)ceil_div(g.C[q].rows, 64) * ceil_div(g.C[q].cols, 64) < gemm_sm_count();
  if (!tiny) {  // mixed shapes: one launch per product, as gemm_f64
    for (int q = 0; q < g.n; ++q)
      gemm_f64(g.A[q], a_kcontig, g.B[q], b_kcontig, g.C[q], g.alpha[q], g.beta[q], g.mode[q], false,
               st);
    return;
  }
  if (!a_kcontig && b_kcontig) return launch_gemm_grouped<CfgTnMK>(g, st);
  if (a_kcontig && b_kcontig) return launch_gemm_grouped<CfgTnKK>(g, st);
  if (!a_kcontig && !b_kcontig) return launch_gemm_grouped<CfgTnMM>(g, st);
  return launch_gemm_grouped<CfgTnKM>(g, st);
}

void gemm_f64(const Opnd& A, bool a_kcontig, const Opnd& B, bool b_kcontig, const OutDesc& C,
              double alpha, double beta, int mode, bool big, cudaStream_t st) {
  if (big && !a_kcontig && b_kcontig) return launch_gemm_cfg<CfgBigMK>(A, B, C, alpha, beta, mode, st);
  if (big && a_kcontig && b_kcontig) return launch_gemm_cfg<CfgBigKT>(A, B, C, alpha, beta, mode, st);
  if (!big && (long long)ceil_div(C.rows, 64) * ceil_div(C.cols, 64) < gemm_sm_count()) {
    if (!a_kcontig && b_kcontig) return launch_gemm_cfg<CfgTnMK>(A, B, C, alpha, beta, mode, st);
    if (a_kcontig && b_kcontig) return launch_gemm_cfg<CfgTnKK>(A, B, C, alpha, beta, mode, st);
    if (!a_kcontig && !b_kcontig) return launch_gemm_cfg<CfgTnMM>(A, B, C, alpha, beta, mode, st);
    return launch_gemm_cfg<CfgTnKM>(A, B, C, alpha, beta, mode, st);
  }
  if (!a_kcontig && b_kcontig) return launch_gemm_cfg<CfgSmMK>(A, B, C, alpha, beta, mode, st);
  if (a_kcontig && b_kcontig) return launch_gemm_cfg<CfgSmKK>(A, B, C, alpha, beta, mode, st);
  if (!a_kcontig && !b_kcontig) return launch_gemm_cfg<CfgSmMM>(A, B, C, alpha, beta, mode, st);
  return launch_gemm_cfg<CfgSmKM>(A, B, C, alpha, beta, mode, st);
}

void trmm_right_lower_inplace_f64(const Opnd& T, const Opnd& L, const OutDesc& C, cudaStream_t st) {
  using Cfg = CfgBigMK;
  ensure_smem(k_trmm_right_lower_inplace<Cfg>, Cfg::SMEM_BYTES);
  int grid = ceil_div(C.rows, Cfg::BM);
  if (grid == 0) return;
  k_trmm_right_lower_inplace<Cfg><<<grid, Cfg::NT, Cfg::SMEM_BYTES, st>>>(T, L, C);
  SDPX_LAUNCH_CHECK();
}

SyrkPlan plan_syrk_f64(int m, long long K, int sm_count) {
  SyrkPlan p;
  p.bm = CfgBigKT::BM;
  int nt = ceil_div(m, p.bm);
  p.ntri = nt * (nt + 1) / 2;
  // Choose the number of K chunks so the unit count fills whole waves of one
  // CTA per SM, with at least 256 rows of K per chunk.
  int best_c = 1;
  double best_eff = 0.0;
  long long max_c = K / 256;
  if (max_c < 1) max_c = 1;
  if (max_c > 16) max_c = 16;
  for (int c = 1; c <= max_c; ++c) {
    long long units = (long long)p.ntri * c;
    double waves = (double)units / sm_count;
    double eff = waves / std::ceil(waves);
    // Prefer more work per wave up to ~4 waves; past that, only efficiency counts.
    double score = eff * std::min(1.0, waves / 4.0);
    if (score > best_eff + 1e-9) {
      best_eff = score;
      best_c = c;
    }
  }
  long long kc = (K + best_c - 1) / best_c;
  kc = ((kc + 15) / 16) * 16;
  p.kchunk = (int)kc;
  p.nchunk = (int)((K + kc - 1) / kc);
  p.partial_doubles = (size_t)p.nchunk * p.ntri * p.bm * p.bm;
  return p;
}

void syrk_lower_f64(const Opnd& P, const SyrkPlan& plan, double* partial, double* S, long long lds,
                    int m, double beta, cudaStream_t st) {
  using Cfg = CfgBigKT;
  ensure_smem(k_syrk_splitk<Cfg>, Cfg::SMEM_BYTES);
  int units = plan.ntri * plan.nchunk;
  k_syrk_splitk<Cfg><<<units, Cfg::NT, Cfg::SMEM_BYTES, st>>>(P, plan.ntri, plan.kchunk, partial);
  SDPX_LAUNCH_CHECK();
  k_syrk_reduce<Cfg::BM, Cfg::BN><<<plan.ntri, 256, 0, st>>>(partial, plan.ntri, plan.nchunk, m, S,
                                                             lds, beta);
  SDPX_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the split-K lower Gram product S = PᵀP.
//
// The split-K partial tiles live in a fixed file-scope device array instead of
// caller- or library-allocated memory.  One K chunk of every lower 128×128 tile
// must fit (ntri·128·128 doubles, ntri = t(t+1)/2, t = ceil(m/128)): the stated
// limit m ≤ 2048 (t = 16, 2.2 Mi doubles) leaves room for a second chunk.  K is
// bounded by the int32 K indexing of the tile loop: chunk starts plus a chunk
// length must stay below 2³¹, which K ≤ 2³⁰ guarantees.  Every GPU that loads
// the library holds the array until the process exits, and all calls share it.
// ---------------------------------------------------------------------------
static constexpr size_t kNoAllocScratchDoubles = (size_t)4 << 20;  // 32 MiB
static constexpr int kNoAllocMaxM = 2048;
static constexpr long long kNoAllocMaxK = 1LL << 30;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[64] = {};

// Device address of the scratch array on the current device.  The array's
// host-side name is only a stand-in, so the address is looked up once per
// device with that device current and cached; a failed lookup is reported.
static double* noalloc_scratch_address() {
  int dev = 0;
  SDPX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw std::runtime_error("device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw CudaError(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  return g_noalloc_ptr[dev];
}

size_t gram_noalloc_capacity_doubles() { return kNoAllocScratchDoubles; }

void syrk_lower_f64_noalloc(const double* P, long long K, int m, double* S, cudaStream_t st) {
  using Cfg = CfgBigKT;
  const int nt = ceil_div(m, Cfg::BM);
  const long long ntri = (long long)nt * (nt + 1) / 2;
  const long long tile = (long long)Cfg::BM * Cfg::BN;
  if (m <= 0 || K <= 0) throw std::invalid_argument("gram: m and K must be positive");
  if (m > kNoAllocMaxM)
    throw std::invalid_argument("gram (allocation-free): m = " + std::to_string(m) +
                                " exceeds the fixed scratch (m ≤ 2048)");
  if (K > kNoAllocMaxK)
    throw std::invalid_argument("gram (allocation-free): K = " + std::to_string(K) +
                                " exceeds the int32 K indexing (K ≤ 2^30)");
  if (ntri * tile > (long long)kNoAllocScratchDoubles)
    throw std::logic_error("gram (allocation-free): scratch smaller than one chunk");
  double* scratch = noalloc_scratch_address();
  int dev = 0, sms = 148;
  SDPX_CUDA(cudaGetDevice(&dev));
  SDPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // As many K chunks as the scratch holds, capped by the normal plan.
  SyrkPlan plan = plan_syrk_f64(m, K, sms);
  long long max_chunks = (long long)kNoAllocScratchDoubles / (ntri * tile);
  int nchunk = (int)std::max<long long>(1, std::min<long long>(plan.nchunk, max_chunks));
  long long kc = (K + nchunk - 1) / nchunk;
  kc = ((kc + 15) / 16) * 16;
  plan.kchunk = (int)kc;
  plan.nchunk = (int)((K + kc - 1) / kc);
  Opnd Pd;
  Pd.base = P;
  Pd.kstride = 1;
  Pd.inner = 1 << 30;
  Pd.inner_stride = K;
  Pd.outer_stride = 0;
  Pd.mn_extent = m;
  Pd.k_extent = (int)K;
  syrk_lower_f64(Pd, plan, scratch, S, m, m, 0.0, st);
}

}  // namespace sdpx
