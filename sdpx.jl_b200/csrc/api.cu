// C ABI of the SDPX B200 core: handle lifecycle, device-resident workspace and
// the hot-path operations of one Newton iteration.  See include/sdpx_b200.h.
//
// Device layout.  All blocks share one "stacked" row space of length K: dense
// blocks (k ≥ 2) occupy k² consecutive rows each (column-major k×k), followed
// by one row per 1×1 block.  The constraint matrix 𝒜 is K×m column-major, so
// column i holds vec(A_i) of every block contiguously; every block matrix
// (X, Y, C, P, R, Z, dX, dY, factors) is a K-vector with the same offsets.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <deque>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "../../include/sdpx_b200.h"
#include "blas_f64.h"
#include "certificate.h"
#include "chol.h"
#include "dbuf.h"
#include "equality.h"
#include "sparse_schur.h"
#include "dd_kernels.h"
#include "mixed.h"
#include "ozaki.h"
#include "schur_bf16.h"
#include "vec_kernels.h"

namespace sdpx {

static std::atomic<unsigned long long> g_launches{0};
void note_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(); }

static std::mutex g_attr_mu;
static std::map<std::pair<const void*, int>, size_t> g_attr_done;
// True when `kern` on the current device has not yet been opted in to at
// least `bytes` of dynamic shared memory (records the new size).
// Raises the kernel's dynamic shared-memory limit on the current device once.
// The attribute is set while the lock is held, so a concurrent caller never
// sees the kernel recorded before the attribute is in place.
void smem_attr_ensure(const void* kern, size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_attr_mu);
  size_t& have = g_attr_done[{kern, dev}];
  if (have >= bytes) return;
  SDPX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  have = bytes;
}


struct DenseBlk {
  int user;
  int k;
  long long off;  // stacked row offset
};

static constexpr double kEps = 2.220446049250313e-16;
static const double kSqrtEps = std::sqrt(2.220446049250313e-16);
int mixed_steps_for(double cond);  // mixed_api.inc

struct Handle {
  dcache::ReleaseScope release_scope;  // first member: destroyed after every buffer
  int dev = 0;
  cudaStream_t st = nullptr;
  int sms = 148;
  std::string err;
  int precision = SDPX_B200_FP64;

  int m = 0, L = 0;
  std::vector<int> k;              // user block orders
  std::vector<long long> user_off; // offset of block l in the host stacked layout
  long long Ku = 0;                // host stacked length Σ k_l²
  std::vector<DenseBlk> dense;
  int nd = 0;                      // number of 1×1 blocks
  long long od = 0;                // stacked offset of the 1×1 group
  std::vector<int> diag_user;      // user index of each 1×1 entry
  long long K = 0;                 // stacked length
  int kmax = 0;

  // device metadata
  DBuf<long long> d_map;           // internal stacked index → host stacked index
  DBuf<long long> d_doff, d_dlen;  // dense block offsets / lengths (k²)
  DBuf<int> d_dk;                  // dense block orders
  DBuf<long long> d_uoff, d_ulen;  // per-user-block segments (internal offsets) for dots
  DBuf<int> d_uk;                  // user block orders
  DBuf<int> d_diag_user;
  std::vector<long long> seg_off, seg_len;  // host copies (user order, internal offsets)

  // problem data
  DBuf<double> A, A0, Pc;          // K×m
  DBuf<double> c, c0;
  DBuf<double> Cst, C0st;          // stacked C
  bool have_original = false;

  // iterate and workspaces
  DBuf<double> x, dx, d, v, r, rho, work_m, work_m2, xbest, keptx, dxbest;
  DBuf<double> X, Y, P, R, Z, dX, dY, LX, MY, W, T1, T2, Xbest, Ybest, tmpK, tmpK2;
  DBuf<double> gemv_part;
  int gemv_chunks = 8;
  // Lower-triangle copy of 𝒜 for the memory-bound operator passes (𝒜v and
  // 𝒜ᵀz read half the bytes): every dense A_i keeps its entries p ≥ c, column
  // by column, the 1×1 group follows.  ap_lo[q] / ap_up[q] are the stacked rows
  // of (p, c) and (c, p), equal on the diagonal and in the 1×1 group.  a_ver
  // counts changes of 𝒜 (equilibration, reset); the copy is rebuilt when stale.
  DBuf<double> Ap, kt_fold;
  DBuf<long long> ap_lo, ap_up;
  long long Kt = 0;
  unsigned long long a_ver = 1, ap_ver = 0;
  // adx = 𝒜·dx of the dx version adx_ver (the mixed operator computes it; the
  // block directions reuse it when dx has not changed since).
  DBuf<double> adx;
  unsigned long long dx_ver = 1, adx_ver = 0;
  void a_changed() {
    ++a_ver;
    adx_ver = 0;
  }
  void dx_written() { ++dx_ver; }
  void restore_dx_best() {  // the last accepted direction (dx, and dy with equality rows)
    d2d(dx.p, dxbest.p, m * sizeof(double));
    if (n_eq) d2d(dyv.p, dybest.p, n_eq * sizeof(double));
    dx_written();
  }
  bool use_packed = true;  // false when the copy did not fit: passes read 𝒜 itself
  void amul(const double* xv, double* out) {  // out = 𝒜·xv (stacked, symmetric blocks)
    if (!use_packed) return gemv_n(A.p, K, m, xv, out, gemv_part.p, gemv_chunks, st);
    ensure_packed();
    gemv_n_sym(Ap.p, Kt, m, xv, ap_lo.p, ap_up.p, out, gemv_part.p, gemv_chunks, st);
  }
  // out = alpha·𝒜ᵀz + beta·base; z need not be symmetric (⟨A_i, Z⟩ = ⟨A_i, sym Z⟩).
  void atmul(const double* z, double alpha, const double* base, double beta, double* out) {
    if (!use_packed) return gemv_t(A.p, K, m, z, alpha, base, beta, out, st);
    ensure_packed();
    fold_sym(Kt, z, ap_lo.p, ap_up.p, kt_fold.p, st);
    gemv_t(Ap.p, Kt, m, kt_fold.p, alpha, base, beta, out, st);
  }
  // The residuals P = 𝒜x − X − C and d = c − 𝒜ᵀY with every entry rounded
  // once from compensated (Dot2) sums: near convergence they sit at the
  // rounding floor, where the controller's centring test compares them, and
  // this makes them independent of the device's summation order.
  void primal_residual(const double* xv, double* out) {
    if (!use_packed)
      return gemv_n_acc(A.p, K, m, xv, X.p, Cst.p, out, gemv_part.p, gemv_chunks, st);
    ensure_packed();
    gemv_n_sym_acc(Ap.p, Kt, m, xv, ap_lo.p, ap_up.p, X.p, Cst.p, out, gemv_part.p, gemv_chunks,
                   st);
  }
  void dual_residual(const double* Yv, double* out) {
    if (!use_packed) return gemv_t_acc(A.p, K, m, Yv, -1.0, c.p, 1.0, out, st);
    ensure_packed();
    fold_sym(Kt, Yv, ap_lo.p, ap_up.p, kt_fold.p, st);
    gemv_t_acc(Ap.p, Kt, m, kt_fold.p, -1.0, c.p, 1.0, out, st);
  }
  void ensure_packed() {
    if (ap_ver == a_ver) return;
    pack_rows(A.p, K, m, ap_lo.p, Kt, Ap.p, st);
    ap_ver = a_ver;
  }
  void adx_current() {  // adx ← 𝒜·dx unless it already holds it
    if (adx_ver == dx_ver) return;
    amul(dx.p, adx.p);
    adx_ver = dx_ver;
  }
  DBuf<double> S, Sf, Dinv;
  DBuf<double> Linv, tmp_mm;       // explicit inverse of the FP64 factor, its scratch
  // FP64 Gram engine of the Schur SYRK: 0 = FP64 DMMA tiles, 1 = exact int8
  // digit products (48-bit digits, int32 accumulation, FP64 level sums).
  int gram_engine = 1;
  // Sparse Schur engine (SDPX's SparseCons path): per dense block the active
  // variables (ascending) and their flat coordinate entries, rebuilt from 𝒜
  // when 𝒜 changes; the 1×1 group keeps its rank-nd Gram on the FP64 tiles.
  bool sparse_schur = false;
  unsigned long long coo_ver = 0;
  std::vector<int> sp_na;
  std::vector<long long> sp_act_off;
  long long sp_active = 0, sp_nnz = 0;
  DBuf<int> sp_cnt, sp_ids, sp_lin;
  DBuf<long long> sp_ptr;
  DBuf<double> sp_val, Xinv, diag_partial;
  SyrkPlan diag_syrk{};
  OzakiPlan oz_plan;
  DBuf<int8_t> oz_digits;
  DBuf<int> oz_exps, oz_err;
  DBuf<double> oz_partial;
  // FP64 block products on the same digit engine: T_i = W·A_i is written
  // row-major into Pc's block region, its rows are cut into digits and
  // P_i = T_i·M_Y overwrites the region column-major (the Gram's layout).  The
  // digits of the constraint matrices are cut once per version of 𝒜.
  struct OzBlock {
    long long kp = 0;
    size_t dig_off = 0;
    long long exp_off = 0;
  };
  std::vector<OzBlock> ozb;
  DBuf<int8_t> oz_adig, oz_tdig, oz_wdig;
  DBuf<int> oz_aexp, oz_texp, oz_wexp;
  DBuf<unsigned> oz_colmax;  // per Schur column: largest high word of |P| over the dense rows
  unsigned long long oz_a_ver = 0;
  int oz_blk_state = 0;  // 0 = not planned, 1 = digit products, -1 = DMMA tiles (memory)
  DBuf<double> partial;
  SyrkPlan syrk;
  DBuf<double> red;                // small reduction scratch
  double* h_red = nullptr;         // pinned mirror
  DBuf<double> mu_user, target_user, work_L;
  DBuf<double> seg_part;           // seg_dot partials
  int seg_parts = 8;
  double last_bpr = 0.0;
  int mixed_predicted_steps = 32;  // from the last FP32 factor's condition estimate
  long long mixed_guard_steps = 0;
  long long operator_applications = 0;  // matrix-free FP64 Newton operator (mixed mode)
  long long schur_builds = 0;
  // The current S is the identity-metric S = 𝒜ᵀ𝒜 of the KKT cold start (so
  // the matrix-free operator of the mixed guard is 𝒜ᵀ𝒜, and an FP64 rebuild
  // must rebuild that same matrix).
  bool identity_metric = false;
  int mixed_fallbacks = 0;

  // batched Cholesky workspace (dense blocks X, Y and line-search trials)
  DBuf<MatDesc<double>> d_descs;
  DBuf<int> d_info;
  DBuf<unsigned> coop_bar;  // grid-barrier state of the single-launch Schur Cholesky
  DBuf<double> d_dmin, d_dmax;
  size_t desc_cap = 0;
  DBuf<double> trials;
  DBuf<long long> d_trial_off;
  DBuf<double> d_tcand;
  DBuf<TrialDesc> d_trial_desc;
  DBuf<int> d_fail;
  std::vector<double> lx_dmin, lx_dmax, my_dmin, my_dmax;
  bool diag_factor_ok = true;

  // Gershgorin scratch
  DBuf<double> g_cand, g_scale;
  DBuf<double> cert_part, cert_rows, cert_cols, cert_sym, cert_stats, cert_shift;
  DBuf<long long> g_cand_off;
  DBuf<int> g_nonfinite;

  // mixed precision state
  std::unique_ptr<MixedWorkspace> mixed;

  // phase timing
  struct PendingEv {
    int phase;
    cudaEvent_t a, b;
  };
  std::vector<PendingEv> pending;
  std::vector<cudaEvent_t> ev_pool;
  double phase_ms[7] = {0, 0, 0, 0, 0, 0, 0};

  // Last device duration (ms) of the Schur kernels: [0] split-BF16 SYRK kernel,
  // [1] split-BF16 block products (all blocks), [2] FP64 SYRK (split-K kernel and
  // reduction), [3] FP64 block products (all blocks).
  cudaEvent_t kt_ev[4][2] = {};
  bool kt_armed[4] = {};
  double kt_ms[4] = {0, 0, 0, 0};
  void kt_create(int k) {
    for (int j = 0; j < 2; ++j)
      if (!kt_ev[k][j]) SDPX_CUDA(cudaEventCreate(&kt_ev[k][j]));
  }
  void kt_begin(int k) {
    kt_create(k);
    SDPX_CUDA(cudaEventRecord(kt_ev[k][0], st));
  }
  void kt_end(int k) {
    SDPX_CUDA(cudaEventRecord(kt_ev[k][1], st));
    kt_armed[k] = true;
  }
  void kt_harvest() {
    for (int k = 0; k < 4; ++k) {
      if (!kt_armed[k]) continue;
      float ms = 0.f;
      SDPX_CUDA(cudaEventSynchronize(kt_ev[k][1]));
      SDPX_CUDA(cudaEventElapsedTime(&ms, kt_ev[k][0], kt_ev[k][1]));
      kt_ms[k] = ms;
      kt_armed[k] = false;
    }
  }

  ~Handle() {
    // All of the handle's device work runs on st: once st is idle its buffers
    // can return to the cache without a device-wide synchronisation.
    if (st && cudaStreamSynchronize(st) == cudaSuccess) release_scope.begin();
    for (auto& row : kt_ev)
      for (auto e : row)
        if (e) cudaEventDestroy(e);
    for (auto& p : pending) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    for (auto e : ev_pool) cudaEventDestroy(e);
    if (h_red) cudaFreeHost(h_red);
    if (h_pin) cudaFreeHost(h_pin);
    mixed.reset();
    if (st) cudaStreamDestroy(st);
  }

  // ---------------------------------------------------------------- utils --
  cudaEvent_t get_event() {
    if (!ev_pool.empty()) {
      cudaEvent_t e = ev_pool.back();
      ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    SDPX_CUDA(cudaEventCreate(&e));
    return e;
  }
  struct PhaseScope {
    Handle* h;
    int phase;
    cudaEvent_t a;
    PhaseScope(Handle* hh, int ph) : h(hh), phase(ph) {
      a = h->get_event();
      SDPX_CUDA(cudaEventRecord(a, h->st));
    }
    ~PhaseScope() {
      cudaEvent_t b = h->get_event();
      cudaEventRecord(b, h->st);
      h->pending.push_back({phase, a, b});
    }
  };
  void harvest_phases() {
    for (auto& p : pending) {
      float ms = 0.f;
      if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess)
        phase_ms[p.phase] += ms;
      ev_pool.push_back(p.a);
      ev_pool.push_back(p.b);
    }
    pending.clear();
  }

  void sync() { SDPX_CUDA(cudaStreamSynchronize(st)); }

  // Residual reuse across consecutive C-ABI calls.  Every entry point bumps
  // call_seq; a call that leaves ρ = r − S·dx consistent with dx records
  // rho_seq = call_seq and the norm.  Only the very next call, and only the
  // refinement and the acceptance-gate residual, may take that norm instead of
  // applying the operator again (the operator is deterministic, so the value is
  // identical).
  unsigned long long call_seq = 0, rho_seq = ~0ull;
  double rho_norm = 0.0;
  void mark_rho_fresh(double norm) {
    rho_seq = call_seq;
    rho_norm = norm;
  }
  bool take_rho_cache(double* norm) {
    bool hit = rho_seq + 1 == call_seq;
    rho_seq = ~0ull;
    if (hit) *norm = rho_norm;
    return hit;
  }
  void d2h(void* dst, const void* src, size_t bytes) {
    SDPX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
  }
  void h2d(void* dst, const void* src, size_t bytes) {
    SDPX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
  }
  void d2d(void* dst, const void* src, size_t bytes) {
    SDPX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st));
  }
  double read_red(int slot) {
    d2h(h_red + slot, red.p + slot, sizeof(double));
    sync();
    return h_red[slot];
  }
  void clear_red(int slot, int count = 1) {
    SDPX_CUDA(cudaMemsetAsync(red.p + slot, 0, sizeof(double) * count, st));
  }

  // Operand descriptors for a dense block matrix M stored at stacked offset o.
  static Opnd blk_as_A(const double* base, long long o, int kk) {  // (mm=r, kk=c) → M[r,c]
    Opnd q;
    q.base = base + o;
    q.kstride = kk;
    q.inner_stride = 1;
    q.outer_stride = 0;
    q.inner = 1 << 30;
    q.mn_extent = kk;
    q.k_extent = kk;
    return q;
  }
  static Opnd blk_as_At(const double* base, long long o, int kk) {  // (mm=r, kk=c) → M[c,r]
    Opnd q = blk_as_A(base, o, kk);
    q.kstride = 1;
    q.inner_stride = kk;
    return q;
  }
  static Opnd blk_as_B(const double* base, long long o, int kk) {  // (kk=p, nn=c) → M[p,c]
    Opnd q = blk_as_A(base, o, kk);
    q.kstride = 1;
    q.inner_stride = kk;
    return q;
  }
  static OutDesc blk_out(double* base, long long o, int kk) {
    OutDesc c;
    c.base = base + o;
    c.row_inner_stride = 1;
    c.row_outer_stride = 0;
    c.row_inner = 1 << 30;
    c.col_inner_stride = kk;
    c.col_outer_stride = 0;
    c.col_inner = 1 << 30;
    c.rows = kk;
    c.cols = kk;
    return c;
  }

  // The same product on every dense block, C_b = alpha·op(A_b)·op(B_b) +
  // beta·C_b (operands from opA(b), opB(b)), as one grouped launch per eight
  // blocks: the blocks' products are independent and each tile is computed
  // as gemm_f64 computes it for one block.
  template <class FA, class FB>
  void blk_gemm_all(FA opA, bool akc, FB opB, bool bkc, double* out, double alpha, double beta,
                    int mode) {
    GemmGroups g;
    for (auto& b : dense) {
      if (g.n == kGemmGroups) {
        gemm_f64_grouped(g, akc, bkc, st);
        g.n = 0;
      }
      g.A[g.n] = opA(b);
      g.B[g.n] = opB(b);
      g.C[g.n] = blk_out(out, b.off, b.k);
      g.alpha[g.n] = alpha;
      g.beta[g.n] = beta;
      g.mode[g.n] = mode;
      ++g.n;
    }
    gemm_f64_grouped(g, akc, bkc, st);
  }

  // M ← X⁻¹·M for every dense block using W = L_X⁻¹ (Z = Wᵀ (W M)); M is read
  // from `in` and the result written to `out` (distinct from T2).
  void dense_cholsolve(const double* in, double* out) {
    blk_gemm_all([&](const DenseBlk& b) { return blk_as_A(W.p, b.off, b.k); }, false,
                 [&](const DenseBlk& b) { return blk_as_B(in, b.off, b.k); }, true, T2.p, 1.0, 0.0,
                 KR_A_LOWER);
    blk_gemm_all([&](const DenseBlk& b) { return blk_as_At(W.p, b.off, b.k); }, true,
                 [&](const DenseBlk& b) { return blk_as_B(T2.p, b.off, b.k); }, true, out, 1.0, 0.0,
                 KR_A_UPPER);
  }

  void ensure_descs(size_t n) {
    if (n <= desc_cap) return;
    desc_cap = std::max<size_t>(n, 2 * desc_cap);
    d_descs.alloc(desc_cap);
    d_info.alloc(desc_cap);
    d_dmin.alloc(desc_cap);
    d_dmax.alloc(desc_cap);
    d_stats.alloc(3 * desc_cap);
  }
  // Pinned staging for the per-round uploads (descriptor lists) and the
  // packed read-back of the batched Cholesky results: asynchronous copies
  // instead of staged pageable ones.  Only grown right after a sync.
  DBuf<double> d_stats;  // one round's dmin | dmax | info, contiguous
  unsigned char* h_pin = nullptr;
  size_t pin_cap = 0;
  unsigned char* pinned(size_t bytes) {
    if (bytes > pin_cap) {
      sync();
      if (h_pin) cudaFreeHost(h_pin);
      h_pin = nullptr;
      pin_cap = std::max<size_t>(bytes, 2 * pin_cap);
      SDPX_CUDA(cudaMallocHost(&h_pin, pin_cap));
    }
    return h_pin;
  }

  // Batched Cholesky of host-described matrices; fills info/dmin/dmax (host).
  // zero_upper = false for positive-definiteness tests that read only
  // info/dmin/dmax (the factor's strict upper triangle is then left as is).
  void potrf_host_list(const std::vector<MatDesc<double>>& mats, std::vector<int>& info,
                       std::vector<double>& dmin, std::vector<double>& dmax,
                       bool zero_upper = true) {
    size_t n = mats.size();
    info.assign(n, 0);
    dmin.assign(n, 0.0);
    dmax.assign(n, 0.0);
    if (n == 0) return;
    ensure_descs(n);
    int nmax = 0;
    for (auto& q : mats) nmax = std::max(nmax, q.n);
    // Pinned layout: [descriptors | dmin (n) | dmax (n) | info (n)], the last
    // three read back in one copy from d_stats.
    const size_t dbytes = (n * sizeof(MatDesc<double>) + 15) / 16 * 16;
    const size_t sbytes = 2 * n * sizeof(double) + n * sizeof(int);
    unsigned char* hp = pinned(dbytes + sbytes);
    std::memcpy(hp, mats.data(), n * sizeof(MatDesc<double>));
    h2d(d_descs.p, hp, n * sizeof(MatDesc<double>));
    double* sdmin = d_stats.p;
    double* sdmax = d_stats.p + n;
    int* sinfo = reinterpret_cast<int*>(d_stats.p + 2 * n);
    if (nmax >= 192 && zero_upper)
      potrf_batched<double, 64>(d_descs.p, (int)n, nmax, sinfo, sdmin, sdmax, st, zero_upper);
    else if (nmax >= 192)
      potrf_batched<double, 48>(d_descs.p, (int)n, nmax, sinfo, sdmin, sdmax, st, zero_upper);
    else
      potrf_batched<double, 32>(d_descs.p, (int)n, nmax, sinfo, sdmin, sdmax, st, zero_upper);
    d2h(hp + dbytes, d_stats.p, sbytes);
    sync();
    const double* hs = reinterpret_cast<const double*>(hp + dbytes);
    std::memcpy(dmin.data(), hs, n * sizeof(double));
    std::memcpy(dmax.data(), hs + n, n * sizeof(double));
    std::memcpy(info.data(), hs + 2 * n, n * sizeof(int));
  }

  // ------------------------------------------------------------ create ----
  void create(const sdpx_b200_problem* p, int device) {
    dev = device;
    SDPX_CUDA(cudaSetDevice(dev));
    SDPX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    SDPX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (p->m <= 0 || p->nblocks <= 0) throw std::invalid_argument("problem needs m > 0 and L > 0");
    if (p->m > (1 << 30)) throw std::invalid_argument("m too large");
    m = (int)p->m;
    L = p->nblocks;
    k.assign(p->block_order, p->block_order + L);
    user_off.resize(L);
    Ku = 0;
    long long dense_rows = 0;
    for (int l = 0; l < L; ++l) {
      if (k[l] <= 0) throw std::invalid_argument("block orders must be positive");
      user_off[l] = Ku;
      Ku += (long long)k[l] * k[l];
      if (k[l] >= 2) {
        dense.push_back({l, k[l], dense_rows});
        dense_rows += (long long)k[l] * k[l];
        kmax = std::max(kmax, k[l]);
      } else {
        diag_user.push_back(l);
      }
    }
    nd = (int)diag_user.size();
    od = dense_rows;
    K = dense_rows + nd;

    // Stacked index map and per-user-block segments.
    std::vector<long long> map(K);
    seg_off.assign(L, 0);
    seg_len.assign(L, 0);
    for (auto& b : dense) {
      for (long long e = 0; e < (long long)b.k * b.k; ++e) map[b.off + e] = user_off[b.user] + e;
      seg_off[b.user] = b.off;
      seg_len[b.user] = (long long)b.k * b.k;
    }
    for (int j = 0; j < nd; ++j) {
      map[od + j] = user_off[diag_user[j]];
      seg_off[diag_user[j]] = od + j;
      seg_len[diag_user[j]] = 1;
    }
    d_map.alloc(K);
    h2d(d_map.p, map.data(), K * sizeof(long long));
    std::vector<long long> doff, dlen;
    std::vector<int> dk;
    for (auto& b : dense) {
      doff.push_back(b.off);
      dlen.push_back((long long)b.k * b.k);
      dk.push_back(b.k);
    }
    d_doff.alloc(dense.size());
    d_dlen.alloc(dense.size());
    d_dk.alloc(dense.size());
    if (!dense.empty()) {
      h2d(d_doff.p, doff.data(), doff.size() * sizeof(long long));
      h2d(d_dlen.p, dlen.data(), dlen.size() * sizeof(long long));
      h2d(d_dk.p, dk.data(), dk.size() * sizeof(int));
    }
    d_uoff.alloc(L);
    d_ulen.alloc(L);
    d_uk.alloc(L);
    h2d(d_uoff.p, seg_off.data(), L * sizeof(long long));
    h2d(d_ulen.p, seg_len.data(), L * sizeof(long long));
    h2d(d_uk.p, k.data(), L * sizeof(int));
    d_diag_user.alloc(nd);
    if (nd) h2d(d_diag_user.p, diag_user.data(), nd * sizeof(int));

    // Constraint matrix upload: dense blocks by 2-D copies, 1×1 blocks packed.
    A.alloc((size_t)K * m);
    for (auto& b : dense) {
      size_t kk2 = (size_t)b.k * b.k;
      SDPX_CUDA(cudaMemcpy2DAsync(A.p + b.off, (size_t)K * sizeof(double), p->Av[b.user],
                                  kk2 * sizeof(double), kk2 * sizeof(double), (size_t)m,
                                  cudaMemcpyHostToDevice, st));
    }
    if (nd) {
      std::vector<double> pack((size_t)nd * m);
      for (int j = 0; j < nd; ++j) {
        const double* src = p->Av[diag_user[j]];
        for (int i = 0; i < m; ++i) pack[(size_t)i * nd + j] = src[i];
      }
      SDPX_CUDA(cudaMemcpy2DAsync(A.p + od, (size_t)K * sizeof(double), pack.data(),
                                  (size_t)nd * sizeof(double), (size_t)nd * sizeof(double),
                                  (size_t)m, cudaMemcpyHostToDevice, st));
      sync();  // `pack` is a host temporary
    }
    c.alloc(m);
    h2d(c.p, p->c, m * sizeof(double));
    std::vector<double> Cu(Ku);
    for (int l = 0; l < L; ++l)
      std::memcpy(Cu.data() + user_off[l], p->C[l], sizeof(double) * k[l] * k[l]);
    tmpK.alloc(std::max<long long>(K, Ku));
    Cst.alloc(K);
    h2d(tmpK.p, Cu.data(), Ku * sizeof(double));
    gather(K, d_map.p, tmpK.p, Cst.p, st);
    sync();

    // Workspaces.
    for (auto* b : {&x, &dx, &d, &v, &r, &rho, &work_m, &work_m2, &xbest, &keptx, &dxbest})
      b->alloc(m), b->zero(st);
    for (auto* b : {&X, &Y, &P, &R, &Z, &dX, &dY, &LX, &MY, &W, &T1, &T2, &Xbest, &Ybest, &tmpK2})
      b->alloc(K), b->zero(st);
    oz_err.alloc(1);
    oz_err.zero(st);
    gemv_chunks = std::max(1, std::min(16, m / 64));
    gemv_part.alloc((size_t)2 * gemv_chunks * std::max<long long>(K, m));  // Dot2 partials: 2×
    {
      std::vector<long long> lo, up;
      for (auto& b : dense)
        for (int cc = 0; cc < b.k; ++cc)
          for (int pp = cc; pp < b.k; ++pp) {
            lo.push_back(b.off + pp + (long long)cc * b.k);
            up.push_back(b.off + cc + (long long)pp * b.k);
          }
      for (int j = 0; j < nd; ++j) {
        lo.push_back(od + j);
        up.push_back(od + j);
      }
      Kt = (long long)lo.size();
      ap_lo.alloc(std::max<long long>(Kt, 1));
      ap_up.alloc(std::max<long long>(Kt, 1));
      if (Kt) {
        h2d(ap_lo.p, lo.data(), Kt * sizeof(long long));
        h2d(ap_up.p, up.data(), Kt * sizeof(long long));
      }
      // The copy is an accelerator: it is made only when it fits beside 4 GB of
      // headroom (the solve's remaining buffers are allocated later).
      size_t freeb = 0, totb = 0;
      SDPX_CUDA(cudaMemGetInfo(&freeb, &totb));
      freeb += dcache::idle_bytes(dev);
      const size_t apb = sizeof(double) * (size_t)std::max<long long>(Kt, 1) * m;
      use_packed = apb + (4ull << 30) <= freeb;
      if (use_packed) Ap.alloc((size_t)std::max<long long>(Kt, 1) * m);
      kt_fold.alloc(std::max<long long>(Kt, 1));
      adx.alloc(K);
      adx.zero(st);
      sync();  // lo/up are host temporaries
    }
    Pc.alloc((size_t)K * m);
    S.alloc((size_t)m * m);
    Sf.alloc((size_t)m * m);
    Dinv.alloc((size_t)ceil_div(m, 64) * 64 * 64);
    syrk = plan_syrk_f64(m, K, sms);
    partial.alloc(syrk.partial_doubles);
    red.alloc(64);
    SDPX_CUDA(cudaMallocHost(&h_red, 64 * sizeof(double)));
    mu_user.alloc(L);
    target_user.alloc(L);
    work_L.alloc(2 * std::max<size_t>((size_t)L, dense.size()) + 2);
    seg_parts = 8;
    seg_part.alloc((size_t)seg_parts * L);
    ensure_descs(std::max<size_t>(16, 2 * dense.size()));
    d_fail.alloc(64);
    d_tcand.alloc(64);
    // Gershgorin scratch
    std::vector<long long> coff(dense.size());
    long long tot = 0;
    for (size_t b = 0; b < dense.size(); ++b) coff[b] = tot, tot += dense[b].k;
    g_cand.alloc(tot);
    g_cand_off.alloc(dense.size());
    if (!dense.empty()) h2d(g_cand_off.p, coff.data(), coff.size() * sizeof(long long));
    g_scale.alloc(dense.size());
    g_nonfinite.alloc(dense.size());
    lx_dmin.assign(dense.size(), 1.0);
    lx_dmax.assign(dense.size(), 1.0);
    my_dmin.assign(dense.size(), 1.0);
    my_dmax.assign(dense.size(), 1.0);
    // Start at X = Y = I.
    fixed_start(1.0, 1.0);
    sync();
  }

  // ----------------------------------------------------------- scaling ----
  void equilibrate(double* E_out, double* s_out, double* objscale, int32_t* passes) {
    if (mixed) mixed->a_planes_valid = false;
    // keep the original data for final slack/residual reconstruction
    if (!have_original) {
      A0.alloc((size_t)K * m);
      d2d(A0.p, A.p, sizeof(double) * K * m);
      C0st.alloc(K);
      d2d(C0st.p, Cst.p, sizeof(double) * K);
      c0.alloc(m);
      d2d(c0.p, c.p, sizeof(double) * m);
      have_original = true;
    }
    std::vector<std::vector<double>> E(L);
    for (int l = 0; l < L; ++l) E[l].assign(k[l], 1.0);
    std::vector<int> used(L, 0);
    std::vector<char> active(L, 1);
    DBuf<double> rn_d, e_d;
    long long rows_total = 0;
    for (auto& b : dense) rows_total += b.k;
    rows_total += nd;
    rn_d.alloc(rows_total);
    e_d.alloc(rows_total);
    std::vector<double> Chost(K);
    for (int it = 1; it <= 8; ++it) {
      bool any = false;
      for (int l = 0; l < L; ++l) any = any || active[l];
      if (!any) break;
      // C row maxima on the host (C is small), A row maxima on the device.
      d2h(Chost.data(), Cst.p, K * sizeof(double));
      rn_d.zero(st);
      long long ro = 0;
      for (auto& b : dense) {
        if (active[b.user]) ruiz_rowmax_dense(A.p, K, m, b.off, b.k, rn_d.p + ro, st);
        ro += b.k;
      }
      if (nd) ruiz_rowmax_diag(A.p, K, m, od, nd, rn_d.p + ro, st);
      std::vector<double> rn(rows_total);
      d2h(rn.data(), rn_d.p, rows_total * sizeof(double));
      sync();
      std::vector<double> e(rows_total, 1.0);
      ro = 0;
      auto handle_block = [&](int l, int kk, long long rowoff, const double* Cblk, long long cstride,
                              bool is_diag) {
        // rn[r] = max(rn[r], max_c |C[r,c]|)
        for (int r0 = 0; r0 < kk; ++r0) {
          double mx = rn[rowoff + r0];
          for (int cc = 0; cc < kk; ++cc) {
            double vv = std::fabs(Cblk[(is_diag ? 0 : (long long)cc * cstride) + r0]);
            if (std::isnan(vv)) vv = INFINITY;
            mx = std::max(mx, vv);
          }
          rn[rowoff + r0] = mx;
        }
        bool conv = false;
        if (it >= 2) {
          double dev = 0.0;
          bool finite = true;
          for (int r0 = 0; r0 < kk; ++r0) {
            double vv = rn[rowoff + r0];
            if (!(vv > 0)) continue;
            if (!std::isfinite(vv)) {
              finite = false;
              break;
            }
            dev = std::max(dev, std::fabs(std::log(vv)));
          }
          conv = finite && dev <= 1.0 / 20.0;
        }
        for (int r0 = 0; r0 < kk; ++r0) {
          double vv = rn[rowoff + r0];
          e[rowoff + r0] = vv > 0 ? 1.0 / std::sqrt(vv) : 1.0;
          E[l][r0] *= e[rowoff + r0];
        }
        used[l] = it;
        if (conv) active[l] = 0;
      };
      for (auto& b : dense) {
        if (active[b.user]) handle_block(b.user, b.k, ro, Chost.data() + b.off, b.k, false);
        ro += b.k;
      }
      for (int j = 0; j < nd; ++j) {
        int l = diag_user[j];
        if (active[l]) handle_block(l, 1, ro + j, Chost.data() + od + j, 1, true);
        else e[ro + j] = 1.0;
      }
      h2d(e_d.p, e.data(), rows_total * sizeof(double));
      ro = 0;
      for (auto& b : dense) {
        if (active[b.user] || used[b.user] == it) ruiz_congruence_dense(A.p, K, m, b.off, b.k, e_d.p + ro, st);
        ro += b.k;
      }
      if (nd) ruiz_congruence_diag(A.p, K, m, od, nd, e_d.p + ro, st);
      // C ← E C E on the host copy, uploaded back
      ro = 0;
      for (auto& b : dense) {
        for (int cc = 0; cc < b.k; ++cc)
          for (int r0 = 0; r0 < b.k; ++r0)
            Chost[b.off + (long long)cc * b.k + r0] *= e[ro + r0] * e[ro + cc];
        ro += b.k;
      }
      for (int j = 0; j < nd; ++j) Chost[od + j] *= e[ro + j] * e[ro + j];
      h2d(Cst.p, Chost.data(), K * sizeof(double));
      sync();
    }
    // Per-variable scale s_i = max_l ‖A_i^(l)‖∞ (1 when zero), objective scale.
    std::vector<double> mx(m), s(m), ch(m);
    colmax(A.p, K, m, work_m.p, st);
    d2h(mx.data(), work_m.p, m * sizeof(double));
    d2h(ch.data(), c.p, m * sizeof(double));
    sync();
    double osc = 0.0;
    for (int i = 0; i < m; ++i) {
      s[i] = mx[i] > 0 ? mx[i] : 1.0;
      ch[i] = ch[i] / s[i];
      osc = std::max(osc, std::fabs(ch[i]));
    }
    if (!(osc > 0 && std::isfinite(osc))) osc = 1.0;
    for (int i = 0; i < m; ++i) ch[i] /= osc;
    h2d(work_m.p, s.data(), m * sizeof(double));
    scale_cols(A.p, K, m, work_m.p, st);
    if (n_eq) {  // `_scale_equality_rows!` (src/ingest.jl:1176-1184); b is unchanged
      if (!eq_have_original) {
        Beq0.alloc((size_t)m * n_eq);
        d2d(Beq0.p, Beq.p, sizeof(double) * m * n_eq);
        eq_have_original = true;
      }
      eq_scale_rows(m, n_eq, Beq.p, work_m.p, st);
    }
    h2d(c.p, ch.data(), m * sizeof(double));
    sync();
    if (E_out) {
      long long o = 0;
      for (int l = 0; l < L; ++l)
        for (int r0 = 0; r0 < k[l]; ++r0) E_out[o++] = E[l][r0];
    }
    if (s_out) std::memcpy(s_out, s.data(), m * sizeof(double));
    if (objscale) *objscale = osc;
    if (passes)
      for (int l = 0; l < L; ++l) passes[l] = used[l];
    a_changed();
  }

  void reset() {
    if (mixed) mixed->a_planes_valid = false;
    mixed_fallbacks = 0;
    mixed_guard_steps = 0;
    identity_metric = false;
    operator_applications = 0;
    schur_builds = 0;
    mixed_predicted_steps = 32;
    a_changed();
    if (have_original) {
      d2d(A.p, A0.p, sizeof(double) * K * m);
      d2d(Cst.p, C0st.p, sizeof(double) * K);
      d2d(c.p, c0.p, sizeof(double) * m);
    }
    if (eq_have_original) d2d(Beq.p, Beq0.p, sizeof(double) * m * n_eq);
    eq_kind = 0;
    eq_qr_sticky = false;
    precision = SDPX_B200_FP64;
    fixed_start(1.0, 1.0);
    sync();
    harvest_phases();
    for (double& v : phase_ms) v = 0.0;
  }

  void data_norms(double* maxC, double* cnorm) {
    clear_red(0, 2);
    absmax(K, Cst.p, red.p + 0, st);
    absmax(m, c.p, red.p + 1, st);
    d2h(h_red, red.p, 2 * sizeof(double));
    sync();
    *maxC = h_red[0];
    *cnorm = h_red[1];
  }

  // -------------------------------------------------------- iterate I/O --
  void set_iterate(const double* hx, const double* hX, const double* hY) {
    if (hx) h2d(x.p, hx, m * sizeof(double));
    if (hX) {
      h2d(tmpK.p, hX, Ku * sizeof(double));
      gather(K, d_map.p, tmpK.p, X.p, st);
    }
    if (hY) {
      h2d(tmpK2.p, hY, Ku * sizeof(double));
      gather(K, d_map.p, tmpK2.p, Y.p, st);
    }
    sync();
  }
  void get_stacked(const double* dev_src, double* host_dst) {
    scatter(K, d_map.p, dev_src, tmpK.p, st);
    d2h(host_dst, tmpK.p, Ku * sizeof(double));
    sync();
  }
  void fixed_start(double wp, double wd) {
    x.zero(st);
    if (n_eq) yv.zero(st);
    X.zero(st);
    Y.zero(st);
    if (!dense.empty()) {
      add_diag(d_doff.p, d_dk.p, (int)dense.size(), kmax, X.p, nullptr, wp, st);
      add_diag(d_doff.p, d_dk.p, (int)dense.size(), kmax, Y.p, nullptr, wd, st);
    }
    if (nd) {
      std::vector<double> ones(nd, wp), ones2(nd, wd);
      h2d(X.p + od, ones.data(), nd * sizeof(double));
      h2d(Y.p + od, ones2.data(), nd * sizeof(double));
      sync();
    }
  }

  // ------------------------------------------------------ block factors --
  bool factor_blocks() {
    // LX = chol(X), MY = chol(Y) for every dense block (batched), 1×1 by sqrt.
    std::vector<MatDesc<double>> mats;
    for (auto& b : dense) {
      d2d(LX.p + b.off, X.p + b.off, sizeof(double) * b.k * b.k);
      d2d(MY.p + b.off, Y.p + b.off, sizeof(double) * b.k * b.k);
    }
    for (auto& b : dense) mats.push_back({LX.p + b.off, b.k, b.k});
    for (auto& b : dense) mats.push_back({MY.p + b.off, b.k, b.k});
    std::vector<int> info;
    std::vector<double> dmn, dmx;
    int fail_h = 0;
    if (nd) {
      SDPX_CUDA(cudaMemsetAsync(d_fail.p, 0, sizeof(int), st));
      diag_factor(nd, od, X.p, Y.p, LX.p, MY.p, d_fail.p, st);
    }
    potrf_host_list(mats, info, dmn, dmx);
    if (nd) {
      d2h(&fail_h, d_fail.p, sizeof(int));
      sync();
    }
    bool ok = fail_h == 0;
    size_t nb = dense.size();
    for (size_t b = 0; b < nb; ++b) {
      ok = ok && info[b] == 0 && info[nb + b] == 0;
      lx_dmin[b] = dmn[b];
      lx_dmax[b] = dmx[b];
      my_dmin[b] = dmn[nb + b];
      my_dmax[b] = dmx[nb + b];
    }
    diag_factor_ok = fail_h == 0;
    if (ok && !dense.empty()) {
      // W = L_X^{-1} for the Schur products and the block solves.
      W.zero(st);
      std::vector<MatDesc<double>> Ls, Ws;
      for (auto& b : dense) {
        Ls.push_back({LX.p + b.off, b.k, b.k});
        Ws.push_back({W.p + b.off, b.k, b.k});
      }
      ensure_descs(2 * nb);
      h2d(d_descs.p, Ls.data(), nb * sizeof(MatDesc<double>));
      h2d(d_descs.p + nb, Ws.data(), nb * sizeof(MatDesc<double>));
      trinv_batched<double, 32>(d_descs.p, d_descs.p + nb, (int)nb, kmax, st);
      sync();
    }
    return ok;
  }

  void block_margins(double* primal, double* dual) {
    // `_cholesky_diagonal_quality` per block; 1×1 blocks contribute 1.
    double p = 1.0, q = 1.0;
    for (size_t b = 0; b < dense.size(); ++b) {
      auto qual = [](double lo, double hi) {
        return (hi > 0 && std::isfinite(hi)) ? std::min(1.0, std::max(0.0, lo / hi)) : 0.0;
      };
      p = std::min(p, qual(lx_dmin[b], lx_dmax[b]));
      q = std::min(q, qual(my_dmin[b], my_dmax[b]));
    }
    *primal = p;
    *dual = q;
  }

  // ---------------------------------------------------------- residuals --
  void residuals(const double* mu, int use_affine, int factor, double* p_res, double* d_res,
                 int* ok) {
    PhaseScope ps(this, 0);
    primal_residual(x.p, P.p);  // P = 𝒜x − X − C
    dual_residual(Y.p, d.p);    // d = c − 𝒜ᵀ vec(Y)
    clear_red(0, 3);
    if (n_eq) {
      // d −= B·y, p = b − Bᵀx (src/step.jl:41-51)
      gemv_n(Beq.p, m, n_eq, yv.p, eq_tm.p, gemv_part.p, gemv_chunks, st);
      axpbypcz(m, 1.0, d.p, -1.0, eq_tm.p, 0.0, nullptr, d.p, st);
      gemv_t(Beq.p, m, n_eq, x.p, -1.0, beq.p, 1.0, pv.p, st);
      absmax(n_eq, pv.p, red.p + 2, st);
    }
    absmax(K, P.p, red.p + 0, st);
    absmax(m, d.p, red.p + 1, st);
    // R = −XY (+ μ I)
    h2d(mu_user.p, mu, L * sizeof(double));
    blk_gemm_all([&](const DenseBlk& b) { return blk_as_A(X.p, b.off, b.k); }, false,
                 [&](const DenseBlk& b) { return blk_as_B(Y.p, b.off, b.k); }, true, R.p, -1.0, 0.0,
                 KR_FULL);
    if (!use_affine && !dense.empty()) {
      std::vector<double> shifts(dense.size());
      for (size_t b = 0; b < dense.size(); ++b) shifts[b] = mu[dense[b].user];
      h2d(work_L.p, shifts.data(), shifts.size() * sizeof(double));
      add_diag(d_doff.p, d_dk.p, (int)dense.size(), kmax, R.p, work_L.p, 0.0, st);
    }
    diag_residual_R(nd, od, X.p, Y.p, mu_user.p, d_diag_user.p, use_affine, R.p, st);
    d2h(h_red, red.p, 3 * sizeof(double));
    sync();
    *p_res = std::max(h_red[0], h_red[2]);
    *d_res = h_red[1];
    last_bpr = h_red[0];
    *ok = 1;
    if (factor) *ok = factor_blocks() ? 1 : 0;
  }

  // ------------------------------------------------------------- Schur ----
  void schur_build(int identity) {
    ++schur_builds;
    PhaseScope ps(this, 1);
    identity_metric = identity != 0;
    if (precision == SDPX_B200_MIXED && mixed) {
      schur_split_bf16(identity != 0);
      return;
    }
    schur_build_fp64(identity);
  }
  bool oz_blocks_ready() {
    if (oz_blk_state == 0) {
      size_t adig = 0, tdig = 0, wdig = 0;
      long long aexp = 0, texp = 0, wexp = 0;
      ozb.clear();
      bool fits_int = true;  // the digit GEMM indexes k·m rows with 32-bit ints
      for (auto& b : dense) fits_int = fits_int && (long long)b.k * m < (1LL << 31) - 128;
      for (auto& b : dense) {
        OzBlock o;
        o.kp = oz_kpad(b.k);
        o.dig_off = adig;
        o.exp_off = aexp;
        const size_t rows = (size_t)b.k * m;
        adig += (size_t)OZ_DIGITS * rows * (size_t)o.kp;
        aexp += (long long)rows;
        tdig = std::max(tdig, (size_t)OZ_DIGITS * rows * (size_t)o.kp);
        texp = std::max(texp, (long long)rows);
        wdig = std::max(wdig, (size_t)2 * OZ_DIGITS * (size_t)b.k * (size_t)o.kp);
        wexp = std::max(wexp, 2LL * b.k);
        ozb.push_back(o);
      }
      // Room for the cached constraint digits, the per-build scratch and the
      // Gram's digit planes (same size as the FP64 panel), with 2 GB to spare.
      size_t freeb = 0, totb = 0;
      SDPX_CUDA(cudaMemGetInfo(&freeb, &totb));
      freeb += dcache::idle_bytes(dev);  // idle cached blocks are ours to reuse
      const size_t gram = oz_plan.m == m && oz_plan.K == K ? 0 : (size_t)OZ_DIGITS * m * (K + 64);
      const size_t need = adig + tdig + wdig + 4 * (size_t)(aexp + texp + wexp) + gram;
      if (dense.empty() || !fits_int || need + (2ull << 30) > freeb) {
        oz_blk_state = -1;
      } else {
        oz_adig.alloc(adig);
        oz_tdig.alloc(tdig);
        oz_wdig.alloc(wdig);
        oz_aexp.alloc(aexp);
        oz_texp.alloc(texp);
        oz_wexp.alloc(wexp);
        oz_colmax.alloc(m);
        oz_a_ver = 0;
        oz_blk_state = 1;
      }
    }
    return oz_blk_state == 1;
  }
  void oz_block_products() {
    if (oz_a_ver != a_ver) {
      for (size_t bi = 0; bi < dense.size(); ++bi) {
        const DenseBlk& b = dense[bi];
        const OzBlock& o = ozb[bi];
        OzRows r;  // row (i, c): A_i[p, c] at off + i·K + c·k + p
        r.base = A.p + b.off;
        r.rows = (long long)b.k * m;
        r.inner = b.k;
        r.is = b.k;
        r.os = K;
        r.len = b.k;
        ozaki_digits_rows(r, o.kp, r.rows * o.kp, oz_adig.p + o.dig_off, oz_aexp.p + o.exp_off, st);
      }
      oz_a_ver = a_ver;
    }
    SDPX_CUDA(cudaMemsetAsync(oz_colmax.p, 0, sizeof(unsigned) * m, st));
    for (size_t bi = 0; bi < dense.size(); ++bi) {
      const DenseBlk& b = dense[bi];
      const OzBlock& o = ozb[bi];
      const long long rows = (long long)b.k * m;
      const long long aplane = rows * o.kp, wplane = (long long)b.k * o.kp;
      int8_t* wd = oz_wdig.p;
      int8_t* yd = oz_wdig.p + OZ_DIGITS * wplane;
      int* we = oz_wexp.p;
      int* ye = oz_wexp.p + b.k;
      OzRows w;  // row r of W: W[r, p] at off + r + p·k, p ≤ r
      w.base = W.p + b.off;
      w.rows = b.k;
      w.is = 1;
      w.es = b.k;
      w.len = b.k;
      w.tri = 1;
      ozaki_digits_rows(w, o.kp, wplane, wd, we, st);
      OzRows y;  // column c' of M_Y: M_Y[c, c'] at off + c + c'·k, c ≥ c'
      y.base = MY.p + b.off;
      y.rows = b.k;
      y.is = b.k;
      y.len = b.k;
      y.tri = 2;
      ozaki_digits_rows(y, o.kp, wplane, yd, ye, st);
      OzGemm g;  // T_i[r, c] = Σ_p A_i[p, c]·W[r, p] → Pc[off + i·K + r·k + c]
      g.xd = oz_adig.p + o.dig_off;
      g.x_plane = aplane;
      g.rows_a = (int)rows;
      g.ea = oz_aexp.p + o.exp_off;
      g.yd = wd;
      g.y_plane = wplane;
      g.rows_b = b.k;
      g.eb = we;
      g.Kp = o.kp;
      g.kmode = 1;
      g.out = Pc.p + b.off;
      g.a_inner = b.k;
      g.a_is = 1;
      g.a_os = K;
      g.b_stride = b.k;
      ozaki_gemm(g, sms, oz_err.p, st);
      OzRows t;  // row (i, r) of T: T_i[r, c] at off + i·K + r·k + c
      t.base = Pc.p + b.off;
      t.rows = rows;
      t.inner = b.k;
      t.is = b.k;
      t.os = K;
      t.len = b.k;
      ozaki_digits_rows(t, o.kp, aplane, oz_tdig.p, oz_texp.p, st);
      OzGemm h = g;  // P_i[r, c'] = Σ_c T_i[r, c]·M_Y[c, c'] → Pc[off + i·K + c'·k + r]
      h.xd = oz_tdig.p;
      h.ea = oz_texp.p;
      h.yd = yd;
      h.eb = ye;
      h.kmode = 2;
      h.colmax = oz_colmax.p;  // the Gram's column exponents over the dense rows
      ozaki_gemm(h, sms, oz_err.p, st);
    }
  }
  // Flat coordinate form of every dense block's coefficients (the
  // `SparseBlockCOO` of src/types/constraints.jl:60-101 with `schur_order`
  // ascending): count the stored entries of each (block, variable) slab on the
  // device, scan on the host, compact on the device in linear-index order.
  void build_coo() {
    const int nb = (int)dense.size();
    for (auto& b : dense)
      if (b.k > kSparseSchurMaxK)
        throw std::invalid_argument("sparse Schur: block order " + std::to_string(b.k) +
                                    " exceeds 160");
    sp_cnt.alloc(std::max<size_t>(1, (size_t)nb * m));
    for (int b = 0; b < nb; ++b)
      coo_count(A.p, K, m, dense[b].off, dense[b].k * dense[b].k, sp_cnt.p + (size_t)b * m, st);
    std::vector<int> cnt((size_t)nb * m);
    if (!cnt.empty()) d2h(cnt.data(), sp_cnt.p, cnt.size() * sizeof(int));
    sync();
    std::vector<int> ids;
    std::vector<long long> ptr(1, 0);
    sp_na.assign(nb, 0);
    sp_act_off.assign(nb, 0);
    for (int b = 0; b < nb; ++b) {
      sp_act_off[b] = (long long)ids.size();
      for (int i = 0; i < m; ++i) {
        const int c = cnt[(size_t)b * m + i];
        if (c == 0) continue;
        ids.push_back(i);
        ptr.push_back(ptr.back() + c);
        ++sp_na[b];
      }
    }
    sp_active = (long long)ids.size();
    sp_nnz = ptr.back();
    sp_ids.alloc(std::max<long long>(1, sp_active));
    sp_ptr.alloc(sp_active + 1);
    sp_lin.alloc(std::max<long long>(1, sp_nnz));
    sp_val.alloc(std::max<long long>(1, sp_nnz));
    if (sp_active) h2d(sp_ids.p, ids.data(), ids.size() * sizeof(int));
    h2d(sp_ptr.p, ptr.data(), ptr.size() * sizeof(long long));
    for (int b = 0; b < nb; ++b)
      coo_fill(A.p, K, dense[b].off, dense[b].k * dense[b].k, sp_ids.p + sp_act_off[b],
               sp_ptr.p + sp_act_off[b], sp_na[b], sp_lin.p, sp_val.p, st);
    sync();
    coo_ver = a_ver;
  }
  // S from the current block factors by the sparse engine: the 1×1 group's
  // Gram first, then every dense block's active pairs in block order (one
  // launch per block, so each entry of S sums its block terms in a fixed order).
  void schur_sparse() {
    if (coo_ver != a_ver) build_coo();
    if (nd) {
      diag_panel(K, m, nd, od, A.p, LX.p, MY.p, Pc.p, st);
      if (diag_syrk.ntri == 0 || diag_syrk.bm == 0) {
        diag_syrk = plan_syrk_f64(m, nd, sms);
        diag_partial.alloc(diag_syrk.partial_doubles);
      }
      Opnd Pd;
      Pd.base = Pc.p + od;
      Pd.kstride = 1;
      Pd.inner = 1 << 30;
      Pd.inner_stride = K;
      Pd.outer_stride = 0;
      Pd.mn_extent = m;
      Pd.k_extent = nd;
      syrk_lower_f64(Pd, diag_syrk, diag_partial.p, S.p, m, m, 0.0, st);
    } else {
      SDPX_CUDA(cudaMemsetAsync(S.p, 0, sizeof(double) * (size_t)m * m, st));
    }
    if (!dense.empty()) {
      Xinv.alloc(K);
      // X⁻¹ = WᵀW with W = L_X⁻¹
      blk_gemm_all([&](const DenseBlk& b) { return blk_as_At(W.p, b.off, b.k); }, true,
                   [&](const DenseBlk& b) { return blk_as_B(W.p, b.off, b.k); }, true, Xinv.p, 1.0,
                   0.0, KR_FULL);
      for (size_t b = 0; b < dense.size(); ++b)
        sparse_schur_block(Y.p + dense[b].off, Xinv.p + dense[b].off, dense[b].k,
                           sp_ptr.p + sp_act_off[b], sp_lin.p, sp_val.p, sp_ids.p + sp_act_off[b],
                           sp_na[b], S.p, m, st);
    }
    mirror_lower(m, S.p, st);
  }

  void schur_build_fp64(int identity) {
    if (!identity && sparse_schur) return schur_sparse();
    const double* panel = A.p;
    if (!identity) {
      kt_begin(3);
      if (gram_engine == 1 && oz_blocks_ready()) oz_block_products();
      else for (auto& b : dense) {
        // T = W · [A_1 … A_m]  (W lower ⇒ K range [0, row-tile end))
        Opnd Wd = blk_as_A(W.p, b.off, b.k);
        Opnd Ap;  // (kk = p, nn = (i, c)) → A[off + c·k + p, i]
        Ap.base = A.p + b.off;
        Ap.kstride = 1;
        Ap.inner = b.k;
        Ap.inner_stride = b.k;
        Ap.outer_stride = K;
        Ap.mn_extent = b.k * m;
        Ap.k_extent = b.k;
        OutDesc Tout;
        Tout.base = Pc.p + b.off;
        Tout.row_inner_stride = 1;
        Tout.row_outer_stride = 0;
        Tout.row_inner = 1 << 30;
        Tout.col_inner = b.k;
        Tout.col_inner_stride = b.k;
        Tout.col_outer_stride = K;
        Tout.rows = b.k;
        Tout.cols = b.k * m;
        gemm_f64(Wd, false, Ap, true, Tout, 1.0, 0.0, KR_A_LOWER, true, st);
        // P_i = T_i · M_Y in place (rows (i, r) two-level, columns c)
        Opnd Tst;
        Tst.base = Pc.p + b.off;
        Tst.kstride = b.k;
        Tst.inner = b.k;
        Tst.inner_stride = 1;
        Tst.outer_stride = K;
        Tst.mn_extent = b.k * m;
        Tst.k_extent = b.k;
        Opnd My = blk_as_B(MY.p, b.off, b.k);
        OutDesc Pout;
        Pout.base = Pc.p + b.off;
        Pout.row_inner = b.k;
        Pout.row_inner_stride = 1;
        Pout.row_outer_stride = K;
        Pout.col_inner = 1 << 30;
        Pout.col_inner_stride = b.k;
        Pout.col_outer_stride = 0;
        Pout.rows = b.k * m;
        Pout.cols = b.k;
        trmm_right_lower_inplace_f64(Tst, My, Pout, st);
      }
      kt_end(3);
      diag_panel(K, m, nd, od, A.p, LX.p, MY.p, Pc.p, st);
      panel = Pc.p;
    }
    Opnd Pd;
    Pd.base = panel;
    Pd.kstride = 1;
    Pd.inner = 1 << 30;
    Pd.inner_stride = K;
    Pd.outer_stride = 0;
    Pd.mn_extent = m;
    Pd.k_extent = (int)K;
    kt_begin(2);
    if (gram_engine == 1) {
      if (oz_plan.m != m || oz_plan.K != K) {
        oz_plan = plan_ozaki_syrk(m, K, sms);
        oz_digits.alloc(oz_plan.digit_bytes);
        oz_exps.alloc(m);
        oz_partial.alloc(oz_plan.partial_alloc_doubles);
      }
      // After the digit block products every dense row of P̂ carries its column
      // maximum already; the Gram's digit pass scans only the 1×1 rows for it.
      const bool known = !identity && oz_blk_state == 1;
      ozaki_syrk(panel, oz_plan, oz_digits.p, oz_exps.p, oz_partial.p, S.p, oz_err.p, st, nullptr,
                 nullptr, known ? oz_colmax.p : nullptr, od);
      kt_end(2);
      int e = 0;
      d2h(&e, oz_err.p, sizeof(int));
      sync();
      if (e) throw CudaError("int8 Gram kernel: a bounded wait gave up");
    } else {
      syrk_lower_f64(Pd, syrk, partial.p, S.p, m, m, 0.0, st);
      kt_end(2);
    }
    mirror_lower(m, S.p, st);
  }

  // ------------------------------------------------------- factorisation --
  void factorize(int* ok, int* attempts, double* quality) {
    PhaseScope ps(this, 2);
    if (precision == SDPX_B200_MIXED && mixed) {
      mixed_factorize(ok, attempts, quality);
      if (*ok && n_eq) {
        // Equality block on the low-precision factor (`_try_factor_mixed_kkt!`,
        // src/kernels/mixed_precision_kkt.jl:1045-1082): its condition estimate
        // joins the refinement-budget gate; a Q that stays indefinite rejects
        // the mixed factor for this iteration.
        double cond_q = INFINITY, quality_q = 0.0;
        if (factor_equality_mixed(&cond_q, &quality_q)) {
          mixed->cond_estimate = std::max(mixed->cond_estimate, cond_q);
          mixed_predicted_steps = mixed_steps_for(mixed->cond_estimate);
          *quality = std::min(*quality, quality_q);
        } else {
          mixed_predicted_steps = 1 << 30;
        }
      }
      if (*ok && mixed_predicted_steps <= 32) return;
      // Static rejection: the FP32 factor of the split-assembled S is not
      // predicted to converge in ≤ 32 refinements (or failed) — FP64 from here.
      precision = SDPX_B200_FP64;
      ++mixed_fallbacks;
      schur_build_fp64(identity_metric ? 1 : 0);
    }
    MatDesc<double> md{Sf.p, m, m};
    std::vector<MatDesc<double>> one{md};
    std::vector<int> info;
    std::vector<double> dmn, dmx;
    double reg = 0.0;
    int att = 0;
    while (true) {
      copy_reg(m, S.p, Sf.p, att == 0 ? 0.0 : reg, st);
      if (potrf_single_pays<double, 64>(m)) {
        if (coop_bar.n < 4) coop_bar.alloc(4);
        potrf_single<double, 64>(Sf.p, m, m, d_info.p, d_dmin.p, d_dmax.p,
                                 reinterpret_cast<CoopBar*>(coop_bar.p), true, st);
      } else {
        ensure_descs(1);
        h2d(d_descs.p, &md, sizeof(md));
        potrf_batched<double, 64>(d_descs.p, 1, m, d_info.p, d_dmin.p, d_dmax.p, st);
      }
      info.resize(1);
      dmn.resize(1);
      dmx.resize(1);
      d2h(info.data(), d_info.p, sizeof(int));
      d2h(dmn.data(), d_dmin.p, sizeof(double));
      d2h(dmx.data(), d_dmax.p, sizeof(double));
      sync();
      if (info[0] < 0) throw CudaError("Schur Cholesky: a grid barrier timed out");
      if (info[0] == 0 || att >= 6) break;
      ++att;
      reg = (att == 1) ? kSqrtEps : reg * 10.0;
    }
    *attempts = att;
    *ok = info[0] == 0 ? 1 : 0;
    double hi = dmx[0], lo = dmn[0];
    *quality = (*ok && hi > 0 && std::isfinite(hi)) ? std::min(1.0, std::max(0.0, lo / hi)) : 0.0;
    if (*ok) {
      // Solves with the FP64 factor are applied 3-5 times per iteration
      // (predictor, corrector, refinement corrections), so L is inverted once
      // (recursive doubling on the DMMA tiles) and each solve is two GEMVs
      // instead of 2·ceil(m/64) dependent substitution launches; the FP64
      // refinement against S follows as before.
      if (Linv.n < (size_t)m * m) {
        Linv.alloc((size_t)m * m);
        tmp_mm.alloc((size_t)m * m);
      }
      trinv_recursive_f64(Sf.p, m, Linv.p, Dinv.p, tmp_mm.p, st);
      if (n_eq) {
        bool rank_deficient = false;
        if (!factor_equality(&rank_deficient)) {
          *ok = 0;
          *quality = 0.0;
          return;
        }
        // `_kkt_factorization_quality` (src/step.jl:338-345, 797-801)
        if (eq_kind == 2) *quality = std::min(*quality, eq_quality);
        if (rank_deficient) *quality = 0.0;
      }
    }
  }

  // ------------------------------------------------------------- solves ----
  void solve_into(double* vec) {  // vec ← S⁻¹ vec with the current factor
    if (precision == SDPX_B200_MIXED && mixed) {
      mixed_solve(vec);
      return;
    }
    gemv_n(Linv.p, m, m, vec, work_m2.p, gemv_part.p, gemv_chunks, st);
    gemv_t(Linv.p, m, m, work_m2.p, 1.0, nullptr, 0.0, vec, st);
  }
  void solve() {
    PhaseScope ps(this, 3);
    d2d(dx.p, r.p, m * sizeof(double));
    solve_kkt_into(dx.p, pv.p, dyv.p);
    dx_written();
    if (precision == SDPX_B200_MIXED && mixed) mixed_guard();
  }
  // Mixed-precision solve guard (the reference's `_solve_mixed_kkt_guarded!`,
  // src/kernels/mixed_precision_kkt.jl:1431-1586): refine the low-precision
  // solution against the FP64 Newton operator until ‖r − S dx‖∞ ≤ 1e-8·max(‖r‖∞,1),
  // at most min(predicted, 32) corrections, stopping when a correction does
  // not reduce the residual.  On failure the iteration continues on the FP64
  // path: S is reassembled and factored in FP64 and dx re-solved.
  void mixed_guard() {
    double res, rn;
    direction_residual(&res, &rn, false);
    rho_seq = ~0ull;  // re-marked below only if dx ends consistent with ρ
    const double target = 1e-8 * std::max(rn, 1.0);
    if (std::isfinite(res) && res <= target) {
      mark_rho_fresh(res);
      return;
    }
    int cap = std::min(mixed_predicted_steps, 32);
    bool ok = false;
    if (std::isfinite(res)) {
      for (int s = 0; s < cap; ++s) {
        d2d(dxbest.p, dx.p, m * sizeof(double));
        if (n_eq) d2d(dybest.p, dyv.p, n_eq * sizeof(double));
        d2d(work_m.p, rho.p, m * sizeof(double));
        solve_kkt_into(work_m.p, rho_p.p, eq_ddy.p);
        combine(m, dx.p, 1.0, work_m.p, st);
        if (n_eq) combine(n_eq, dyv.p, 1.0, eq_ddy.p, st);
        dx_written();
        double corr = residual_norm_only();
        ++mixed_guard_steps;
        if (!std::isfinite(corr) || corr >= res) {
          restore_dx_best();
          break;
        }
        res = corr;
        if (res <= target) {
          ok = true;
          break;
        }
      }
    }
    if (!ok)
      switch_to_fp64_now();
    else
      mark_rho_fresh(res);
  }
  // Leave mixed mode for good within the current iteration: FP64 Schur,
  // FP64 factor, and re-solve of the current right-hand side.
  void switch_to_fp64_now() {
    precision = SDPX_B200_FP64;
    ++mixed_fallbacks;
    schur_build_fp64(identity_metric ? 1 : 0);
    int ok = 0, att = 0;
    double q = 0.0;
    factorize(&ok, &att, &q);
    if (!ok) throw CudaError("FP64 fallback factorisation failed");
    d2d(dx.p, r.p, m * sizeof(double));
    solve_kkt_into(dx.p, pv.p, dyv.p);
    dx_written();
  }
  // ρ = r − S·dx  (FP64 Newton operator)
  void apply_residual() {
    if (precision == SDPX_B200_MIXED && mixed) {
      mixed_residual();
      return;
    }
    symv_full(m, S.p, dx.p, -1.0, r.p, 1.0, rho.p, st);
    if (n_eq) eq_residual_terms();
  }
  void direction_residual(double* res, double* rnorm, bool allow_cache = true) {
    PhaseScope ps(this, 3);
    double cached = 0.0;
    const bool hit = allow_cache && take_rho_cache(&cached);
    if (!hit) apply_residual();
    clear_red(0, 4);
    if (!hit) absmax(m, rho.p, red.p + 0, st);
    absmax(m, r.p, red.p + 1, st);
    if (n_eq) {  // ρ_p and p enter the residual and the gate scale (src/kkt.jl:3670-3708)
      if (!hit) absmax(n_eq, rho_p.p, red.p + 2, st);
      absmax(n_eq, pv.p, red.p + 3, st);
    }
    d2h(h_red, red.p, 4 * sizeof(double));
    sync();
    *res = hit ? cached : std::max(h_red[0], h_red[2]);
    *rnorm = std::max(h_red[1], h_red[3]);
    mark_rho_fresh(*res);
  }
  double residual_norm_only(bool allow_cache = false) {
    double cached = 0.0;
    if (allow_cache && take_rho_cache(&cached)) return cached;
    apply_residual();
    clear_red(0, 2);
    absmax(m, rho.p, red.p, st);
    if (!n_eq) return read_red(0);
    absmax(n_eq, rho_p.p, red.p + 1, st);
    d2h(h_red, red.p, 2 * sizeof(double));
    sync();
    return std::max(h_red[0], h_red[1]);
  }
  void refine(int policy, double tol, int cap, int fixed_steps, int* steps_out, double* res_out) {
    PhaseScope ps(this, 3);
    auto correction = [&]() {  // `_apply_kkt_correction!` (src/kkt.jl:3762-3780)
      d2d(dxbest.p, dx.p, m * sizeof(double));
      if (n_eq) d2d(dybest.p, dyv.p, n_eq * sizeof(double));
      d2d(work_m.p, rho.p, m * sizeof(double));
      solve_kkt_into(work_m.p, rho_p.p, eq_ddy.p);
      combine(m, dx.p, 1.0, work_m.p, st);
      if (n_eq) combine(n_eq, dyv.p, 1.0, eq_ddy.p, st);
      dx_written();
    };
    int steps = 0;
    double residual;
    if (precision == SDPX_B200_MIXED && mixed) {
      // `_refine_mixed_direction!` (src/kernels/mixed_precision_kkt.jl:1634-1680)
      double rel = tol > 0 ? tol : 64.0 * kEps;
      clear_red(1, 1);
      absmax(m, r.p, red.p + 1, st);
      double abstol = rel * std::max(read_red(1), 1.0);
      residual = residual_norm_only(true);
      bool consistent = true;
      for (int s = 0; s < 32; ++s) {
        if (residual <= abstol) break;
        correction();
        double corr = residual_norm_only();
        if (!std::isfinite(corr) || corr >= residual) {
          restore_dx_best();
          consistent = false;
          break;
        }
        ++steps;
        residual = corr;
      }
      if (consistent) mark_rho_fresh(residual);
      *steps_out = steps;
      *res_out = residual;
      return;
    }
    bool consistent = true;
    if (policy == 0) {
      residual = residual_norm_only(true);
      for (int s = 0; s < fixed_steps; ++s) {
        correction();
        double corr = residual_norm_only();
        if (!std::isfinite(corr) || corr > residual) {
          restore_dx_best();
          consistent = false;
          break;
        }
        ++steps;
        residual = corr;
      }
    } else {
      if (cap <= 0) {
        *steps_out = 0;
        *res_out = 0.0;
        return;
      }
      double rel = tol > 0 ? tol : 64.0 * kEps;
      clear_red(1, 1);
      absmax(m, r.p, red.p + 1, st);
      double rn = read_red(1);
      double abstol = rel * std::max(rn, 1.0);
      residual = residual_norm_only(true);
      for (int s = 0; s < cap; ++s) {
        if (residual <= abstol) break;
        correction();
        double corr = residual_norm_only();
        if (!std::isfinite(corr) || corr > residual) {
          restore_dx_best();
          consistent = false;
          break;
        }
        ++steps;
        bool small = corr > residual * 0.5;
        residual = corr;
        if (small) break;
      }
    }
    if (consistent) mark_rho_fresh(residual);
    *steps_out = steps;
    *res_out = residual;
  }

  // -------------------------------------------------------- right sides ---
  void rhs_from_R() {
    // Z = X⁻¹(P·Y − R); v = 𝒜ᵀ vec(Z); r = −(d + v)
    for (auto& b : dense) d2d(T1.p + b.off, R.p + b.off, sizeof(double) * b.k * b.k);
    blk_gemm_all([&](const DenseBlk& b) { return blk_as_A(P.p, b.off, b.k); }, false,
                 [&](const DenseBlk& b) { return blk_as_B(Y.p, b.off, b.k); }, true, T1.p, 1.0,
                 -1.0, KR_FULL);  // T1 = P·Y − R
    dense_cholsolve(T1.p, Z.p);
    diag_rhs_Z(nd, od, P.p, Y.p, R.p, LX.p, Z.p, st);
    atmul(Z.p, -1.0, d.p, -1.0, r.p);  // r = −v − d
  }
  void rhs_predictor() {
    PhaseScope ps(this, 4);
    rhs_from_R();
  }
  void rhs_corrector_mehrotra(double sigma, double mu, int block_local) {
    PhaseScope ps(this, 4);
    std::vector<double> target(L, sigma * mu);
    if (block_local) {
      std::vector<double> dots(L);
      seg_dot(d_uoff.p, d_ulen.p, L, seg_parts, X.p, nullptr, 0.0, Y.p, nullptr, 0.0, seg_part.p,
              work_L.p, st);
      d2h(dots.data(), work_L.p, L * sizeof(double));
      sync();
      for (int l = 0; l < L; ++l) target[l] = sigma * dots[l] / k[l];
    }
    build_corrector_R(target);
    rhs_from_R();
  }
  void rhs_corrector_fixed(double beta, const double* mu) {
    PhaseScope ps(this, 4);
    std::vector<double> aff(L), target(L);
    seg_dot(d_uoff.p, d_ulen.p, L, seg_parts, X.p, dX.p, 1.0, Y.p, dY.p, 1.0, seg_part.p,
            work_L.p, st);
    d2h(aff.data(), work_L.p, L * sizeof(double));
    sync();
    for (int l = 0; l < L; ++l) {
      double rl = aff[l] / mu[l] / k[l];
      double gl = std::max(rl < 1 ? rl * rl : rl, beta);
      target[l] = gl * mu[l];
    }
    build_corrector_R(target);
    rhs_from_R();
  }
  void build_corrector_R(const std::vector<double>& target) {
    // R = target·I − X·Y − dX·dY
    blk_gemm_all([&](const DenseBlk& b) { return blk_as_A(X.p, b.off, b.k); }, false,
                 [&](const DenseBlk& b) { return blk_as_B(Y.p, b.off, b.k); }, true, R.p, -1.0, 0.0,
                 KR_FULL);
    blk_gemm_all([&](const DenseBlk& b) { return blk_as_A(dX.p, b.off, b.k); }, false,
                 [&](const DenseBlk& b) { return blk_as_B(dY.p, b.off, b.k); }, true, R.p, -1.0,
                 1.0, KR_FULL);
    if (!dense.empty()) {
      std::vector<double> sh(dense.size());
      for (size_t b = 0; b < dense.size(); ++b) sh[b] = target[dense[b].user];
      h2d(work_L.p, sh.data(), sh.size() * sizeof(double));
      add_diag(d_doff.p, d_dk.p, (int)dense.size(), kmax, R.p, work_L.p, 0.0, st);
    }
    h2d(target_user.p, target.data(), L * sizeof(double));
    diag_corrector_R(nd, od, X.p, Y.p, dX.p, dY.p, target_user.p, d_diag_user.p, R.p, st);
  }
  void set_rhs(int which) {
    if (which == 0) atmul(Cst.p, 1.0, nullptr, 0.0, r.p);
    else d2d(r.p, c.p, m * sizeof(double));
    // equality right-hand side: b for the primal solve, 0 for the dual one
    // (src/solver/interior_point.jl:817-861)
    if (n_eq) {
      if (which == 0) d2d(pv.p, beq.p, n_eq * sizeof(double));
      else pv.zero(st);
    }
  }

  // ---------------------------------------------------------- directions --
  void direction_blocks() {
    PhaseScope ps(this, 4);
    adx_current();
    axpbypcz(K, 1.0, adx.p, 1.0, P.p, 0.0, nullptr, dX.p, st);  // dX = 𝒜dx + P
    for (auto& b : dense) d2d(T1.p + b.off, R.p + b.off, sizeof(double) * b.k * b.k);
    blk_gemm_all([&](const DenseBlk& b) { return blk_as_A(dX.p, b.off, b.k); }, false,
                 [&](const DenseBlk& b) { return blk_as_B(Y.p, b.off, b.k); }, true, T1.p, -1.0,
                 1.0, KR_FULL);  // T1 = R − dX·Y
    dense_cholsolve(T1.p, dY.p);
    if (!dense.empty()) symmetrize(d_doff.p, d_dk.p, (int)dense.size(), kmax, dY.p, st);
    diag_dY(nd, od, R.p, dX.p, Y.p, LX.p, dY.p, st);
  }

  // ------------------------------------------------- step length helpers --
  // Host copies of the k = 2 blocks (closed-form tests as in the reference).
  struct Small2 {
    double X[4], dX[4];
  };
  std::vector<Small2> fetch_k2(const double* M, const double* dM) {
    std::vector<Small2> out;
    for (auto& b : dense) {
      if (b.k != 2) continue;
      Small2 s;
      d2h(s.X, M + b.off, 4 * sizeof(double));
      d2h(s.dX, dM + b.off, 4 * sizeof(double));
      out.push_back(s);
    }
    if (!out.empty()) sync();
    return out;
  }
  static bool isposdef2(const Small2& s, double t) {
    double a = s.X[0] + t * s.dX[0];
    if (!(a > 0)) return false;
    double bb = s.X[1] + t * s.dX[1];
    double dd = s.X[3] + t * s.dX[3];
    return a * dd > bb * bb;
  }
  static bool margin2(const Small2& s, double t, double ratio) {
    if (!(ratio > 0)) return isposdef2(s, t);
    double a = s.X[0] + t * s.dX[0];
    double a21 = s.X[1] + t * s.dX[1];
    double a22 = s.X[3] + t * s.dX[3];
    if (!(a > 0)) return false;
    double l11 = std::sqrt(a), l21 = a21 / l11, d22 = a22 - l21 * l21;
    if (!(d22 > 0)) return false;
    double l22 = std::sqrt(d22);
    double lo = std::min(std::fabs(l11), std::fabs(l22)), hi = std::max(std::fabs(l11), std::fabs(l22));
    return std::isfinite(lo) && std::isfinite(hi) && hi > 0 && lo > ratio * hi;
  }
  static double ftb2(const Small2& s) {
    // src/kernels/generic.jl:358-398 (2×2 closed form, bisection fallback)
    double a = s.X[0], bb = s.X[2], dd = s.X[3];
    double da = s.dX[0], db = (s.dX[2] + s.dX[1]) / 2.0, ddd = s.dX[3];
    double a1 = a + da, b1 = bb + db, d1 = dd + ddd;
    if (a1 > 0 && a1 * d1 > b1 * b1) return 1.0;
    double c0 = a * dd - bb * bb;
    double c1 = da * dd + a * ddd - 2.0 * bb * db;
    double c2 = da * ddd - db * db;
    double root = 1.0;
    bool found = false;
    if (c2 == 0) {
      if (c1 < 0) {
        double cand = -c0 / c1;
        if (0 < cand && cand <= 1) root = cand, found = true;
      }
    } else {
      double disc = c1 * c1 - 4.0 * c2 * c0;
      if (disc >= 0) {
        double sd = std::sqrt(disc), den = 2.0 * c2;
        double q1 = (-c1 - sd) / den, q2 = (-c1 + sd) / den;
        if (0 < q1 && q1 <= root) root = q1, found = true;
        if (0 < q2 && q2 <= root) root = q2, found = true;
      }
    }
    if (found) return root;
    double lo = 0.0, hi = 1.0;
    for (int i = 0; i < 64; ++i) {
      double mid = (lo + hi) / 2.0;
      if (isposdef2(s, mid)) lo = mid;
      else hi = mid;
    }
    return lo;
  }

  // PD(+margin) tests of X_b + t·dX_b for every dense block with k > 2 and
  // every candidate t; returns pass[cand] (all blocks pass).
  std::vector<char> dense_trials(const double* M, const double* dM, const std::vector<double>& t,
                                 double ratio) {
    std::vector<char> pass(t.size(), 1);
    std::vector<int> idx;
    for (size_t b = 0; b < dense.size(); ++b)
      if (dense[b].k > 2) idx.push_back((int)b);
    if (idx.empty() || t.empty()) return pass;
    // trial buffer: per block, |t| matrices
    std::vector<long long> toff(dense.size(), 0);
    long long need = 0;
    for (size_t b = 0; b < dense.size(); ++b)
      toff[b] = need, need += (long long)t.size() * dense[b].k * dense[b].k;
    if ((size_t)need > trials.n) trials.alloc(need);
    if (d_trial_off.n < dense.size()) d_trial_off.alloc(dense.size());
    h2d(d_trial_off.p, toff.data(), dense.size() * sizeof(long long));
    if (d_tcand.n < t.size()) d_tcand.alloc(t.size());
    h2d(d_tcand.p, t.data(), t.size() * sizeof(double));
    make_trials(d_doff.p, d_dk.p, d_trial_off.p, (int)dense.size(), kmax, M, dM, d_tcand.p,
                (int)t.size(), trials.p, st);
    // (blocks with k ≤ 2 also get trial copies above; they are ignored here)
    std::vector<MatDesc<double>> mats;
    for (int b : idx)
      for (size_t c2 = 0; c2 < t.size(); ++c2)
        mats.push_back({trials.p + toff[b] + (long long)c2 * dense[b].k * dense[b].k, dense[b].k,
                        dense[b].k});
    std::vector<int> info;
    std::vector<double> dmn, dmx;
    potrf_host_list(mats, info, dmn, dmx, false);
    size_t q = 0;
    for (size_t bi = 0; bi < idx.size(); ++bi)
      for (size_t c2 = 0; c2 < t.size(); ++c2, ++q) {
        bool ok = info[q] == 0;
        if (ok && ratio > 0)
          ok = std::isfinite(dmn[q]) && std::isfinite(dmx[q]) && dmx[q] > 0 && dmn[q] > ratio * dmx[q];
        if (!ok) pass[c2] = 0;
      }
    return pass;
  }
  std::vector<char> diag_trials(const double* M, const double* dM, const std::vector<double>& t,
                                double ratio) {
    std::vector<char> pass(t.size(), 1);
    if (!nd || t.empty()) return pass;
    if (d_tcand.n < t.size()) d_tcand.alloc(t.size());
    if (d_fail.n < t.size()) d_fail.alloc(t.size());
    h2d(d_tcand.p, t.data(), t.size() * sizeof(double));
    SDPX_CUDA(cudaMemsetAsync(d_fail.p, 0, t.size() * sizeof(int), st));
    diag_trial(nd, od, M, dM, d_tcand.p, (int)t.size(), ratio > 0 ? 1 : 0, d_fail.p, st);
    std::vector<int> f(t.size());
    d2h(f.data(), d_fail.p, t.size() * sizeof(int));
    sync();
    for (size_t c2 = 0; c2 < t.size(); ++c2) pass[c2] = f[c2] == 0;
    return pass;
  }
  std::vector<char> all_trials(const double* M, const double* dM, const std::vector<double>& t,
                               double ratio, const std::vector<Small2>& k2) {
    auto p1 = dense_trials(M, dM, t, ratio);
    auto p2 = diag_trials(M, dM, t, ratio);
    for (size_t c2 = 0; c2 < t.size(); ++c2) {
      bool ok = p1[c2] && p2[c2];
      for (auto& s : k2) ok = ok && margin2(s, t[c2], ratio);
      p1[c2] = ok;
    }
    return p1;
  }

  // One trial matrix  out = M_b + t·dM_b  of dense block b (side-specific M, dM).
  struct TrialReq {
    const double* M;
    const double* dM;
    int b;
    double t;
  };
  // Build all requested trial matrices, factor them in one batch and return
  // (info == 0, min |L_ii|, max |L_ii|) per request.
  void run_trials(const std::vector<TrialReq>& reqs, std::vector<int>& info,
                  std::vector<double>& dmn, std::vector<double>& dmx) {
    size_t n = reqs.size();
    info.clear();
    dmn.clear();
    dmx.clear();
    if (n == 0) return;
    std::vector<long long> off(n);
    long long need = 0;
    int nmax = 0;
    for (size_t q = 0; q < n; ++q) {
      int kk = dense[reqs[q].b].k;
      off[q] = need;
      need += (long long)kk * kk;
      nmax = std::max(nmax, kk);
    }
    if ((size_t)need > trials.n) trials.alloc(std::max<size_t>(need, trials.n * 2));
    std::vector<TrialDesc> td(n);
    for (size_t q = 0; q < n; ++q) {
      const DenseBlk& B = dense[reqs[q].b];
      td[q] = {reqs[q].M + B.off, reqs[q].dM + B.off, trials.p + off[q], reqs[q].t, B.k};
    }
    if (d_trial_desc.n < n) d_trial_desc.alloc(std::max<size_t>(n, 2 * d_trial_desc.n));
    // Staged at the end of the pinned area: potrf_host_list below uses its
    // start, and this copy is ordered before that call's final sync.
    const size_t tail = (n * (sizeof(MatDesc<double>) + 2 * sizeof(double) + sizeof(int)) + 64 + 15) / 16 * 16;
    unsigned char* hp = pinned(tail + n * sizeof(TrialDesc)) + tail;
    std::memcpy(hp, td.data(), n * sizeof(TrialDesc));
    h2d(d_trial_desc.p, hp, n * sizeof(TrialDesc));
    make_trials_list(d_trial_desc.p, (int)n, nmax, st);
    std::vector<MatDesc<double>> mats(n);
    for (size_t q = 0; q < n; ++q) mats[q] = {trials.p + off[q], dense[reqs[q].b].k, dense[reqs[q].b].k};
    potrf_host_list(mats, info, dmn, dmx, false);
  }

  // Fraction-to-boundary bounds of both sides (src/kernels/generic.jl:350-422):
  // closed forms for 1×1 and 2×2 blocks, otherwise a full-step Cholesky test
  // followed by 64 bisection steps.  Every (side, block) bisection advances in
  // the same rounds: each round factors, in one batch, the complete 4-level
  // subtree of midpoints of every unfinished interval, and the sequential
  // bisection path is replayed through it — the result equals the sequential one.
  long long ftb_rounds = 0, ftb_trials = 0;  // batched trial rounds / trials of the bisections
  void ftb_bounds(double* boundX, double* boundY) {
    double b2[2] = {1.0, 1.0};
    const double* Ms[2] = {X.p, Y.p};
    const double* dMs[2] = {dX.p, dY.p};
    for (int side = 0; side < 2; ++side) {
      if (nd) {
        diag_ftb(nd, od, Ms[side], dMs[side], red.p + 8 + side, st);
      }
      for (auto& s2 : fetch_k2(Ms[side], dMs[side])) b2[side] = std::min(b2[side], ftb2(s2));
    }
    if (nd) {
      d2h(h_red + 8, red.p + 8, 2 * sizeof(double));
      sync();
      b2[0] = std::min(b2[0], h_red[8]);
      b2[1] = std::min(b2[1], h_red[9]);
    }
    struct Bis {
      int side, b;
      double lo = 0.0, hi = 1.0;
      int done = 0;
      bool first = true, finished = false;
      double result = 1.0;
    };
    std::vector<Bis> probs;
    for (int side = 0; side < 2; ++side)
      for (size_t b = 0; b < dense.size(); ++b)
        if (dense[b].k > 2) {
          Bis q;
          q.side = side;
          q.b = (int)b;
          probs.push_back(q);
        }
    // Each round evaluates a complete tree of the next `depth` bisection steps
    // of every unfinished problem in one batched Cholesky; the deepest tree
    // that keeps the batch within about one trial matrix per SM is used (a
    // round costs about the same for any batch up to one wave).
    while (true) {
      int active = 0;
      for (auto& P : probs) active += P.finished ? 0 : 1;
      int DEPTH = 4;
      while (DEPTH < 7 && active * ((1 << (DEPTH + 1)) - 1) <= sms - 16) ++DEPTH;
      std::vector<TrialReq> reqs;
      std::vector<std::vector<double>> pts(probs.size());
      std::vector<size_t> first_req(probs.size());
      for (size_t q = 0; q < probs.size(); ++q) {
        Bis& P = probs[q];
        if (P.finished) continue;
        int depth = std::min(DEPTH, 64 - P.done);
        int npts = (1 << depth) - 1;
        std::vector<double> los(npts), his(npts);
        pts[q].assign(npts, 0.0);
        los[0] = P.lo;
        his[0] = P.hi;
        for (int n2 = 0; n2 < npts; ++n2) {
          pts[q][n2] = (los[n2] + his[n2]) / 2.0;
          int l2 = 2 * n2 + 1, r2 = 2 * n2 + 2;
          if (l2 < npts) los[l2] = los[n2], his[l2] = pts[q][n2];
          if (r2 < npts) los[r2] = pts[q][n2], his[r2] = his[n2];
        }
        first_req[q] = reqs.size();
        for (double t : pts[q]) reqs.push_back({Ms[P.side], dMs[P.side], P.b, t});
        if (P.first) reqs.push_back({Ms[P.side], dMs[P.side], P.b, 1.0});
      }
      if (reqs.empty()) break;
      std::vector<int> info;
      std::vector<double> dmn, dmx;
      run_trials(reqs, info, dmn, dmx);
      ++ftb_rounds;
      ftb_trials += (long long)reqs.size();
      for (size_t q = 0; q < probs.size(); ++q) {
        Bis& P = probs[q];
        if (P.finished) continue;
        const size_t f = first_req[q];
        const int npts = (int)pts[q].size();
        if (P.first) {
          P.first = false;
          if (info[f + npts] == 0) {  // full step stays positive definite
            P.finished = true;
            P.result = 1.0;
            continue;
          }
        }
        int node = 0, depth = 0;
        while (node < npts) {
          double mid = pts[q][node];
          if (info[f + node] == 0) {
            P.lo = mid;
            node = 2 * node + 2;
          } else {
            P.hi = mid;
            node = 2 * node + 1;
          }
          ++depth;
        }
        P.done += depth;
        // Once [lo, hi] holds no double strictly inside, every remaining
        // midpoint equals hi (a failing point: the full step or a failed trial)
        // or lo > 0 (a passing trial), so the remaining steps leave lo as it is.
        const double mid = (P.lo + P.hi) / 2.0;
        if (P.done >= 64 || mid == P.hi || (mid == P.lo && P.lo > 0.0)) {
          P.finished = true;
          P.result = P.lo;
        }
      }
    }
    for (auto& P : probs) b2[P.side] = std::min(b2[P.side], P.result);
    *boundX = b2[0];
    *boundY = b2[1];
  }

  void affine_diagnostics(int adaptive, double* out, double* block_compl) {
    PhaseScope ps(this, 5);
    double tX = 1.0, tY = 1.0;
    if (adaptive) {
      double bX, bY;
      ftb_bounds(&bX, &bY);
      tX = bX < 1 ? bX : 1.0;
      tY = bY < 1 ? bY : 1.0;
    }
    std::vector<double> c12(2 * (size_t)L);
    seg_dot(d_uoff.p, d_ulen.p, L, seg_parts, X.p, nullptr, 0.0, Y.p, nullptr, 0.0, seg_part.p,
            work_L.p, st);
    seg_dot(d_uoff.p, d_ulen.p, L, seg_parts, X.p, dX.p, tX, Y.p, dY.p, tY, seg_part.p,
            work_L.p + L, st);
    d2h(c12.data(), work_L.p, 2 * L * sizeof(double));  // both in one read-back
    sync();
    const double* c1 = c12.data();
    const double* c2 = c12.data() + L;
    double s1 = 0, s2 = 0;
    for (int l = 0; l < L; ++l) s1 += c1[l], s2 += c2[l];
    out[0] = s1;
    out[1] = s2;
    out[2] = tX;
    out[3] = tY;
    if (block_compl) std::memcpy(block_compl, c1, L * sizeof(double));
  }

  void line_search(int rule, double fp, double fd, double gamma, double min_step, double margin,
                   double* tX_out, double* tY_out) {
    PhaseScope ps(this, 5);
    if (rule == 1) {
      double bX, bY;
      ftb_bounds(&bX, &bY);
      *tX_out = bX < 1 ? fp * bX : 1.0;
      *tY_out = bY < 1 ? fd * bY : 1.0;
      return;
    }
    // Backtracking (src/kernels/threaded.jl:1751-1818): the first t in 1, γ, γ², …
    // whose trial passes every block (Cholesky + diagonal-ratio margin), or the
    // first t below min_step.  Candidates of both sides are factored together,
    // eight per side per round.
    const double* Ms[2] = {X.p, Y.p};
    const double* dMs[2] = {dX.p, dY.p};
    std::vector<Small2> k2[2] = {fetch_k2(X.p, dX.p), fetch_k2(Y.p, dY.p)};
    double t_next[2] = {1.0, 1.0};
    double result[2] = {1.0, 1.0};
    bool done[2] = {false, false};
    constexpr int J = 8;
    while (!(done[0] && done[1])) {
      std::vector<double> cand[2];
      for (int side = 0; side < 2; ++side) {
        if (done[side]) continue;
        double tt = t_next[side];
        for (int j = 0; j < J; ++j) {
          cand[side].push_back(tt);
          if (tt < min_step) break;
          tt *= gamma;
        }
      }
      // dense blocks with k > 2: one batch for both sides
      std::vector<TrialReq> reqs;
      std::vector<int> big;
      for (size_t b = 0; b < dense.size(); ++b)
        if (dense[b].k > 2) big.push_back((int)b);
      for (int side = 0; side < 2; ++side)
        for (int b : big)
          for (double t : cand[side]) reqs.push_back({Ms[side], dMs[side], b, t});
      std::vector<int> info;
      std::vector<double> dmn, dmx;
      run_trials(reqs, info, dmn, dmx);
      size_t q = 0;
      for (int side = 0; side < 2; ++side) {
        if (done[side]) continue;
        std::vector<char> pass(cand[side].size(), 1);
        for (size_t bi = 0; bi < big.size(); ++bi)
          for (size_t c2 = 0; c2 < cand[side].size(); ++c2, ++q) {
            bool ok = info[q] == 0;
            if (ok && margin > 0)
              ok = std::isfinite(dmn[q]) && std::isfinite(dmx[q]) && dmx[q] > 0 &&
                   dmn[q] > margin * dmx[q];
            if (!ok) pass[c2] = 0;
          }
        auto pd = diag_trials(Ms[side], dMs[side], cand[side], margin);
        for (size_t c2 = 0; c2 < cand[side].size(); ++c2) {
          bool ok = pass[c2] && pd[c2];
          for (auto& s2 : k2[side]) ok = ok && margin2(s2, cand[side][c2], margin);
          if (ok || cand[side][c2] < min_step) {
            result[side] = cand[side][c2];
            done[side] = true;
            break;
          }
        }
        if (!done[side]) t_next[side] = cand[side].back() * gamma;
      }
    }
    *tX_out = result[0];
    *tY_out = result[1];
  }

  // -------------------------------------------------------------- update --
  void update(double tX, double tY, double* compl_total, int* finite, double* block_dots) {
    PhaseScope ps(this, 6);
    combine(K, X.p, tX, dX.p, st);
    combine(K, Y.p, tY, dY.p, st);
    combine(m, x.p, tX, dx.p, st);
    if (n_eq) combine(n_eq, yv.p, tY, dyv.p, st);  // src/solver/interior_point.jl:2228-2229
    std::vector<double> dots(L);
    seg_dot(d_uoff.p, d_ulen.p, L, seg_parts, X.p, nullptr, 0.0, Y.p, nullptr, 0.0, seg_part.p,
            work_L.p, st);
    d2h(dots.data(), work_L.p, L * sizeof(double));
    clear_red(0, 4);
    absmax(K, X.p, red.p + 0, st);
    absmax(K, Y.p, red.p + 1, st);
    absmax(m, x.p, red.p + 2, st);
    if (n_eq) absmax(n_eq, yv.p, red.p + 3, st);
    d2h(h_red, red.p, 4 * sizeof(double));
    sync();
    double s = 0;
    for (int l = 0; l < L; ++l) s += dots[l];
    *compl_total = s;
    *finite = std::isfinite(h_red[0]) && std::isfinite(h_red[1]) && std::isfinite(h_red[2]) &&
              std::isfinite(h_red[3]);
    if (block_dots) std::memcpy(block_dots, dots.data(), L * sizeof(double));
  }
  void accepted_residuals(double bpr, double tX, double tY, double* pa, double* da) {
    *pa = std::fabs(1.0 - tX) * bpr;
    axpbypcz(m, 1.0 - tY, d.p, -tY, rho.p, 0.0, nullptr, d.p, st);
    clear_red(0, 2);
    absmax(m, d.p, red.p, st);
    if (n_eq) {  // p+ = (1 − tX)p + tX·ρ_p (src/solver/interior_point.jl:1298-1305)
      axpbypcz(n_eq, tX, rho_p.p, 1.0 - tX, pv.p, 0.0, nullptr, pv.p, st);
      absmax(n_eq, pv.p, red.p + 1, st);
    }
    d2h(h_red, red.p, 2 * sizeof(double));
    sync();
    *da = h_red[0];
    if (n_eq) *pa = std::max(*pa, h_red[1]);
  }
  void objectives(double* po, double* dobj) {
    std::vector<double> dots(2);
    // pObj = cᵀx ; dObj = Σ⟨C_l, Y_l⟩
    seg_dot(d_uoff.p, d_ulen.p, L, seg_parts, Cst.p, nullptr, 0.0, Y.p, nullptr, 0.0, seg_part.p,
            work_L.p, st);
    std::vector<double> cy(L);
    d2h(cy.data(), work_L.p, L * sizeof(double));
    std::vector<double> hc(m), hx(m);
    d2h(hc.data(), c.p, m * sizeof(double));
    d2h(hx.data(), x.p, m * sizeof(double));
    sync();
    double p = 0;
    for (int i = 0; i < m; ++i) p += hc[i] * hx[i];
    double dd = 0;
    for (int l = 0; l < L; ++l) dd += cy[l];
    if (n_eq) {  // + bᵀy (src/kernels/threaded.jl:833)
      eq_dot(n_eq, beq.p, yv.p, red.p, st);
      dd += read_red(0);
    }
    *po = p;
    *dobj = dd;
  }
  void solution_residuals(double* pr, double* dr) {
    primal_residual(x.p, tmpK2.p);
    dual_residual(Y.p, work_m.p);
    clear_red(0, 3);
    if (n_eq) {
      gemv_n(Beq.p, m, n_eq, yv.p, eq_tm.p, gemv_part.p, gemv_chunks, st);
      axpbypcz(m, 1.0, work_m.p, -1.0, eq_tm.p, 0.0, nullptr, work_m.p, st);
      gemv_t(Beq.p, m, n_eq, x.p, -1.0, beq.p, 1.0, eq_q.p, st);
      absmax(n_eq, eq_q.p, red.p + 2, st);
    }
    absmax(K, tmpK2.p, red.p + 0, st);
    absmax(m, work_m.p, red.p + 1, st);
    d2h(h_red, red.p, 3 * sizeof(double));
    sync();
    *pr = std::max(h_red[0], h_red[2]);
    *dr = h_red[1];
  }

  // ---------------------------------------------------------- cold start --
  void cold_start_iterate() {
    d2d(x.p, keptx.p, m * sizeof(double));
    amul(x.p, tmpK.p);
    axpbypcz(K, 1.0, tmpK.p, -1.0, Cst.p, 0.0, nullptr, X.p, st);
    amul(dx.p, Y.p);
    if (n_eq) axpbypcz(n_eq, -1.0, dyv.p, 0.0, nullptr, 0.0, nullptr, yv.p, st);  // y = −q
  }
  // Per-block certified shift (src/cold_start.jl:287-308) for all blocks at once.
  void psd_shift(int which, int* ok_out) {
    double* M = which == 0 ? X.p : Y.p;
    std::vector<double> applied(L, 0.0);
    std::vector<char> done(L, 0), bad(L, 0);
    for (int round = 0; round <= 16; ++round) {
      // stats for every block: finite, scale (max |lower|), lower eigen bound
      std::vector<double> scale(L, 0.0), margin(L, 0.0);
      std::vector<char> finite(L, 1);
      size_t nb = dense.size();
      if (nb) {
        long long tot = 0;
        for (auto& b : dense) tot += b.k;
        g_scale.zero(st);
        g_nonfinite.zero(st);
        gershgorin(d_doff.p, d_dk.p, (int)nb, kmax, M, g_cand.p, g_cand_off.p, g_scale.p,
                   g_nonfinite.p, st);
        std::vector<double> cand(tot), sc(nb);
        std::vector<int> nf(nb);
        d2h(cand.data(), g_cand.p, tot * sizeof(double));
        d2h(sc.data(), g_scale.p, nb * sizeof(double));
        d2h(nf.data(), g_nonfinite.p, nb * sizeof(int));
        sync();
        long long o = 0;
        for (size_t b = 0; b < nb; ++b) {
          int l = dense[b].user, kk = dense[b].k;
          scale[l] = sc[b];
          finite[l] = nf[b] == 0;
          double bound;
          if (kk == 2) {
            // exact eigenvalue (lower authoritative)
            double h4[4];
            d2h(h4, M + dense[b].off, 4 * sizeof(double));
            sync();
            double cc = (h4[0] + h4[3]) / 2, rr = std::hypot((h4[0] - h4[3]) / 2, h4[1]);
            bound = cc - rr;
          } else {
            bound = cand[o];
            for (int i = 1; i < kk; ++i) bound = std::min(bound, cand[o + i]);
          }
          margin[l] = bound;
          o += kk;
        }
      }
      if (nd) {
        std::vector<double> dv(nd);
        d2h(dv.data(), M + od, nd * sizeof(double));
        sync();
        for (int j = 0; j < nd; ++j) {
          int l = diag_user[j];
          finite[l] = std::isfinite(dv[j]);
          scale[l] = std::fabs(dv[j]);
          margin[l] = dv[j];
        }
      }
      // decide shifts
      std::vector<double> shifts(L, 0.0);
      bool any = false;
      for (int l = 0; l < L; ++l) {
        if (done[l] || bad[l]) continue;
        if (!finite[l]) {
          bad[l] = 1;
          continue;
        }
        double safety = kSqrtEps * std::max(1.0, scale[l]);
        if (margin[l] > safety) {
          done[l] = 1;
          continue;
        }
        if (round == 16) {
          bad[l] = 1;
          continue;
        }
        double slack = 8.0 * kEps * std::max(1.0, scale[l]);
        double sh = safety - margin[l] + slack;
        if (!std::isfinite(sh)) {
          bad[l] = 1;
          continue;
        }
        shifts[l] = sh;
        applied[l] += sh;
        any = true;
      }
      if (!any) break;
      apply_block_shifts(M, shifts);
    }
    bool ok = true;
    for (int l = 0; l < L; ++l) ok = ok && !bad[l] && done[l];
    *ok_out = ok ? 1 : 0;
  }
  void apply_block_shifts(double* M, const std::vector<double>& shifts) {
    if (!dense.empty()) {
      std::vector<double> sh(dense.size());
      for (size_t b = 0; b < dense.size(); ++b) sh[b] = shifts[dense[b].user];
      h2d(work_L.p, sh.data(), sh.size() * sizeof(double));
      add_diag(d_doff.p, d_dk.p, (int)dense.size(), kmax, M, work_L.p, 0.0, st);
    }
    if (nd) {
      std::vector<double> dv(nd);
      d2h(dv.data(), M + od, nd * sizeof(double));
      sync();
      for (int j = 0; j < nd; ++j) dv[j] += shifts[diag_user[j]];
      h2d(M + od, dv.data(), nd * sizeof(double));
    }
    sync();
  }
  void add_identity(int which, double shift) {
    std::vector<double> sh(L, shift);
    apply_block_shifts(which == 0 ? X.p : Y.p, sh);
  }
  void block_dots(double* dots, double* trX, double* trY) {
    seg_dot(d_uoff.p, d_ulen.p, L, seg_parts, X.p, nullptr, 0.0, Y.p, nullptr, 0.0, seg_part.p,
            work_L.p, st);
    d2h(dots, work_L.p, L * sizeof(double));
    sync();
    block_trace(d_uoff.p, d_uk.p, L, X.p, work_L.p, st);
    d2h(trX, work_L.p, L * sizeof(double));
    sync();
    block_trace(d_uoff.p, d_uk.p, L, Y.p, work_L.p, st);
    d2h(trY, work_L.p, L * sizeof(double));
    sync();
  }

  // -------------------------------------------------------- original data --
  void rebuild_slack(const double* hx, double* hX) {
    const double* Ause = have_original ? A0.p : A.p;
    const double* Cuse = have_original ? C0st.p : Cst.p;
    h2d(work_m.p, hx, m * sizeof(double));
    gemv_n(Ause, K, m, work_m.p, tmpK2.p, gemv_part.p, gemv_chunks, st);
    axpbypcz(K, 1.0, tmpK2.p, -1.0, Cuse, 0.0, nullptr, tmpK2.p, st);
    get_stacked(tmpK2.p, hX);
  }
  void original_residuals(const double* hx, const double* hX, const double* hY, double* pr,
                          double* dr, const double* hy = nullptr) {
    const double* Ause = have_original ? A0.p : A.p;
    const double* Cuse = have_original ? C0st.p : Cst.p;
    const double* cuse = have_original ? c0.p : c.p;
    h2d(work_m.p, hx, m * sizeof(double));
    // X → T1, Y → T2 (scratch stacked buffers)
    h2d(tmpK.p, hX, Ku * sizeof(double));
    gather(K, d_map.p, tmpK.p, T1.p, st);
    h2d(tmpK.p, hY, Ku * sizeof(double));
    gather(K, d_map.p, tmpK.p, T2.p, st);
    gemv_n(Ause, K, m, work_m.p, tmpK2.p, gemv_part.p, gemv_chunks, st);
    axpbypcz(K, 1.0, tmpK2.p, -1.0, T1.p, -1.0, Cuse, tmpK2.p, st);
    gemv_t(Ause, K, m, T2.p, -1.0, cuse, 1.0, work_m2.p, st);
    clear_red(0, 3);
    if (n_eq) {  // d −= B·y, p = b − Bᵀx on the original equality rows
      if (!hy) throw std::invalid_argument("equality multipliers y are required when n > 0");
      const double* Buse = eq_have_original ? Beq0.p : Beq.p;
      h2d(eq_z.p, hy, n_eq * sizeof(double));
      gemv_n(Buse, m, n_eq, eq_z.p, eq_tm.p, gemv_part.p, gemv_chunks, st);
      axpbypcz(m, 1.0, work_m2.p, -1.0, eq_tm.p, 0.0, nullptr, work_m2.p, st);
      gemv_t(Buse, m, n_eq, work_m.p, -1.0, beq.p, 1.0, eq_q.p, st);
      absmax(n_eq, eq_q.p, red.p + 2, st);
    }
    absmax(K, tmpK2.p, red.p + 0, st);
    absmax(m, work_m2.p, red.p + 1, st);
    d2h(h_red, red.p, 3 * sizeof(double));
    sync();
    *pr = std::max(h_red[0], h_red[2]);
    *dr = h_red[1];
  }

  // ---------------------------------------------------------- certificate --
  // Per-block PSD check of `_block_psd_certificate` (src/validation.jl:765-904).
  struct PsdDetail {
    bool ok = true, finite = true, resolved = true;
    double symmetry = 0.0, allowed = 0.0, required = 0.0;
  };
  // Lower Cholesky pass/fail of (M + Mᵀ)/2 + shift·I for a small block (host,
  // the unblocked column algorithm; a pivot that is not > 0 fails).
  static bool small_shifted_chol(const double* M, int k, double shift) {
    double S[16];
    for (int c = 0; c < k; ++c)
      for (int r = 0; r < k; ++r) S[r + c * k] = (M[r + c * k] + M[c + r * k]) / 2.0;
    for (int i = 0; i < k; ++i) S[i + i * k] += shift;
    for (int j = 0; j < k; ++j) {
      double d = S[j + j * k];
      for (int p = 0; p < j; ++p) d -= S[j + p * k] * S[j + p * k];
      if (!(d > 0.0)) return false;
      d = std::sqrt(d);
      S[j + j * k] = d;
      for (int i = j + 1; i < k; ++i) {
        double v = S[i + j * k];
        for (int p = 0; p < j; ++p) v -= S[i + p * k] * S[j + p * k];
        S[i + j * k] = v / d;
      }
    }
    return true;
  }
  // PSD details of every user block of the stacked device matrix M.
  std::vector<PsdDetail> psd_certificate(const double* M, double tol) {
    const double base = std::max(tol, 128.0 * kEps);
    std::vector<PsdDetail> det(L);
    size_t nb = dense.size();
    std::vector<double> stats(3 * nb);
    if (nb) {
      cert_block_stats(d_doff.p, d_dk.p, (int)nb, M, cert_stats.p, st);
      d2h(stats.data(), cert_stats.p, 3 * nb * sizeof(double));
    }
    std::vector<double> dv(nd);
    if (nd) d2h(dv.data(), M + od, nd * sizeof(double));
    sync();
    for (int j = 0; j < nd; ++j) {
      PsdDetail& d = det[diag_user[j]];
      d.finite = std::isfinite(dv[j]);
      d.allowed = base * std::max(std::fabs(dv[j]), 1.0);
      if (!d.finite) {
        d.ok = false;
        d.resolved = false;
        d.required = d.allowed;
        continue;
      }
      d.required = std::max(0.0, -dv[j]);
      d.ok = d.required <= d.allowed;
    }
    std::vector<size_t> chol0;
    for (size_t b = 0; b < nb; ++b) {
      PsdDetail& d = det[dense[b].user];
      const int kk = dense[b].k;
      d.finite = stats[3 * b] == 0.0;
      d.allowed = base * std::max(stats[3 * b + 1], 1.0);
      d.symmetry = stats[3 * b + 2];
      if (!d.finite) {
        d.ok = false;
        d.resolved = false;
        d.required = d.allowed;
        continue;
      }
      if (kk == 2) {
        double h4[4];
        d2h(h4, M + dense[b].off, 4 * sizeof(double));
        sync();
        double off = (h4[2] + h4[1]) / 2.0, center = (h4[0] + h4[3]) / 2.0;
        double radius = std::hypot((h4[0] - h4[3]) / 2.0, off);
        d.required = std::max(0.0, -(center - radius));
        d.ok = d.required <= d.allowed && d.symmetry <= d.allowed;
        continue;
      }
      chol0.push_back(b);
    }
    // Cholesky of the symmetrised blocks at shift 0, then at the allowed shift.
    auto factor_with = [&](const std::vector<size_t>& sel, const std::vector<double>& shift_of,
                           std::vector<int>& info) {
      std::vector<double> sh(nb, 0.0);
      for (size_t q = 0; q < sel.size(); ++q) sh[sel[q]] = shift_of[q];
      h2d(cert_shift.p, sh.data(), nb * sizeof(double));
      cert_sym_shift(d_doff.p, d_dk.p, (int)nb, kmax, M, cert_shift.p, cert_sym.p, st);
      std::vector<MatDesc<double>> mats;
      for (size_t b : sel) mats.push_back({cert_sym.p + dense[b].off, dense[b].k, dense[b].k});
      std::vector<double> dmn, dmx;
      potrf_host_list(mats, info, dmn, dmx, false);
    };
    std::vector<int> info;
    factor_with(chol0, std::vector<double>(chol0.size(), 0.0), info);
    std::vector<size_t> large_fail;
    std::vector<double> large_shift;
    for (size_t q = 0; q < chol0.size(); ++q) {
      size_t b = chol0[q];
      PsdDetail& d = det[dense[b].user];
      if (info[q] == 0) {
        d.required = 0.0;
        d.ok = d.symmetry <= d.allowed;
        continue;
      }
      const int kk = dense[b].k;
      if (kk > 4) {
        large_fail.push_back(b);
        large_shift.push_back(d.allowed);
        continue;
      }
      // order 3 or 4: allowed-shift test, doubling and 48-step bisection on the host
      double h16[16];
      d2h(h16, M + dense[b].off, kk * kk * sizeof(double));
      sync();
      bool allowed_ok = small_shifted_chol(h16, kk, d.allowed);
      double lower = 0.0, upper = d.allowed;
      bool resolved = allowed_ok;
      if (!resolved) {
        lower = upper;
        for (int it = 0; it < 64; ++it) {
          double cand = upper + upper;
          if (!std::isfinite(cand)) break;
          upper = cand;
          if (small_shifted_chol(h16, kk, upper)) {
            resolved = true;
            break;
          }
          lower = upper;
        }
      }
      if (resolved)
        for (int it = 0; it < 48; ++it) {
          double mid = (lower + upper) / 2.0;
          if (small_shifted_chol(h16, kk, mid))
            upper = mid;
          else
            lower = mid;
        }
      d.ok = allowed_ok && d.symmetry <= d.allowed;
      d.required = upper;
      d.resolved = resolved;
    }
    if (!large_fail.empty()) {
      factor_with(large_fail, large_shift, info);
      for (size_t q = 0; q < large_fail.size(); ++q) {
        PsdDetail& d = det[dense[large_fail[q]].user];
        d.ok = info[q] == 0 && d.symmetry <= d.allowed;
        d.required = d.allowed;
        d.resolved = false;
      }
    }
    return det;
  }
  static double psd_violation(const std::vector<PsdDetail>& det, int* failing) {
    double v = 0.0;
    *failing = 0;
    for (const auto& d : det) {
      if (d.ok) continue;
      ++*failing;
      if (!d.finite) v = INFINITY;
      if (std::isinf(v)) continue;
      double excess = std::max(0.0, d.symmetry - d.allowed);
      double shift = d.resolved ? d.required : d.allowed;
      v = std::max(v, std::max(excess, shift));
    }
    return v;
  }

  void certificate(const double* hx, const double* hX, const double* hY, double ep, double ed,
                   double eg, int legacy, sdpx_b200_certificate_result* out,
                   const double* hy = nullptr) {
    const double* Ause = have_original ? A0.p : A.p;
    const double* Cuse = have_original ? C0st.p : Cst.p;
    const double* cuse = have_original ? c0.p : c.p;
    if (cert_rows.n < (size_t)(3 * K)) {
      cert_part.alloc((size_t)3 * gemv_chunks * K);
      cert_rows.alloc((size_t)3 * K);
      cert_cols.alloc((size_t)3 * m);
      cert_sym.alloc(K);
      cert_stats.alloc(3 * std::max<size_t>(dense.size(), 1));
      cert_shift.alloc(std::max<size_t>(dense.size(), 1));
    }
    h2d(work_m.p, hx, m * sizeof(double));
    h2d(tmpK.p, hX, Ku * sizeof(double));
    gather(K, d_map.p, tmpK.p, T1.p, st);
    h2d(tmpK.p, hY, Ku * sizeof(double));
    gather(K, d_map.p, tmpK.p, T2.p, st);
    double* rows = cert_rows.p;
    double* cols = cert_cols.p;
    cert_primal_rows(Ause, K, m, work_m.p, T1.p, Cuse, cert_part.p, gemv_chunks, rows, rows + K,
                     rows + 2 * K, st);
    // Equality rows (n > 0): their terms of the dual residual and backward
    // errors, the equality backward errors and bᵀy (src/validation.jl:454-482,
    // 629-644, 666-740; `dual_objective`, src/solver/interior_point.jl:7-14).
    const double* Buse = eq_have_original ? Beq0.p : Beq.p;
    if (n_eq) {
      if (!hy) throw std::invalid_argument("equality multipliers y are required when n > 0");
      h2d(eq_z.p, hy, n_eq * sizeof(double));
    }
    cert_dual_cols(Ause, K, m, T2.p, cuse, cols, cols + m, cols + 2 * m, st,
                   n_eq ? Buse : nullptr, n_eq, n_eq ? eq_z.p : nullptr);
    clear_red(0, 20);
    if (n_eq) {
      cert_equality_rows(Buse, m, n_eq, work_m.p, beq.p, eq_cert.p, eq_cert.p + n_eq,
                         eq_cert.p + 2 * n_eq, st);
      absmax(n_eq, eq_cert.p, red.p + 14, st);
      absmax(n_eq, eq_cert.p + n_eq, red.p + 15, st);
      absmax(n_eq, eq_cert.p + 2 * n_eq, red.p + 16, st);
      absmax(n_eq, beq.p, red.p + 17, st);
      cert_dot(n_eq, eq_z.p, beq.p, red.p + 18, st);  // bᵀy, non-finite y
    }
    absmax(K, rows, red.p + 0, st);
    absmax(K, rows + K, red.p + 1, st);
    absmax(K, rows + 2 * K, red.p + 2, st);
    absmax(m, cols, red.p + 3, st);
    absmax(m, cols + m, red.p + 4, st);
    absmax(m, cols + 2 * m, red.p + 5, st);
    absmax(K, Cuse, red.p + 6, st);
    absmax(m, cuse, red.p + 7, st);
    cert_dot(m, work_m.p, cuse, red.p + 8, st);  // c·x, non-finite x
    cert_dot(K, T2.p, Cuse, red.p + 10, st);     // Σ⟨C_l, Y_l⟩, non-finite Y
    cert_dot(K, T1.p, T2.p, red.p + 12, st);     // Σ⟨X_l, Y_l⟩, non-finite X
    double r[20];
    d2h(r, red.p, sizeof(r));
    sync();
    int pfail = 0, dfail = 0;
    double pviol = psd_violation(psd_certificate(T1.p, std::max(ep, eg)), &pfail);
    double dviol = psd_violation(psd_certificate(T2.p, std::max(ed, eg)), &dfail);

    sdpx_b200_certificate_result cr{};
    cr.primal_objective = r[8];
    cr.dual_objective = r[10] + r[18];
    cr.gap = cr.primal_objective - cr.dual_objective;
    double oscale =
        std::max(1.0, (std::fabs(cr.primal_objective) + std::fabs(cr.dual_objective)) / 2.0);
    cr.gap_relative = std::fabs(cr.gap) / oscale;
    cr.complementarity = r[12];
    cr.complementarity_relative = std::fabs(cr.complementarity) / oscale;
    cr.primal_affine_residual = std::max(r[0], r[14]);
    cr.dual_affine_residual = r[3];
    cr.primal_cone_violation = pviol;
    cr.dual_cone_violation = dviol;
    cr.primal_residual = std::max(cr.primal_affine_residual, pviol);
    cr.dual_residual = std::max(r[3], dviol);
    cr.primal_residual_scaled = cr.primal_residual / (1.0 + std::max(r[6], r[17]));
    cr.dual_residual_scaled = cr.dual_residual / (1.0 + r[7]);
    cr.equality_backward_error = r[15];
    cr.equality_strict_backward_error = r[16];
    cr.primal_block_backward_error = r[1];
    cr.primal_block_strict_backward_error = r[2];
    cr.dual_backward_error = r[4];
    cr.dual_strict_backward_error = r[5];
    cr.primal_psd_failing_blocks = pfail;
    cr.dual_psd_failing_blocks = dfail;
    bool primal_finite = std::isfinite(cr.primal_objective) && std::isfinite(cr.primal_residual) &&
                         r[9] == 0.0 && r[13] == 0.0;
    bool dual_finite = std::isfinite(cr.dual_objective) && std::isfinite(cr.dual_residual) &&
                       r[11] == 0.0 && r[19] == 0.0;
    bool finite = primal_finite && dual_finite && std::isfinite(cr.gap_relative) &&
                  std::isfinite(cr.complementarity);
    bool gap_ok = legacy ? (0.0 <= cr.gap && cr.gap <= eg) : (cr.gap_relative <= eg);
    int f = 0;
    if (!finite) f |= SDPX_B200_CERT_NONFINITE;
    if (!(cr.primal_residual_scaled <= ep)) f |= SDPX_B200_CERT_PRIMAL_RESIDUAL;
    if (!(cr.equality_backward_error <= ep)) f |= SDPX_B200_CERT_EQUALITY_BACKWARD_ERROR;
    if (!(cr.primal_block_backward_error <= ep)) f |= SDPX_B200_CERT_PRIMAL_BLOCK_BACKWARD_ERROR;
    if (!(cr.dual_residual_scaled <= ed)) f |= SDPX_B200_CERT_DUAL_RESIDUAL;
    if (!(cr.dual_backward_error <= ed)) f |= SDPX_B200_CERT_DUAL_BACKWARD_ERROR;
    if (!gap_ok) f |= SDPX_B200_CERT_DUALITY_GAP;
    if (pfail) f |= SDPX_B200_CERT_PRIMAL_PSD;
    if (dfail) f |= SDPX_B200_CERT_DUAL_PSD;
    cr.failures = f;
    cr.valid = f == 0;
    *out = cr;
  }

  // ------------------------------------------------------- mixed precision --
  void mixed_init();
  void mixed_check_err();
  void schur_split_bf16(bool identity);
  void mixed_factorize(int* ok, int* attempts, double* quality);
  void mixed_solve(double* vec);
  void mixed_residual();

  // ------------------------------------------- equality rows (n > 0) ------
  // Bᵀx = b with B m×n column-major (SDPX's `SDPProblem.B`, `.b`), multipliers
  // y.  p = b − Bᵀx, ρ_p = p − Bᵀdx.  The equality factor is either the
  // Cholesky of Q = B̂ᵀB̂ (eq_kind 1) or the column-pivoted QR of B̂ (eq_kind
  // 2, kept for the rest of the solve once used), B̂ = L_S⁻¹B·D with D the
  // column scales.  In mixed mode L_S is the FP32 factor and Q's Cholesky takes
  // regularisation retries instead of the rank test.
  int n_eq = 0;
  DBuf<double> Beq, Beq0, beq;
  DBuf<double> yv, dyv, pv, rho_p, ybest, dybest, eq_dyh, eq_ddy, eq_q, eq_z, eq_tm;
  DBuf<double> Bt, Qf, Bqr, eq_scale, eq_rdiag, eq_colnorm, eq_partial, eq_cert;
  DBuf<int> eq_perm, eq_pairs, eq_equal;
  DBuf<unsigned long long> eq_fp;
  SyrkPlan eq_syrk;
  bool eq_have_original = false;
  double eq_requested = kSqrtEps;
  int eq_solver = 0;  // 0 = automatic, 1 = rank-revealing QR from the start
  int eq_kind = 0;    // 0 = none, 1 = normal equations, 2 = rank-revealing QR
  int eq_rank = 0;
  double eq_quality = 0.0;
  bool eq_qr_sticky = false;
  void set_equality(int n, const double* hB, const double* hb);
  bool factor_equality(bool* rank_deficient);
  bool factor_equality_mixed(double* cond_q, double* quality_q);
  // ------------------------------------------------ adjoint (adjoint_api.inc)
  DBuf<double> adj_D, adj_W, adj_G, adj_L, adj_Z, adj_zero, adj_w, adj_p, adj_dy;
  void adj_xinv_m_y(const double* Mst, double* Zout);
  // Double-double (Float64x2) workspace of the refined adjoint: pairs
  // (hi, lo) of stacked K-vectors and m-vectors.
  DBuf<double> ddXi_h, ddXi_l, ddT_h, ddT_l, ddU_h, ddU_l, ddV_h, ddV_l, ddD_h, ddD_l;
  DBuf<double> ddp_h, ddp_l, ddw_h, ddw_l, ddlam_h, ddlam_l, ddu_h, ddu_l, ddlb_h, ddlb_l;
  DBuf<double> ddcg_ph, ddcg_pl, ddcg_qh, ddcg_ql;  // conjugate-gradient directions
  void dd_prepare_inverse();
  void dd_xinv_m_y(const double* Mh, const double* Ml, double* Zh, double* Zl);
  void dd_schur_apply(const double* vh, const double* vl, double* oh, double* ol);
  void adjoint_refined(const double* hwx, const double* hWX, const double* hWY, double* gc,
                       double* gC, int nA, const int32_t* Aidx, double* gA, int steps,
                       double* residual);
  void adjoint(const double* hwx, const double* hwy, const double* hWX, const double* hWY,
               double* gc, double* gb, double* gC, int nA, const int32_t* Aidx, double* gA);
  void equality_panel(const double* Li);
  DBuf<double> Qs;
  void solve_kkt_into(double* vec, const double* prhs, double* dy_out);
  void eq_residual_terms();
};

}  // namespace sdpx

// Mixed-precision members live in mixed_api.inc, the equality block's in
// equality_api.inc (same translation unit).
#include "mixed_api.inc"
#include "equality_api.inc"
#include "adjoint_api.inc"
#include "driver_api.inc"

// ============================================================================
//                                   C ABI
// ============================================================================
using sdpx::Handle;

struct sdpx_b200_handle {
  Handle h;
  std::unique_ptr<sdpx::CoreLoop> loop;  // declared after h: destroyed first
};

static thread_local std::string g_create_error;

#define GUARD(hh, body)                                   \
  do {                                                    \
    if (!(hh)) return -1;                                 \
    try {                                                 \
      ++(hh)->h.call_seq;                                 \
      SDPX_CUDA(cudaSetDevice((hh)->h.dev));              \
      body;                                               \
      return 0;                                           \
    } catch (const std::exception& ex) {                  \
      (hh)->h.err = ex.what();                            \
      return -2;                                          \
    } catch (...) {                                       \
      (hh)->h.err = "unknown error";                      \
      return -3;                                          \
    }                                                     \
  } while (0)

extern "C" {

int sdpx_b200_abi_version(void) { return SDPX_B200_ABI_VERSION; }
const char* sdpx_b200_create_error(void) { return g_create_error.c_str(); }

int sdpx_b200_create(const sdpx_b200_problem* problem, int device, sdpx_b200_handle** out) {
  if (!problem || !out) return -1;
  *out = nullptr;
  auto* hh = new (std::nothrow) sdpx_b200_handle();
  if (!hh) return -4;
  try {
    hh->h.create(problem, device);
  } catch (const std::exception& ex) {
    g_create_error = ex.what();
    delete hh;
    return -2;
  }
  *out = hh;
  return 0;
}
void sdpx_b200_destroy(sdpx_b200_handle* h) {
  if (!h) return;
  cudaSetDevice(h->h.dev);
  cudaStreamSynchronize(h->h.st);
  delete h;
}
const char* sdpx_b200_last_error(const sdpx_b200_handle* h) { return h ? h->h.err.c_str() : "null handle"; }
int sdpx_b200_set_precision(sdpx_b200_handle* h, int mode) {
  GUARD(h, {
    if (mode != SDPX_B200_FP64 && mode != SDPX_B200_MIXED) throw std::invalid_argument("bad precision mode");
    h->h.precision = mode;
    if (mode == SDPX_B200_MIXED) h->h.mixed_init();
  });
}
int sdpx_b200_equilibrate(sdpx_b200_handle* h, double* E, double* s, double* osc, int32_t* passes) {
  GUARD(h, h->h.equilibrate(E, s, osc, passes));
}
int sdpx_b200_data_norms(sdpx_b200_handle* h, double* a, double* b) { GUARD(h, h->h.data_norms(a, b)); }
int sdpx_b200_set_iterate(sdpx_b200_handle* h, const double* x, const double* X, const double* Y) {
  GUARD(h, h->h.set_iterate(x, X, Y));
}
int sdpx_b200_get_iterate(sdpx_b200_handle* h, double* x, double* X, double* Y) {
  GUARD(h, {
    if (x) {
      h->h.d2h(x, h->h.x.p, h->h.m * sizeof(double));
      h->h.sync();
    }
    if (X) h->h.get_stacked(h->h.X.p, X);
    if (Y) h->h.get_stacked(h->h.Y.p, Y);
  });
}
int sdpx_b200_get_direction(sdpx_b200_handle* h, double* dx, double* dX, double* dY) {
  GUARD(h, {
    if (dx) {
      h->h.d2h(dx, h->h.dx.p, h->h.m * sizeof(double));
      h->h.sync();
    }
    if (dX) h->h.get_stacked(h->h.dX.p, dX);
    if (dY) h->h.get_stacked(h->h.dY.p, dY);
  });
}
int sdpx_b200_get_rhs(sdpx_b200_handle* h, double* r) {
  GUARD(h, {
    h->h.d2h(r, h->h.r.p, h->h.m * sizeof(double));
    h->h.sync();
  });
}
int sdpx_b200_fixed_start(sdpx_b200_handle* h, double wp, double wd) {
  GUARD(h, {
    h->h.fixed_start(wp, wd);
    h->h.sync();
  });
}
int sdpx_b200_residuals(sdpx_b200_handle* h, const double* mu, int use_affine, int factor,
                        double* p_res, double* d_res, int* ok) {
  GUARD(h, h->h.residuals(mu, use_affine, factor, p_res, d_res, ok));
}
int sdpx_b200_block_primal_residual(sdpx_b200_handle* h, double* v) { GUARD(h, *v = h->h.last_bpr); }
int sdpx_b200_block_margins(sdpx_b200_handle* h, double* p, double* d) {
  GUARD(h, h->h.block_margins(p, d));
}
int sdpx_b200_schur_build(sdpx_b200_handle* h, int identity) {
  GUARD(h, {
    if (identity) {
      // cold start: factors of the identity
      h->h.schur_build(1);
    } else {
      h->h.schur_build(0);
    }
  });
}
int sdpx_b200_get_schur(sdpx_b200_handle* h, double* S) {
  GUARD(h, {
    h->h.d2h(S, h->h.S.p, sizeof(double) * h->h.m * h->h.m);
    h->h.sync();
  });
}
int sdpx_b200_factorize(sdpx_b200_handle* h, int* ok, int* att, double* q) {
  GUARD(h, h->h.factorize(ok, att, q));
}
int sdpx_b200_rhs_predictor(sdpx_b200_handle* h) { GUARD(h, h->h.rhs_predictor()); }
int sdpx_b200_rhs_corrector_mehrotra(sdpx_b200_handle* h, double sigma, double mu, int bl) {
  GUARD(h, h->h.rhs_corrector_mehrotra(sigma, mu, bl));
}
int sdpx_b200_rhs_corrector_fixed(sdpx_b200_handle* h, double beta, const double* mu) {
  GUARD(h, h->h.rhs_corrector_fixed(beta, mu));
}
int sdpx_b200_set_rhs(sdpx_b200_handle* h, int which) { GUARD(h, h->h.set_rhs(which)); }
int sdpx_b200_solve(sdpx_b200_handle* h) { GUARD(h, h->h.solve()); }
int sdpx_b200_direction_residual(sdpx_b200_handle* h, double* res, double* rn) {
  GUARD(h, h->h.direction_residual(res, rn));
}
int sdpx_b200_refine(sdpx_b200_handle* h, int policy, double tol, int cap, int fixed_steps,
                     int* steps, double* res) {
  GUARD(h, h->h.refine(policy, tol, cap, fixed_steps, steps, res));
}
int sdpx_b200_direction_blocks(sdpx_b200_handle* h) { GUARD(h, h->h.direction_blocks()); }
int sdpx_b200_affine_diagnostics(sdpx_b200_handle* h, int adaptive, double* out, double* bc) {
  GUARD(h, h->h.affine_diagnostics(adaptive, out, bc));
}
int sdpx_b200_line_search(sdpx_b200_handle* h, int rule, double fp, double fd, double gamma,
                          double min_step, double margin, double* tX, double* tY) {
  GUARD(h, h->h.line_search(rule, fp, fd, gamma, min_step, margin, tX, tY));
}
int sdpx_b200_update(sdpx_b200_handle* h, double tX, double tY, double* c, int* f, double* bd) {
  GUARD(h, h->h.update(tX, tY, c, f, bd));
}
int sdpx_b200_accepted_residuals(sdpx_b200_handle* h, double bpr, double tX, double tY, double* pa,
                                 double* da) {
  GUARD(h, h->h.accepted_residuals(bpr, tX, tY, pa, da));
}
int sdpx_b200_objectives(sdpx_b200_handle* h, double* p, double* d) { GUARD(h, h->h.objectives(p, d)); }
int sdpx_b200_solution_residuals(sdpx_b200_handle* h, double* p, double* d) {
  GUARD(h, h->h.solution_residuals(p, d));
}
int sdpx_b200_keep_direction(sdpx_b200_handle* h) {
  GUARD(h, h->h.d2d(h->h.keptx.p, h->h.dx.p, h->h.m * sizeof(double)));
}
int sdpx_b200_cold_start_iterate(sdpx_b200_handle* h) {
  GUARD(h, {
    h->h.cold_start_iterate();
    h->h.sync();
  });
}
int sdpx_b200_psd_shift(sdpx_b200_handle* h, int which, int* ok) { GUARD(h, h->h.psd_shift(which, ok)); }
int sdpx_b200_add_identity(sdpx_b200_handle* h, int which, double shift) {
  GUARD(h, h->h.add_identity(which, shift));
}
int sdpx_b200_block_dots(sdpx_b200_handle* h, double* d, double* tx, double* ty) {
  GUARD(h, h->h.block_dots(d, tx, ty));
}
int sdpx_b200_scale_iterate(sdpx_b200_handle* h, int which, double f) {
  GUARD(h, {
    sdpx::scale(h->h.K, which == 0 ? h->h.X.p : h->h.Y.p, f, h->h.st);
    h->h.sync();
  });
}
int sdpx_b200_store_best(sdpx_b200_handle* h) {
  GUARD(h, {
    auto& H = h->h;
    H.d2d(H.xbest.p, H.x.p, H.m * sizeof(double));
    H.d2d(H.Xbest.p, H.X.p, H.K * sizeof(double));
    H.d2d(H.Ybest.p, H.Y.p, H.K * sizeof(double));
    if (H.n_eq) H.d2d(H.ybest.p, H.yv.p, H.n_eq * sizeof(double));
  });
}
int sdpx_b200_restore_best(sdpx_b200_handle* h) {
  GUARD(h, {
    auto& H = h->h;
    H.d2d(H.x.p, H.xbest.p, H.m * sizeof(double));
    H.d2d(H.X.p, H.Xbest.p, H.K * sizeof(double));
    H.d2d(H.Y.p, H.Ybest.p, H.K * sizeof(double));
    if (H.n_eq) H.d2d(H.yv.p, H.ybest.p, H.n_eq * sizeof(double));
    H.sync();
  });
}
int sdpx_b200_rebuild_slack(sdpx_b200_handle* h, const double* x, double* X) {
  GUARD(h, h->h.rebuild_slack(x, X));
}
int sdpx_b200_certificate(sdpx_b200_handle* h, const double* x, const double* X, const double* Y,
                          double eps_primal, double eps_dual, double eps_gap, int32_t legacy_gap,
                          sdpx_b200_certificate_result* out) {
  GUARD(h, {
    if (!x || !X || !Y || !out) throw std::invalid_argument("certificate: NULL argument");
    h->h.certificate(x, X, Y, eps_primal, eps_dual, eps_gap, legacy_gap, out);
  });
}
int sdpx_b200_original_residuals(sdpx_b200_handle* h, const double* x, const double* X,
                                 const double* Y, double* p, double* d) {
  GUARD(h, h->h.original_residuals(x, X, Y, p, d));
}
int sdpx_b200_original_residuals_eq(sdpx_b200_handle* h, const double* x, const double* X,
                                    const double* y, const double* Y, double* p, double* d) {
  GUARD(h, h->h.original_residuals(x, X, Y, p, d, y));
}
int sdpx_b200_certificate_eq(sdpx_b200_handle* h, const double* x, const double* X,
                             const double* y, const double* Y, double eps_primal,
                             double eps_dual, double eps_gap, int32_t legacy_gap,
                             sdpx_b200_certificate_result* out) {
  GUARD(h, h->h.certificate(x, X, Y, eps_primal, eps_dual, eps_gap, legacy_gap, out, y));
}
int sdpx_b200_set_equality(sdpx_b200_handle* h, int32_t n, const double* B, const double* b) {
  GUARD(h, h->h.set_equality(n, B, b));
}
int sdpx_b200_set_equality_options(sdpx_b200_handle* h, double requested_accuracy, int solver) {
  GUARD(h, {
    if (solver != 0 && solver != 1) throw std::invalid_argument("bad equality solver");
    h->h.eq_requested = requested_accuracy;
    h->h.eq_solver = solver;
  });
}
int sdpx_b200_get_multipliers(sdpx_b200_handle* h, double* y, double* dy, double* p) {
  GUARD(h, {
    auto& H = h->h;
    const size_t bytes = (size_t)H.n_eq * sizeof(double);
    if (H.n_eq) {
      if (y) H.d2h(y, H.yv.p, bytes);
      if (dy) H.d2h(dy, H.dyv.p, bytes);
      if (p) H.d2h(p, H.pv.p, bytes);
      H.sync();
    }
  });
}
int sdpx_b200_set_multipliers(sdpx_b200_handle* h, const double* y) {
  GUARD(h, {
    auto& H = h->h;
    if (H.n_eq && y) {
      H.h2d(H.yv.p, y, (size_t)H.n_eq * sizeof(double));
      H.sync();
    }
  });
}
int sdpx_b200_equality_info(sdpx_b200_handle* h, int* kind, int* rank, double* quality) {
  GUARD(h, {
    if (kind) *kind = h->h.eq_kind;
    if (rank) *rank = h->h.eq_rank;
    if (quality) *quality = h->h.eq_quality;
  });
}
int sdpx_b200_adjoint(sdpx_b200_handle* h, const double* wx, const double* wy, const double* WX,
                      const double* WY, double* grad_c, double* grad_b, double* grad_C,
                      int32_t nA, const int32_t* A_index, double* grad_A) {
  GUARD(h, h->h.adjoint(wx, wy, WX, WY, grad_c, grad_b, grad_C, nA, A_index, grad_A));
}
int sdpx_b200_adjoint_refined(sdpx_b200_handle* h, const double* wx, const double* WX,
                              const double* WY, double* grad_c, double* grad_C, int32_t nA,
                              const int32_t* A_index, double* grad_A, int32_t refine_steps,
                              double* residual) {
  GUARD(h, h->h.adjoint_refined(wx, WX, WY, grad_c, grad_C, nA, A_index, grad_A, refine_steps,
                                residual));
}
void sdpx_b200_default_options(sdpx_b200_solve_options* o) {
  if (!o) return;
  *o = sdpx_b200_solve_options{};
  o->beta = 0.1;
  o->gamma = 0.9;
  o->omega_p = o->omega_d = 1.0;
  o->eps_gap = o->eps_primal = o->eps_dual = 1e-10;
  o->iter_max = 200;
  o->restart = 1;
  o->min_step = 1e-10;
  o->omega_step = 1e5;
  o->max_restarts = 5;
  o->max_centering = 4;
  o->stall_iterations = 15;
  o->stall_tolerance = 1e-3;
  o->step_rule = 0;
  o->refine_steps = 1;
  o->refine_policy = 2;
  o->refine_max_steps = 8;
  o->refine_tol = 0.0;
  o->max_time = INFINITY;
  o->parameter_policy = 0;
  o->parameter_strategy = 0;
  o->adaptive_sigma_max = 0.0;
  o->scaling = 0;
  o->precision = SDPX_B200_FP64;
  o->equality_solver = 0;
}
int sdpx_b200_optimize_begin(sdpx_b200_handle* h, const sdpx_b200_solve_options* o) {
  GUARD(h, {
    if (!o) throw std::invalid_argument("options are required");
    h->h.reset();
    h->loop = std::make_unique<sdpx::CoreLoop>(h->h);
    h->loop->begin(*o);
  });
}
int sdpx_b200_newton_step(sdpx_b200_handle* h, int32_t* running, int32_t* iteration,
                          double* p_obj, double* d_obj, double* p_res, double* d_res) {
  GUARD(h, {
    if (!h->loop) throw std::logic_error("sdpx_b200_optimize_begin was not called");
    const bool more = h->loop->step();
    if (running) *running = more ? 1 : 0;
    if (iteration) *iteration = h->loop->iter;
    if (p_obj) *p_obj = h->loop->pObj;
    if (d_obj) *d_obj = h->loop->dObj;
    if (p_res) *p_res = h->loop->p_res;
    if (d_res) *d_res = h->loop->d_res;
  });
}
int sdpx_b200_optimize_end(sdpx_b200_handle* h, sdpx_b200_solve_result* out) {
  GUARD(h, {
    if (!h->loop) throw std::logic_error("sdpx_b200_optimize_begin was not called");
    if (!out) throw std::invalid_argument("result is required");
    while (h->loop->step()) {
    }
    h->loop->end(out);
  });
}
int sdpx_b200_optimize(sdpx_b200_handle* h, const sdpx_b200_solve_options* o,
                       sdpx_b200_solve_result* out) {
  GUARD(h, {
    if (!o || !out) throw std::invalid_argument("options and result are required");
    h->h.reset();
    h->loop = std::make_unique<sdpx::CoreLoop>(h->h);
    h->loop->begin(*o);
    while (h->loop->step()) {
    }
    h->loop->end(out);
  });
}
int sdpx_b200_loop_state(sdpx_b200_handle* h, double* out8) {
  GUARD(h, {
    if (!h->loop) throw std::logic_error("sdpx_b200_optimize_begin was not called");
    auto& L = *h->loop;
    out8[0] = L.pObj;
    out8[1] = L.dObj;
    out8[2] = L.p_res;
    out8[3] = L.d_res;
    out8[4] = L.scale_p;
    out8[5] = L.scale_d;
    out8[6] = L.term_tol;
    out8[7] = L.current_compl;
  });
}
int sdpx_b200_get_solution(sdpx_b200_handle* h, double* x, double* X, double* y, double* Y) {
  GUARD(h, {
    if (!h->loop || h->loop->sx.empty()) throw std::logic_error("no solution: optimize first");
    auto& L = *h->loop;
    if (x) std::memcpy(x, L.sx.data(), L.sx.size() * sizeof(double));
    if (X) std::memcpy(X, L.sX.data(), L.sX.size() * sizeof(double));
    if (y && !L.sy.empty()) std::memcpy(y, L.sy.data(), L.sy.size() * sizeof(double));
    if (Y) std::memcpy(Y, L.sY.data(), L.sY.size() * sizeof(double));
  });
}
int sdpx_b200_get_trace(sdpx_b200_handle* h, int32_t* modes, int32_t cap, int32_t* count) {
  GUARD(h, {
    const int n = h->loop ? (int)h->loop->trace.size() : 0;
    if (count) *count = n;
    for (int i = 0; i < n && i < cap && modes; ++i) modes[i] = h->loop->trace[i];
  });
}
int sdpx_b200_step_stats(sdpx_b200_handle* h, int64_t* rounds, int64_t* trials) {
  GUARD(h, {
    if (rounds) *rounds = h->h.ftb_rounds;
    if (trials) *trials = h->h.ftb_trials;
  });
}
int sdpx_b200_reset(sdpx_b200_handle* h) { GUARD(h, h->h.reset()); }
int sdpx_b200_get_precision(sdpx_b200_handle* h, int* mode, int* fallbacks, double* cond_estimate) {
  GUARD(h, {
    *mode = h->h.precision;
    if (fallbacks) *fallbacks = h->h.mixed_fallbacks;
    if (cond_estimate) *cond_estimate = h->h.mixed ? h->h.mixed->cond_estimate : 0.0;
  });
}
int sdpx_b200_counters(sdpx_b200_handle* h, int64_t* out4) {
  GUARD(h, {
    if (!out4) throw std::invalid_argument("counters: NULL output");
    out4[0] = h->h.operator_applications;
    out4[1] = h->h.mixed_guard_steps;
    out4[2] = h->h.mixed_fallbacks;
    out4[3] = h->h.schur_builds;
  });
}
int sdpx_b200_get_stream(sdpx_b200_handle* h, void** stream) { GUARD(h, *stream = (void*)h->h.st); }
int sdpx_b200_trim_device_cache(void) {
  sdpx::dcache::trim(-1);
  return 0;
}
int sdpx_b200_launch_count(uint64_t* count) {
  if (!count) return -1;
  *count = sdpx::launch_count();
  return 0;
}
static thread_local std::string g_noalloc_error;
const char* sdpx_b200_gram_noalloc_error(void) { return g_noalloc_error.c_str(); }
int sdpx_b200_gram_noalloc(const double* P, int64_t K, int32_t m, double* S, void* stream) {
  if (!P || !S) {
    g_noalloc_error = "gram (allocation-free): NULL operand";
    return -1;
  }
  try {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    sdpx::syrk_lower_f64_noalloc(P, K, m, S, st);
    sdpx::mirror_lower(m, S, st);
    return 0;
  } catch (const std::invalid_argument& ex) {
    g_noalloc_error = ex.what();
    return -1;
  } catch (const std::exception& ex) {
    g_noalloc_error = ex.what();
    return -2;
  }
}
int sdpx_b200_set_sparse_schur(sdpx_b200_handle* h, int enable) {
  GUARD(h, {
    if (enable != 0 && enable != 1) throw std::invalid_argument("enable must be 0 or 1");
    if (enable) {
      for (auto& b : h->h.dense)
        if (b.k > sdpx::kSparseSchurMaxK)
          throw std::invalid_argument("sparse Schur: block order " + std::to_string(b.k) +
                                      " exceeds 160");
    }
    h->h.sparse_schur = enable == 1;
  });
}
int sdpx_b200_sparse_schur_info(sdpx_b200_handle* h, int64_t* active_positions,
                                int64_t* stored_entries) {
  GUARD(h, {
    if (h->h.coo_ver != h->h.a_ver) h->h.build_coo();
    if (active_positions) *active_positions = h->h.sp_active;
    if (stored_entries) *stored_entries = h->h.sp_nnz;
  });
}
int sdpx_b200_set_gram_engine(sdpx_b200_handle* h, int engine) {
  GUARD(h, {
    if (engine != 0 && engine != 1) throw std::invalid_argument("gram engine must be 0 or 1");
    h->h.gram_engine = engine;
  });
}
int sdpx_b200_kernel_times(sdpx_b200_handle* h, double* ms4) {
  GUARD(h, {
    if (!ms4) throw std::invalid_argument("kernel_times: NULL output");
    h->h.kt_harvest();
    for (int i = 0; i < 4; ++i) ms4[i] = h->h.kt_ms[i];
  });
}
int sdpx_b200_phase_times(sdpx_b200_handle* h, double* ms7, int reset) {
  GUARD(h, {
    h->h.harvest_phases();
    for (int i = 0; i < 7; ++i) ms7[i] = h->h.phase_ms[i];
    if (reset)
      for (int i = 0; i < 7; ++i) h->h.phase_ms[i] = 0.0;
  });
}

}  // extern "C"
