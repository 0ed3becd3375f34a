/*
 * SDPX-B200 batched small-SDP engine — C ABI (libsdpx_b200.so, sm_100a).
 *
 * Solves many independent dense SDPs of SDPX's form
 *     min cᵀx  s.t.  X = Σ_i x_i A_i − C ⪰ 0
 * (one PSD block each, DenseCons layout of src/types/constraints.jl:12-27:
 * A is a k²×m column-major matrix whose column i is vec(A_i)) in lockstep on
 * one GPU: every interior-point phase is one kernel launch over all instances
 * still running, one CTA per instance, while each instance keeps its own
 * scalar controller on the host.  Each instance follows SDPX's dense loop
 * (`_solve_sdp_core!`, src/solver/interior_point.jl:1742-2333, with
 * `newton_step!`, src/step.jl:643-1023) exactly as sdpx_b200_optimize does
 * for the same options, so its status, iteration count and objectives are
 * the single-instance solve's up to floating-point summation order.  SDPX
 * itself has no batch solver; this replaces a host loop of
 * sdpx_b200_create / sdpx_b200_optimize / sdpx_b200_destroy per instance.
 *
 * Supported options: parameter_policy = 1 (fixed start x = 0, X = ω_p·I,
 * Y = ω_d·I), scaling = 1 (none), precision = SDPX_B200_FP64 or
 * SDPX_B200_FLOAT64X2 (below), step_rule 0 or
 * 1 (backtracking; every block has k ≥ 3), max_time = ∞ per batch.  Sizes:
 * 3 ≤ k ≤ 64 and 1 ≤ m ≤ 256 per instance.  Anything else is a usage error
 * (return < 0, message from sdpx_b200_batch_last_error).
 */
#ifndef SDPX_B200_BATCH_H
#define SDPX_B200_BATCH_H

#include <stdint.h>

#include "sdpx_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sdpx_b200_batch sdpx_b200_batch;

typedef struct {
  int32_t count;               /* number of instances                         */
  const int32_t* block_order;  /* k per instance                              */
  const int32_t* m;            /* m per instance                              */
  const double* const* Av;     /* per instance: k²·m doubles (column i = vec A_i) */
  const double* const* C;      /* per instance: k² doubles                    */
  const double* const* c;      /* per instance: m doubles                     */
} sdpx_b200_batch_problem;

/* Precision mode of the batched engine only (sdpx_b200_solve_options.precision):
 * the Newton system — block residuals, X⁻¹, the Schur matrix and its
 * Cholesky factor, right-hand sides, solves, refinement residuals and the
 * direction blocks — in double-double (Float64x2), the iterate in FP64. */
#define SDPX_B200_FLOAT64X2 2

/* Largest block order and constraint count an instance may have. */
#define SDPX_B200_BATCH_MAX_K 64
#define SDPX_B200_BATCH_MAX_M 256

/* Uploads every instance into one pooled device workspace. */
int sdpx_b200_batch_create(const sdpx_b200_batch_problem* problem, int device,
                           sdpx_b200_batch** out);
void sdpx_b200_batch_destroy(sdpx_b200_batch* b);
const char* sdpx_b200_batch_last_error(const sdpx_b200_batch* b);
/* Message of the last failed sdpx_b200_batch_create on this thread. */
const char* sdpx_b200_batch_create_error(void);

/* Solves every instance; results[i] (count entries) as sdpx_b200_optimize
 * reports them (objectives and residuals on the original data). */
int sdpx_b200_batch_optimize(sdpx_b200_batch* b, const sdpx_b200_solve_options* opts,
                             sdpx_b200_solve_result* results);

/* Solution of instance i after sdpx_b200_batch_optimize: x (m), X and Y
 * (k² column-major).  Any pointer may be NULL. */
int sdpx_b200_batch_get_solution(sdpx_b200_batch* b, int32_t i, double* x, double* X, double* Y);

/* Every instance's solution in one read-back: x receives Σ m_i doubles
 * (instance i at Σ_{j<i} m_j), X and Y Σ k_i² doubles each (instance i's
 * k_i² column-major entries at Σ_{j<i} k_j²).  Any pointer may be NULL. */
int sdpx_b200_batch_get_solutions(sdpx_b200_batch* b, double* x, double* X, double* Y);

/* Replaces instance i's current iterate with host x (m), X and Y (k²
 * column-major), e.g. to certify solutions computed elsewhere; NULL keeps
 * that part.  Certificates need every instance's x, X and Y set (or a solve). */
int sdpx_b200_batch_set_solution(sdpx_b200_batch* b, int32_t i, const double* x,
                                 const double* X, const double* Y);

/* Result certificates of every instance's current solution (after
 * sdpx_b200_batch_optimize: the returned iterate) against its data, computed
 * for all instances by one kernel and read back once — SDPX's
 * `result_certificate` (src/validation.jl:948-1115), optimality kind, n = 0,
 * with the fields and failure bits of sdpx_b200_certificate (results: count
 * entries; the block counts are 0 or 1).  legacy_gap = 1 selects the
 * 0 ≤ gap ≤ eps_gap test. */
int sdpx_b200_batch_certificate(sdpx_b200_batch* b, double eps_primal, double eps_dual,
                                double eps_gap, int32_t legacy_gap,
                                sdpx_b200_certificate_result* results);

/* Counters of the last optimize: out[0] loop passes, out[1] phase kernel
 * launches, out[2] seconds in the loop, out[3] seconds in the Schur phase,
 * out[4] seconds in the Schur factorisation phase, out[5] seconds in the step
 * length phases, out[6] instance-iterations, out[7] Schur FLOPs
 * (Σ per instance-iteration of 2·k³·m + k²·m²). */
int sdpx_b200_batch_stats(sdpx_b200_batch* b, double* out8);

/* How the affine predictor's fraction-to-boundary bounds (the step lengths
 * that set σ, `fraction_to_boundary_bound!`, src/kernels/generic.jl:350-422)
 * are computed: mode 1 (default) t* = −1/λ_min(L⁻¹·dM·L⁻ᵀ) from the block's
 * Cholesky factor L (1 when the full step stays interior), by a Householder
 * tridiagonalisation and a Sturm-count multisection; mode 0 the reference's
 * bisection of Cholesky trials of M + t·dM (up to 64 steps).  The two agree up
 * to the rounding of the trials near t*.  The backtracking line search always
 * runs Cholesky trials. */
int sdpx_b200_batch_set_step_bounds(sdpx_b200_batch* b, int32_t mode);

/* Launch shape of the Schur phase: threads per CTA (128, 256 or 512), the
 * SYRK tile (16 or 32; 512 threads need 32; tile 64 with 128 threads selects
 * the FP64 tensor-core (DMMA) products, which tile each instance by 32 or 64
 * as its k and m need) and the Schur work per CTA in
 * FLOPs (an instance's panel and SYRK are split over ceil(work / grain) CTAs;
 * grain ≤ 0: one CTA per instance). */
int sdpx_b200_batch_set_schur_shape(sdpx_b200_batch* b, int32_t threads, int32_t tile,
                                    double grain);

/* Times every candidate Schur launch shape (24: five scalar shapes and the
 * DMMA path, each at four work grains) on the current iterate of all
 * instances (the fixed start when no solve ran) and keeps the fastest.
 * table (may be NULL) receives `capacity` rows of (threads, tile, grain,
 * milliseconds); *count = number of candidates timed. */
int sdpx_b200_batch_autotune(sdpx_b200_batch* b, const sdpx_b200_solve_options* opts,
                             double* table, int32_t capacity, int32_t* count);

#ifdef __cplusplus
}
#endif

#endif /* SDPX_B200_BATCH_H */
