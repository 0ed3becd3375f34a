/*
 * SDPX-B200 C ABI — the boundary between SDPX's Julia host code and the B200
 * dense-SDP interior-point core (libsdpx_b200.so, sm_100a).
 *
 * Every function returns an int status: 0 = ok, > 0 = numerical outcome the
 * caller must interpret (documented per call), < 0 = usage or CUDA error with a
 * message available from sdpx_b200_last_error().  Nothing throws or aborts
 * across the boundary.  Host arrays are only read/written during the call.
 *
 * Data conventions (SDPX's DenseCons, src/types/constraints.jl:12-27):
 *   - block l has order k_l; A^(l) is a k_l²×m column-major matrix whose
 *     column i is vec(A_i^(l)) (column-major vec); every A_i^(l) is symmetric;
 *   - "stacked" host matrices (X, Y, dX, dY, C) concatenate the k_l×k_l
 *     column-major blocks in block order: Σ_l k_l² doubles;
 *   - the core solves SDPX's form min cᵀx s.t. X_l = Σ_i x_i A_i^(l) − C_l ⪰ 0
 *     and, when sdpx_b200_set_equality attached them, Bᵀx = b (n > 0).
 *
 * One handle = one solve = one CUDA stream.  A handle is not reentrant; use
 * one handle per concurrent solve (SDPX: "Concurrent factorization must use
 * distinct solver/provider workspaces", docs/src/providers.md).
 */
#ifndef SDPX_B200_H
#define SDPX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SDPX_B200_ABI_VERSION 1

typedef struct sdpx_b200_handle sdpx_b200_handle;

typedef struct {
  int64_t m;                  /* number of variables x_i                       */
  int32_t nblocks;            /* L                                             */
  const int32_t* block_order; /* k_l, length L                                 */
  const double* const* Av;    /* per block: k_l²·m doubles (column i = vec A_i) */
  const double* const* C;     /* per block: k_l² doubles                       */
  const double* c;            /* m                                             */
} sdpx_b200_problem;

/* Precision modes of the Newton system. */
#define SDPX_B200_FP64 0  /* plain FP64 Schur assembly and Cholesky                */
#define SDPX_B200_MIXED 1 /* split-BF16 Schur assembly, FP32 Cholesky, FP64 refine  */

int sdpx_b200_abi_version(void);
/* Message of the last failed sdpx_b200_create on this thread. */
const char* sdpx_b200_create_error(void);

/* Problem upload and workspace allocation.  Replaces the provider
 * instantiation SDPX performs through `instantiate_la_backend`
 * (src/la_backend.jl:508-570) and `Workspace(prob)` (src/workspace.jl:779). */
int sdpx_b200_create(const sdpx_b200_problem* problem, int device, sdpx_b200_handle** out);
void sdpx_b200_destroy(sdpx_b200_handle* h);
const char* sdpx_b200_last_error(const sdpx_b200_handle* h);
int sdpx_b200_set_precision(sdpx_b200_handle* h, int mode);
/* Current precision mode (mixed mode switches itself to FP64 when the guard
 * fails), number of such switches, and the last FP32-factor condition estimate. */
int sdpx_b200_get_precision(sdpx_b200_handle* h, int* mode, int* fallbacks, double* cond_estimate);

/* Ruiz + per-variable + objective scaling of the resident data in place
 * (`equilibrate`, src/ingest.jl:1431-1519).  Outputs: E (Σ k_l, per block
 * congruence factors), s (m), objective scale, passes (L).  The original data
 * is retained for sdpx_b200_rebuild_slack / sdpx_b200_original_residuals. */
int sdpx_b200_equilibrate(sdpx_b200_handle* h, double* E, double* s, double* objective_scale,
                          int32_t* passes);
/* max_l ‖C_l‖∞ and ‖c‖∞ of the working (scaled) data. */
int sdpx_b200_data_norms(sdpx_b200_handle* h, double* max_C, double* c_norm);

/* Iterate I/O (stacked layout). */
int sdpx_b200_set_iterate(sdpx_b200_handle* h, const double* x, const double* X, const double* Y);
int sdpx_b200_get_iterate(sdpx_b200_handle* h, double* x, double* X, double* Y);
int sdpx_b200_get_direction(sdpx_b200_handle* h, double* dx, double* dX, double* dY);
int sdpx_b200_get_rhs(sdpx_b200_handle* h, double* r);
/* x = 0, X = ω_p I, Y = ω_d I (fixed-policy start, src/solver/interior_point.jl:1600-1612). */
int sdpx_b200_fixed_start(sdpx_b200_handle* h, double omega_p, double omega_d);

/* Residuals P_l, d, R_l and (factor != 0) the block Cholesky factors of X, Y
 * (`threaded_compute_residuals!`, src/kernels/threaded.jl:423-506).
 * blocks_ok = 0 when a block factorization failed.  mu: L targets. */
int sdpx_b200_residuals(sdpx_b200_handle* h, const double* mu, int use_affine, int factor,
                        double* p_res, double* d_res, int* blocks_ok);
/* max_l ‖P_l‖∞ of the last residual evaluation (src/step.jl:74-80). */
int sdpx_b200_block_primal_residual(sdpx_b200_handle* h, double* value);
/* min/max diagonal ratios of the X and Y factors (src/step.jl:273-281). */
int sdpx_b200_block_margins(sdpx_b200_handle* h, double* primal, double* dual);

/* Schur complement S_ij = tr(A_i X⁻¹ A_j Y) from the current block factors
 * (`schur_build!` DenseCons, src/schur.jl:511-562).  identity != 0 uses X = Y = I
 * (KKT cold start, src/solver/interior_point.jl:709-723). */
int sdpx_b200_schur_build(sdpx_b200_handle* h, int identity);
int sdpx_b200_get_schur(sdpx_b200_handle* h, double* S /* m×m, full symmetric */);

/* Cholesky of S with ≤ 6 relative diagonal regularisation retries
 * (`_factor_dense_kkt_native!`, src/kkt.jl:1404-1445).  Returns 0 and ok = 0
 * when S stays indefinite.  quality = min/max |L_ii|. */
int sdpx_b200_factorize(sdpx_b200_handle* h, int* ok, int* reg_attempts, double* quality);

/* Right-hand sides: predictor (src/step.jl:95-108), corrector (Mehrotra,
 * src/kernels/threaded.jl:916-1067; fixed-policy, :837-901), cold start
 * (which = 0: r = Σ_l A^(l)ᵀ vec C_l, which = 1: r = c). */
int sdpx_b200_rhs_predictor(sdpx_b200_handle* h);
int sdpx_b200_rhs_corrector_mehrotra(sdpx_b200_handle* h, double sigma, double mu, int block_local);
int sdpx_b200_rhs_corrector_fixed(sdpx_b200_handle* h, double beta, const double* mu);
int sdpx_b200_set_rhs(sdpx_b200_handle* h, int which);

/* dx = S⁻¹ r with the current factor (`_solve_dense_kkt_owned!`, src/kkt.jl:2570-2595);
 * with equality rows also dy, from S·dx − B·dy = r, Bᵀdx = p. */
int sdpx_b200_solve(sdpx_b200_handle* h);
/* ρ = r − S·dx; residual = ‖ρ‖∞, rnorm = ‖r‖∞ (src/kkt.jl:3689-3708).  With
 * equality rows ρ += B·dy, ρ_p = p − Bᵀdx, residual = max(‖ρ‖∞, ‖ρ_p‖∞) and
 * rnorm = max(‖r‖∞, ‖p‖∞). */
int sdpx_b200_direction_residual(sdpx_b200_handle* h, double* residual, double* rnorm);
/* Residual-driven refinement with rollback (`_refine_native_direction!`,
 * src/kkt.jl:3891-3963).  policy: 0 fixed, 1 adaptive/auto; tol ≤ 0 selects
 * 64·eps.  In mixed mode the correction solves use the FP32 factor and the
 * residual is the FP64 Newton residual. */
int sdpx_b200_refine(sdpx_b200_handle* h, int policy, double tol, int cap, int fixed_steps,
                     int* steps, double* residual);
/* dX_l = mat(A^(l)·dx) + P_l, dY_l = sym(X_l⁻¹(R_l − dX_l Y_l))
 * (`threaded_direction_blocks!`, src/kernels/threaded.jl:574-663). */
int sdpx_b200_direction_blocks(sdpx_b200_handle* h);

/* Affine predictor step bounds and complementarity (src/step.jl:546-619).
 * out[0] = Σ⟨X_l,Y_l⟩, out[1] = Σ⟨X_l+tX dX_l, Y_l+tY dY_l⟩, out[2] = tX,
 * out[3] = tY;  block_compl: L values ⟨X_l,Y_l⟩.  adaptive = 0 uses unit steps. */
int sdpx_b200_affine_diagnostics(sdpx_b200_handle* h, int adaptive, double* out,
                                 double* block_compl);

/* Step lengths (`threaded_line_search!`, src/kernels/threaded.jl:1602-1818).
 * rule: 0 backtrack, 1 fraction-to-boundary. */
int sdpx_b200_line_search(sdpx_b200_handle* h, int rule, double primal_fraction,
                          double dual_fraction, double gamma, double min_step, double margin,
                          double* tX, double* tY);

/* X += tX dX, Y += tY dY, x += tX dx; returns Σ⟨X_l,Y_l⟩, finiteness and the
 * L block values (`threaded_update_blocks!`, src/kernels/threaded.jl:665-754). */
int sdpx_b200_update(sdpx_b200_handle* h, double tX, double tY, double* compl_total, int* finite,
                     double* block_dots);
/* d ← (1−tY)d − tY ρ ; p_after = |1−tX|·block_primal_residual
 * (`_accepted_sdp_trial_residuals!`, src/solver/interior_point.jl:1287-1321). */
int sdpx_b200_accepted_residuals(sdpx_b200_handle* h, double block_primal_residual, double tX,
                                 double tY, double* p_after, double* d_after);
int sdpx_b200_objectives(sdpx_b200_handle* h, double* p_obj, double* d_obj);
/* Exact residual recomputation on the working data (src/validation.jl:15-60). */
int sdpx_b200_solution_residuals(sdpx_b200_handle* h, double* p_res, double* d_res);

/* KKT cold-start helpers (src/solver/interior_point.jl:699-1287, src/cold_start.jl). */
int sdpx_b200_keep_direction(sdpx_b200_handle* h);
int sdpx_b200_cold_start_iterate(sdpx_b200_handle* h);
/* Certified strictly-interior identity shift of every block of X (which = 0)
 * or Y (which = 1) (`_cold_start_psd_shift!`); ok = 0 when a block fails. */
int sdpx_b200_psd_shift(sdpx_b200_handle* h, int which, int* ok);
int sdpx_b200_add_identity(sdpx_b200_handle* h, int which, double shift);
int sdpx_b200_block_dots(sdpx_b200_handle* h, double* dots, double* trace_X, double* trace_Y);
int sdpx_b200_scale_iterate(sdpx_b200_handle* h, int which, double factor);
int sdpx_b200_store_best(sdpx_b200_handle* h);
int sdpx_b200_restore_best(sdpx_b200_handle* h);

/* Original (unscaled) data: slack X = Σ x_i A_i − C and residuals. */
int sdpx_b200_rebuild_slack(sdpx_b200_handle* h, const double* x, double* X);
int sdpx_b200_original_residuals(sdpx_b200_handle* h, const double* x, const double* X,
                                 const double* Y, double* p_res, double* d_res);

/* ---- Equality rows Bᵀx = b (n > 0) ------------------------------------
 * SDPX's `SDPProblem.B` (m×n, one column per equality) and `.b`
 * (src/types/problems.jl) with their multipliers y; the KKT factor and solve
 * replace the n > 0 branches of `_factor_dense_kkt_native!`
 * (src/kkt.jl:1466-1680: B̃ = L_S⁻¹B, unit ∞-norm columns, Q = B̃ᵀB̃ by
 * Cholesky with the rank test, column-pivoted QR of B̃ when it fails) and of
 * `_solve_dense_kkt_owned!` (src/kkt.jl:2570-2595).  Residuals, refinement,
 * update, objectives, the cold start and the equilibration carry the B, b, y
 * terms of src/step.jl:25-72, src/kkt.jl:3689-3708 and
 * src/solver/interior_point.jl:699-1311 once they are set.  In the mixed
 * precision mode B̃ comes from the FP32 factor and Q is factored in FP64 with
 * up to 8 diagonal regularisations (src/kernels/mixed_precision_kkt.jl:481-520,
 * 1045-1082); the guard refines against the FP64 KKT operator with the B terms. */

/* B column-major m×n, b length n; call after create and before
 * sdpx_b200_equilibrate.  n = 0 removes the equality rows. */
int sdpx_b200_set_equality(sdpx_b200_handle* h, int32_t n, const double* B, const double* b);
/* Rank tolerance input min(ϵ_gap, ϵ_primal, ϵ_dual) (`_requested_accuracy`,
 * src/kkt.jl:518-521) and `equality_solver`: 0 = automatic (normal
 * equations, rank-revealing QR once they lose rank), 1 = QR from the start. */
int sdpx_b200_set_equality_options(sdpx_b200_handle* h, double requested_accuracy, int solver);
/* y, dy and p = b − Bᵀx (p as last updated: residuals, cold-start right-hand
 * side or accepted-step carry); any pointer may be NULL. */
int sdpx_b200_get_multipliers(sdpx_b200_handle* h, double* y, double* dy, double* p);
int sdpx_b200_set_multipliers(sdpx_b200_handle* h, const double* y);
/* Current equality factor: kind 0 = none, 1 = normal equations (Cholesky of
 * Q), 2 = rank-revealing QR; its numerical rank and quality (min/max |R_jj|
 * over the rank for QR, 1 for the normal equations). */
int sdpx_b200_equality_info(sdpx_b200_handle* h, int* kind, int* rank, double* quality);
/* sdpx_b200_original_residuals with the equality terms: d −= B·y and
 * p = b − Bᵀx on the original rows. */
int sdpx_b200_original_residuals_eq(sdpx_b200_handle* h, const double* x, const double* X,
                                    const double* y, const double* Y, double* p_res,
                                    double* d_res);

/* ---- Adjoint of the solution map -----------------------------------------
 * Gradient of L = ⟨wx, x⟩ + ⟨wy, y⟩ + Σ_l⟨WX_l, X_l⟩ + Σ_l⟨WY_l, Y_l⟩ at the
 * current iterate with respect to the data c (m), b (n), C (stacked, Σk_l²)
 * and the coefficients A_i for the nA indices in A_index (grad_A: nA stacked
 * layouts, one per index, each Σk_l²).  SDPX has no adjoint: this is the
 * implicit-function derivative of the HKM-linearised KKT conditions, reusing
 * the Newton system's factor — call it after sdpx_b200_residuals (factor = 1),
 * sdpx_b200_schur_build and sdpx_b200_factorize at the iterate, in the FP64
 * precision mode.  Any seed may be NULL (zero); any output may be NULL.
 *   λ from one KKT solve with right-hand side (wx + 𝒜ᵀWX − 𝒜ᵀG, −wy),
 *   G = X⁻¹·sym(WY)·Y;  ∂L/∂c = −λx, ∂L/∂b = λy,
 *   ∂L/∂C_l = sym(X⁻¹ΛY) − sym(WX_l − G_l) with Λ = mat(𝒜λx),
 *   ∂L/∂A_i = λx_i·Y − x_i·∂L/∂C. */
int sdpx_b200_adjoint(sdpx_b200_handle* h, const double* wx, const double* wy, const double* WX,
                      const double* WY, double* grad_c, double* grad_b, double* grad_C,
                      int32_t nA, const int32_t* A_index, double* grad_A);

/* The same gradient (no equality rows: n = 0) with the linear system solved
 * to double-double (Float64x2) accuracy: X⁻¹ by Newton–Schulz steps from the
 * FP64 inverse, every product of S·v = 𝒜ᵀ(X⁻¹ mat(𝒜v) Y) and of the seeds in
 * double-double, and λ solved by up to refine_steps (≤ 64) conjugate-gradient
 * steps in double-double preconditioned by the FP64 factor (the
 * low-precision factor / high-precision residual scheme of
 * `_solve_mixed_kkt_guarded!`, src/kernels/mixed_precision_kkt.jl:1475-1586,
 * one level up; CG keeps converging when κ(S)·eps ≥ 1 near a solution, where
 * plain refinement on the FP64 factor stops contracting).  The FP64 solve is
 * returned when CG does not reduce the true residual.  residual (may be
 * NULL) = ‖w − S·λ‖∞ / ‖w‖∞ of the returned λ, in double-double. */
int sdpx_b200_adjoint_refined(sdpx_b200_handle* h, const double* wx, const double* WX,
                              const double* WY, double* grad_c, double* grad_C, int32_t nA,
                              const int32_t* A_index, double* grad_A, int32_t refine_steps,
                              double* residual);

/* ---- The whole interior-point solve inside the library -------------------
 * SDPX's `_solve_pipeline!` for the dense route (src/solver/interior_point.jl:
 * 3131-3571: Ruiz scaling, KKT cold start :699-1287, core loop :1323-2687 with
 * `newton_step!` src/step.jl:643-1023, the guarded Mehrotra controller
 * src/adaptive_parameters.jl and the stagnation detector src/stagnation.jl,
 * unscaling and original-coordinate residuals) run on the host side of the
 * library: one call per solve, or begin / one loop pass per newton_step / end. */
typedef struct {
  double beta, gamma, omega_p, omega_d, eps_gap, eps_primal, eps_dual;
  int32_t iter_max, restart;
  double min_step, omega_step;
  int32_t max_restarts, max_centering, stall_iterations;
  double stall_tolerance;
  int32_t step_rule;         /* 0 auto, 1 backtrack, 2 fraction to boundary      */
  int32_t refine_steps;
  int32_t refine_policy;     /* 0 fixed, 1 adaptive, 2 auto                      */
  int32_t refine_max_steps;
  double refine_tol, max_time;
  int32_t parameter_policy;  /* 0 auto (KKT cold start), 1 fixed start           */
  int32_t parameter_strategy; /* 0 adaptive, 1 fixed                             */
  double adaptive_sigma_max;
  int32_t scaling;           /* 0 auto, 1 none, 2 equilibrate                    */
  int32_t precision;         /* SDPX_B200_FP64 or SDPX_B200_MIXED                */
  int32_t equality_solver;   /* 0 automatic, 1 rank-revealing QR                 */
} sdpx_b200_solve_options;

#define SDPX_B200_STATUS_OPTIMAL 1
#define SDPX_B200_STATUS_ITER_LIMIT 2
#define SDPX_B200_STATUS_STALLED 3
#define SDPX_B200_STATUS_INSUFFICIENT_PRECISION 4
#define SDPX_B200_STATUS_NUMERICAL_BREAKDOWN 5
#define SDPX_B200_STATUS_MAX_RESTARTS 6
#define SDPX_B200_STATUS_TIME_LIMIT 7

typedef struct {
  int32_t status;            /* SDPX_B200_STATUS_*                               */
  int32_t iterations, restarts;
  int32_t mixed_iterations, fp64_iterations;
  double p_obj, d_obj;       /* original data                                    */
  double p_res, d_res;       /* original data                                    */
  double seconds;
  char message[256];
} sdpx_b200_solve_result;

/* SDPX's SolverOptions{Float64} defaults (src/types/workspaces.jl:101-185),
 * tolerances 1e-10. */
void sdpx_b200_default_options(sdpx_b200_solve_options* opts);
int sdpx_b200_optimize(sdpx_b200_handle* h, const sdpx_b200_solve_options* opts,
                       sdpx_b200_solve_result* result);
int sdpx_b200_optimize_begin(sdpx_b200_handle* h, const sdpx_b200_solve_options* opts);
/* One pass of the loop body: termination tests, then one Newton step with step
 * length and update (a1–a13), or a restart / centering / FP64-switch pass.
 * running = 0 once the loop has ended. */
int sdpx_b200_newton_step(sdpx_b200_handle* h, int32_t* running, int32_t* iteration,
                          double* p_obj, double* d_obj, double* p_res, double* d_res);
int sdpx_b200_optimize_end(sdpx_b200_handle* h, sdpx_b200_solve_result* result);
/* The solution of the last sdpx_b200_optimize(_end), original coordinates
 * (stacked X, Y; y of length n).  Any pointer may be NULL. */
int sdpx_b200_get_solution(sdpx_b200_handle* h, double* x, double* X, double* y, double* Y);
/* Loop state after begin or a step: pObj, dObj, p_res, d_res (working
 * data), the primal and dual residual scales, the gap tolerance and Σ⟨X_l,Y_l⟩. */
int sdpx_b200_loop_state(sdpx_b200_handle* h, double* out8);
/* Precision of each Newton step of the last solve: 1 mixed, 0 FP64. */
int sdpx_b200_get_trace(sdpx_b200_handle* h, int32_t* modes, int32_t capacity, int32_t* count);

/* Batched trial rounds and trials the fraction-to-boundary bisections
 * (src/kernels/generic.jl:350-422) have run on this handle. */
int sdpx_b200_step_stats(sdpx_b200_handle* h, int64_t* rounds, int64_t* trials);

/* Restore the data as uploaded (undo sdpx_b200_equilibrate) and reset the
 * iterate to x = 0, X = Y = I, so one handle can run repeated solves. */
int sdpx_b200_reset(sdpx_b200_handle* h);
/* The handle's CUDA stream (cudaStream_t), for callers that time or order work on it. */
int sdpx_b200_get_stream(sdpx_b200_handle* h, void** stream);
/* Number of kernels this library has launched in this process. */
int sdpx_b200_launch_count(uint64_t* count);

/* Sparse Schur engine — SDPX's `SparseCons` path (`sparse = :on`,
 * src/types/constraints.jl:26-101; `sparse_schur_block!` src/schur.jl:936-1032,
 * `_two_sided_coo_product!` :601-656, `_dot_dense_coo` :566-579, the serial
 * block-order reduction :1173-1197).  enable = 1 makes every FP64 Schur build
 * (not the identity-metric one of the cold start, not the mixed mode) take
 * the coefficients as flat coordinate entries per dense block and active
 * variable, S_ij += ⟨Y_l·A_i·X_l⁻¹, A_j⟩ over the active pairs, work
 * Σ_p nnz_p·k² + Σ_{p≤r} nnz_r per block; 1×1 blocks keep their Gram on the
 * FP64 tiles.  Every dense block order must be ≤ 160 (else -2 and a message).
 * The entries are extracted from the device copy of 𝒜 (after equilibration)
 * on the first build. */
int sdpx_b200_set_sparse_schur(sdpx_b200_handle* h, int enable);
/* Active (block, variable) positions and stored entries of that form. */
int sdpx_b200_sparse_schur_info(sdpx_b200_handle* h, int64_t* active_positions,
                                int64_t* stored_entries);

/* Allocation-free Gram (Schur) product — no counterpart in the reference.
 *
 * S = Pᵀ P for a K×m column-major FP64 matrix P already in device memory
 * (column i is one variable's stacked vector, as in the Schur assembly with
 * the identity metric), written as the full symmetric m×m column-major S.
 * It performs no allocation: the split-K partial tiles use a fixed 32 MiB
 * device array compiled into the library, so it suits callers that cannot
 * call cudaMalloc — runtimes that own all device memory through their own
 * pool (e.g. a Julia or Python caching allocator) or serving loops where an
 * implicit cudaMalloc/cudaFree would synchronise the device.
 *   - m ≤ 2048 (the array holds one K chunk of every lower 128×128 tile) and
 *     K ≤ 2^30 (the tile loop indexes K in int32); larger m or K, and NULL
 *     P or S, return -1 with a message and leave S untouched.
 *   - The first call on each device looks up the array's device address with
 *     that device current; make that first call before any stream capture.
 *   - Every call on a device shares the one array: calls that overlap on the
 *     GPU (different streams, or different host threads) race.  Serialise them.
 *   - stream: a cudaStream_t (NULL = legacy default stream); the call is
 *     asynchronous with respect to the host.
 * Every GPU that loads the library keeps the array until the process exits. */
int sdpx_b200_gram_noalloc(const double* P, int64_t K, int32_t m, double* S, void* stream);
const char* sdpx_b200_gram_noalloc_error(void);

/* Cold-path result certificate in original coordinates — SDPX's
 * `result_certificate` (src/validation.jl:948-1115), optimality kind, n = 0.
 * Residuals and componentwise backward errors are one device pass each over
 * the original constraint data; block PSD checks factor symmetrised, shifted
 * copies with the batched Cholesky (closed forms for 1×1 and 2×2 blocks,
 * shift bisection for blocks of order ≤ 4, as the reference).  A NaN
 * residual is reported as +inf (the certificate is invalid either way). */
typedef struct {
  int32_t valid;                     /* 1 when failures == 0                       */
  int32_t failures;                  /* bitmask of SDPX_B200_CERT_*                */
  int32_t primal_psd_failing_blocks; /* number of X blocks failing the PSD check   */
  int32_t dual_psd_failing_blocks;   /* number of Y blocks failing the PSD check   */
  double primal_objective, dual_objective, gap, gap_relative;
  double primal_residual, dual_residual;               /* max(affine, cone violation) */
  double primal_affine_residual, dual_affine_residual;
  double primal_cone_violation, dual_cone_violation;
  double primal_residual_scaled, dual_residual_scaled;
  double equality_backward_error, equality_strict_backward_error; /* 0 when n = 0 */
  double primal_block_backward_error, primal_block_strict_backward_error;
  double dual_backward_error, dual_strict_backward_error;
  double complementarity, complementarity_relative;
} sdpx_b200_certificate_result;

#define SDPX_B200_CERT_NONFINITE 1
#define SDPX_B200_CERT_PRIMAL_RESIDUAL 2
#define SDPX_B200_CERT_EQUALITY_BACKWARD_ERROR 4
#define SDPX_B200_CERT_PRIMAL_BLOCK_BACKWARD_ERROR 8
#define SDPX_B200_CERT_DUAL_RESIDUAL 16
#define SDPX_B200_CERT_DUAL_BACKWARD_ERROR 32
#define SDPX_B200_CERT_DUALITY_GAP 64
#define SDPX_B200_CERT_PRIMAL_PSD 128
#define SDPX_B200_CERT_DUAL_PSD 256

/* x (m), X and Y (stacked, original coordinates).  legacy_gap = 1 selects the
 * `termination = :legacy` gap test 0 ≤ gap ≤ eps_gap, else gap_rel ≤ eps_gap. */
int sdpx_b200_certificate(sdpx_b200_handle* h, const double* x, const double* X, const double* Y,
                          double eps_primal, double eps_dual, double eps_gap, int32_t legacy_gap,
                          sdpx_b200_certificate_result* out);
/* The same certificate with the equality rows' terms (n > 0): y enters the
 * dual objective (bᵀy), the dual residual and its backward errors (B·y), and
 * b − Bᵀx the primal residual and the equality backward errors
 * (src/validation.jl:454-482, 629-644, 666-740). */
int sdpx_b200_certificate_eq(sdpx_b200_handle* h, const double* x, const double* X,
                             const double* y, const double* Y, double eps_primal,
                             double eps_dual, double eps_gap, int32_t legacy_gap,
                             sdpx_b200_certificate_result* out);

/* Engine of the FP64 Schur assembly — the Gram S = P̂ᵀP̂ and the block
 * products T_i = L_X⁻¹·A_i, P_i = T_i·L_Y (no counterpart in the reference,
 * whose Float64 products are BLAS): 0 = FP64 DMMA tiles, 1 = exact int8
 * (default) digit products on the tensor cores — every operand row or column
 * scaled by a power of two and cut into eight int8 digits (55 significant
 * bits), digit products accumulated exactly in int32 and the levels summed in
 * FP64. */
int sdpx_b200_set_gram_engine(sdpx_b200_handle* h, int engine);

/* Instrumentation (no counterpart in the reference): device time (ms) of the
 * most recent launch of the Schur kernels, measured with events on the
 * handle's stream: [0] split-BF16 SYRK kernel, [1] split-BF16 block products
 * of all blocks, [2] FP64 SYRK (split-K kernel and reduction), [3] FP64 block
 * products of all blocks; 0 where none ran yet. */
int sdpx_b200_kernel_times(sdpx_b200_handle* h, double* ms4);

/* Device memory (no counterpart in the reference): buffers released by
 * destroyed handles stay cached in this process for reuse by later handles
 * (allocation and release cost ≈ 1.8 and 2.9 ms per GB on the B200; a handle of
 * the m = 2000 workload holds ≈ 25 GB).  This call returns every idle cached
 * block to the driver.  Always 0. */
int sdpx_b200_trim_device_cache(void);

/* Instrumentation (no counterpart in the reference), counts since the last
 * reset: [0] applications of the matrix-free FP64 Newton operator (mixed-mode
 * residuals), [1] mixed-guard correction steps, [2] switches from mixed to
 * FP64, [3] Schur builds. */
int sdpx_b200_counters(sdpx_b200_handle* h, int64_t* out4);

/* Cumulative device time per phase (ms) since the last reset:
 * [0] residual+block factor, [1] Schur assembly, [2] KKT factor,
 * [3] solves+refinement, [4] directions+RHS, [5] step length, [6] update. */
int sdpx_b200_phase_times(sdpx_b200_handle* h, double* ms7, int reset);

#ifdef __cplusplus
}
#endif
#endif /* SDPX_B200_H */
