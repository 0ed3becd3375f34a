/*
 * SDPX-B200 C ABI — reduced normal system of SDPX's LP standard form and of
 * Lorentz (second-order) cones: NT scaling, the scaled normal matrix
 * Q = B̂ᵀB̂ + δI, its Cholesky factor and the direction recovery.
 *
 * Status codes follow sdpx_b200.h: 0 = ok, > 0 = numerical outcome, < 0 =
 * usage or CUDA error with a message from sdpx_b200_normal_last_error().
 *
 * Data conventions (SDPX's LPStandardFormSystem, src/lp_solver.jl:85-100):
 *   - B is n × m_eq column-major (variable-major rows, one column per
 *     equality), n = n_lp + Σ cone_dims;
 *   - variables are ordered [n_lp LP variables | cone 1 | cone 2 | …]; cone k
 *     occupies cone_dims[k] consecutive variables, head coordinate first;
 *   - LP variable j reads weights[row_for_variable[j]] (0-based) and the
 *     diagonal coefficient g_j of the permutation-diagonal G.
 * The Hessian of the eliminated primal block is D = blockdiag(diag(w_row·g² + δ),
 * Hs_1, …) with Hs_k = W_kᵀW_k the Nesterov–Todd metric of cone k.
 */
#ifndef SDPX_B200_NORMAL_H
#define SDPX_B200_NORMAL_H

#include <stdint.h>

#include "sdpx_b200.h" /* sdpx_b200_solve_options, sdpx_b200_solve_result */

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sdpx_b200_normal sdpx_b200_normal;

/* Upload B and the LP row map.  Replaces the construction of
 * LPStandardFormSystem (src/lp_solver.jl:85-100,1858-1890) and of the
 * NativeSOC workspace's NT buffers filled by `_native_soc_scaling!`
 * (src/soc_native.jl:1083-1098). */
int sdpx_b200_normal_create(int32_t n_lp, int32_t n_cones, const int32_t* cone_dims, int32_t m_eq,
                            const double* B, const int32_t* row_for_variable,
                            const double* diagonal_coefficient, int32_t n_weights, int device,
                            sdpx_b200_normal** out);
void sdpx_b200_normal_destroy(sdpx_b200_normal* h);
const char* sdpx_b200_normal_last_error(const sdpx_b200_normal* h);
/* Message of the last failed sdpx_b200_normal_create on this thread. */
const char* sdpx_b200_normal_create_error(void);

/* NT scaling point of every cone from the slack s and dual z (cone part, Σq
 * doubles each) — `_soc_nt_scaling!` (src/soc_lorentz_kernels.jl:72-185),
 * evaluated per cone in the reference's operation order.  ok[k] (n_cones) is 1
 * when cone k's scaling exists; the scalings are kept for the next
 * assemble/solve.  Optional outputs (NULL to skip): w, lambda (Σq), eta,
 * eta_squared (n_cones).  Returns 1 when any cone failed. */
int sdpx_b200_normal_nt_scaling(sdpx_b200_normal* h, const double* s, const double* z, int32_t* ok,
                                double* w, double* lambda, double* eta, double* eta_squared);

/* Apply a per-cone NT map to v (Σq) with the kept scalings: which = 0 → W
 * (`_soc_nt_apply_w!`, src/soc_lorentz_kernels.jl:187-206), 1 → W⁻¹
 * (`_soc_nt_apply_winv!`, :208-227), 2 → Hs⁻¹ = (WᵀW)⁻¹
 * (`_soc_nt_apply_hs_inverse!`, :229-255). */
int sdpx_b200_normal_nt_apply(sdpx_b200_normal* h, int32_t which, const double* v, double* out);

/* LP pack `_lp_standard_pack_range!` (src/lp_solver.jl:1892-1915):
 * D_j = weights[row_j]·g_j² + δ, D⁻¹, D^{-1/2} (n_lp each; NULL to skip). */
int sdpx_b200_normal_pack(sdpx_b200_normal* h, const double* weights, double regularization,
                          double* D, double* inverse_diagonal, double* inverse_sqrt);

/* Assemble Q = B̂ᵀB̂ + δI, B̂ = [D^{-1/2}B_LP ; W_k⁻¹B_k] (so Q = Bᵀ D⁻¹ B + δI),
 * one FP64 SYRK on the tensor cores — `_lp_assemble_reduced_schur!`
 * (src/lp_solver.jl:1998-2040) with the Lorentz blocks' metric
 * Aᵀ Hs⁻¹ A of `_native_soc_add_metric!` (src/soc_native.jl:1119-1218).
 * Requires nt_scaling first when n_cones > 0. */
int sdpx_b200_normal_assemble(sdpx_b200_normal* h, const double* weights, double regularization);

/* Assemble and factor with regularization retries: up to max_attempts tries,
 * δ ×10 after each non-positive-definite factor (src/lp_solver.jl:4090-4115,
 * `_lp_factor_reduced!` :2321-2343).  Returns 1 when every attempt failed. */
int sdpx_b200_normal_factorize(sdpx_b200_normal* h, const double* weights, double regularization,
                               int32_t max_attempts, int32_t* attempts,
                               double* regularization_used);

/* m_eq×m_eq column-major copy of the last assembled Q (full symmetric),
 * or of its lower Cholesky factor when which = 1. */
int sdpx_b200_normal_get_matrix(sdpx_b200_normal* h, int32_t which, double* out);

/* rhs = [rx (n); ry (m_eq)] → [dx; dy] in place — `_lp_solve_factor!`
 * (src/lp_solver.jl:2177-2213): t = D⁻¹rx, dy = Q⁻¹(ry − Bᵀt),
 * dx = t + D⁻¹B·dy.  Returns 1 when no successful factor is held. */
int sdpx_b200_normal_solve(sdpx_b200_normal* h, double* rhs);

/* Primal-dual interior-point solve of the standard-form LP + Lorentz-cone
 * problem  min cᵀx  s.t.  Bᵀx = b,  x ∈ R₊^{n_lp} × L^{q_1} × …  (dual
 * max bᵀy s.t. By + z = c, z in the same cone) on this handle's B, every
 * vector and matrix operation on the device.  SDPX's LP loop `solve_lp!`
 * (src/lp_solver.jl:3651-4400: residuals and best snapshot, termination, the
 * regularised reduced factor with ×10 retries decaying to √(eps·√eps),
 * Mehrotra predictor-corrector under the adaptive controller of
 * src/adaptive_parameters.jl, fraction-to-boundary steps, the regularisation-
 * aware direction gate) with the Lorentz cones entering through their
 * Nesterov–Todd scaling (src/soc_lorentz_kernels.jl:72-255).  Start x = z = e,
 * y = 0.  The options' beta, gamma, eps_*, iter_max, max_time and
 * parameter_strategy apply.  x, z (n) and y (m_eq) receive the solution (the
 * best iterate when not Optimal; NULL to skip).  Requires the standard LP
 * layout (identity row_for_variable, g = 1). */
int sdpx_b200_normal_optimize(sdpx_b200_normal* h, const double* b, const double* c,
                              const sdpx_b200_solve_options* opts, sdpx_b200_solve_result* result,
                              double* x, double* y, double* z);

/* Device time (ms) of the last assemble (pack + scale + SYRK) and factor. */
int sdpx_b200_normal_times(sdpx_b200_normal* h, double* assemble_ms, double* factor_ms);
/* CUDA stream of the handle (cudaStream_t). */
int sdpx_b200_normal_get_stream(sdpx_b200_normal* h, void** stream);

#ifdef __cplusplus
}
#endif
#endif /* SDPX_B200_NORMAL_H */
