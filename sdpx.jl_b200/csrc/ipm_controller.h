// Scalar interior-point controller shared by the dense-SDP loop
// (driver_api.inc) and the LP + Lorentz-cone loop (cone_ipm.inc): the guarded
// Mehrotra controller of src/adaptive_parameters.jl:19-782, the stagnation
// detector of src/stagnation.jl:56-175 and their constants.  Only scalars.
#pragma once
#include <cmath>
#include <deque>
#include <string>
#include <utility>
#include <vector>

#include "../../include/sdpx_b200.h"

namespace sdpx {
namespace ipm {

constexpr double kEpsD = 2.220446049250313e-16;
constexpr double kRefineUlps = 64.0;        // src/kkt.jl:3634-3637
constexpr double kFloorUlps = 16.0;         // src/stagnation.jl:13
constexpr double kProjectionSlack = 10.0;   // src/stagnation.jl:26
constexpr double kNearSolutionMerit = 100.0;  // src/solver/interior_point.jl:2703-2709
constexpr double kCenteringBetaStep = 4.0;
constexpr double kCenteringBetaMax = 0.5;
inline double sqrt_eps() { return std::sqrt(kEpsD); }

struct Params {  // IterationParameters, src/adaptive_parameters.jl:95-110
  double sigma = 0, primal_fraction = 0, dual_fraction = 0, backtracking = 0;
  double primal_reg = 0, dual_reg = 0, refinement_tolerance = 0;
  int refinement_max_count = 0;
  double minimum_step = 0, restart_scale = 0, centrality_target = 0;
  bool fallback = false;
};

struct Diag {  // IterationDiagnostics, src/adaptive_parameters.jl:66-86
  int iteration = 0;
  double primal_residual = INFINITY, dual_residual = INFINITY, relative_gap = INFINITY;
  double mu = INFINITY, mu_aff = INFINITY, affine_primal_step = 0, affine_dual_step = 0;
  double previous_primal_step = 1, previous_dual_step = 1;
  long long backtracking_count = 0;
  double regularization = 0;
  int refinement_count = 0;
  double factorization_quality = 1, achieved_residual_reduction = 1;
  double primal_psd_margin = 1, dual_psd_margin = 1;
  bool precision_floor = false;
};

struct Fixed {  // FixedParameterPolicy, src/adaptive_parameters.jl:19-30, :112-130
  double sigma, pf, df, bt, pr, dr, rtol;
  int rcount;
  double min_step, restart_scale;
  static Fixed from(const sdpx_b200_solve_options& o) {
    const double tol = o.refine_tol > 0 ? o.refine_tol : kRefineUlps * kEpsD;
    const int count = o.refine_policy == 0 ? o.refine_steps : o.refine_max_steps;
    return Fixed{o.beta, o.gamma, o.gamma, o.gamma, 0.0, 0.0, tol, count, o.min_step,
                 o.omega_step};
  }
  Params params(bool fallback = false) const {  // src/adaptive_parameters.jl:156-177
    Params p;
    p.sigma = sigma;
    p.primal_fraction = pf;
    p.dual_fraction = df;
    p.backtracking = bt;
    p.primal_reg = pr;
    p.dual_reg = dr;
    p.refinement_tolerance = rtol;
    p.refinement_max_count = rcount;
    p.minimum_step = min_step;
    p.restart_scale = restart_scale;
    p.centrality_target = sigma;
    p.fallback = fallback;
    return p;
  }
};

struct Adaptive {  // AdaptiveParameterPolicy, src/adaptive_parameters.jl:39-52, :132-154
  Fixed fb;
  double sigma_min, sigma_max, fraction_min, fraction_max, bt_min, bt_max;
  double centrality_floor, severe_floor, refinement_floor, requested;
  int instability_limit;
  static Adaptive from(const sdpx_b200_solve_options& o) {
    Adaptive a;
    a.fb = Fixed::from(o);
    const double req = std::min(o.eps_gap, std::min(o.eps_primal, o.eps_dual));
    a.refinement_floor = std::max(kRefineUlps * kEpsD, req > 0 ? req * req : 0.0);
    const double general = std::max(0.5, a.fb.sigma);
    a.sigma_max = o.adaptive_sigma_max > 0 ? std::max(o.adaptive_sigma_max, a.fb.sigma) : general;
    a.sigma_min = std::min(1.0 / 50.0, a.fb.sigma);
    a.fraction_min = std::min(4.0 / 5.0, a.fb.pf);
    a.fraction_max = std::max(99.0 / 100.0, a.fb.pf);
    a.bt_min = std::min(11.0 / 20.0, a.fb.bt);
    a.bt_max = std::max(9.0 / 10.0, a.fb.bt);
    a.centrality_floor = 2.0 / 25.0;
    a.severe_floor = 1.0 / 5.0;
    a.requested = req;
    a.instability_limit = 2;
    return a;
  }
};

inline double clampd(double v, double lo, double hi) { return std::min(std::max(v, lo), hi); }

// src/adaptive_parameters.jl:220-244
inline double adaptive_fraction(const Adaptive& p, double affine, double previous, long long bt,
                                double ratio) {
  double c;
  if (affine < 1.0 / 20.0) c = 21.0 / 25.0;
  else if (affine < 1.0 / 5.0) c = 9.0 / 10.0;
  else if (affine < 7.0 / 10.0) c = 19.0 / 20.0;
  else c = 99.0 / 100.0;
  if (previous < 1.0 / 10.0) c = std::min(c, 9.0 / 10.0);
  if (bt >= 4) c = std::min(c, 22.0 / 25.0);
  if (ratio < 1.0 / 1000000.0) c = std::min(c, 9.0 / 10.0);
  return std::min(std::max(c, p.fraction_min), p.fraction_max);
}

struct HistRow {
  int iteration;
  double sigma, primal_step, dual_step;
  long long backtracking_count;
  int refinement_count;
  double primal_residual, dual_residual, achieved;
  bool unstable;
};

// `select_parameters(::AdaptiveParameterPolicy, ...)`, src/adaptive_parameters.jl:246-424
inline Params select_adaptive(const Adaptive& p, const Diag& d, const std::vector<HistRow>& hist) {
  const double vals[] = {d.primal_residual, d.dual_residual, d.mu, d.mu_aff,
                         d.affine_primal_step, d.affine_dual_step, d.factorization_quality,
                         d.primal_psd_margin, d.dual_psd_margin};
  bool finite = d.mu > 0 && d.mu_aff >= 0;
  for (double v : vals) finite = finite && std::isfinite(v);
  if (!finite) return p.fb.params(true);
  if (d.factorization_quality <= 0) return p.fb.params(true);
  int recent = 0;
  for (auto it = hist.rbegin(); it != hist.rend(); ++it) {
    if (it->unstable) ++recent;
    else break;
  }
  if (recent >= p.instability_limit) return p.fb.params(true);
  const double cold_merit = std::max(d.primal_residual, std::max(d.dual_residual, d.relative_gap));
  if (cold_merit >= 1.0) return p.fb.params();
  const double ratio = clampd(d.mu_aff / d.mu, 0.0, 1.0);
  const double affine_min = std::min(d.affine_primal_step, d.affine_dual_step);
  double sigma_c = std::pow(ratio, affine_min >= 3.0 / 4.0 ? 3.0 : 2.0);
  double floor;
  if (affine_min < 1.0 / 20.0 || d.achieved_residual_reduction > 5.0 / 4.0 ||
      d.factorization_quality < sqrt_eps())
    floor = p.severe_floor;
  else if (affine_min < 1.0 / 4.0 || d.backtracking_count >= 4 ||
           d.refinement_count >= std::max(p.fb.rcount - 1, 1))
    floor = p.centrality_floor;
  else
    floor = 0.0;
  sigma_c = std::max(sigma_c, floor);
  if (d.iteration <= 1) sigma_c = std::max(sigma_c, std::min(p.fb.sigma, p.sigma_max));
  const double previous_sigma = hist.empty() ? p.fb.sigma : hist.back().sigma;
  const double sigma =
      clampd(4.0 / 5.0 * sigma_c + 1.0 / 5.0 * previous_sigma, p.sigma_min, p.sigma_max);
  const double pfrac = adaptive_fraction(p, d.affine_primal_step, d.previous_primal_step,
                                         d.backtracking_count, ratio);
  const double dfrac = adaptive_fraction(p, d.affine_dual_step, d.previous_dual_step,
                                         d.backtracking_count, ratio);
  double bt;
  if (d.backtracking_count >= 6 || d.achieved_residual_reduction > 5.0 / 4.0) bt = 13.0 / 20.0;
  else if (d.backtracking_count >= 3) bt = 18.0 / 25.0;
  else if (affine_min > 4.0 / 5.0) bt = 17.0 / 20.0;
  else bt = 4.0 / 5.0;
  bt = clampd(bt, p.bt_min, p.bt_max);
  const double reg = d.regularization > 0 ? std::max(d.regularization / 10.0, sqrt_eps()) : 0.0;
  const double rtol = std::max(p.refinement_floor, p.fb.rtol);
  const int rcount = (d.factorization_quality < sqrt_eps() || d.refinement_count > 0)
                         ? p.fb.rcount
                         : std::min(p.fb.rcount, 2);
  const double requested = p.requested > 0 ? p.requested : sqrt_eps();
  const double step_floor = std::max(100.0 * kEpsD, std::min(p.fb.min_step, requested / 100.0));
  const double min_step = (d.factorization_quality < sqrt_eps() || d.backtracking_count >= 8)
                              ? p.fb.min_step
                              : step_floor;
  const double feas_min = std::max(std::min(d.primal_residual, d.dual_residual), requested);
  const double feas_ratio = std::max(d.primal_residual, d.dual_residual) / feas_min;
  double restart_c;
  if (feas_ratio > 1000000.0) restart_c = 1000.0;
  else if (feas_ratio > 1000.0) restart_c = 100.0;
  else restart_c = 10.0;
  Params out;
  out.sigma = sigma;
  out.primal_fraction = pfrac;
  out.dual_fraction = dfrac;
  out.backtracking = bt;
  out.primal_reg = reg;
  out.dual_reg = reg;
  out.refinement_tolerance = rtol;
  out.refinement_max_count = rcount;
  out.minimum_step = min_step;
  out.restart_scale = clampd(restart_c, 10.0, p.fb.restart_scale);
  out.centrality_target = sigma;
  return out;
}

// src/adaptive_parameters.jl:574-608; returns (unstable, severe)
inline std::pair<bool, bool> outcome_unstable(int iteration, double compl_red, double feas_ratio,
                                              double tX, double tY) {
  const bool nonfinite = !(std::isfinite(compl_red) && std::isfinite(feas_ratio) &&
                           std::isfinite(tX) && std::isfinite(tY));
  const bool compl_growth = iteration > 3 && compl_red > 2;
  const bool feas_growth = iteration > 3 && feas_ratio > 3;
  const double min_step = std::min(tX, tY);
  const bool tiny = iteration > 3 && tX < 1e-6 && tY < 1e-6 && feas_ratio >= 1.0;
  const bool stalled = iteration > 5 && min_step < 1.0 / 50.0 && feas_ratio > 49.0 / 50.0 &&
                       compl_red > 49.0 / 50.0;
  const bool severe = nonfinite || compl_growth || feas_growth;
  return {severe || tiny || stalled, severe};
}

// src/adaptive_parameters.jl:523-531
inline long long estimate_backtracking(double step, double gamma, bool backtrack_rule) {
  if (!backtrack_rule) return 0;
  if (!std::isfinite(step) || step <= 0 || step >= 1 || gamma <= 0 || gamma >= 1) return 0;
  const double ratio = std::log(step) / std::log(gamma);
  if (std::isnan(ratio) || ratio <= 0) return 0;
  if (!std::isfinite(ratio)) return 1LL << 62;
  return std::max(0LL, (long long)std::nearbyint(ratio));
}

struct Controller {  // AdaptiveIPMController, src/adaptive_parameters.jl:440-782
  bool adaptive_strategy = true;
  double default_beta = 0.1, default_gamma = 0.9, beta = 0.1, gamma = 0.9;
  double previous_feasibility = NAN;
  int instability_count = 0;
  bool fallback = false;
  std::vector<HistRow> history;
  Fixed fixed{};
  Adaptive adaptive{};
  Params parameters;
  void init(const sdpx_b200_solve_options& o) {
    adaptive_strategy = o.parameter_strategy == 0;
    default_beta = beta = o.beta;
    default_gamma = gamma = o.gamma;
    previous_feasibility = NAN;
    instability_count = 0;
    fallback = false;
    history.clear();
    fixed = Fixed::from(o);
    if (adaptive_strategy) adaptive = Adaptive::from(o);
    parameters = fixed.params();
  }
  Params select(const Diag& d) {  // src/adaptive_parameters.jl:533-572
    Params p;
    if (fallback) {
      Fixed pol{default_beta, default_gamma, default_gamma, default_gamma, 0.0, 0.0,
                parameters.refinement_tolerance, parameters.refinement_max_count,
                parameters.minimum_step, parameters.restart_scale};
      p = pol.params(true);
    } else if (adaptive_strategy) {
      p = select_adaptive(adaptive, d, history);
    } else {
      p = fixed.params();
    }
    parameters = p;
    beta = p.sigma;
    gamma = std::min(p.primal_fraction, p.dual_fraction);
    if (p.fallback) {
      fallback = true;
      beta = default_beta;
      gamma = default_gamma;
    }
    return p;
  }
  // `record_and_update!`, src/adaptive_parameters.jl:617-760 (the fields the
  // selection reads back)
  void record(int iteration, double compl_before, double compl_after, double p_res,
              double d_res, double tX, double tY, double p_after, double d_after,
              long long bt_count, int refinement_count, const Params& selected) {
    const double reduction = compl_before > 0 ? compl_after / compl_before : 1.0;
    const double feasibility = std::max(p_res, d_res);
    const double prev = previous_feasibility;
    const double feas_ratio = (std::isfinite(prev) && prev > 0) ? feasibility / prev : 1.0;
    const auto un = outcome_unstable(iteration, reduction, feas_ratio, tX, tY);
    if (adaptive_strategy && !fallback) {
      if (un.second) instability_count = 2;
      else if (un.first) ++instability_count;
      else instability_count = std::max(instability_count - 1, 0);
      if (instability_count >= 2) {
        beta = default_beta;
        gamma = default_gamma;
        fallback = true;
      }
    }
    const double residual_before = std::max(p_res, std::max(d_res, kEpsD));
    const double achieved = std::max(p_after, d_after) / residual_before;
    history.push_back(HistRow{iteration, selected.sigma, tX, tY, bt_count, refinement_count,
                              p_res, d_res, achieved, un.first});
    previous_feasibility = feasibility;
  }
  bool strategy_adaptive() const { return adaptive_strategy && !fallback; }
};

struct Stagnation {  // src/stagnation.jl:56-175
  int window = 15;
  double tolerance = 1e-3;
  std::deque<double> merits;
  std::deque<bool> at_floor;
  int reason = 0;  // 0 none, 1 precision_floor, 2 no_progress, 3 too_slow
  double rate = 0.0;
  void init(int w, double tol) {
    window = std::max(w, 0);
    tolerance = std::max(tol, 0.0);
    merits.clear();
    at_floor.clear();
    reason = 0;
    rate = 0.0;
  }
  bool all_floor() const {
    for (bool b : at_floor)
      if (!b) return false;
    return true;
  }
  bool observe(double merit, bool floor_reached, long long remaining) {
    if (window <= 0) return false;
    merits.push_back(merit);
    at_floor.push_back(floor_reached);
    if ((int)merits.size() > window + 1) {
      merits.pop_front();
      at_floor.pop_front();
    }
    if ((int)merits.size() <= window) return false;
    const double ref = merits.front();
    if (!(std::isfinite(ref) && std::isfinite(merit) && ref > 0 && merit > 0)) return false;
    const double progress = std::log(ref) - std::log(merit);
    rate = progress / window;
    if (!(progress > tolerance)) {
      reason = all_floor() ? 1 : 2;
      return true;
    }
    if (merit <= 1.0) return false;
    const double projected = std::log(merit) / rate;
    if (projected > kProjectionSlack * std::max(remaining, 1LL)) {
      reason = all_floor() ? 1 : 3;
      return true;
    }
    return false;
  }
};

// src/stagnation.jl:89-100
inline double merit_of(const sdpx_b200_solve_options& o, double p_res, double d_res,
                       double gap_rel, double cmpl, double scale_p, double scale_d,
                       double objective_scale) {
  auto safe = [](double e) { return e > 0 ? e : kEpsD; };
  double m = (p_res / scale_p) / safe(o.eps_primal);
  m = std::max(m, (d_res / scale_d) / safe(o.eps_dual));
  m = std::max(m, gap_rel / safe(o.eps_gap));
  if (std::isfinite(cmpl) && cmpl > 0)
    m = std::max(m, cmpl / (safe(o.eps_gap) * std::max(1.0, objective_scale)));
  return m;
}
// Compensated (Neumaier) sum of the per-block scalars added on the host; the
// Python driver's `_seq_sum` is the same algorithm.
inline double comp_sum(const std::vector<double>& v) {
  double total = 0.0, comp = 0.0;
  for (double x : v) {
    const double t = total + x;
    if (std::fabs(total) >= std::fabs(x)) comp += (total - t) + x;
    else comp += (x - t) + total;
    total = t;
  }
  if (comp != 0.0 && std::isfinite(comp)) total += comp;
  return total;
}

// src/stagnation.jl:108-114
inline bool precision_floor(double p_res, double d_res, double gap_rel, double sp, double sd) {
  const double f = kFloorUlps * kEpsD;
  return (p_res / sp) <= f && (d_res / sd) <= f && gap_rel <= f;
}
// src/step.jl:383-394
inline double relative_regularization(int attempts) {
  if (attempts <= 0) return 0.0;
  double v = sqrt_eps();
  for (int i = 2; i <= attempts; ++i) v *= 10.0;
  return v;
}

}  // namespace ipm

}  // namespace sdpx
