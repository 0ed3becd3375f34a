"""Scalar host-side control of the interior-point loop.

These are the parts of SDPX's iteration that never touch a matrix: the guarded
Mehrotra parameter controller (src/adaptive_parameters.jl) and the rolling
stagnation detector (src/stagnation.jl).  They run on the host between device
launches and decide sigma, step fractions, the backtracking factor, refinement
caps and when to stop.  Every constant and branch follows the cited lines so
that the device path sees exactly the parameters SDPX would choose.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import List, Optional

EPS = 2.220446049250313e-16
SQRT_EPS = math.sqrt(EPS)

# src/kkt.jl:3634-3637
REFINE_MIN_DECREASE = 0.5
REFINE_DEFAULT_TOL_ULPS = 64
# src/stagnation.jl:13, :26
PRECISION_FLOOR_ULPS = 16
PROJECTION_SLACK = 10.0
# src/solver/interior_point.jl:2703-2709
NEAR_SOLUTION_MERIT = 100.0
CENTERING_BETA_STEP = 4.0
CENTERING_BETA_MAX = 0.5


@dataclass
class SolverOptions:
    """Subset of `SolverOptions{Float64}` (src/types/workspaces.jl:101-170) the
    dense core reads, with the same defaults."""

    beta: float = 0.1
    gamma: float = 0.9
    omega_p: float = 1.0
    omega_d: float = 1.0
    eps_gap: float = 1e-10
    eps_primal: float = 1e-10
    eps_dual: float = 1e-10
    iter_max: int = 200
    restart: bool = True
    min_step: float = 1e-10
    omega_step: float = 1e5
    max_restarts: int = 5
    max_centering: int = 4
    stall_iterations: int = 15
    stall_tolerance: float = 1e-3
    step_rule: str = "auto"              # backtrack | fraction_to_boundary | auto
    refine_steps: int = 1
    refine_policy: str = "auto"          # fixed | adaptive | auto
    refine_max_steps: int = 8
    refine_tol: float = 0.0
    max_time: float = math.inf
    parameter_policy: str = "auto"       # fixed | auto
    parameter_strategy: str = "adaptive"  # fixed | adaptive
    adaptive_sigma_max: float = 0.0
    scaling: str = "auto"                # auto | none | equilibrate
    # Equality block of the KKT system (src/types/workspaces.jl:181):
    # "auto" = normal equations, rank-revealing QR once they lose rank;
    # "qr" = rank-revealing QR from the first factorization.
    equality_solver: str = "auto"
    verbosity: int = 0
    # B200 precision mode: "fp64" (plain FP64 device path) or "mixed"
    # (split-BF16 Schur assembly + FP32 factor + FP64 refinement, FP64 switch).
    precision: str = "fp64"
    mixed_condition_limit: float = 1e8

    def with_tolerance(self, tol: float) -> "SolverOptions":
        return replace(self, eps_gap=tol, eps_primal=tol, eps_dual=tol)


@dataclass
class IterationDiagnostics:
    """src/adaptive_parameters.jl:66-86."""

    iteration: int = 0
    primal_residual: float = math.inf
    dual_residual: float = math.inf
    relative_gap: float = math.inf
    mu: float = math.inf
    mu_aff: float = math.inf
    affine_primal_step: float = 0.0
    affine_dual_step: float = 0.0
    previous_primal_step: float = 1.0
    previous_dual_step: float = 1.0
    backtracking_count: int = 0
    regularization: float = 0.0
    refinement_count: int = 0
    factorization_quality: float = 1.0
    predicted_residual_reduction: float = 1.0
    achieved_residual_reduction: float = 1.0
    primal_psd_margin: float = 1.0
    dual_psd_margin: float = 1.0
    precision_floor: bool = False


@dataclass
class IterationParameters:
    """src/adaptive_parameters.jl:95-110."""

    sigma: float
    primal_fraction_to_boundary: float
    dual_fraction_to_boundary: float
    backtracking_factor: float
    minimum_step: float
    restart_scale: float
    primal_regularization: float = 0.0
    dual_regularization: float = 0.0
    refinement_tolerance: float = 0.0
    refinement_max_count: int = 0
    centrality_target: float = 0.0
    fallback: bool = False
    fallback_reason: str = "none"


@dataclass
class FixedParameterPolicy:
    """src/adaptive_parameters.jl:19-30, constructor :112-130."""

    sigma: float
    primal_fraction_to_boundary: float
    dual_fraction_to_boundary: float
    backtracking_factor: float
    primal_regularization: float
    dual_regularization: float
    refinement_tolerance: float
    refinement_max_count: int
    minimum_step: float
    restart_scale: float

    @staticmethod
    def from_options(opts: SolverOptions) -> "FixedParameterPolicy":
        tol = opts.refine_tol if opts.refine_tol > 0 else REFINE_DEFAULT_TOL_ULPS * EPS
        count = opts.refine_steps if opts.refine_policy == "fixed" else opts.refine_max_steps
        return FixedParameterPolicy(opts.beta, opts.gamma, opts.gamma, opts.gamma, 0.0, 0.0,
                                    tol, count, opts.min_step, opts.omega_step)

    def parameters(self, fallback: bool = False, reason: str = "none") -> IterationParameters:
        """`_fixed_iteration_parameters` (src/adaptive_parameters.jl:156-177)."""
        return IterationParameters(
            sigma=self.sigma,
            primal_fraction_to_boundary=self.primal_fraction_to_boundary,
            dual_fraction_to_boundary=self.dual_fraction_to_boundary,
            backtracking_factor=self.backtracking_factor,
            primal_regularization=self.primal_regularization,
            dual_regularization=self.dual_regularization,
            refinement_tolerance=self.refinement_tolerance,
            refinement_max_count=self.refinement_max_count,
            minimum_step=self.minimum_step,
            restart_scale=self.restart_scale,
            centrality_target=self.sigma,
            fallback=fallback,
            fallback_reason=reason,
        )


@dataclass
class AdaptiveParameterPolicy:
    """src/adaptive_parameters.jl:39-52, constructor :132-154."""

    fallback: FixedParameterPolicy
    sigma_min: float
    sigma_max: float
    fraction_min: float
    fraction_max: float
    backtracking_min: float
    backtracking_max: float
    centrality_floor: float
    severe_centrality_floor: float
    refinement_floor: float
    requested_tolerance: float
    instability_limit: int

    @staticmethod
    def from_options(opts: SolverOptions) -> "AdaptiveParameterPolicy":
        fixed = FixedParameterPolicy.from_options(opts)
        requested = min(opts.eps_gap, opts.eps_primal, opts.eps_dual)
        refinement_floor = max(REFINE_DEFAULT_TOL_ULPS * EPS,
                               requested * requested if requested > 0 else 0.0)
        general = max(0.5, fixed.sigma)
        sigma_max = max(opts.adaptive_sigma_max, fixed.sigma) if opts.adaptive_sigma_max > 0 else general
        return AdaptiveParameterPolicy(
            fixed,
            min(1.0 / 50.0, fixed.sigma),
            sigma_max,
            min(4.0 / 5.0, fixed.primal_fraction_to_boundary),
            max(99.0 / 100.0, fixed.primal_fraction_to_boundary),
            min(11.0 / 20.0, fixed.backtracking_factor),
            max(9.0 / 10.0, fixed.backtracking_factor),
            2.0 / 25.0,
            1.0 / 5.0,
            refinement_floor,
            requested,
            2,
        )


def _finite_diagnostics(d: IterationDiagnostics) -> bool:
    """src/adaptive_parameters.jl:203-218."""
    values = (d.primal_residual, d.dual_residual, d.mu, d.mu_aff, d.affine_primal_step,
              d.affine_dual_step, d.factorization_quality, d.primal_psd_margin, d.dual_psd_margin)
    return all(math.isfinite(v) for v in values) and d.mu > 0 and d.mu_aff >= 0


def _adaptive_fraction(p: AdaptiveParameterPolicy, affine_step: float, previous_step: float,
                       backtracking_count: int, ratio: float) -> float:
    """src/adaptive_parameters.jl:220-244."""
    if affine_step < 1.0 / 20.0:
        cand = 21.0 / 25.0
    elif affine_step < 1.0 / 5.0:
        cand = 9.0 / 10.0
    elif affine_step < 7.0 / 10.0:
        cand = 19.0 / 20.0
    else:
        cand = 99.0 / 100.0
    if previous_step < 1.0 / 10.0:
        cand = min(cand, 9.0 / 10.0)
    if backtracking_count >= 4:
        cand = min(cand, 22.0 / 25.0)
    if ratio < 1.0 / 1_000_000.0:
        cand = min(cand, 9.0 / 10.0)
    return min(max(cand, p.fraction_min), p.fraction_max)


def _clamp(v: float, lo: float, hi: float) -> float:
    return min(max(v, lo), hi)


def select_adaptive_parameters(p: AdaptiveParameterPolicy, d: IterationDiagnostics,
                               history: List[dict]) -> IterationParameters:
    """`select_parameters(::AdaptiveParameterPolicy, ...)`, src/adaptive_parameters.jl:246-424."""
    if not _finite_diagnostics(d):
        return p.fallback.parameters(True, "nonfinite_diagnostics")
    if d.factorization_quality <= 0:
        return p.fallback.parameters(True, "degraded_factorization")
    recent = 0
    for row in reversed(history):
        if row.get("unstable", False):
            recent += 1
        else:
            break
    if recent >= p.instability_limit:
        return p.fallback.parameters(True, "repeated_instability")
    cold_merit = max(d.primal_residual, d.dual_residual, d.relative_gap)
    if cold_merit >= 1.0:
        return p.fallback.parameters()

    ratio = _clamp(d.mu_aff / d.mu, 0.0, 1.0)
    affine_min = min(d.affine_primal_step, d.affine_dual_step)
    exponent = 3 if affine_min >= 3.0 / 4.0 else 2
    sigma_candidate = ratio ** exponent
    if (affine_min < 1.0 / 20.0 or d.achieved_residual_reduction > 5.0 / 4.0
            or d.factorization_quality < SQRT_EPS):
        floor = p.severe_centrality_floor
    elif (affine_min < 1.0 / 4.0 or d.backtracking_count >= 4
          or d.refinement_count >= max(p.fallback.refinement_max_count - 1, 1)):
        floor = p.centrality_floor
    else:
        floor = 0.0
    sigma_candidate = max(sigma_candidate, floor)
    if d.iteration <= 1:
        sigma_candidate = max(sigma_candidate, min(p.fallback.sigma, p.sigma_max))
    previous_sigma = history[-1]["sigma"] if history else p.fallback.sigma
    sigma = _clamp(4.0 / 5.0 * sigma_candidate + 1.0 / 5.0 * previous_sigma, p.sigma_min, p.sigma_max)

    primal_fraction = _adaptive_fraction(p, d.affine_primal_step, d.previous_primal_step,
                                         d.backtracking_count, ratio)
    dual_fraction = _adaptive_fraction(p, d.affine_dual_step, d.previous_dual_step,
                                       d.backtracking_count, ratio)
    if d.backtracking_count >= 6 or d.achieved_residual_reduction > 5.0 / 4.0:
        backtracking = 13.0 / 20.0
    elif d.backtracking_count >= 3:
        backtracking = 18.0 / 25.0
    elif affine_min > 4.0 / 5.0:
        backtracking = 17.0 / 20.0
    else:
        backtracking = 4.0 / 5.0
    backtracking = _clamp(backtracking, p.backtracking_min, p.backtracking_max)

    regularization = max(d.regularization / 10.0, SQRT_EPS) if d.regularization > 0 else 0.0
    refinement_tolerance = max(p.refinement_floor, p.fallback.refinement_tolerance)
    if d.factorization_quality < SQRT_EPS or d.refinement_count > 0:
        refinement_max_count = p.fallback.refinement_max_count
    else:
        refinement_max_count = min(p.fallback.refinement_max_count, 2)
    requested = p.requested_tolerance if p.requested_tolerance > 0 else SQRT_EPS
    precision_step_floor = max(100.0 * EPS, min(p.fallback.minimum_step, requested / 100.0))
    if d.factorization_quality < SQRT_EPS or d.backtracking_count >= 8:
        minimum_step = p.fallback.minimum_step
    else:
        minimum_step = precision_step_floor
    feasibility_min = max(min(d.primal_residual, d.dual_residual), requested)
    feasibility_ratio = max(d.primal_residual, d.dual_residual) / feasibility_min
    if feasibility_ratio > 1_000_000.0:
        restart_candidate = 1_000.0
    elif feasibility_ratio > 1_000.0:
        restart_candidate = 100.0
    else:
        restart_candidate = 10.0
    restart_scale = _clamp(restart_candidate, 10.0, p.fallback.restart_scale)
    return IterationParameters(
        sigma=sigma,
        primal_fraction_to_boundary=primal_fraction,
        dual_fraction_to_boundary=dual_fraction,
        backtracking_factor=backtracking,
        primal_regularization=regularization,
        dual_regularization=regularization,
        refinement_tolerance=refinement_tolerance,
        refinement_max_count=refinement_max_count,
        minimum_step=minimum_step,
        restart_scale=restart_scale,
        centrality_target=sigma,
    )


def _outcome_is_unstable(iteration, compl_red, feas_ratio, tX, tY):
    """src/adaptive_parameters.jl:574-608."""
    nonfinite = not (math.isfinite(compl_red) and math.isfinite(feas_ratio)
                     and math.isfinite(tX) and math.isfinite(tY))
    compl_growth = iteration > 3 and compl_red > 2
    feas_growth = iteration > 3 and feas_ratio > 3
    min_step = min(tX, tY)
    tiny = iteration > 3 and tX < 1e-6 and tY < 1e-6 and feas_ratio >= 1.0
    stalled = (iteration > 5 and min_step < 1.0 / 50.0 and feas_ratio > 49.0 / 50.0
               and compl_red > 49.0 / 50.0)
    if nonfinite:
        reason = "nonfinite_outcome"
    elif compl_growth:
        reason = "complementarity_growth"
    elif feas_growth:
        reason = "feasibility_growth"
    elif tiny:
        reason = "repeated_tiny_step"
    elif stalled:
        reason = "stalled_progress"
    else:
        reason = "none"
    return reason != "none", reason


def estimate_backtracking_count(step: float, gamma: float, rule: str) -> int:
    """src/adaptive_parameters.jl:523-531."""
    if rule != "backtrack":
        return 0
    if (not math.isfinite(step)) or step <= 0 or step >= 1 or gamma <= 0 or gamma >= 1:
        return 0
    ratio = math.log(step) / math.log(gamma)
    if math.isnan(ratio) or ratio <= 0:
        return 0
    if not math.isfinite(ratio):
        return 2 ** 62
    return max(0, int(round(ratio)))


class AdaptiveIPMController:
    """`AdaptiveIPMController` (src/adaptive_parameters.jl:440-480, :533-572, :617-770)."""

    def __init__(self, opts: SolverOptions):
        self.strategy = opts.parameter_strategy
        self.default_beta = opts.beta
        self.default_gamma = opts.gamma
        self.beta = opts.beta
        self.gamma = opts.gamma
        self.previous_complementarity = math.nan
        self.previous_feasibility = math.nan
        self.instability_count = 0
        self.fallback = False
        self.history: List[dict] = []
        self.fixed_policy = FixedParameterPolicy.from_options(opts)
        self.adaptive_policy = (AdaptiveParameterPolicy.from_options(opts)
                                if opts.parameter_strategy == "adaptive" else None)
        self.parameters = self.fixed_policy.parameters()

    def history_value(self, name, default):
        return self.history[-1].get(name, default) if self.history else default

    def select(self, d: IterationDiagnostics) -> IterationParameters:
        """`select_iteration_parameters!` (src/adaptive_parameters.jl:533-572)."""
        if self.fallback:
            pol = FixedParameterPolicy(self.default_beta, self.default_gamma, self.default_gamma,
                                       self.default_gamma, 0.0, 0.0,
                                       self.parameters.refinement_tolerance,
                                       self.parameters.refinement_max_count,
                                       self.parameters.minimum_step,
                                       self.parameters.restart_scale)
            params = pol.parameters(True, "previous_instability")
        elif self.adaptive_policy is not None:
            params = select_adaptive_parameters(self.adaptive_policy, d, self.history)
        else:
            params = self.fixed_policy.parameters()
        self.parameters = params
        self.beta = params.sigma
        self.gamma = min(params.primal_fraction_to_boundary, params.dual_fraction_to_boundary)
        if params.fallback:
            self.fallback = True
            self.beta = self.default_beta
            self.gamma = self.default_gamma
        return params

    def record(self, *, iteration, predictor_quality, complementarity_before,
               complementarity_after, primal_residual, dual_residual, primal_step,
               dual_step, primal_residual_after, dual_residual_after, backtracking_count,
               affine_primal_step, affine_dual_step, mu_before, mu_affine, relative_gap,
               regularization, refinement_count, refinement_residual,
               factorization_quality, primal_psd_margin, dual_psd_margin, precision_floor,
               selected: IterationParameters):
        """`record_and_update!` (src/adaptive_parameters.jl:617-760)."""
        reduction = (complementarity_after / complementarity_before
                     if complementarity_before > 0 else 1.0)
        feasibility = max(primal_residual, dual_residual)
        prev = self.previous_feasibility
        feas_ratio = feasibility / prev if (math.isfinite(prev) and prev > 0) else 1.0
        unstable, reason = _outcome_is_unstable(iteration, reduction, feas_ratio,
                                                primal_step, dual_step)
        if self.strategy == "adaptive" and not self.fallback:
            severe = reason in ("nonfinite_outcome", "complementarity_growth", "feasibility_growth")
            if severe:
                self.instability_count = 2
            elif unstable:
                self.instability_count += 1
            else:
                self.instability_count = max(self.instability_count - 1, 0)
            if self.instability_count >= 2:
                self.beta = self.default_beta
                self.gamma = self.default_gamma
                self.fallback = True
        residual_before = max(primal_residual, dual_residual, EPS)
        achieved = max(primal_residual_after, dual_residual_after) / residual_before
        self.history.append(dict(
            iteration=iteration, sigma=selected.sigma,
            primal_step=primal_step, dual_step=dual_step,
            backtracking_count=backtracking_count, refinement_count=refinement_count,
            primal_residual=primal_residual, dual_residual=dual_residual,
            achieved_residual_reduction=achieved, unstable=unstable,
            predictor_quality=predictor_quality, mu=mu_before, mu_aff=mu_affine,
            affine_primal_step=affine_primal_step, affine_dual_step=affine_dual_step,
            relative_gap=relative_gap, refinement_residual=refinement_residual,
            fallback=self.fallback or selected.fallback,
        ))
        self.previous_complementarity = complementarity_after
        self.previous_feasibility = feasibility

    def iteration_beta_gamma_strategy(self):
        """`controller_options` (src/adaptive_parameters.jl:771-782)."""
        return self.beta, self.gamma, ("fixed" if self.fallback else self.strategy)


class StagnationDetector:
    """src/stagnation.jl:56-175."""

    def __init__(self, window: int, tolerance: float):
        self.window = max(window, 0)
        self.tolerance = max(tolerance, 0.0)
        self.merits: List[float] = []
        self.at_floor: List[bool] = []
        self.reason = "none"
        self.rate = 0.0
        self.projected = math.inf

    def observe(self, merit: float, floor_reached: bool, remaining: int) -> bool:
        if self.window <= 0:
            return False
        self.merits.append(merit)
        self.at_floor.append(floor_reached)
        if len(self.merits) > self.window + 1:
            self.merits.pop(0)
            self.at_floor.pop(0)
        if len(self.merits) <= self.window:
            return False
        ref = self.merits[0]
        if not (math.isfinite(ref) and math.isfinite(merit) and ref > 0 and merit > 0):
            return False
        progress = math.log(ref) - math.log(merit)
        self.rate = progress / self.window
        if not (progress > self.tolerance):
            self.reason = "precision_floor" if all(self.at_floor) else "no_progress"
            self.projected = math.inf
            return True
        if merit <= 1.0:
            return False
        self.projected = math.log(merit) / self.rate
        if self.projected > PROJECTION_SLACK * max(remaining, 1):
            self.reason = "precision_floor" if all(self.at_floor) else "too_slow"
            return True
        return False


def stagnation_merit(opts: SolverOptions, p_res, d_res, gap_rel, compl, scale_p, scale_d,
                     objective_scale) -> float:
    """src/stagnation.jl:89-100."""
    def safe(e):
        return e if e > 0 else EPS
    merit = (p_res / scale_p) / safe(opts.eps_primal)
    merit = max(merit, (d_res / scale_d) / safe(opts.eps_dual))
    merit = max(merit, gap_rel / safe(opts.eps_gap))
    if math.isfinite(compl) and compl > 0:
        merit = max(merit, compl / (safe(opts.eps_gap) * max(1.0, objective_scale)))
    return merit


def at_precision_floor(p_res, d_res, gap_rel, scale_p, scale_d) -> bool:
    """src/stagnation.jl:108-114."""
    f = PRECISION_FLOOR_ULPS * EPS
    return (p_res / scale_p) <= f and (d_res / scale_d) <= f and gap_rel <= f
