"""Interior-point driver: SDPX's dense SDP core loop over a device backend.

This is the host half of the B200 provider.  It restates the control flow of
SDPX's `_solve_sdp_core!` (src/solver/interior_point.jl:1323-2687), its KKT
cold start (:699-1287) and `newton_step!` (src/step.jl:643-1023).  All matrix
work is delegated to a backend object whose methods are the hot-path seams of
the reference (residuals, Schur assembly, KKT factor/solve/refine, direction
recovery, line search, update); only scalars cross back to the host.

The product backend is `CudaBackend` (C-ABI library of sm_100a kernels).  Any
object with the same methods can drive the loop; the test-suite uses a NumPy
restatement of the reference kernels to pin this driver against SDPX's own
golden solves.
"""
from __future__ import annotations

import enum
import math
import time
from dataclasses import dataclass, field, replace
from typing import Any, Dict, List, Optional

import numpy as np

from .controller import (
    CENTERING_BETA_MAX, CENTERING_BETA_STEP, EPS, NEAR_SOLUTION_MERIT, SQRT_EPS,
    AdaptiveIPMController, IterationDiagnostics, IterationParameters, SolverOptions,
    StagnationDetector, at_precision_floor, estimate_backtracking_count, stagnation_merit,
)
from .problem import Equilibration, SDPProblem, unequilibrate


class Status(enum.Enum):
    """Subset of SDPX's `SolveStatus` reachable from the dense SDP core."""

    Optimal = "Optimal"
    IterLimit = "IterLimit"
    Stalled = "Stalled"
    InsufficientPrecision = "InsufficientPrecision"
    NumericalBreakdown = "NumericalBreakdown"
    MaxRestartsExceeded = "MaxRestartsExceeded"
    TimeLimit = "TimeLimit"


@dataclass
class SDPResult:
    status: Status
    message: str
    x: np.ndarray
    X: List[np.ndarray]
    y: np.ndarray
    Y: List[np.ndarray]
    pObj: float
    dObj: float
    p_res: float
    d_res: float
    iterations: int
    restarts: int
    history: List[Dict[str, Any]] = field(default_factory=list)
    precision_trace: List[str] = field(default_factory=list)
    seconds: float = 0.0
    certificate: Optional[Dict[str, Any]] = None

    @property
    def relative_gap(self) -> float:
        return abs(self.pObj - self.dObj) / max(1.0, (abs(self.pObj) + abs(self.dObj)) / 2)


def _seq_sum(values) -> float:
    """Compensated (Neumaier) sum of the per-block scalars the loop adds on
    the host (block traces and ⟨X_l, Y_l⟩ for the cold-start shifts and the
    stagnation merit), written out so that it is the same in every interpreter
    and in the library's own loop (sdpx_b200_optimize, `ipm::comp_sum`)."""
    total, comp = 0.0, 0.0
    for v in values:
        v = float(v)
        t = total + v
        if abs(total) >= abs(v):
            comp += (total - t) + v
        else:
            comp += (v - t) + total
        total = t
    if comp and math.isfinite(comp):
        total += comp
    return total


def _relative_regularization(attempts: int) -> float:
    """src/step.jl:383-394."""
    if attempts <= 0:
        return 0.0
    value = SQRT_EPS
    for _ in range(2, attempts + 1):
        value *= 10.0
    return value


def resolved_step_rule(k: List[int], rule: str) -> str:
    """src/kernels/threaded.jl:1589-1600."""
    if rule == "auto":
        return "fraction_to_boundary" if all(kl <= 2 for kl in k) else "backtrack"
    return rule


# --------------------------------------------------------------------------
#   Newton step (src/step.jl:643-1023)
# --------------------------------------------------------------------------

def newton_step(be, opts: SolverOptions, ctl: AdaptiveIPMController, mu: List[float], *,
                iteration: int, relative_gap: float, primal_scale: float,
                dual_scale: float) -> Dict[str, Any]:
    beta, gamma, strategy = ctl.iteration_beta_gamma_strategy()
    use_affine = strategy == "adaptive"
    p_res, d_res, blocks_ok = be.compute_residuals(mu, use_affine, True)
    if not blocks_ok:
        return dict(status="breakdown",
                    reason="Cholesky factorization of X or Y failed (iterate left the interior)",
                    p_res=p_res, d_res=d_res, reg_attempts=0)
    be.schur_build()
    kkt = be.factorize()
    if not kkt["ok"]:
        return dict(status="breakdown",
                    reason=("Schur complement not positive definite after "
                            f"{kkt['reg_attempts']} regularization attempt(s)"),
                    p_res=p_res, d_res=d_res, reg_attempts=kkt["reg_attempts"])
    # ---- predictor ----
    be.predictor_rhs()
    be.solve_direction()
    be.direction_blocks()

    adaptive = strategy == "adaptive" and not ctl.fallback
    pd = be.affine_diagnostics(adaptive)
    prev_tX = ctl.history_value("primal_step", 1.0)
    prev_tY = ctl.history_value("dual_step", 1.0)
    prev_bt = ctl.history_value("backtracking_count", 0)
    prev_ref = ctl.history_value("refinement_count", 0)
    cur_feas = max(p_res / max(primal_scale, 1.0), d_res / max(dual_scale, 1.0))
    if not ctl.history:
        prev_achieved = 1.0
    else:
        row = ctl.history[-1]
        prev_feas = max(row["primal_residual"] / max(primal_scale, 1.0),
                        row["dual_residual"] / max(dual_scale, 1.0), EPS)
        prev_achieved = cur_feas / prev_feas
    primal_margin, dual_margin = be.block_margins()
    quality = kkt["quality"]
    regularization = _relative_regularization(kkt["reg_attempts"])
    diag = IterationDiagnostics(
        iteration=iteration,
        primal_residual=p_res / max(primal_scale, 1.0),
        dual_residual=d_res / max(dual_scale, 1.0),
        relative_gap=relative_gap,
        mu=pd["mu"], mu_aff=pd["mu_aff"],
        affine_primal_step=pd["tX"], affine_dual_step=pd["tY"],
        previous_primal_step=prev_tX, previous_dual_step=prev_tY,
        backtracking_count=prev_bt, regularization=regularization,
        refinement_count=prev_ref, factorization_quality=quality,
        predicted_residual_reduction=max(abs(1.0 - pd["tX"]), abs(1.0 - pd["tY"])),
        achieved_residual_reduction=prev_achieved,
        primal_psd_margin=primal_margin, dual_psd_margin=dual_margin,
        precision_floor=at_precision_floor(p_res, d_res, relative_gap, primal_scale, dual_scale),
    )
    params = ctl.select(diag)

    # ---- corrector ----
    if adaptive and not params.fallback:
        be.mehrotra_corrector_rhs(params.sigma, pd["mu"], not pd["uniform"])
    else:
        be.fixed_corrector_rhs(beta, mu)
    be.solve_direction()
    if adaptive and not params.fallback:
        refine_tol, refine_cap = params.refinement_tolerance, params.refinement_max_count
    else:
        refine_tol, refine_cap = opts.refine_tol, opts.refine_max_steps
    refine_steps, _ = be.refine(opts.refine_policy, refine_tol, refine_cap, opts.refine_steps)
    # Acceptance gate, src/step.jl:911-930 and src/kkt.jl:3670-3687.
    residual, r_norm = be.direction_residual()
    direction_tol = max(SQRT_EPS, opts.eps_primal, opts.eps_dual) * max(r_norm, 1.0)
    if not math.isfinite(residual) or residual > direction_tol:
        return dict(status="breakdown",
                    reason=(f"final structured KKT direction residual {residual} "
                            f"exceeded the accepted tolerance {direction_tol}"),
                    p_res=p_res, d_res=d_res, reg_attempts=kkt["reg_attempts"])
    block_primal_residual = be.block_primal_residual()
    be.direction_blocks()
    return dict(status="ok", p_res=p_res, d_res=d_res,
                block_primal_residual=block_primal_residual,
                reg_attempts=kkt["reg_attempts"], predictor_quality=pd["quality"],
                complementarity=pd["complementarity"], mu=pd["mu"], mu_aff=pd["mu_aff"],
                affine_primal_step=pd["tX"], affine_dual_step=pd["tY"],
                factorization_quality=quality, primal_psd_margin=primal_margin,
                dual_psd_margin=dual_margin, regularization=regularization,
                precision_floor=diag.precision_floor, params=params,
                refine_steps=refine_steps, refine_residual=residual)


# --------------------------------------------------------------------------
#   KKT cold start (src/solver/interior_point.jl:699-1287, src/cold_start.jl)
# --------------------------------------------------------------------------

def kkt_cold_start(be, opts: SolverOptions, scale_p: float, scale_d: float):
    k = be.k
    L = len(k)
    total_degree = sum(k)
    be.schur_build(identity=True)
    kkt = be.factorize()
    if not kkt["ok"]:
        return dict(ok=False, reason="identity_kkt_factorization")
    threshold = max(SQRT_EPS, opts.eps_primal, opts.eps_dual)

    def solve_cold(which: str):
        be.set_rhs(which)
        be.solve_direction()
        initial, r_norm = be.direction_residual()
        scale = max(r_norm, 1.0)
        normalized = initial / scale
        if math.isfinite(normalized) and normalized > threshold:
            be.refine(opts.refine_policy, opts.refine_tol, opts.refine_max_steps, opts.refine_steps)
            final, _ = be.direction_residual()
            normalized = final / scale
        return math.isfinite(normalized) and normalized <= threshold

    if not solve_cold("cold_primal"):
        return dict(ok=False, reason="kkt_cold_start_solve")
    be.keep_direction_as("x")
    if not solve_cold("cold_dual"):
        return dict(ok=False, reason="kkt_cold_start_solve")
    be.cold_start_iterate()     # X = mat(Av x) - C, Y = mat(Av v), y = -q
    p_res, d_res, _ = be.compute_residuals([0.0] * L, opts.parameter_strategy == "adaptive", False)
    np_, nd_ = p_res / scale_p, d_res / scale_d
    if not (math.isfinite(np_) and math.isfinite(nd_) and np_ <= threshold and nd_ <= threshold):
        return dict(ok=False, reason="kkt_cold_start_residuals")
    # Per-block certified identity shifts (`_cold_start_psd_shift!`,
    # src/cold_start.jl:287-308).  Blocks are independent, so shifting every X
    # block and then every Y block equals the reference's interleaved loop.
    if not (be.psd_shift("X") and be.psd_shift("Y")):
        return dict(ok=False, reason="cold_start_psd_shift")
    dots, trX, trY = be.block_dots()
    primal_mass, dual_mass = _seq_sum(trX), _seq_sum(trY)
    # _cold_start_identity_mass_shifts (src/cold_start.jl:338-360)
    if not (total_degree > 0 and math.isfinite(primal_mass) and math.isfinite(dual_mass)):
        return dict(ok=False, reason="cold_start_identity_mass_floor")
    target = float(total_degree)
    p_floor = max(0.0, (target - primal_mass) / target)
    d_floor = max(0.0, (target - dual_mass) / target)
    if p_floor > 0:
        be.add_identity("X", p_floor)
    if d_floor > 0:
        be.add_identity("Y", d_floor)
    dots, trX, trY = be.block_dots()
    kappa = _seq_sum(dots)
    pm, dm = _seq_sum(trX), _seq_sum(trY)
    # _cold_start_centering_shifts (src/cold_start.jl:407-430)
    ok = (math.isfinite(kappa) and kappa > 0 and math.isfinite(pm) and pm > 0
          and math.isfinite(dm) and dm > 0)
    if not ok:
        return dict(ok=False, reason="cold_start_centering_shifts")
    p_center = kappa / (2.0 * dm)
    d_center = kappa / (2.0 * pm)
    if p_center > 0:
        be.add_identity("X", p_center)
    if d_center > 0:
        be.add_identity("Y", d_center)
    # The margin pass re-runs the certified shift (src/solver/interior_point.jl:1166-1169).
    be.psd_shift("X")
    be.psd_shift("Y")
    dots, _, _ = be.block_dots()
    mu = [opts.beta * dots[l] / k[l] for l in range(L)]
    return dict(ok=True, mu=mu)


# --------------------------------------------------------------------------
#   Core loop (src/solver/interior_point.jl:1323-2687)
# --------------------------------------------------------------------------

def solve_core(be, opts: SolverOptions, *, termination_gap_tolerance: Optional[float] = None,
               trace: Optional[List[Dict[str, Any]]] = None) -> Dict[str, Any]:
    """Run the interior-point loop on the (already scaled) problem held by `be`.

    Returns the final status, scaled iterate objectives and counters; the
    iterate itself stays on the device and is read with `be.get_iterate()`.
    """
    t0 = time.perf_counter()
    k = be.k
    L = len(k)
    if termination_gap_tolerance is None:
        termination_gap_tolerance = opts.eps_gap
    max_C, c_norm, b_norm = be.data_norms()
    scale_p = 1.0 + max(max_C, b_norm if be.n > 0 else 0.0)
    scale_d = 1.0 + c_norm

    fully_cold = opts.parameter_policy == "auto"
    if fully_cold:
        cs = kkt_cold_start(be, opts, scale_p, scale_d)
        if not cs["ok"]:
            return dict(status=Status.NumericalBreakdown,
                        message=f"Cold-start KKT initialization failed ({cs['reason']}).",
                        iterations=0, restarts=0, pObj=0.0, dObj=0.0, p_res=math.inf,
                        d_res=math.inf, seconds=time.perf_counter() - t0)
        mu = cs["mu"]
    else:
        be.fixed_start(opts.omega_p, opts.omega_d)
        dots, _, _ = be.block_dots()
        mu = [opts.beta * dots[l] / k[l] for l in range(L)]

    # After the automatic resolver the solve runs with the fixed parameter
    # *policy* but the adaptive *strategy* (src/solver/interior_point.jl:1424-1434).
    ctl = AdaptiveIPMController(opts)
    iter_ = 0
    restarts = 0
    centering_attempts = 0
    pObj, dObj = be.objectives()
    p_res, d_res, _ = be.compute_residuals(mu, ctl.strategy == "adaptive", False)
    status: Optional[Status] = None
    message = ""
    best_merit = math.inf
    initial_merit = math.inf
    stagnation = StagnationDetector(opts.stall_iterations, opts.stall_tolerance)
    dots, _, _ = be.block_dots()
    current_compl = _seq_sum(dots)
    best = None
    step_rule = resolved_step_rule(k, opts.step_rule)
    adaptive_margin = SQRT_EPS if opts.parameter_strategy == "adaptive" else 0.0

    while True:
        gap = pObj - dObj
        gap_rel = abs(gap) / max(1.0, (abs(pObj) + abs(dObj)) / 2)
        term_ok = p_res / scale_p <= opts.eps_primal and d_res / scale_d <= opts.eps_dual
        gap_ok = gap_rel <= termination_gap_tolerance
        if term_ok and gap_ok:
            p_res, d_res = be.solution_residuals()
            term_ok = p_res / scale_p <= opts.eps_primal and d_res / scale_d <= opts.eps_dual
        objective_scale = max(abs(pObj), abs(dObj))
        merit = stagnation_merit(opts, p_res, d_res, gap_rel, current_compl, scale_p, scale_d,
                                 objective_scale)
        floor_reached = at_precision_floor(p_res, d_res, gap_rel, scale_p, scale_d)
        stagnated = stagnation.observe(merit, floor_reached, opts.iter_max - iter_)
        if math.isfinite(merit) and not math.isfinite(initial_merit):
            initial_merit = merit
        if math.isfinite(merit) and merit < best_merit:
            best_merit = merit
            be.store_best()
            best = dict(pObj=pObj, dObj=dObj, p_res=p_res, d_res=d_res, iter=iter_)
        if trace is not None:
            trace.append(dict(iter=iter_, pObj=pObj, dObj=dObj, gap_rel=gap_rel, p_res=p_res,
                              d_res=d_res, merit=merit, precision=be.precision_label()))
        if term_ok and gap_ok:
            status, message = Status.Optimal, "Optimal"
            break
        if iter_ >= opts.iter_max:
            status = Status.IterLimit
            message = f"Cannot reach optimality within {opts.iter_max} iterations."
            break
        if stagnated:
            status = (Status.InsufficientPrecision if stagnation.reason == "precision_floor"
                      else Status.Stalled)
            message = f"Convergence stagnated ({stagnation.reason})."
            break
        if time.perf_counter() - t0 > opts.max_time:
            status, message = Status.TimeLimit, "Time limit exceeded."
            break

        be.begin_iteration(dict(gap_rel=gap_rel, p_res=p_res / scale_p, d_res=d_res / scale_d,
                                stagnated=False, stagnation_rate=stagnation.rate,
                                window_full=len(stagnation.merits) > stagnation.window))
        res = newton_step(be, opts, ctl, mu, iteration=iter_ + 1, relative_gap=gap_rel,
                          primal_scale=scale_p, dual_scale=scale_d)
        if res["status"] == "breakdown":
            if be.fallback_to_fp64(res["reason"]):
                continue
            status, message = Status.NumericalBreakdown, res["reason"]
            break
        p_res, d_res = res["p_res"], res["d_res"]
        params: IterationParameters = res["params"]
        tX, tY = be.line_search(step_rule, params.primal_fraction_to_boundary,
                                params.dual_fraction_to_boundary, params.backtracking_factor,
                                params.minimum_step, adaptive_margin)
        bt_count = (estimate_backtracking_count(tX, params.backtracking_factor, step_rule)
                    + estimate_backtracking_count(tY, params.backtracking_factor, step_rule))

        primal_feasible = p_res / scale_p <= opts.eps_primal
        dual_feasible = d_res / scale_d <= opts.eps_dual
        x_stuck = tX < params.minimum_step
        y_stuck = tY < params.minimum_step
        if x_stuck and primal_feasible and not y_stuck:
            tX, x_stuck = 0.0, False
        if y_stuck and dual_feasible and not x_stuck:
            tY, y_stuck = 0.0, False
        if x_stuck or y_stuck:
            if x_stuck and y_stuck and be.fallback_to_fp64("outer_step_collapse"):
                continue
            near_tol = 1000.0
            gap_now = abs(pObj - dObj) / max(1.0, (abs(pObj) + abs(dObj)) / 2)
            if (gap_now < near_tol * termination_gap_tolerance
                    and p_res / scale_p < near_tol * opts.eps_primal
                    and d_res / scale_d < near_tol * opts.eps_dual):
                status = Status.Stalled
                message = "Step size collapsed near, but not within, the requested tolerance."
                break
            omega_step = params.restart_scale
            made_progress = (math.isfinite(initial_merit) and best_merit < initial_merit * 1e-3
                             and best_merit < NEAR_SOLUTION_MERIT)
            if opts.stall_iterations > 0 and made_progress:
                status = Status.InsufficientPrecision
                message = "Step size collapsed after the solve had already converged (precision exhaustion)."
                break
            if centering_attempts < opts.max_centering and ctl.beta < CENTERING_BETA_MAX:
                centering_attempts += 1
                ctl.beta = min(ctl.beta * CENTERING_BETA_STEP, CENTERING_BETA_MAX)
                dots, _, _ = be.block_dots()
                mu = [ctl.beta * dots[l] / k[l] for l in range(L)]
                continue
            rescale_X = x_stuck and not primal_feasible
            rescale_Y = y_stuck and not dual_feasible
            if opts.restart and restarts < opts.max_restarts and (rescale_X or rescale_Y):
                restarts += 1
                if rescale_X:
                    be.scale_iterate("X", omega_step)
                if rescale_Y:
                    be.scale_iterate("Y", omega_step)
                dots, _, _ = be.block_dots()
                current_compl = _seq_sum(dots)
                mu = [ctl.beta * dots[l] / k[l] for l in range(L)]
                continue
            elif opts.restart and restarts < opts.max_restarts:
                status = Status.Stalled
                message = "Step size collapsed while both residuals were already within tolerance."
                break
            else:
                status = (Status.MaxRestartsExceeded if restarts >= opts.max_restarts
                          else Status.NumericalBreakdown)
                message = "Step size collapsed."
                break

        compl_after, finite, block_dots = be.update(tX, tY)
        if not finite:
            status, message = Status.NumericalBreakdown, "non-finite primal or dual iterate detected"
            break
        p_after, d_after = be.accepted_trial_residuals(res["block_primal_residual"], tX, tY)
        ctl.record(iteration=iter_ + 1, predictor_quality=res["predictor_quality"],
                   complementarity_before=res["complementarity"],
                   complementarity_after=compl_after, primal_residual=p_res,
                   dual_residual=d_res, primal_step=tX, dual_step=tY,
                   primal_residual_after=p_after, dual_residual_after=d_after,
                   backtracking_count=bt_count, affine_primal_step=res["affine_primal_step"],
                   affine_dual_step=res["affine_dual_step"], mu_before=res["mu"],
                   mu_affine=res["mu_aff"], relative_gap=gap_rel,
                   regularization=res["regularization"], refinement_count=res["refine_steps"],
                   refinement_residual=res["refine_residual"],
                   factorization_quality=res["factorization_quality"],
                   primal_psd_margin=res["primal_psd_margin"],
                   dual_psd_margin=res["dual_psd_margin"],
                   precision_floor=res["precision_floor"], selected=params)
        current_compl = compl_after
        # threaded_update_mu! (src/kernels/threaded.jl:756-801)
        if ctl.strategy == "adaptive" and not ctl.fallback:
            target = ctl.beta * compl_after / max(sum(k), 1)
            mu = [target] * L
        else:
            mu = [ctl.beta * block_dots[l] / k[l] for l in range(L)]
        if not all(math.isfinite(v) for v in mu):
            status, message = Status.NumericalBreakdown, "non-finite complementarity target detected"
            break
        pObj, dObj = be.objectives()
        if not (math.isfinite(pObj) and math.isfinite(dObj)):
            status, message = Status.NumericalBreakdown, "non-finite primal or dual objective detected"
            break
        iter_ += 1
        p_res, d_res = p_after, d_after
        if trace is not None:
            trace[-1].update(tX=tX, tY=tY, sigma=params.sigma,
                             refine_steps=res["refine_steps"], reg=res["reg_attempts"])

    if status is not Status.Optimal and best is not None:
        final_merit = stagnation_merit(opts, p_res, d_res,
                                       abs(pObj - dObj) / max(1.0, (abs(pObj) + abs(dObj)) / 2),
                                       current_compl, scale_p, scale_d, max(abs(pObj), abs(dObj)))
        if not math.isfinite(final_merit) or best_merit < final_merit / 2:
            be.restore_best()
            pObj, dObj = best["pObj"], best["dObj"]
            p_res, d_res = best["p_res"], best["d_res"]
            message += f" Returned the best iterate found (iteration {best['iter']})."
    return dict(status=status, message=message, iterations=iter_, restarts=restarts,
                pObj=pObj, dObj=dObj, p_res=p_res, d_res=d_res,
                seconds=time.perf_counter() - t0)


def solve_with_backend(be, opts: SolverOptions, *, trace=None) -> SDPResult:
    """`_solve_pipeline!` restricted to the dense SDP route
    (src/solver/interior_point.jl:3131-3571): Ruiz scaling (plan.scaling ===
    :sdp_ruiz for `scaling=:auto`), the core loop, unscaling, slack rebuild and
    original-coordinate residuals."""
    t0 = time.perf_counter()
    if be.n > 0:
        # `_requested_accuracy` (src/kkt.jl:518-521) sets the rank tolerance of
        # the equality factor; `equality_solver` picks its first method.
        requested = min(opts.eps_gap, opts.eps_primal, opts.eps_dual)
        be.configure_equality(requested if requested > 0 else SQRT_EPS, opts.equality_solver)
    eq: Optional[Equilibration] = None
    if opts.scaling in ("auto", "equilibrate"):
        eq = be.equilibrate()
    term_tol = opts.eps_gap
    if eq is not None and eq.objective_scale > 1.0:
        term_tol = opts.eps_gap / eq.objective_scale
    core = solve_core(be, opts, termination_gap_tolerance=term_tol, trace=trace)
    x, X, y, Y = be.get_iterate()
    if eq is not None:
        x, X, y, Y = unequilibrate(eq, x, X, y, Y)
    be.restore_original()
    X = be.rebuild_slack(x)
    pObj = float(be.original_c() @ x)
    dObj = float(sum(np.sum(Cl * Yl) for Cl, Yl in zip(be.original_C(), Y)))
    if be.n > 0:
        dObj += float(np.asarray(be.original_b()) @ np.asarray(y))
    p_res, d_res = be.original_residuals(x, X, y, Y)
    return SDPResult(status=core["status"], message=core["message"], x=x, X=X, y=y, Y=Y,
                     pObj=pObj, dObj=dObj, p_res=p_res, d_res=d_res,
                     iterations=core["iterations"], restarts=core["restarts"],
                     history=trace if trace is not None else [],
                     precision_trace=be.precision_history(),
                     seconds=time.perf_counter() - t0)
