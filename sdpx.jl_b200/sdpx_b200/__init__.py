"""SDPX-B200: a B200-native dense-SDP interior-point core for SDPX.

Public surface mirrors SDPX's qualified entry points:

* `ingest(c, A, C, B, b)`  ↔ `SDPX.ingest` (src/ingest.jl:620,797)
* `solve(prob; tolerance)` ↔ `SDPX.solve(prob; tolerance)` (src/solver/interior_point.jl:3654)
* `certificate(prob, result)` ↔ `result_certificate(prob, result)` (src/validation.jl:948)
* `normal.NormalSystem`     ↔ the LP standard-form reduced system and Lorentz NT
  scaling (src/lp_solver.jl, src/soc_lorentz_kernels.jl, src/soc_native.jl)
* `adjoint(prob, result, …)` gradients of a loss of the solution with respect
  to the data, and `batch.solve_batch` for many independent instances (no
  counterpart in SDPX)

`solve` runs on the CUDA backend (`libsdpx_b200.so`, sm_100a) and raises if
the library or a GPU is unavailable; there is no CPU fallback.
"""
from .controller import SolverOptions
from .driver import SDPResult, Status, solve_with_backend
from .problem import Equilibration, SDPProblem, ingest, unequilibrate
from .batch import batch_instances, solve_batch

__all__ = ["SolverOptions", "SDPResult", "Status", "SDPProblem", "Equilibration", "ingest",
           "unequilibrate", "solve", "solve_with_backend", "certificate", "adjoint",
           "solve_batch", "batch_instances"]


def solve(prob: SDPProblem, *, tolerance: float = 1e-8, precision: str = "fp64",
          maximum_iterations: int = 200, scaling: str = "auto", device: int = 0,
          trace=None, certificate: bool = False, driver: str = "native",
          sparse_schur: bool = False, **kwargs) -> SDPResult:
    """Solve `prob` on the B200 (mirrors `SDPX.solve(prob; tolerance)`).

    `precision="fp64"` is the plain FP64 device path; `precision="mixed"`
    assembles the Schur complement with split-BF16 tensor-core products, factors
    it in FP32 and refines the Newton system in FP64, switching to the FP64 path
    when the condition estimate or the stagnation detector calls for it.
    `certificate=True` attaches the device-computed cold-path certificate
    (`result.certificate`) before the device data is released.  The loop runs
    inside the library (`driver="native"`, sdpx_b200_optimize) unless
    `driver="python"` or a `trace` list asks for the Python driver.
    `sparse_schur=True` builds the FP64 Schur complement from the coefficients'
    stored entries (SDPX's `sparse = :on`), for structurally sparse A_i.
    """
    from .cuda_backend import CudaBackend
    opts = SolverOptions(iter_max=maximum_iterations, scaling=scaling, precision=precision,
                         **kwargs).with_tolerance(tolerance)
    with CudaBackend(prob, precision=precision, device=device,
                     condition_limit=opts.mixed_condition_limit) as be:
        if sparse_schur:
            be.set_sparse_schur(True)
        if driver == "native" and trace is None:
            result = be.optimize(opts)
        else:
            result = solve_with_backend(be, opts, trace=trace)
        if certificate:
            result.certificate = be.certificate(result.x, result.X, result.Y, opts.eps_primal,
                                                opts.eps_dual, opts.eps_gap, y=result.y)
        return result


def adjoint(prob: SDPProblem, result: SDPResult, *, wx=None, wy=None, WX=None, WY=None,
            A_index=(), device: int = 0, refine: int = 0) -> dict:
    """Gradient of L = ⟨wx, x⟩ + ⟨wy, y⟩ + Σ⟨WX_l, X_l⟩ + Σ⟨WY_l, Y_l⟩ at the
    returned solution with respect to the original data c, b, C and the
    coefficients A_i of `A_index` (no counterpart in SDPX).  The Newton system
    is factored once more at the solution, on the original (unscaled) data in
    FP64, and one KKT solve gives every gradient (sdpx_b200_adjoint).  With
    `refine` > 0 (no equality rows) the system is solved to double-double
    accuracy with that many refinement steps (sdpx_b200_adjoint_refined): near
    a solution the Schur matrix is ill-conditioned enough that one FP64 solve
    is accurate to only ~1e-5."""
    from .cuda_backend import CudaBackend
    with CudaBackend(prob, precision="fp64", device=device) as be:
        be.set_iterate(result.x, result.X, result.Y, y=result.y)
        be.compute_residuals([0.0] * prob.L, True, True)
        be.schur_build()
        if not be.factorize()["ok"]:
            raise RuntimeError("the Newton system at the solution could not be factored")
        if refine > 0:
            if prob.n or wy is not None:
                raise ValueError("the refined adjoint has no equality rows")
            return be.adjoint_refined(wx, WX, WY, A_index, steps=refine)
        return be.adjoint(wx, wy, WX, WY, A_index)


def certificate(prob: SDPProblem, result: SDPResult, *, eps_primal: float = 1e-10,
                eps_dual: float = 1e-10, eps_gap: float = 1e-10, legacy_gap: bool = False,
                device: int = 0) -> dict:
    """`result_certificate(prob, result, opts)` (src/validation.jl:948-1115) for the
    optimality kind, recomputed on the B200 from the original data."""
    from .cuda_backend import CudaBackend
    with CudaBackend(prob, device=device) as be:
        return be.certificate(result.x, result.X, result.Y, eps_primal, eps_dual, eps_gap,
                              legacy_gap, y=result.y)
