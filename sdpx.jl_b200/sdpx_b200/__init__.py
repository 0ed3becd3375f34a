"""SDPX-B200: a B200-native dense-SDP interior-point core for SDPX.

Public surface mirrors SDPX's qualified entry points:

* `ingest(c, A, C, B, b)`  ↔ `SDPX.ingest` (src/ingest.jl:620,797)
* `solve(prob; tolerance)` ↔ `SDPX.solve(prob; tolerance)` (src/solver/interior_point.jl:3654)

`solve` runs on the CUDA backend (`libsdpx_b200.so`, sm_100a) and raises if
the library or a GPU is unavailable; there is no CPU fallback.
"""
from .controller import SolverOptions
from .driver import SDPResult, Status, solve_with_backend
from .problem import Equilibration, SDPProblem, ingest, unequilibrate

__all__ = ["SolverOptions", "SDPResult", "Status", "SDPProblem", "Equilibration", "ingest",
           "unequilibrate", "solve", "solve_with_backend"]


def solve(prob: SDPProblem, *, tolerance: float = 1e-8, precision: str = "fp64",
          maximum_iterations: int = 200, scaling: str = "auto", device: int = 0,
          trace=None, **kwargs) -> SDPResult:
    """Solve `prob` on the B200 (mirrors `SDPX.solve(prob; tolerance)`).

    `precision="fp64"` is the plain FP64 device path; `precision="mixed"`
    assembles the Schur complement with split-BF16 tensor-core products, factors
    it in FP32 and refines the Newton system in FP64, switching to the FP64 path
    when the condition estimate or the stagnation detector calls for it.
    """
    from .cuda_backend import CudaBackend
    opts = SolverOptions(iter_max=maximum_iterations, scaling=scaling, precision=precision,
                         **kwargs).with_tolerance(tolerance)
    with CudaBackend(prob, precision=precision, device=device,
                     condition_limit=opts.mixed_condition_limit) as be:
        return solve_with_backend(be, opts, trace=trace)
