"""ctypes binding of libsdpx_b200.so and the device backend of the host driver.

Every method maps onto one C-ABI entry point of include/sdpx_b200.h; matrices
stay resident on the GPU and only scalars (or the final iterate) come back.
The library is loaded from this package's directory; if it is missing, or no
CUDA device is usable, construction raises — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import List, Optional

import numpy as np

from .problem import Equilibration, SDPProblem

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libsdpx_b200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Problem(C.Structure):
    _fields_ = [("m", C.c_int64), ("nblocks", C.c_int32), ("block_order", C.POINTER(C.c_int32)),
                ("Av", C.POINTER(_dp)), ("C", C.POINTER(_dp)), ("c", _dp)]


class BatchProblem(C.Structure):
    """`sdpx_b200_batch_problem` (include/sdpx_b200_batch.h)."""
    _fields_ = [("count", C.c_int32), ("block_order", C.POINTER(C.c_int32)),
                ("m", C.POINTER(C.c_int32)), ("Av", C.POINTER(_dp)), ("C", C.POINTER(_dp)),
                ("c", C.POINTER(_dp))]


class CertificateResult(C.Structure):
    """Mirror of sdpx_b200_certificate_result (include/sdpx_b200.h)."""
    _fields_ = [("valid", C.c_int32), ("failures", C.c_int32),
                ("primal_psd_failing_blocks", C.c_int32), ("dual_psd_failing_blocks", C.c_int32)] + [
        (name, C.c_double) for name in (
            "primal_objective", "dual_objective", "gap", "gap_relative", "primal_residual",
            "dual_residual", "primal_affine_residual", "dual_affine_residual",
            "primal_cone_violation", "dual_cone_violation", "primal_residual_scaled",
            "dual_residual_scaled", "equality_backward_error", "equality_strict_backward_error",
            "primal_block_backward_error", "primal_block_strict_backward_error",
            "dual_backward_error", "dual_strict_backward_error", "complementarity",
            "complementarity_relative")]


# Failure bits of the certificate, named as SDPX's failure symbols (src/validation.jl:1069-1096).
CERTIFICATE_FAILURES = (
    (1, "nonfinite"), (2, "primal_residual"), (4, "equality_backward_error"),
    (8, "primal_block_backward_error"), (16, "dual_residual"), (32, "dual_backward_error"),
    (64, "duality_gap"), (128, "primal_psd"), (256, "dual_psd"))

class SolveOptions(C.Structure):
    """`sdpx_b200_solve_options` (include/sdpx_b200.h)."""
    _fields_ = [("beta", C.c_double), ("gamma", C.c_double), ("omega_p", C.c_double),
                ("omega_d", C.c_double), ("eps_gap", C.c_double), ("eps_primal", C.c_double),
                ("eps_dual", C.c_double), ("iter_max", C.c_int32), ("restart", C.c_int32),
                ("min_step", C.c_double), ("omega_step", C.c_double),
                ("max_restarts", C.c_int32), ("max_centering", C.c_int32),
                ("stall_iterations", C.c_int32), ("stall_tolerance", C.c_double),
                ("step_rule", C.c_int32), ("refine_steps", C.c_int32),
                ("refine_policy", C.c_int32), ("refine_max_steps", C.c_int32),
                ("refine_tol", C.c_double), ("max_time", C.c_double),
                ("parameter_policy", C.c_int32), ("parameter_strategy", C.c_int32),
                ("adaptive_sigma_max", C.c_double), ("scaling", C.c_int32),
                ("precision", C.c_int32), ("equality_solver", C.c_int32)]


class SolveResult(C.Structure):
    """`sdpx_b200_solve_result` (include/sdpx_b200.h)."""
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("restarts", C.c_int32),
                ("mixed_iterations", C.c_int32), ("fp64_iterations", C.c_int32),
                ("p_obj", C.c_double), ("d_obj", C.c_double), ("p_res", C.c_double),
                ("d_res", C.c_double), ("seconds", C.c_double), ("message", C.c_char * 256)]


STATUS_NAMES = {1: "Optimal", 2: "IterLimit", 3: "Stalled", 4: "InsufficientPrecision",
                5: "NumericalBreakdown", 6: "MaxRestartsExceeded", 7: "TimeLimit"}


def native_options(o) -> SolveOptions:
    """SolverOptions → sdpx_b200_solve_options."""
    return SolveOptions(
        o.beta, o.gamma, o.omega_p, o.omega_d, o.eps_gap, o.eps_primal, o.eps_dual,
        int(o.iter_max), int(bool(o.restart)), o.min_step, o.omega_step, int(o.max_restarts),
        int(o.max_centering), int(o.stall_iterations), o.stall_tolerance,
        {"auto": 0, "backtrack": 1, "fraction_to_boundary": 2}[o.step_rule],
        int(o.refine_steps), {"fixed": 0, "adaptive": 1, "auto": 2}[o.refine_policy],
        int(o.refine_max_steps), o.refine_tol, o.max_time,
        {"auto": 0, "fixed": 1}[o.parameter_policy],
        {"adaptive": 0, "fixed": 1}[o.parameter_strategy], o.adaptive_sigma_max,
        {"auto": 0, "none": 1, "equilibrate": 2}[o.scaling],
        {"fp64": 0, "mixed": 1, "float64x2": 2}[o.precision],
        {"auto": 0, "qr": 1}[o.equality_solver])


# name -> argtypes (restype is int unless noted)
_SIGS = {
    "sdpx_b200_abi_version": [],
    "sdpx_b200_create": [C.POINTER(_Problem), C.c_int, C.POINTER(C.c_void_p)],
    "sdpx_b200_set_precision": [C.c_void_p, C.c_int],
    "sdpx_b200_equilibrate": [C.c_void_p, _dp, _dp, _dp, C.POINTER(C.c_int32)],
    "sdpx_b200_data_norms": [C.c_void_p, _dp, _dp],
    "sdpx_b200_set_iterate": [C.c_void_p, _dp, _dp, _dp],
    "sdpx_b200_get_iterate": [C.c_void_p, _dp, _dp, _dp],
    "sdpx_b200_get_direction": [C.c_void_p, _dp, _dp, _dp],
    "sdpx_b200_get_rhs": [C.c_void_p, _dp],
    "sdpx_b200_fixed_start": [C.c_void_p, C.c_double, C.c_double],
    "sdpx_b200_residuals": [C.c_void_p, _dp, C.c_int, C.c_int, _dp, _dp, _ip],
    "sdpx_b200_block_primal_residual": [C.c_void_p, _dp],
    "sdpx_b200_block_margins": [C.c_void_p, _dp, _dp],
    "sdpx_b200_schur_build": [C.c_void_p, C.c_int],
    "sdpx_b200_get_schur": [C.c_void_p, _dp],
    "sdpx_b200_factorize": [C.c_void_p, _ip, _ip, _dp],
    "sdpx_b200_rhs_predictor": [C.c_void_p],
    "sdpx_b200_rhs_corrector_mehrotra": [C.c_void_p, C.c_double, C.c_double, C.c_int],
    "sdpx_b200_rhs_corrector_fixed": [C.c_void_p, C.c_double, _dp],
    "sdpx_b200_set_rhs": [C.c_void_p, C.c_int],
    "sdpx_b200_solve": [C.c_void_p],
    "sdpx_b200_direction_residual": [C.c_void_p, _dp, _dp],
    "sdpx_b200_refine": [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, _ip, _dp],
    "sdpx_b200_direction_blocks": [C.c_void_p],
    "sdpx_b200_affine_diagnostics": [C.c_void_p, C.c_int, _dp, _dp],
    "sdpx_b200_line_search": [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double,
                              C.c_double, C.c_double, _dp, _dp],
    "sdpx_b200_update": [C.c_void_p, C.c_double, C.c_double, _dp, _ip, _dp],
    "sdpx_b200_accepted_residuals": [C.c_void_p, C.c_double, C.c_double, C.c_double, _dp, _dp],
    "sdpx_b200_objectives": [C.c_void_p, _dp, _dp],
    "sdpx_b200_solution_residuals": [C.c_void_p, _dp, _dp],
    "sdpx_b200_keep_direction": [C.c_void_p],
    "sdpx_b200_cold_start_iterate": [C.c_void_p],
    "sdpx_b200_psd_shift": [C.c_void_p, C.c_int, _ip],
    "sdpx_b200_add_identity": [C.c_void_p, C.c_int, C.c_double],
    "sdpx_b200_block_dots": [C.c_void_p, _dp, _dp, _dp],
    "sdpx_b200_scale_iterate": [C.c_void_p, C.c_int, C.c_double],
    "sdpx_b200_store_best": [C.c_void_p],
    "sdpx_b200_restore_best": [C.c_void_p],
    "sdpx_b200_rebuild_slack": [C.c_void_p, _dp, _dp],
    "sdpx_b200_original_residuals": [C.c_void_p, _dp, _dp, _dp, _dp, _dp],
    "sdpx_b200_certificate": [C.c_void_p, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double,
                              C.c_int32, C.POINTER(CertificateResult)],
    "sdpx_b200_phase_times": [C.c_void_p, _dp, C.c_int],
    "sdpx_b200_kernel_times": [C.c_void_p, _dp],
    "sdpx_b200_set_gram_engine": [C.c_void_p, C.c_int],
    "sdpx_b200_set_sparse_schur": [C.c_void_p, C.c_int],
    "sdpx_b200_sparse_schur_info": [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
    "sdpx_b200_counters": [C.c_void_p, C.POINTER(C.c_int64)],
    "sdpx_b200_reset": [C.c_void_p],
    "sdpx_b200_get_precision": [C.c_void_p, _ip, _ip, _dp],
    "sdpx_b200_get_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
    "sdpx_b200_launch_count": [C.POINTER(C.c_uint64)],
    "sdpx_b200_set_equality": [C.c_void_p, C.c_int32, _dp, _dp],
    "sdpx_b200_set_equality_options": [C.c_void_p, C.c_double, C.c_int],
    "sdpx_b200_get_multipliers": [C.c_void_p, _dp, _dp, _dp],
    "sdpx_b200_set_multipliers": [C.c_void_p, _dp],
    "sdpx_b200_equality_info": [C.c_void_p, _ip, _ip, _dp],
    "sdpx_b200_original_residuals_eq": [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp],
    "sdpx_b200_optimize": [C.c_void_p, C.POINTER(SolveOptions), C.POINTER(SolveResult)],
    "sdpx_b200_optimize_begin": [C.c_void_p, C.POINTER(SolveOptions)],
    "sdpx_b200_newton_step": [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _dp,
                              _dp, _dp, _dp],
    "sdpx_b200_optimize_end": [C.c_void_p, C.POINTER(SolveResult)],
    "sdpx_b200_get_solution": [C.c_void_p, _dp, _dp, _dp, _dp],
    "sdpx_b200_loop_state": [C.c_void_p, _dp],
    "sdpx_b200_step_stats": [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
    "sdpx_b200_get_trace": [C.c_void_p, C.POINTER(C.c_int32), C.c_int32,
                            C.POINTER(C.c_int32)],
    "sdpx_b200_adjoint": [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int32,
                          C.POINTER(C.c_int32), _dp],
    "sdpx_b200_adjoint_refined": [C.c_void_p, _dp, _dp, _dp, _dp, _dp, C.c_int32,
                                  C.POINTER(C.c_int32), _dp, C.c_int32, _dp],
    "sdpx_b200_certificate_eq": [C.c_void_p, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                 C.c_double, C.c_int32, C.POINTER(CertificateResult)],
    # batched small-SDP engine (include/sdpx_b200_batch.h)
    "sdpx_b200_batch_create": [C.POINTER(BatchProblem), C.c_int, C.POINTER(C.c_void_p)],
    "sdpx_b200_batch_optimize": [C.c_void_p, C.POINTER(SolveOptions), C.POINTER(SolveResult)],
    "sdpx_b200_batch_get_solution": [C.c_void_p, C.c_int32, _dp, _dp, _dp],
    "sdpx_b200_batch_get_solutions": [C.c_void_p, _dp, _dp, _dp],
    "sdpx_b200_batch_set_solution": [C.c_void_p, C.c_int32, _dp, _dp, _dp],
    "sdpx_b200_batch_certificate": [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int32,
                                    C.POINTER(CertificateResult)],
    "sdpx_b200_batch_stats": [C.c_void_p, _dp],
    "sdpx_b200_batch_set_step_bounds": [C.c_void_p, C.c_int32],
    "sdpx_b200_batch_set_schur_shape": [C.c_void_p, C.c_int32, C.c_int32, C.c_double],
    "sdpx_b200_batch_autotune": [C.c_void_p, C.POINTER(SolveOptions), _dp, C.c_int32,
                                 C.POINTER(C.c_int32)],
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libsdpx_b200.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} not found: build it with `python sdpx.jl_b200/build.py`")
    lib = C.CDLL(path)
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    lib.sdpx_b200_destroy.argtypes = [C.c_void_p]
    lib.sdpx_b200_destroy.restype = None
    lib.sdpx_b200_last_error.argtypes = [C.c_void_p]
    lib.sdpx_b200_last_error.restype = C.c_char_p
    lib.sdpx_b200_create_error.argtypes = []
    lib.sdpx_b200_create_error.restype = C.c_char_p
    lib.sdpx_b200_batch_destroy.argtypes = [C.c_void_p]
    lib.sdpx_b200_batch_destroy.restype = None
    lib.sdpx_b200_batch_last_error.argtypes = [C.c_void_p]
    lib.sdpx_b200_batch_last_error.restype = C.c_char_p
    lib.sdpx_b200_batch_create_error.argtypes = []
    lib.sdpx_b200_batch_create_error.restype = C.c_char_p
    _lib = lib
    return lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class SDPXB200Error(RuntimeError):
    pass


class CudaBackend:
    """Device backend of `sdpx_b200.driver` (all numerics on the B200)."""

    PHASES = ("residual_and_block_factor", "schur_assembly", "kkt_factorization",
              "solve_and_refinement", "rhs_and_directions", "step_length", "update")

    def __init__(self, prob: SDPProblem, *, precision: str = "fp64", device: int = 0,
                 condition_limit: float = 1e8):
        self.lib = load_library()
        self.prob0 = prob
        self.k = list(prob.k)
        self.m = prob.m
        self.n = prob.n
        self.L = len(self.k)
        self.Ku = int(sum(kl * kl for kl in self.k))
        self.offsets = np.cumsum([0] + [kl * kl for kl in self.k])
        self._keep = []
        order = (C.c_int32 * self.L)(*self.k)
        av_ptrs = (_dp * self.L)()
        c_ptrs = (_dp * self.L)()
        for l in range(self.L):
            # Av[l] is (m, k*k) C-ordered == k²×m column-major (column i = vec A_i)
            a = np.ascontiguousarray(prob.Av[l], dtype=np.float64)
            cm = np.ascontiguousarray(np.asfortranarray(prob.C[l]).reshape(-1, order="F"))
            self._keep += [a, cm]
            av_ptrs[l] = _p(a)
            c_ptrs[l] = _p(cm)
        cvec = np.ascontiguousarray(prob.c, dtype=np.float64)
        self._keep.append(cvec)
        pr = _Problem(self.m, self.L, order, av_ptrs, c_ptrs, _p(cvec))
        h = C.c_void_p()
        rc = self.lib.sdpx_b200_create(C.byref(pr), device, C.byref(h))
        if rc != 0:
            raise SDPXB200Error("sdpx_b200_create failed: " +
                                self.lib.sdpx_b200_create_error().decode())
        self._keep = []     # host data has been copied to the device
        self.h = h
        if self.n > 0:
            # Equality rows (SDPX `SDPProblem.B`, `.b`).
            Bm = np.asfortranarray(np.asarray(prob.B, dtype=np.float64).reshape(self.m, self.n))
            bv = np.ascontiguousarray(prob.b, dtype=np.float64)
            self._call("sdpx_b200_set_equality", self.n, _p(Bm), _p(bv))
        self.requested = precision
        self.condition_limit = condition_limit
        self.mode = "fp64"
        self._history: List[str] = []
        self._switch_reason: Optional[str] = None
        self._in_loop = False

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.sdpx_b200_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int, what: str):
        if rc != 0:
            msg = self.lib.sdpx_b200_last_error(self.h)
            raise SDPXB200Error(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def _call(self, name, *args):
        self._ck(getattr(self.lib, name)(self.h, *args), name)

    # -- stacked <-> per-block --------------------------------------------
    def _split(self, flat):
        return [flat[self.offsets[l]:self.offsets[l + 1]].reshape(self.k[l], self.k[l], order="F").copy()
                for l in range(self.L)]

    def _join(self, blocks):
        return np.ascontiguousarray(np.concatenate(
            [np.asarray(b, dtype=np.float64).reshape(-1, order="F") for b in blocks]))

    # -- precision control --------------------------------------------------
    def _set_mode(self, mode: str):
        self._call("sdpx_b200_set_precision", 1 if mode == "mixed" else 0)
        self.mode = mode

    def _sync_mode(self):
        mode, fb, cond = C.c_int(), C.c_int(), C.c_double()
        self._call("sdpx_b200_get_precision", C.byref(mode), C.byref(fb), C.byref(cond))
        self.mode = "mixed" if mode.value == 1 else "fp64"
        self.fallbacks = fb.value
        self.cond_estimate = cond.value
        return self.mode

    def precision_label(self):
        return self._sync_mode() if getattr(self, "h", None) else self.mode

    def precision_history(self):
        return list(self._history)

    def begin_iteration(self, info):
        """Called at every loop top.  Enters mixed mode after the cold start and
        leaves it for good when the condition estimate of S passes the limit or
        the stagnation rate says the mixed directions stopped paying."""
        if not self._in_loop:
            self._in_loop = True
            if self.requested == "mixed":
                self._set_mode("mixed")
        self._history.append(self._sync_mode())

    def fallback_to_fp64(self, reason: str) -> bool:
        if self.mode == "mixed":
            self._switch_reason = reason
            self._set_mode("fp64")
            return True
        return False

    # -- problem level -------------------------------------------------------
    def equilibrate(self) -> Equilibration:
        E = np.zeros(sum(self.k))
        s = np.zeros(self.m)
        osc = C.c_double()
        passes = (C.c_int32 * self.L)()
        self._call("sdpx_b200_equilibrate", _p(E), _p(s), C.byref(osc), passes)
        Es, o = [], 0
        for kl in self.k:
            Es.append(E[o:o + kl].copy())
            o += kl
        return Equilibration(Es, s, osc.value, list(passes))

    def data_norms(self):
        a, b = C.c_double(), C.c_double()
        self._call("sdpx_b200_data_norms", C.byref(a), C.byref(b))
        bn = float(np.max(np.abs(self.prob0.b))) if self.n else 0.0
        return a.value, b.value, bn

    def configure_equality(self, requested_accuracy, solver):
        """Rank tolerance input and `equality_solver` of the equality factor."""
        if solver not in ("auto", "qr"):
            raise NotImplementedError(f"equality_solver={solver!r}")
        self._call("sdpx_b200_set_equality_options", float(requested_accuracy),
                   0 if solver == "auto" else 1)

    def optimize(self, opts, steps: bool = False):
        """The whole solve inside the library (sdpx_b200_optimize: the C++ loop
        of the same driver); with `steps` the loop is driven one
        sdpx_b200_newton_step at a time.  Returns an SDPResult in the original
        coordinates."""
        from .driver import SDPResult, Status
        no = native_options(opts)
        res = SolveResult()
        if steps:
            self._call("sdpx_b200_optimize_begin", C.byref(no))
            running = C.c_int32(1)
            while running.value:
                self._call("sdpx_b200_newton_step", C.byref(running), None, None, None, None,
                           None)
            self._call("sdpx_b200_optimize_end", C.byref(res))
        else:
            self._call("sdpx_b200_optimize", C.byref(no), C.byref(res))
        x, Xs, Ys = np.zeros(self.m), np.zeros(self.Ku), np.zeros(self.Ku)
        y = np.zeros(self.n)
        self._call("sdpx_b200_get_solution", _p(x), _p(Xs), _p(y) if self.n else None, _p(Ys))
        cnt = C.c_int32()
        self._call("sdpx_b200_get_trace", None, 0, C.byref(cnt))
        modes = (C.c_int32 * max(1, cnt.value))()
        self._call("sdpx_b200_get_trace", modes, len(modes), C.byref(cnt))
        trace = ["mixed" if modes[i] else "fp64" for i in range(cnt.value)]
        self._history = trace
        return SDPResult(status=Status(STATUS_NAMES[res.status]),
                         message=res.message.decode(errors="replace"), x=x, X=self._split(Xs),
                         y=y, Y=self._split(Ys), pObj=res.p_obj, dObj=res.d_obj,
                         p_res=res.p_res, d_res=res.d_res, iterations=res.iterations,
                         restarts=res.restarts, precision_trace=trace, seconds=res.seconds)

    def adjoint(self, wx=None, wy=None, WX=None, WY=None, A_index=()):
        """Gradient of ⟨wx, x⟩ + ⟨wy, y⟩ + Σ⟨WX_l, X_l⟩ + Σ⟨WY_l, Y_l⟩ at the current
        iterate (after residuals with factors, schur_build and factorize) with
        respect to c, b, C and the A_i of `A_index` (see sdpx_b200_adjoint)."""
        def vec(a, size):
            return None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(size)
        wxv, wyv = vec(wx, self.m), (vec(wy, self.n) if self.n else None)
        WXs = None if WX is None else self._join(WX)
        WYs = None if WY is None else self._join(WY)
        idx = np.ascontiguousarray(A_index, dtype=np.int32)
        gc, gb, gC = np.zeros(self.m), np.zeros(self.n), np.zeros(self.Ku)
        gA = np.zeros(max(1, idx.size) * self.Ku)
        ptr = lambda a: None if a is None else _p(a)
        self._call("sdpx_b200_adjoint", ptr(wxv), ptr(wyv), ptr(WXs), ptr(WYs), _p(gc),
                   _p(gb) if self.n else None, _p(gC), int(idx.size),
                   idx.ctypes.data_as(C.POINTER(C.c_int32)), _p(gA))
        return dict(grad_c=gc, grad_b=gb, grad_C=self._split(gC),
                    grad_A=[self._split(gA[q * self.Ku:(q + 1) * self.Ku])
                            for q in range(idx.size)])

    def adjoint_refined(self, wx=None, WX=None, WY=None, A_index=(), steps: int = 3):
        """The adjoint's linear system solved to double-double accuracy
        (sdpx_b200_adjoint_refined; no equality rows).  Adds `residual`, the
        relative double-double residual of the refined solve."""
        def vec(a, size):
            return None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(size)
        wxv = vec(wx, self.m)
        WXs = None if WX is None else self._join(WX)
        WYs = None if WY is None else self._join(WY)
        idx = np.ascontiguousarray(A_index, dtype=np.int32)
        gc, gC = np.zeros(self.m), np.zeros(self.Ku)
        gA = np.zeros(max(1, idx.size) * self.Ku)
        res = C.c_double()
        ptr = lambda a: None if a is None else _p(a)
        self._call("sdpx_b200_adjoint_refined", ptr(wxv), ptr(WXs), ptr(WYs), _p(gc), _p(gC),
                   int(idx.size), idx.ctypes.data_as(C.POINTER(C.c_int32)), _p(gA), int(steps),
                   C.byref(res))
        return dict(grad_c=gc, grad_C=self._split(gC),
                    grad_A=[self._split(gA[q * self.Ku:(q + 1) * self.Ku])
                            for q in range(idx.size)], residual=float(res.value))

    def equality_info(self):
        """(kind, rank, quality) of the current equality factor."""
        kind, rank, q = C.c_int(), C.c_int(), C.c_double()
        self._call("sdpx_b200_equality_info", C.byref(kind), C.byref(rank), C.byref(q))
        return (("none", "normal_equations", "rank_revealing_qr")[kind.value], rank.value,
                q.value)

    def get_equality_direction(self):
        dy = np.zeros(self.n)
        if self.n:
            self._call("sdpx_b200_get_multipliers", None, _p(dy), None)
        return dy

    def fixed_start(self, omega_p, omega_d):
        self._call("sdpx_b200_fixed_start", omega_p, omega_d)

    def set_iterate(self, x, X, Y, y=None):
        x = np.ascontiguousarray(x, dtype=np.float64)
        Xs, Ys = self._join(X), self._join(Y)
        self._call("sdpx_b200_set_iterate", _p(x), _p(Xs), _p(Ys))
        if self.n:
            yv = np.zeros(self.n) if y is None else np.ascontiguousarray(y, dtype=np.float64)
            self._call("sdpx_b200_set_multipliers", _p(yv))

    def get_iterate(self):
        x = np.zeros(self.m)
        Xs = np.zeros(self.Ku)
        Ys = np.zeros(self.Ku)
        self._call("sdpx_b200_get_iterate", _p(x), _p(Xs), _p(Ys))
        y = np.zeros(self.n)
        if self.n:
            self._call("sdpx_b200_get_multipliers", _p(y), None, None)
        return x, self._split(Xs), y, self._split(Ys)

    def get_direction(self):
        dx = np.zeros(self.m)
        dXs = np.zeros(self.Ku)
        dYs = np.zeros(self.Ku)
        self._call("sdpx_b200_get_direction", _p(dx), _p(dXs), _p(dYs))
        return dx, self._split(dXs), self._split(dYs)

    def get_rhs(self):
        r = np.zeros(self.m)
        self._call("sdpx_b200_get_rhs", _p(r))
        return r

    def schur_matrix(self):
        S = np.zeros((self.m, self.m))
        self._call("sdpx_b200_get_schur", _p(S))
        return S

    # -- hot path --------------------------------------------------------------
    def compute_residuals(self, mu, use_affine, factor):
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        p, d, ok = C.c_double(), C.c_double(), C.c_int()
        self._call("sdpx_b200_residuals", _p(mu), int(bool(use_affine)), int(bool(factor)),
                   C.byref(p), C.byref(d), C.byref(ok))
        return p.value, d.value, bool(ok.value)

    def block_primal_residual(self):
        v = C.c_double()
        self._call("sdpx_b200_block_primal_residual", C.byref(v))
        return v.value

    def schur_build(self, identity=False):
        self._call("sdpx_b200_schur_build", int(bool(identity)))

    def factorize(self):
        ok, att, q = C.c_int(), C.c_int(), C.c_double()
        self._call("sdpx_b200_factorize", C.byref(ok), C.byref(att), C.byref(q))
        return dict(ok=bool(ok.value), reg_attempts=att.value, quality=q.value)

    def predictor_rhs(self):
        self._call("sdpx_b200_rhs_predictor")

    def solve_direction(self):
        self._call("sdpx_b200_solve")

    def direction_blocks(self):
        self._call("sdpx_b200_direction_blocks")

    def direction_residual(self):
        a, b = C.c_double(), C.c_double()
        self._call("sdpx_b200_direction_residual", C.byref(a), C.byref(b))
        return a.value, b.value

    def refine(self, policy, tol, cap, fixed_steps):
        steps, res = C.c_int(), C.c_double()
        self._call("sdpx_b200_refine", 0 if policy == "fixed" else 1, float(tol), int(cap),
                   int(fixed_steps), C.byref(steps), C.byref(res))
        return steps.value, res.value

    def affine_diagnostics(self, adaptive):
        out = np.zeros(4)
        blk = np.zeros(self.L)
        self._call("sdpx_b200_affine_diagnostics", int(bool(adaptive)), _p(out), _p(blk))
        compl, aff, tX, tY = out
        uniform = bool(adaptive)
        ref = None
        if adaptive:
            for l, kl in enumerate(self.k):
                val = float(blk[l])
                if not math.isfinite(val):
                    uniform = False
                elif ref is None:
                    ref = (val, kl)
                elif not ((kl == ref[1] and val == ref[0]) or
                          (kl != ref[1] and val / kl == ref[0] / ref[1])):
                    uniform = False
        den = float(max(sum(self.k), 1))
        mu = compl / den
        mu_aff = max(0.0, aff / den)
        if adaptive:
            quality = min(max(mu_aff / mu, 0.0), 2.0) if mu > 0 else 1.0
        else:
            quality = min(max(aff / compl, 0.0), 2.0) if compl > 0 else 1.0
        return dict(complementarity=float(compl), affine_complementarity=float(aff), mu=mu,
                    mu_aff=mu_aff, quality=quality, tX=float(tX), tY=float(tY), uniform=uniform)

    def block_margins(self):
        a, b = C.c_double(), C.c_double()
        self._call("sdpx_b200_block_margins", C.byref(a), C.byref(b))
        return a.value, b.value

    def mehrotra_corrector_rhs(self, sigma, mu, block_local):
        self._call("sdpx_b200_rhs_corrector_mehrotra", float(sigma), float(mu), int(bool(block_local)))

    def fixed_corrector_rhs(self, beta, mu):
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        self._call("sdpx_b200_rhs_corrector_fixed", float(beta), _p(mu))

    def line_search(self, rule, fp, fd, gamma, min_step, margin):
        tX, tY = C.c_double(), C.c_double()
        self._call("sdpx_b200_line_search", 1 if rule == "fraction_to_boundary" else 0,
                   float(fp), float(fd), float(gamma), float(min_step), float(margin),
                   C.byref(tX), C.byref(tY))
        return tX.value, tY.value

    def update(self, tX, tY):
        c, f = C.c_double(), C.c_int()
        dots = np.zeros(self.L)
        self._call("sdpx_b200_update", float(tX), float(tY), C.byref(c), C.byref(f), _p(dots))
        return c.value, bool(f.value), [float(v) for v in dots]

    def accepted_trial_residuals(self, bpr, tX, tY):
        a, b = C.c_double(), C.c_double()
        self._call("sdpx_b200_accepted_residuals", float(bpr), float(tX), float(tY),
                   C.byref(a), C.byref(b))
        return a.value, b.value

    def objectives(self):
        a, b = C.c_double(), C.c_double()
        self._call("sdpx_b200_objectives", C.byref(a), C.byref(b))
        return a.value, b.value

    def solution_residuals(self):
        a, b = C.c_double(), C.c_double()
        self._call("sdpx_b200_solution_residuals", C.byref(a), C.byref(b))
        return a.value, b.value

    # -- cold start ------------------------------------------------------------
    def set_rhs(self, which):
        self._call("sdpx_b200_set_rhs", 0 if which == "cold_primal" else 1)

    def keep_direction_as(self, name):
        self._call("sdpx_b200_keep_direction")

    def cold_start_iterate(self):
        self._call("sdpx_b200_cold_start_iterate")

    def psd_shift(self, which):
        ok = C.c_int()
        self._call("sdpx_b200_psd_shift", 0 if which == "X" else 1, C.byref(ok))
        return bool(ok.value)

    def add_identity(self, which, shift):
        self._call("sdpx_b200_add_identity", 0 if which == "X" else 1, float(shift))

    def block_dots(self):
        d, tx, ty = np.zeros(self.L), np.zeros(self.L), np.zeros(self.L)
        self._call("sdpx_b200_block_dots", _p(d), _p(tx), _p(ty))
        return [float(v) for v in d], [float(v) for v in tx], [float(v) for v in ty]

    def scale_iterate(self, which, factor):
        self._call("sdpx_b200_scale_iterate", 0 if which == "X" else 1, float(factor))

    def store_best(self):
        self._call("sdpx_b200_store_best")

    def restore_best(self):
        self._call("sdpx_b200_restore_best")

    # -- original coordinates ---------------------------------------------------
    def restore_original(self):
        pass

    def original_c(self):
        return self.prob0.c

    def original_C(self):
        return self.prob0.C

    def original_b(self):
        return self.prob0.b

    def rebuild_slack(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        Xs = np.zeros(self.Ku)
        self._call("sdpx_b200_rebuild_slack", _p(x), _p(Xs))
        return self._split(Xs)

    def original_residuals(self, x, X, y, Y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        Xs, Ys = self._join(X), self._join(Y)
        a, b = C.c_double(), C.c_double()
        if self.n:
            yv = np.ascontiguousarray(y, dtype=np.float64)
            self._call("sdpx_b200_original_residuals_eq", _p(x), _p(Xs), _p(yv), _p(Ys),
                       C.byref(a), C.byref(b))
        else:
            self._call("sdpx_b200_original_residuals", _p(x), _p(Xs), _p(Ys), C.byref(a),
                       C.byref(b))
        return a.value, b.value

    def certificate(self, x, X, Y, eps_primal=1e-10, eps_dual=1e-10, eps_gap=1e-10,
                    legacy_gap=False, y=None) -> dict:
        """Cold-path certificate of (x, X, Y) against the original data
        (`result_certificate`, src/validation.jl:948-1115)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        Xs, Ys = self._join(X), self._join(Y)
        out = CertificateResult()
        if self.n:
            if y is None:
                raise ValueError("the equality multipliers y are required when n > 0")
            yv = np.ascontiguousarray(y, dtype=np.float64)
            self._call("sdpx_b200_certificate_eq", _p(x), _p(Xs), _p(yv), _p(Ys),
                       float(eps_primal), float(eps_dual), float(eps_gap),
                       1 if legacy_gap else 0, C.byref(out))
        else:
            self._call("sdpx_b200_certificate", _p(x), _p(Xs), _p(Ys), float(eps_primal),
                       float(eps_dual), float(eps_gap), 1 if legacy_gap else 0, C.byref(out))
        d = {name: getattr(out, name) for name, _ in CertificateResult._fields_}
        d["valid"] = bool(out.valid)
        d["failures"] = [name for bit, name in CERTIFICATE_FAILURES if out.failures & bit]
        d["available"] = True
        d["kind"] = "optimality"
        return d

    def reset(self):
        """Restore the uploaded data and the start iterate for another solve."""
        self._call("sdpx_b200_reset")
        self.mode = "fp64"
        self._in_loop = False
        self._history = []
        self._switch_reason = None

    def set_gram_engine(self, engine: str):
        """FP64 Schur engine (Gram and block products): "dmma" (FP64 tensor
        tiles) or "int8" (exact int8 digit products, eight digits = 55 bits)."""
        self._call("sdpx_b200_set_gram_engine", {"dmma": 0, "int8": 1}[engine])

    def set_sparse_schur(self, enable: bool = True):
        """Schur builds from flat coordinate entries per block and active
        variable (SDPX's `sparse = :on` SparseCons path) instead of the dense
        block products; FP64 precision mode."""
        self._call("sdpx_b200_set_sparse_schur", 1 if enable else 0)

    def sparse_schur_info(self) -> dict:
        a, e = C.c_int64(), C.c_int64()
        self._call("sdpx_b200_sparse_schur_info", C.byref(a), C.byref(e))
        return dict(active_positions=int(a.value), stored_entries=int(e.value))

    def kernel_times(self) -> dict:
        """Device ms of the latest Schur kernel launches (see sdpx_b200_kernel_times)."""
        out = np.zeros(4)
        self._call("sdpx_b200_kernel_times", _p(out))
        return dict(split_syrk=float(out[0]), split_block_products=float(out[1]),
                    fp64_syrk=float(out[2]), fp64_block_products=float(out[3]))

    def counters(self) -> dict:
        """Operator applications, guard steps, FP64 switches, Schur builds since reset."""
        out = (C.c_int64 * 4)()
        self._call("sdpx_b200_counters", out)
        return dict(operator_applications=out[0], guard_steps=out[1], fp64_switches=out[2],
                    schur_builds=out[3])

    def stream_handle(self) -> int:
        p = C.c_void_p()
        self._call("sdpx_b200_get_stream", C.byref(p))
        return int(p.value or 0)

    @staticmethod
    def launch_count() -> int:
        lib = load_library()
        v = C.c_uint64()
        if lib.sdpx_b200_launch_count(C.byref(v)) != 0:
            raise SDPXB200Error("launch_count failed")
        return int(v.value)

    def phase_times(self, reset=False):
        ms = np.zeros(7)
        self._call("sdpx_b200_phase_times", _p(ms), int(bool(reset)))
        return dict(zip(self.PHASES, ms.tolist()))
