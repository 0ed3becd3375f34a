"""Reduced normal system of SDPX's LP standard form and of Lorentz cones, on the B200.

Host mirror of `LPStandardFormSystem` (src/lp_solver.jl:85-100) and of the
NativeSOC NT scaling (src/soc_native.jl:1083-1218), bound to
include/sdpx_b200_normal.h.  Method names follow the reference's functions:

==========================  ==================================================
`soc_nt_scaling`            `_native_soc_scaling!` / `_soc_nt_scaling!`
`soc_nt_apply_w`            `_soc_nt_apply_w!`
`soc_nt_apply_winv`         `_soc_nt_apply_winv!`
`soc_nt_apply_hs_inverse`   `_soc_nt_apply_hs_inverse!`
`lp_standard_pack`          `_lp_standard_pack_range!`
`assemble_reduced_schur`    `_lp_assemble_reduced_schur!` (+ cone metrics)
`factor_reduced`            `_lp_factor_reduced!` + the ×10 retry loop
`solve_factor`              `_lp_solve_factor!`
==========================  ==================================================

Every method runs on the GPU through libsdpx_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence, Tuple

import numpy as np

from .cuda_backend import SDPXB200Error, load_library

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

_SIGS = {
    "sdpx_b200_normal_create": [C.c_int32, C.c_int32, _ip, C.c_int32, _dp, _ip, _dp, C.c_int32,
                                C.c_int, C.POINTER(C.c_void_p)],
    "sdpx_b200_normal_nt_scaling": [C.c_void_p, _dp, _dp, _ip, _dp, _dp, _dp, _dp],
    "sdpx_b200_normal_nt_apply": [C.c_void_p, C.c_int32, _dp, _dp],
    "sdpx_b200_normal_pack": [C.c_void_p, _dp, C.c_double, _dp, _dp, _dp],
    "sdpx_b200_normal_assemble": [C.c_void_p, _dp, C.c_double],
    "sdpx_b200_normal_factorize": [C.c_void_p, _dp, C.c_double, C.c_int32, _ip, _dp],
    "sdpx_b200_normal_get_matrix": [C.c_void_p, C.c_int32, _dp],
    "sdpx_b200_normal_solve": [C.c_void_p, _dp],
    "sdpx_b200_normal_times": [C.c_void_p, _dp, _dp],
    "sdpx_b200_normal_get_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
}
_bound = False


def _lib():
    global _bound
    lib = load_library()
    if not _bound:
        from .cuda_backend import SolveOptions, SolveResult
        _SIGS["sdpx_b200_normal_optimize"] = [C.c_void_p, _dp, _dp, C.POINTER(SolveOptions),
                                              C.POINTER(SolveResult), _dp, _dp, _dp]
        for name, args in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = C.c_int
        lib.sdpx_b200_normal_destroy.argtypes = [C.c_void_p]
        lib.sdpx_b200_normal_destroy.restype = None
        lib.sdpx_b200_normal_last_error.argtypes = [C.c_void_p]
        lib.sdpx_b200_normal_last_error.restype = C.c_char_p
        lib.sdpx_b200_normal_create_error.argtypes = []
        lib.sdpx_b200_normal_create_error.restype = C.c_char_p
        _bound = True
    return lib


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class ConeSolveResult:
    """Outcome of `NormalSystem.optimize` (statuses as `SDPResult`)."""

    def __init__(self, status, iterations, x, y, z, pObj, dObj, p_res, d_res, seconds, message):
        self.status, self.iterations = status, iterations
        self.x, self.y, self.z = x, y, z
        self.pObj, self.dObj, self.p_res, self.d_res = pObj, dObj, p_res, d_res
        self.seconds, self.message = seconds, message

    @property
    def relative_gap(self) -> float:
        return abs(self.pObj - self.dObj) / max(1.0, (abs(self.pObj) + abs(self.dObj)) / 2)


class PosDefError(np.linalg.LinAlgError):
    """The reduced normal matrix stayed indefinite (Julia's PosDefException)."""


class NormalSystem:
    """Device-resident reduced system for variables [n_lp LP | Lorentz cones].

    `B` is n × m_eq (one column per equality, as `LPStandardFormSystem.B`).
    LP variable j reads `weights[row_for_variable[j]]` and the coefficient g_j
    (`diagonal_coefficient`) of the permutation-diagonal G; by default each LP
    variable has its own row and g = 1.
    """

    def __init__(self, B, n_lp: int, cone_dims: Sequence[int] = (), *,
                 row_for_variable=None, diagonal_coefficient=None, n_weights: Optional[int] = None,
                 device: int = 0):
        self.lib = _lib()
        B = np.asarray(B, dtype=np.float64)
        n = int(n_lp) + int(sum(cone_dims))
        if B.ndim != 2 or B.shape[0] != n:
            raise ValueError(f"B must be {n} x m_eq, got {B.shape}")
        self.n_lp, self.n, self.m = int(n_lp), n, int(B.shape[1])
        self.cone_dims = [int(q) for q in cone_dims]
        self.cone_offsets = np.cumsum([0] + self.cone_dims)[:-1] + self.n_lp
        rows = np.arange(self.n_lp) if row_for_variable is None else np.asarray(row_for_variable)
        coef = np.ones(self.n_lp) if diagonal_coefficient is None else diagonal_coefficient
        self.n_weights = int(n_weights if n_weights is not None else
                             (int(rows.max()) + 1 if self.n_lp else 0))
        self._rows = np.ascontiguousarray(rows, dtype=np.int32)
        self._coef = _f64(coef)
        self._dims = np.ascontiguousarray(self.cone_dims, dtype=np.int32)
        Bf = np.asfortranarray(B)
        h = C.c_void_p()
        rc = self.lib.sdpx_b200_normal_create(
            self.n_lp, len(self.cone_dims), self._dims.ctypes.data_as(_ip), self.m,
            Bf.ctypes.data_as(_dp), self._rows.ctypes.data_as(_ip), _p(self._coef),
            self.n_weights, device, C.byref(h))
        if rc != 0:
            raise SDPXB200Error(self.lib.sdpx_b200_normal_create_error().decode())
        self.h = h

    # -- lifecycle --------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.sdpx_b200_normal_destroy(self.h)
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

    def _check(self, rc: int, what: str) -> int:
        if rc < 0:
            raise SDPXB200Error(f"{what}: {self.lib.sdpx_b200_normal_last_error(self.h).decode()}")
        return rc

    # -- cones ------------------------------------------------------------
    def _cone_part(self, v) -> np.ndarray:
        v = _f64(v)
        nq = self.n - self.n_lp
        if v.shape == (self.n,):
            v = np.ascontiguousarray(v[self.n_lp:])
        if v.shape != (nq,):
            raise ValueError(f"expected {nq} cone coordinates, got {v.shape}")
        return v

    def soc_nt_scaling(self, s, z) -> Tuple[bool, int, dict]:
        """NT scaling of every cone from slack s and dual z (cone part or full
        vectors).  Returns (ok, first_failed_cone or -1, {w, lambda, eta,
        eta_squared, ok}) — `_native_soc_scaling!` returns (false, block)."""
        s, z = self._cone_part(s), self._cone_part(z)
        nc, nq = len(self.cone_dims), s.size
        ok = np.zeros(nc, dtype=np.int32)
        w, lam = np.zeros(nq), np.zeros(nq)
        eta, eta2 = np.zeros(nc), np.zeros(nc)
        rc = self._check(self.lib.sdpx_b200_normal_nt_scaling(
            self.h, _p(s), _p(z), ok.ctypes.data_as(_ip), _p(w), _p(lam), _p(eta), _p(eta2)),
            "nt_scaling")
        bad = np.flatnonzero(ok == 0)
        out = {"w": w, "lambda": lam, "eta": eta, "eta_squared": eta2, "ok": ok.astype(bool)}
        return rc == 0, (int(bad[0]) if bad.size else -1), out

    def _apply(self, which: int, v) -> np.ndarray:
        v = self._cone_part(v)
        out = np.empty_like(v)
        self._check(self.lib.sdpx_b200_normal_nt_apply(self.h, which, _p(v), _p(out)), "nt_apply")
        return out

    def soc_nt_apply_w(self, v):
        return self._apply(0, v)

    def soc_nt_apply_winv(self, v):
        return self._apply(1, v)

    def soc_nt_apply_hs_inverse(self, v):
        return self._apply(2, v)

    # -- LP pack, assembly, factor, solve ---------------------------------
    def _weights(self, weights):
        if self.n_lp == 0:
            return np.zeros(1)
        w = _f64(weights)
        if w.shape != (self.n_weights,):
            raise ValueError(f"weights must have {self.n_weights} entries")
        return w

    def lp_standard_pack(self, weights, regularization: float):
        """(D, D⁻¹, D^{-1/2}) of the LP variables."""
        w = self._weights(weights)
        D, Di, Ds = (np.empty(self.n_lp) for _ in range(3))
        self._check(self.lib.sdpx_b200_normal_pack(self.h, _p(w), regularization, _p(D), _p(Di),
                                                   _p(Ds)), "pack")
        return D, Di, Ds

    def assemble_reduced_schur(self, weights, regularization: float) -> np.ndarray:
        """Q = Bᵀ D⁻¹ B + δI (m_eq × m_eq, full symmetric copy)."""
        w = self._weights(weights)
        self._check(self.lib.sdpx_b200_normal_assemble(self.h, _p(w), regularization), "assemble")
        return self.matrix(0)

    def matrix(self, which: int = 0) -> np.ndarray:
        out = np.empty((self.m, self.m), order="F")
        self._check(self.lib.sdpx_b200_normal_get_matrix(self.h, which, _p(out)), "get_matrix")
        return out

    def factor_reduced(self, weights, regularization: float, max_attempts: int = 8):
        """Assemble + Cholesky with δ ×10 retries.  Returns (success, attempts, δ used)."""
        w = self._weights(weights)
        att = C.c_int32(0)
        reg = C.c_double(0.0)
        rc = self._check(self.lib.sdpx_b200_normal_factorize(
            self.h, _p(w), regularization, max_attempts, C.byref(att), C.byref(reg)), "factorize")
        return rc == 0, att.value, reg.value

    def solve_factor(self, rhs) -> np.ndarray:
        """[rx; ry] → [dx; dy] (returns a new array)."""
        v = _f64(rhs).copy()
        if v.shape != (self.n + self.m,):
            raise ValueError(f"rhs must have {self.n + self.m} entries")
        rc = self._check(self.lib.sdpx_b200_normal_solve(self.h, _p(v)), "solve")
        if rc != 0:
            raise PosDefError("no successful factor held")
        return v

    def optimize(self, b, c, *, tolerance: float = 1e-8, **kwargs):
        """Interior-point solve of  min cᵀx  s.t.  Bᵀx = b,  x ∈ R₊^{n_lp} × cones
        on the device (sdpx_b200_normal_optimize): SDPX's LP loop with the
        Lorentz cones through their NT scaling.  `precision="mixed"` assembles
        the normal matrix from split-BF16 planes on the tensor cores and refines
        Δy against the FP64 operator, switching to the FP64 assembly when the
        refinement stalls.  Needs the standard LP layout (one weight row per LP
        variable, g = 1).  Returns a `ConeSolveResult`."""
        from .controller import SolverOptions
        from .cuda_backend import STATUS_NAMES, SolveResult, native_options
        opts = SolverOptions(**kwargs).with_tolerance(tolerance)
        no = native_options(opts)
        res = SolveResult()
        bv, cv = _f64(b), _f64(c)
        if bv.shape != (self.m,) or cv.shape != (self.n,):
            raise ValueError("b must have m_eq entries and c n entries")
        x, y, z = np.zeros(self.n), np.zeros(self.m), np.zeros(self.n)
        self._check(self.lib.sdpx_b200_normal_optimize(self.h, _p(bv), _p(cv), C.byref(no),
                                                       C.byref(res), _p(x), _p(y), _p(z)),
                    "optimize")
        out = ConeSolveResult(STATUS_NAMES[res.status], res.iterations, x, y, z, res.p_obj,
                              res.d_obj, res.p_res, res.d_res, res.seconds,
                              res.message.decode(errors="replace"))
        out.split_iterations, out.fp64_iterations = res.mixed_iterations, res.fp64_iterations
        return out

    def times(self) -> Tuple[float, float]:
        a, f = C.c_double(), C.c_double()
        self._check(self.lib.sdpx_b200_normal_times(self.h, C.byref(a), C.byref(f)), "times")
        return a.value, f.value

    def stream_handle(self) -> int:
        s = C.c_void_p()
        self._check(self.lib.sdpx_b200_normal_get_stream(self.h, C.byref(s)), "get_stream")
        return s.value or 0
