"""Batches of independent dense SDPs (the 4096-instance small-SDP workload).

Two engines:

* ``engine="batched"`` (`BatchSolver`, include/sdpx_b200_batch.h): every
  instance lives in one pooled device workspace and every interior-point phase
  is one kernel launch over all instances still running, one CTA per instance
  (the Schur assembly split into work items of a tuned size).  Each instance
  keeps its own scalar controller, so its status, iterations and objectives are
  those of its single solve with the same options.  It runs SDPX's fixed start
  without equilibration (``parameter_policy="fixed"``, ``scaling="none"``), in
  FP64 or with the Newton system in double-double (``precision="float64x2"``),
  for one PSD block of order 3..64 and m ≤ 256 per instance.
* ``engine="loop"``: one device handle and CUDA stream per instance
  (`sdpx_b200_optimize`), driven by ``threads`` host threads — the
  per-instance loop the batched engine is measured against.

SDPX has no batch solver (its `src/prepared.jl` only reuses structure between
solves of one problem); both engines run SDPX's dense loop per instance.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, List, Optional, Sequence

import numpy as np

from .controller import SolverOptions
from .driver import SDPResult, Status, solve_with_backend
from .problem import SDPProblem

# The options the batched engine serves (fixed start, no equilibration).
BATCH_OPTIONS = {"parameter_policy": "fixed", "scaling": "none"}


def batch_instances(count: int, seed: int = 0, n_range=(4, 64), m_cap: int = 200) -> List[SDPProblem]:
    """Instances of uneven size: block order n ~ U{n_range}, m ~ U{3..min(m_cap,
    n(n+1)/2)}, each from the SDPA-form generator (`generators.sdpa_dense`,
    one PSD block) seeded by (seed, instance id)."""
    from . import generators as G
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        m = int(rng.integers(3, min(m_cap, n * (n + 1) // 2) + 1))
        out.append(G.sdpa_dense(m=m, blocks=[n], lp=0, seed=int(seed) * 1_000_003 + i))
    return out


def batch_options(tolerance: float = 1e-8, **kwargs) -> SolverOptions:
    """SolverOptions of the batched engine (and of the loop it is compared with)."""
    kw = dict(BATCH_OPTIONS)
    kw.update(kwargs)
    return SolverOptions(**kw).with_tolerance(tolerance)


def _tune_cache_path() -> str:
    return os.environ.get("SDPX_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "sdpx_b200",
                                       "batch_schur.json"))


class BatchSolver:
    """All instances in one pooled device workspace (sdpx_b200_batch_*).

    Raises if the library or a GPU is unavailable, or if an instance is outside
    the engine's scope (more than one block, equality rows, k ∉ [3, 64],
    m ∉ [1, 256])."""

    def __init__(self, problems: Sequence[SDPProblem], device: int = 0):
        from .cuda_backend import BatchProblem, SDPXB200Error, load_library
        self._lib = load_library()
        self._err = SDPXB200Error
        self.problems = list(problems)
        if not self.problems:
            raise ValueError("empty batch")
        for i, p in enumerate(self.problems):
            if p.L != 1 or p.n != 0:
                raise ValueError(f"instance {i}: the batched engine takes one PSD block and "
                                 f"no equality rows")
        dp = C.POINTER(C.c_double)
        n = len(self.problems)
        self._keep = []
        ks = (C.c_int32 * n)(*[p.k[0] for p in self.problems])
        ms = (C.c_int32 * n)(*[p.m for p in self.problems])
        Avs, Cs, cs = (dp * n)(), (dp * n)(), (dp * n)()
        for i, p in enumerate(self.problems):
            a = np.ascontiguousarray(p.Av[0], dtype=np.float64)
            cm = np.ascontiguousarray(np.asarray(p.C[0], dtype=np.float64).T)  # column-major
            cv = np.ascontiguousarray(p.c, dtype=np.float64)
            self._keep += [a, cm, cv]
            Avs[i] = a.ctypes.data_as(dp)
            Cs[i] = cm.ctypes.data_as(dp)
            cs[i] = cv.ctypes.data_as(dp)
        prob = BatchProblem(n, ks, ms, Avs, Cs, cs)
        h = C.c_void_p()
        rc = self._lib.sdpx_b200_batch_create(C.byref(prob), device, C.byref(h))
        self._keep = None  # the data is on the device now
        if rc != 0:
            raise SDPXB200Error("sdpx_b200_batch_create: " +
                                self._lib.sdpx_b200_batch_create_error().decode())
        self._h = h
        self.shape = None

    def _call(self, name, *args):
        rc = getattr(self._lib, name)(self._h, *args)
        if rc != 0:
            raise self._err(f"{name}: " + self._lib.sdpx_b200_batch_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sdpx_b200_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def signature(self) -> str:
        """Workload key of the tuning cache: count and size ranges."""
        ks = [p.k[0] for p in self.problems]
        ms = [p.m for p in self.problems]
        return f"n{len(ks)}-k{min(ks)}..{max(ks)}-m{min(ms)}..{max(ms)}"

    def set_step_bounds(self, mode: str):
        """Affine fraction-to-boundary bounds: "eigen" (default, −1/λ_min of
        L⁻¹·dM·L⁻ᵀ) or "bisection" (the reference's Cholesky-trial bisection)."""
        self._call("sdpx_b200_batch_set_step_bounds", {"bisection": 0, "eigen": 1}[mode])

    def set_schur_shape(self, threads: int, tile: int, grain: float):
        self._call("sdpx_b200_batch_set_schur_shape", int(threads), int(tile), float(grain))
        self.shape = (int(threads), int(tile), float(grain))

    def autotune(self, opts: Optional[SolverOptions] = None, cache: bool = True) -> List[tuple]:
        """Time every Schur launch shape on the device and keep the fastest;
        with `cache`, a choice stored for this workload signature is reused
        and a new one is stored (JSON at $SDPX_B200_TUNE_CACHE, default
        ~/.cache/sdpx_b200/batch_schur.json).  Returns the timing table
        [(threads, tile, grain, ms)] (empty when the cache answered)."""
        from .cuda_backend import native_options
        path = _tune_cache_path()
        key = self.signature()
        if cache and os.path.exists(path):
            try:
                with open(path) as f:
                    stored = json.load(f).get(key)
            except (OSError, ValueError):
                stored = None
            if stored:
                self.set_schur_shape(*stored)
                return []
        no = native_options(opts or batch_options())
        cap = 64
        table = np.zeros(4 * cap)
        cnt = C.c_int32()
        self._call("sdpx_b200_batch_autotune", C.byref(no),
                   table.ctypes.data_as(C.POINTER(C.c_double)), cap, C.byref(cnt))
        rows = [tuple(table[4 * i:4 * i + 4]) for i in range(min(cnt.value, cap))]
        best = min(rows, key=lambda r: r[3])
        self.shape = (int(best[0]), int(best[1]), float(best[2]))
        if cache:
            try:
                os.makedirs(os.path.dirname(path), exist_ok=True)
                data = {}
                if os.path.exists(path):
                    with open(path) as f:
                        data = json.load(f)
                data[key] = list(self.shape)
                with open(path, "w") as f:
                    json.dump(data, f, indent=1)
            except (OSError, ValueError):
                pass
        return rows

    def optimize(self, opts: Optional[SolverOptions] = None,
                 solutions: bool = True) -> List[SDPResult]:
        """Solve every instance; results in input order (objectives and
        residuals on the original data, as `sdpx_b200_optimize` reports them)."""
        from .cuda_backend import STATUS_NAMES, SolveResult, native_options
        no = native_options(opts or batch_options())
        n = len(self.problems)
        res = (SolveResult * n)()
        self._call("sdpx_b200_batch_optimize", C.byref(no), res)
        dp = C.POINTER(C.c_double)
        mt = sum(p.m for p in self.problems)
        kt = sum(p.k[0] * p.k[0] for p in self.problems)
        xs, Xs, Ys = np.zeros(mt), np.zeros(kt), np.zeros(kt)
        if solutions:  # one read-back of every instance's x, X, Y
            self._call("sdpx_b200_batch_get_solutions", xs.ctypes.data_as(dp),
                       Xs.ctypes.data_as(dp), Ys.ctypes.data_as(dp))
        out = []
        mo = ko = 0
        for i, p in enumerate(self.problems):
            k = p.k[0]
            x, X, Y = xs[mo:mo + p.m], Xs[ko:ko + k * k], Ys[ko:ko + k * k]
            mo += p.m
            ko += k * k
            r = res[i]
            out.append(SDPResult(
                status=Status(STATUS_NAMES[r.status]), message=r.message.decode(errors="replace"),
                x=x, X=[X.reshape(k, k).T.copy()], y=np.zeros(0), Y=[Y.reshape(k, k).T.copy()],
                pObj=r.p_obj, dObj=r.d_obj, p_res=r.p_res, d_res=r.d_res,
                iterations=r.iterations, restarts=r.restarts,
                precision_trace=["fp64"] * r.fp64_iterations, seconds=r.seconds))
        return out

    def set_solution(self, i: int, x=None, X=None, Y=None):
        """Replace instance i's current iterate (X, Y as k×k matrices); None
        keeps that part (sdpx_b200_batch_set_solution)."""
        dp = C.POINTER(C.c_double)
        keep = []

        def ptr(a, col_major):
            if a is None:
                return None
            a = np.asarray(a, dtype=np.float64)
            a = np.ascontiguousarray(a.T if col_major else a).reshape(-1)
            keep.append(a)
            return a.ctypes.data_as(dp)
        self._call("sdpx_b200_batch_set_solution", int(i), ptr(x, False), ptr(X, True),
                   ptr(Y, True))

    def certificate(self, eps_primal: float = 1e-10, eps_dual: float = 1e-10,
                    eps_gap: float = 1e-10, legacy_gap: bool = False) -> List[dict]:
        """`result_certificate` of every instance's current solution, all
        computed by one device kernel and read back once
        (sdpx_b200_batch_certificate); dicts as `sdpx_b200.certificate`."""
        from .cuda_backend import CERTIFICATE_FAILURES, CertificateResult
        n = len(self.problems)
        out = (CertificateResult * n)()
        self._call("sdpx_b200_batch_certificate", float(eps_primal), float(eps_dual),
                   float(eps_gap), 1 if legacy_gap else 0, out)
        certs = []
        for r in out:
            d = {name: getattr(r, name) for name, _ in CertificateResult._fields_}
            d["valid"] = bool(r.valid)
            d["failures"] = [name for bit, name in CERTIFICATE_FAILURES if r.failures & bit]
            d["available"] = True
            d["kind"] = "optimality"
            certs.append(d)
        return certs

    def stats(self) -> Dict[str, float]:
        """Counters of the last optimize (sdpx_b200_batch_stats)."""
        v = np.zeros(8)
        self._call("sdpx_b200_batch_stats", v.ctypes.data_as(C.POINTER(C.c_double)))
        keys = ("passes", "launches", "seconds", "schur_seconds", "factor_seconds",
                "step_seconds", "instance_iterations", "schur_flops")
        return dict(zip(keys, v.tolist()))


def solve_batch(problems: Sequence[SDPProblem], *, tolerance: float = 1e-8,
                engine: str = "batched", precision: str = "fp64", threads: int = 8,
                device: int = 0, driver: str = "native", autotune: bool = False,
                **kwargs) -> List[SDPResult]:
    """Solve every problem; results in input order.

    ``engine="batched"``: one `BatchSolver` over all problems with the
    batched engine's options (`BATCH_OPTIONS` plus `kwargs`); ``precision``
    "fp64" or "float64x2" (the Newton system in double-double, for tight
    tolerances such as 1e-12).
    ``engine="loop"``: one handle per problem, ``threads`` concurrent solves
    with `SolverOptions(precision, **kwargs)`; with the native driver the whole
    loop runs inside the library, so the threads hold the GIL only to start and
    collect."""
    if engine == "batched":
        if precision not in ("fp64", "float64x2"):
            raise ValueError("the batched engine runs in FP64 or Float64x2")
        opts = batch_options(tolerance, precision=precision, **kwargs)
        with BatchSolver(problems, device=device) as bs:
            if autotune:
                bs.autotune(opts)
            return bs.optimize(opts)
    if engine != "loop":
        raise ValueError(f"unknown engine {engine!r}")
    from .cuda_backend import CudaBackend
    opts = SolverOptions(precision=precision, **kwargs).with_tolerance(tolerance)

    def one(prob):
        with CudaBackend(prob, precision=precision, device=device,
                         condition_limit=opts.mixed_condition_limit) as be:
            if driver == "native":
                return be.optimize(opts)
            return solve_with_backend(be, opts)

    if threads <= 1:
        return [one(p) for p in problems]
    with ThreadPoolExecutor(max_workers=threads) as pool:
        return list(pool.map(one, problems))
