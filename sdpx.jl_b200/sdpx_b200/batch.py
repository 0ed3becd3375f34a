"""Batches of independent dense SDPs (the 4096-instance small-SDP workload).

Every instance gets its own device handle and CUDA stream; `threads` host
threads drive the solves concurrently.  With the native driver each solve is
one library call (sdpx_b200_optimize) that releases the GIL for its whole
duration, so the threads' host loops and device work overlap fully.  Results
are the single-instance solver's: the same kernels in the same order per
instance.  A batched engine that runs one kernel per IPM phase over all
instances is not part of this module.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor
from typing import List, Sequence

import numpy as np

from .controller import SolverOptions
from .driver import SDPResult, solve_with_backend
from .problem import SDPProblem


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


def solve_batch(problems: Sequence[SDPProblem], *, tolerance: float = 1e-8,
                precision: str = "fp64", threads: int = 8, device: int = 0,
                driver: str = "native", **kwargs) -> List[SDPResult]:
    """Solve every problem (one handle each, `threads` concurrent solves);
    results in input order.  With the native driver the whole loop runs inside
    the library, so the threads hold the GIL only to start and collect."""
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
