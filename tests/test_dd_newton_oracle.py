"""The Float64x2 Newton-system oracle (oracle/dd_newton_oracle.py) on CPU.

Its double-double Cholesky and solve are exact to double-double level, and on
small instances of the batch workload it reaches a 1e-12 relative gap where
the FP64 Newton system stops short (direction gate or stagnation) — the
reason the batched engine has a Float64x2 mode.
"""
import numpy as np

from oracle.dd_newton_oracle import dd_cholesky, dd_cholsolve, dd_newton_solve
from oracle.dd_oracle import DD, dd_matmul
from sdpx_b200 import batch_instances
from sdpx_b200.batch import batch_options


def test_dd_cholesky_solve_is_double_double_accurate():
    rng = np.random.default_rng(3)
    G = rng.standard_normal((12, 12))
    S = G @ G.T + 1e-6 * np.eye(12)          # κ ≈ 1e8
    b = rng.standard_normal(12)
    L = dd_cholesky(DD(S))
    x = dd_cholsolve(L, b)
    r = DD(b) - dd_matmul(DD(S), DD(x.hi[:, None], x.lo[:, None])).reshape(-1)
    assert np.max(np.abs(r.to_float())) <= 1e-22 * np.abs(S).max() * np.abs(x.hi).max()
    LLt = dd_matmul(L, L.T) - DD(S)
    assert np.max(np.abs(LLt.to_float())) <= 1e-28 * np.abs(S).max()


def test_dd_newton_reaches_1e12_where_fp64_stops():
    from oracle.sdpx_oracle import oracle_solve
    probs = [p for p in batch_instances(256, seed=1) if p.k[0] <= 12 and p.m <= 30][:3]
    assert len(probs) == 3
    opts = batch_options(1e-12)
    fp64 = [oracle_solve(p, opts) for p in probs]
    dd = [dd_newton_solve(p, opts) for p in probs]
    assert all(r.status.value == "Optimal" and r.relative_gap <= 1e-12 for r in dd)
    assert sum(r.status.value == "Optimal" for r in fp64) < len(probs)
