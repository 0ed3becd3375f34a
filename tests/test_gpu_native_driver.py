"""The interior-point loop inside the library (sdpx_b200_optimize, C++)
against the Python driver (sdpx_b200.driver, pinned to the oracle by the gate
tests) on the same device kernels.

Both loops restate SDPX's `_solve_pipeline!` / `_solve_sdp_core!` /
`newton_step!` and the guarded Mehrotra controller; they must take the same
decisions in the same order: same status, iteration count, restarts and
precision trace, objectives to 1e-12 relative and the returned iterate to
1e-10.  The per-step entry point (sdpx_b200_newton_step) must reproduce the
one-call solve exactly.
"""
import numpy as np
import pytest

from sdpx_b200 import SolverOptions, generators as G
from sdpx_b200.driver import solve_with_backend

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200.cuda_backend import CudaBackend
    return CudaBackend


FIXED = dict(parameter_policy="fixed", parameter_strategy="fixed", scaling="none")
CASES = [
    ("closed_form", G.gate_closed_form, dict(tol=1e-10)),
    ("dense_gate", G.gate_dense, dict(tol=1e-8)),
    ("t1_fixed", G.toy_t1, dict(opts=FIXED)),
    ("t2_fixed", G.toy_t2, dict(opts=FIXED)),
    ("t3_fixed", G.toy_t3, dict(opts=FIXED)),
    ("readme_eq", G.readme_moment_equalities, dict(tol=1e-8)),
    ("sdpa_small", lambda: G.sdpa_dense(m=60, blocks=[12, 5, 2], lp=4, seed=11), dict(tol=1e-8)),
    ("sdpa_eq", lambda: G.sdpa_dense_equalities(m=80, blocks=[12, 6], lp=5, n_eq=5, seed=6),
     dict(tol=1e-8)),
    ("sdpa_mixed", lambda: G.sdpa_dense(m=150, blocks=[70, 33], lp=9, seed=2),
     dict(tol=1e-8, precision="mixed")),
]


def _opts(cfg):
    o = SolverOptions(precision=cfg.get("precision", "fp64"), **cfg.get("opts", {}))
    return o.with_tolerance(cfg["tol"]) if "tol" in cfg else o


def _rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


@pytest.mark.parametrize("name,build,cfg", CASES, ids=[c[0] for c in CASES])
def test_native_loop_matches_python_driver(cuda, name, build, cfg):
    prob = build()
    opts = _opts(cfg)
    with cuda(prob, precision=opts.precision) as be:
        rp = solve_with_backend(be, opts)
    with cuda(prob, precision=opts.precision) as be:
        rn = be.optimize(opts)
    assert rn.status == rp.status, (rn.message, rp.message)
    assert rn.iterations == rp.iterations
    assert rn.restarts == rp.restarts
    assert rn.precision_trace == rp.precision_trace
    assert abs(rn.pObj - rp.pObj) <= 1e-12 * max(1.0, abs(rp.pObj))
    assert abs(rn.dObj - rp.dObj) <= 1e-12 * max(1.0, abs(rp.dObj))
    assert _rel(rn.x, rp.x) <= 1e-10
    assert _rel(rn.y, rp.y) <= 1e-10
    for a, b in zip(rn.X + rn.Y, rp.X + rp.Y):
        assert _rel(a, b) <= 1e-10


def test_newton_step_entry_reproduces_optimize(cuda):
    prob = G.sdpa_dense(m=60, blocks=[12, 5, 2], lp=4, seed=11)
    opts = SolverOptions().with_tolerance(1e-8)
    with cuda(prob) as be:
        r1 = be.optimize(opts)
    with cuda(prob) as be:
        r2 = be.optimize(opts, steps=True)
    assert r1.status == r2.status and r1.iterations == r2.iterations
    assert r1.pObj == r2.pObj and r1.dObj == r2.dObj
    assert np.array_equal(r1.x, r2.x)
