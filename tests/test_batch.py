"""Batches of independent instances (the 4096 small-SDP workload's shape).

CPU: the instance generator's size distribution, the batched engine's scope
checks (made before any device call) and the oracle on the batched engine's
options.  GPU: the per-instance loop (one handle and stream per instance,
host threads) reproduces each instance's single solve exactly — same status,
iterations and objectives — because each instance runs the same
deterministic kernels in the same order.  The batched engine's parity tests
are in test_gpu_batch_engine.py.
"""
import ctypes as C

import numpy as np
import pytest

from sdpx_b200 import batch_instances


def test_batch_instance_sizes():
    probs = batch_instances(64, seed=3)
    assert len(probs) == 64
    for p in probs:
        n = p.k[0]
        assert 4 <= n <= 64 and len(p.k) == 1
        assert 3 <= p.m <= min(200, n * (n + 1) // 2)
    again = batch_instances(4, seed=3)
    assert all(np.array_equal(a.c, b.c) for a, b in zip(probs[:4], again))


def _batch_problem(ks, ms):
    from sdpx_b200.cuda_backend import BatchProblem
    dp = C.POINTER(C.c_double)
    n = len(ks)
    keep = [np.zeros(k * k * m) for k, m in zip(ks, ms)] + [np.zeros(k * k) for k in ks] + \
        [np.zeros(m) for m in ms]
    Av, Cs, cs = (dp * n)(), (dp * n)(), (dp * n)()
    for i in range(n):
        Av[i] = keep[i].ctypes.data_as(dp)
        Cs[i] = keep[n + i].ctypes.data_as(dp)
        cs[i] = keep[2 * n + i].ctypes.data_as(dp)
    prob = BatchProblem(n, (C.c_int32 * n)(*ks), (C.c_int32 * n)(*ms), Av, Cs, cs)
    return prob, keep


@pytest.mark.parametrize("ks, ms, msg", [
    ([5, 2], [4, 3], "block order 2 outside [3, 64]"),
    ([65], [4], "block order 65 outside [3, 64]"),
    ([8, 9], [3, 257], "m = 257 outside [1, 256]"),
    ([8], [0], "m = 0 outside [1, 256]"),
])
def test_batch_create_rejects_out_of_scope_instances(ks, ms, msg):
    """Sizes are checked before the device is touched (runs without a GPU)."""
    from sdpx_b200.cuda_backend import load_library
    lib = load_library()
    prob, keep = _batch_problem(ks, ms)
    h = C.c_void_p()
    assert lib.sdpx_b200_batch_create(C.byref(prob), 0, C.byref(h)) == -2
    assert not h.value
    assert msg in lib.sdpx_b200_batch_create_error().decode()


def test_batch_solver_rejects_multi_block_problems():
    from sdpx_b200 import generators as G
    from sdpx_b200.batch import BatchSolver
    with pytest.raises(ValueError, match="one PSD block"):
        BatchSolver([G.sdpa_dense(m=10, blocks=[5, 4], lp=0, seed=1)])


def test_oracle_solves_batch_instances_with_the_batch_options():
    """The oracle runs the batched engine's options (fixed start, no
    equilibration) to Optimal on small instances of the workload."""
    from oracle.sdpx_oracle import oracle_solve
    from sdpx_b200.batch import batch_options
    probs = [p for p in batch_instances(40, seed=0) if p.k[0] <= 16 and p.m <= 60][:4]
    assert len(probs) >= 2
    for p in probs:
        r = oracle_solve(p, batch_options(1e-8))
        assert r.status.value == "Optimal"
        assert r.relative_gap <= 1e-8


@pytest.mark.gpu
def test_concurrent_batch_equals_single_solves():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200 import solve, solve_batch
    probs = batch_instances(12, seed=5)
    batch = solve_batch(probs, tolerance=1e-8, threads=4, engine="loop")
    for p, rb in zip(probs, batch):
        rs = solve(p, tolerance=1e-8)
        assert rb.status == rs.status
        assert rb.iterations == rs.iterations
        assert rb.pObj == rs.pObj and rb.dObj == rs.dObj
    assert sum(r.status.value == "Optimal" for r in batch) >= 11


def test_bulk_solutions_are_sliced_per_instance(monkeypatch):
    """BatchSolver.optimize reads every solution with one
    sdpx_b200_batch_get_solutions call and slices the concatenated arrays in
    input order (x_i at Σ_{j<i} m_j, X_i and Y_i at Σ_{j<i} k_j², column-major):
    checked against a stand-in for the library that writes position-tagged
    values, so no device is needed."""
    import sdpx_b200.cuda_backend as cb
    from sdpx_b200.batch import BatchSolver, batch_options
    probs = batch_instances(5, seed=1)
    mt = sum(p.m for p in probs)
    kt = sum(p.k[0] ** 2 for p in probs)
    calls = []

    class StandIn:
        def sdpx_b200_batch_create(self, prob, device, h):
            h._obj.value = 1
            return 0

        def sdpx_b200_batch_optimize(self, h, opts, res):
            for i in range(len(probs)):
                res[i].status = 1
                res[i].iterations = i
            return 0

        def sdpx_b200_batch_get_solutions(self, h, x, X, Y):
            calls.append("bulk")
            np.ctypeslib.as_array(x, shape=(mt,))[:] = np.arange(mt)
            np.ctypeslib.as_array(X, shape=(kt,))[:] = np.arange(kt) + 0.5
            np.ctypeslib.as_array(Y, shape=(kt,))[:] = -np.arange(kt, dtype=np.float64)
            return 0

        def sdpx_b200_batch_destroy(self, h):
            return None

        def sdpx_b200_batch_last_error(self, h):
            return b""

    monkeypatch.setattr(cb, "load_library", lambda *a, **k: StandIn())
    with BatchSolver(probs) as bs:
        res = bs.optimize(batch_options(1e-8), solutions=True)
        assert calls == ["bulk"]
        mo = ko = 0
        for i, (p, r) in enumerate(zip(probs, res)):
            k = p.k[0]
            assert r.status.value == "Optimal" and r.iterations == i
            assert np.array_equal(r.x, np.arange(mo, mo + p.m))
            X = (np.arange(ko, ko + k * k) + 0.5).reshape(k, k).T   # column-major → matrix
            assert np.array_equal(r.X[0], X)
            assert np.array_equal(r.Y[0], -np.arange(ko, ko + k * k, dtype=np.float64).reshape(k, k).T)
            mo += p.m
            ko += k * k
        bare = bs.optimize(batch_options(1e-8), solutions=False)
        assert calls == ["bulk"] and all(not r.x.any() for r in bare)
