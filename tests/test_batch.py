"""Batches of independent instances (the 4096 small-SDP workload's shape).

CPU: the instance generator's size distribution.  GPU: a concurrent batch
(one handle and stream per instance, host threads) reproduces each instance's
single solve exactly — same status, iterations and objectives — because each
instance runs the same deterministic kernels in the same order.
"""
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


@pytest.mark.gpu
def test_concurrent_batch_equals_single_solves():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sdpx_b200 import solve, solve_batch
    probs = batch_instances(12, seed=5)
    batch = solve_batch(probs, tolerance=1e-8, threads=4)
    for p, rb in zip(probs, batch):
        rs = solve(p, tolerance=1e-8)
        assert rb.status == rs.status
        assert rb.iterations == rs.iterations
        assert rb.pObj == rs.pObj and rb.dObj == rs.dObj
    assert sum(r.status.value == "Optimal" for r in batch) >= 11
