"""The batched small-SDP engine (sdpx_b200_batch_*) against single-instance
solves with the same options and against the oracle.

Every instance keeps its own controller, so the engine must reproduce each
instance's single solve: same status, objectives within 1e-7 relative (they
differ only by summation order), iterations within one.  The launch shape of
the Schur phase changes no result bit (every Schur entry is one thread's sum
over K in the same order whatever the tiles and work split).
"""
import numpy as np
import pytest

from sdpx_b200 import batch_instances

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def test_batched_engine_matches_single_solves(cuda_ok):
    from sdpx_b200 import solve
    from sdpx_b200.batch import BATCH_OPTIONS, BatchSolver, batch_options
    probs = batch_instances(48, seed=7)
    opts = batch_options(1e-8)
    with BatchSolver(probs) as bs:
        batch = bs.optimize(opts)
        st = bs.stats()
    assert st["launches"] > 0 and st["instance_iterations"] > 0
    mismatch = []
    for i, (p, rb) in enumerate(zip(probs, batch)):
        rs = solve(p, tolerance=1e-8, **BATCH_OPTIONS)
        if rb.status != rs.status or abs(rb.iterations - rs.iterations) > 1 or \
                rel(rb.pObj, rs.pObj) > 1e-7 or rel(rb.dObj, rs.dObj) > 1e-7:
            mismatch.append((i, rb.status.value, rs.status.value, rb.iterations, rs.iterations,
                             rb.pObj, rs.pObj))
    assert not mismatch, mismatch
    assert sum(r.status.value == "Optimal" for r in batch) == len(probs)
    for p, rb in zip(probs, batch):
        assert rb.relative_gap <= 1e-8
        assert rb.p_res / (1 + np.abs(p.C[0]).max()) <= 1e-8
        assert rb.d_res / (1 + np.abs(p.c).max()) <= 1e-8
        # the returned iterate is the solution: X = 𝒜x − C ⪰ 0, Y ⪰ 0
        X = np.tensordot(rb.x, p.Av[0], axes=1).reshape(p.k[0], p.k[0]) - p.C[0]
        assert np.allclose(X, rb.X[0], atol=1e-9 * (1 + np.abs(X).max()))
        assert np.linalg.eigvalsh(rb.Y[0]).min() >= -1e-9 * (1 + np.abs(rb.Y[0]).max())


def test_batched_engine_matches_oracle(cuda_ok):
    from oracle.sdpx_oracle import oracle_solve
    from sdpx_b200.batch import BatchSolver, batch_options
    probs = [p for p in batch_instances(60, seed=11) if p.k[0] <= 24 and p.m <= 80][:6]
    assert len(probs) >= 4
    opts = batch_options(1e-8)
    with BatchSolver(probs) as bs:
        batch = bs.optimize(opts)
    for p, rb in zip(probs, batch):
        ro = oracle_solve(p, opts)
        assert rb.status == ro.status
        assert abs(rb.iterations - ro.iterations) <= 1
        assert rel(rb.pObj, ro.pObj) <= 1e-7 and rel(rb.dObj, ro.dObj) <= 1e-7


def test_schur_launch_shape_changes_no_result(cuda_ok):
    from sdpx_b200.batch import BatchSolver, batch_options
    probs = batch_instances(24, seed=2)
    opts = batch_options(1e-8)
    with BatchSolver(probs) as bs:
        ref = bs.optimize(opts, solutions=False)
        for shape in [(128, 16, 0.0), (512, 32, 1.0e6), (256, 16, 16.0e6)]:
            bs.set_schur_shape(*shape)
            out = bs.optimize(opts, solutions=False)
            for a, b in zip(ref, out):
                assert a.status == b.status and a.iterations == b.iterations
                assert a.pObj == b.pObj and a.dObj == b.dObj


def test_dmma_schur_matches_the_scalar_kernels(cuda_ok):
    """The Schur phase on the FP64 tensor cores (three grouped DMMA products)
    against the scalar kernels: the same solves up to summation order."""
    from sdpx_b200.batch import BatchSolver, batch_options
    probs = batch_instances(48, seed=21)
    opts = batch_options(1e-8)
    with BatchSolver(probs) as bs:
        bs.set_schur_shape(256, 32, 0.0)
        ref = bs.optimize(opts, solutions=False)
        bs.set_schur_shape(128, 64, 0.0)
        dm = bs.optimize(opts, solutions=False)
        bs.set_schur_shape(128, 64, 1.0e6)
        dm2 = bs.optimize(opts, solutions=False)
    diff = [i for i, (a, b) in enumerate(zip(ref, dm))
            if a.status != b.status or abs(a.iterations - b.iterations) > 1 or
            rel(a.pObj, b.pObj) > 1e-7 or rel(a.dObj, b.dObj) > 1e-7]
    assert len(diff) <= 1, diff
    for a, b in zip(dm, dm2):  # the work split changes no bit
        assert a.status == b.status and a.iterations == b.iterations and a.pObj == b.pObj


def test_autotune_picks_a_timed_shape(cuda_ok, tmp_path, monkeypatch):
    from sdpx_b200.batch import BatchSolver, batch_options
    monkeypatch.setenv("SDPX_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    probs = batch_instances(32, seed=4)
    with BatchSolver(probs) as bs:
        table = bs.autotune(batch_options(1e-8))
        assert len(table) == 24
        best = min(table, key=lambda r: r[3])
        assert bs.shape == (int(best[0]), int(best[1]), float(best[2]))
        assert all(r[3] > 0 for r in table)
        res = bs.optimize(batch_options(1e-8), solutions=False)
        assert sum(r.status.value == "Optimal" for r in res) == len(probs)
    with BatchSolver(probs) as bs2:  # the stored choice is reused
        assert bs2.autotune(batch_options(1e-8)) == []
        assert bs2.shape == (int(best[0]), int(best[1]), float(best[2]))


def test_batched_engine_rejects_unsupported_options(cuda_ok):
    from sdpx_b200.batch import BatchSolver
    from sdpx_b200 import SolverOptions
    from sdpx_b200.cuda_backend import SDPXB200Error
    probs = batch_instances(2, seed=1)
    with BatchSolver(probs) as bs:
        with pytest.raises(SDPXB200Error, match="fixed start"):
            bs.optimize(SolverOptions().with_tolerance(1e-8))
        with pytest.raises(SDPXB200Error, match="equilibration"):
            bs.optimize(SolverOptions(parameter_policy="fixed").with_tolerance(1e-8))


def _cert_compare(g, o, scale):
    import math
    assert g["valid"] == o["valid"], (g["failures"], o["failures"])
    assert sorted(g["failures"]) == sorted(o["failures"])
    assert g["primal_psd_failing_blocks"] == len(o["primal_psd_failing_blocks"])
    assert g["dual_psd_failing_blocks"] == len(o["dual_psd_failing_blocks"])
    for f in ("primal_objective", "dual_objective", "complementarity"):
        assert math.isclose(g[f], o[f], rel_tol=1e-12, abs_tol=1e-12 * scale), (f, g[f], o[f])
    for f in ("primal_affine_residual", "dual_affine_residual"):
        assert abs(g[f] - o[f]) <= 1e-12 * scale, (f, g[f], o[f])
    for f in ("primal_block_backward_error", "primal_block_strict_backward_error",
              "dual_backward_error", "dual_strict_backward_error"):
        assert abs(g[f] - o[f]) <= 1e-12, (f, g[f], o[f])
    for f in ("primal_cone_violation", "dual_cone_violation"):
        assert math.isclose(g[f], o[f], rel_tol=1e-9, abs_tol=1e-14), (f, g[f], o[f])


def test_batched_certificate_matches_oracle(cuda_ok):
    """One kernel certifies every instance; each certificate equals the oracle
    restatement of `result_certificate` on the same solution, also with a
    planted indefinite X (order 5: unresolved shift; order 4 and 3: the shift
    bisection) and a non-finite entry."""
    from oracle.certificate_oracle import result_certificate
    from sdpx_b200 import generators as G
    from sdpx_b200.batch import BatchSolver, batch_options
    probs = [p for p in batch_instances(40, seed=9) if p.m <= 60][:5]
    probs += [G.sdpa_dense(m=m, blocks=[k], lp=0, seed=50 + k) for k, m in ((3, 4), (4, 6), (5, 9))]
    with BatchSolver(probs) as bs:
        res = bs.optimize(batch_options(1e-8))
        certs = bs.certificate(1e-8, 1e-8, 1e-8)
        for p, r, g in zip(probs, res, certs):
            o = result_certificate(p.Av, p.C, p.k, p.c, r.x, r.X, r.Y, 1e-8, 1e-8, 1e-8)
            assert g["valid"] and o["valid"], (g["failures"], o["failures"])
            scale = 1 + np.abs(p.C[0]).max() + np.abs(p.c).max() + \
                np.abs(p.Av[0]).max() * np.abs(r.x).sum()
            _cert_compare(g, o, scale)
        planted = {}
        for j, shift in ((len(probs) - 1, 2.0), (len(probs) - 2, 1.5), (len(probs) - 3, 0.75)):
            X = res[j].X[0] - shift * np.eye(probs[j].k[0])
            bs.set_solution(j, X=X)
            planted[j] = X
        x_bad = res[0].x.copy()
        x_bad[1] = np.inf
        bs.set_solution(0, x=x_bad)
        certs = bs.certificate(1e-8, 1e-8, 1e-8)
        for j, p in enumerate(probs):
            X = planted.get(j, res[j].X[0])
            x = x_bad if j == 0 else res[j].x
            o = result_certificate(p.Av, p.C, p.k, p.c, x, [X], res[j].Y, 1e-8, 1e-8, 1e-8)
            if j in planted:
                assert "primal_psd" in certs[j]["failures"]
            if j == 0:  # as the per-handle certificate: invalid, with "nonfinite"
                assert "nonfinite" in certs[j]["failures"] and not certs[j]["valid"]
                continue
            scale = 1 + np.abs(p.C[0]).max() + np.abs(p.c).max() + \
                np.abs(p.Av[0]).max() * np.abs(x).sum()
            _cert_compare(certs[j], o, scale)


def test_float64x2_mode_reaches_1e12_with_valid_certificates(cuda_ok):
    """The double-double Newton system takes every instance of a sample of the
    workload to a 1e-12 gap (FP64 stops short on most) and the batched
    certificate at 1e-12 is valid for all of them."""
    from sdpx_b200.batch import BatchSolver, batch_options
    probs = batch_instances(32, seed=1)
    with BatchSolver(probs) as bs:
        res = bs.optimize(batch_options(1e-12, precision="float64x2"))
        certs = bs.certificate(1e-12, 1e-12, 1e-12)
        fp64 = bs.optimize(batch_options(1e-12), solutions=False)
    assert all(r.status.value == "Optimal" for r in res), [r.message for r in res]
    assert all(r.relative_gap <= 1e-12 for r in res)
    assert all(c["valid"] for c in certs), [c["failures"] for c in certs if not c["valid"]]
    assert sum(r.status.value == "Optimal" for r in fp64) < len(probs) // 2


def test_float64x2_mode_matches_its_oracle(cuda_ok):
    from oracle.dd_newton_oracle import dd_newton_solve
    from sdpx_b200.batch import BatchSolver, batch_options
    probs = [p for p in batch_instances(256, seed=1) if p.k[0] <= 12 and p.m <= 30][:3]
    opts = batch_options(1e-12, precision="float64x2")
    with BatchSolver(probs) as bs:
        res = bs.optimize(opts)
    for p, rb in zip(probs, res):
        ro = dd_newton_solve(p, opts)
        assert rb.status == ro.status
        assert abs(rb.iterations - ro.iterations) <= 1
        assert rel(rb.pObj, ro.pObj) <= 1e-10 and rel(rb.dObj, ro.dObj) <= 1e-10


def test_eigenvalue_step_bounds_match_the_bisection(cuda_ok):
    """The affine bounds from −1/λ_min(L⁻¹·dM·L⁻ᵀ) (the default) and from the
    reference's bisection of Cholesky trials differ only by the trials'
    rounding near t*: same status, objectives within 1e-7, iterations ±1."""
    from sdpx_b200.batch import BatchSolver, batch_options
    probs = batch_instances(64, seed=12)
    opts = batch_options(1e-8)
    with BatchSolver(probs) as bs:
        eig = bs.optimize(opts, solutions=False)
        bs.set_step_bounds("bisection")
        bis = bs.optimize(opts, solutions=False)
    diff = [(i, a.status.value, b.status.value, a.iterations, b.iterations)
            for i, (a, b) in enumerate(zip(eig, bis))
            if a.status != b.status or abs(a.iterations - b.iterations) > 1 or
            rel(a.pObj, b.pObj) > 1e-7]
    assert len(diff) <= 1, diff
    assert sum(r.status.value == "Optimal" for r in eig) >= len(probs) - 1


def test_batched_engine_at_its_size_limits(cuda_ok):
    """The smallest and largest instances the engine takes (k = 3 with m = 1,
    k = 64 with m = 256) mixed with ordinary ones, in both precisions, against
    single-instance solves with the same options."""
    from sdpx_b200 import generators as G, solve
    from sdpx_b200.batch import BATCH_OPTIONS, BatchSolver, batch_options
    probs = [G.sdpa_dense(m=1, blocks=[3], lp=0, seed=31),
             G.sdpa_dense(m=256, blocks=[64], lp=0, seed=32),
             G.sdpa_dense(m=6, blocks=[3], lp=0, seed=33),
             G.sdpa_dense(m=200, blocks=[64], lp=0, seed=34)] + batch_instances(8, seed=35)
    opts = batch_options(1e-8)
    with BatchSolver(probs) as bs:
        res = bs.optimize(opts)
        dd = bs.optimize(batch_options(1e-10, precision="float64x2"), solutions=False)
    for p, rb in zip(probs, res):
        rs = solve(p, tolerance=1e-8, **BATCH_OPTIONS)
        assert rb.status == rs.status, (p.k, p.m, rb.message, rs.message)
        assert abs(rb.iterations - rs.iterations) <= 2
        assert rel(rb.pObj, rs.pObj) <= 1e-7 and rel(rb.dObj, rs.dObj) <= 1e-7
    assert all(r.status.value == "Optimal" for r in res)
    assert all(r.status.value == "Optimal" and r.relative_gap <= 1e-10 for r in dd)


def test_bulk_solution_readback_equals_per_instance(cuda_ok):
    """sdpx_b200_batch_get_solutions (one read-back, instances in input order)
    returns exactly what sdpx_b200_batch_get_solution returns per instance."""
    import ctypes as C
    from sdpx_b200.batch import BatchSolver, batch_options
    probs = batch_instances(12, seed=5)
    dp = C.POINTER(C.c_double)
    with BatchSolver(probs) as bs:
        res = bs.optimize(batch_options(1e-8), solutions=True)
        for i, (p, r) in enumerate(zip(probs, res)):
            k = p.k[0]
            x, X, Y = np.zeros(p.m), np.zeros(k * k), np.zeros(k * k)
            bs._call("sdpx_b200_batch_get_solution", i, x.ctypes.data_as(dp),
                     X.ctypes.data_as(dp), Y.ctypes.data_as(dp))
            assert np.array_equal(r.x, x)
            assert np.array_equal(r.X[0], X.reshape(k, k).T)
            assert np.array_equal(r.Y[0], Y.reshape(k, k).T)
