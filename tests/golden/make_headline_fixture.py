"""Regenerate tests/golden/headline_m2000.json: the CPU oracle's complete solve
of the seeded m = 2000 dense SDP (PSD blocks 400 + 200, 500 nonnegatives,
seed 0) to a 1e-8 relative gap, with its original-coordinate certificate.

The GPU tests and the bench compare the device solves of the same instance
with this record (status, objectives within 1e-7 relative).  Run from the
repository root; it takes a few minutes on a multi-core host:

    python tests/golden/make_headline_fixture.py
"""
import json
import os
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
for p in (ROOT, ROOT / "sdpx.jl_b200"):
    sys.path.insert(0, str(p))

from oracle.certificate_oracle import result_certificate  # noqa: E402
from oracle.sdpx_oracle import oracle_solve  # noqa: E402
from sdpx_b200 import SolverOptions, generators as G  # noqa: E402

SHAPE = dict(m=2000, blocks=[400, 200], lp=500, seed=0)
TOL = 1e-8


def main():
    prob = G.sdpa_dense(**SHAPE)
    opts = SolverOptions().with_tolerance(TOL)
    t0 = time.perf_counter()
    r = oracle_solve(prob, opts)
    dt = time.perf_counter() - t0
    cert = result_certificate(prob.Av, prob.C, prob.k, prob.c, r.x, r.X, r.Y,
                              opts.eps_primal, opts.eps_dual, opts.eps_gap)
    out = {"shape": SHAPE, "tolerance": TOL, "status": r.status.value,
           "iterations": r.iterations, "pObj": r.pObj, "dObj": r.dObj,
           "relative_gap": r.relative_gap, "p_res": r.p_res, "d_res": r.d_res,
           "certificate_valid": bool(cert["valid"]), "certificate_failures": cert["failures"],
           "cpu_seconds": dt, "cpu_count": os.cpu_count()}
    Path(__file__).with_name("headline_m2000.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out))


if __name__ == "__main__":
    main()
