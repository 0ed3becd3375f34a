"""Profiling harness: a few interior-point iterations of one seeded instance.

    python sdpx.jl_b200/sdpx_b200/profile_run.py --m 2000 --blocks 400 200 --lp 500 \
        --mode mixed --iterations 3

Runs the cold start plus `--iterations` Newton iterations on the GPU (the solve
stops with IterLimit) so that a kernel profiler sees a bounded, representative
launch sequence.  Prints the per-phase device time of the run.
"""
import argparse
import json
import os
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=2000)
    ap.add_argument("--blocks", type=int, nargs="+", default=[400, 200])
    ap.add_argument("--lp", type=int, default=500)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--mode", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--iterations", type=int, default=3)
    args = ap.parse_args()
    from sdpx_b200 import SolverOptions, generators as G
    from sdpx_b200.cuda_backend import CudaBackend

    prob = G.sdpa_dense(m=args.m, blocks=args.blocks, lp=args.lp, seed=args.seed)
    opts = SolverOptions(iter_max=args.iterations, precision=args.mode).with_tolerance(1e-8)
    with CudaBackend(prob, precision=args.mode) as be:
        r = be.optimize(opts)  # the loop inside the library, as the product runs it
        phases = be.phase_times()
    print(json.dumps({"status": r.status.value, "iterations": r.iterations,
                      "precision": r.precision_trace, "phase_ms": phases}))


if __name__ == "__main__":
    main()
