"""Regenerate tests/golden/gates.json from the reference's recorded gate
baselines (benchmark/baselines/gates.json of SDPX.jl) and its correctness pins
(test/correctness.jl:236-241).  Run from the repository root with the reference
checkout path as the only argument; the committed JSON is what the tests read.
"""
import json
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_gate_fixture.py <path of the SDPX.jl checkout>")
ref = Path(sys.argv[1])
base = json.loads((ref / "benchmark/baselines/gates.json").read_text())
keep = ("status", "iterations", "objective", "relative_gap", "primal_residual", "dual_residual")
out = {name: {k: base[name][k] for k in keep} for name in ("sdp_closed_form", "sdp_dense")}
out["sdp_closed_form"]["tolerance"] = 1e-10      # benchmark/gates.jl:138
out["sdp_dense"]["tolerance"] = 1e-8             # benchmark/gates.jl:197
out["compare"] = {"iterations": 1, "objective_rel": 1e-9, "residual_factor": 10.0,
                  "absolute_floor": 1e-10}       # benchmark/gates.jl:58-77
out["T1_fixed_policy"] = {"iterations": 19, "iteration_slack": 2,
                          "objective": 4.898979485566356, "objective_abs": 1e-8}
# T2 / T3 (test/correctness.jl:97-135, T6 pin :T2_Float64 => 15 at :230-233):
# the equality x1 = 2 (once, then duplicated), optimum 11/2, tolerance 1e-6.
out["T2_fixed_policy"] = {"iterations": 15, "iteration_slack": 2, "objective": 5.5,
                          "objective_abs": 1e-6}
out["T3_fixed_policy"] = {"objective": 5.5, "objective_abs": 1e-6}
Path(__file__).with_name("gates.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
