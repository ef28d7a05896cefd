"""Profiling run: steps a benchmark workload and records, for every PCG
launch, its iteration count, so that an ncu capture of one launch of
tl::kPcg can be turned into DRAM bytes per PCG iteration.

    python profile_run.py --workload plastic-block --steps 4 --precision mixed

prints one JSON line {"pcg_iterations": [...], ...}; PCG launch i of the
program (0-based, in launch order) made pcg_iterations[i] iterations.  The
same command runs under `ncu -k regex:kPcg -s <i> -c 1`.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.abspath(__file__))


def main():
    sys.path.insert(0, ROOT)
    import talus_b200 as tb
    from talus_b200.workloads import WORKLOADS, make_bodies

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="plastic-block", choices=sorted(WORKLOADS))
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--count", type=int, default=0, help="bodies of a batch workload (0: the workload's own)")
    ap.add_argument("--solver", choices=["auto", "assembled", "assembled-two-phase", "elementwise"], default="auto",
                    help="PCG operator form (tl_system_set_solver)")
    ap.add_argument("--tolerance", type=float, default=1e-3, help="PCG relative tolerance")
    ap.add_argument("--cap", type=int, default=64, help="PCG iteration cap")
    ap.add_argument("--factor", type=int, default=-1,
                    help="hold a solver state with this factor budget (tl_system_use_factor; -1: none)")
    ap.add_argument("--cells", default="", help="plastic-block lattice cells as NX,NY,NZ (default: the workload's)")
    args = ap.parse_args()
    spec = dict(WORKLOADS[args.workload])
    if args.count and spec.get("batch"):
        spec["count"] = args.count
    if args.cells:
        spec["cells"] = tuple(int(c) for c in args.cells.split(","))
    meshes, mats = make_bodies(spec)
    precision = tb.FP32_MIXED if args.precision == "mixed" else tb.FP64
    law = tb.NEO_HOOKEAN if spec["law"] == "snh" else tb.COROTATED
    system = tb.System(meshes, mats, precision)
    system.set_solver(args.solver)
    if args.factor >= 0:
        system.use_factor(True, args.factor)
    for i, m in enumerate(meshes):
        system.set_state(tb.rest_state(m), i)
    settings = tb.Settings(law=law, trace=True, tolerance=args.tolerance, cg_iterations=args.cap)
    reports = [[r.as_dict() for r in system.step(settings)] for _ in range(args.steps)]
    print(json.dumps({"workload": args.workload, "precision": args.precision,
                      "tets": sum(m.tets for m in meshes), "nodes": sum(m.nodes for m in meshes),
                      "pcg_iterations": system.trace(),
                      "tangent_iterations": sum(r[0]["cg_tangent_iterations"] for r in reports),
                      "device_seconds": [r[0]["device_seconds"] for r in reports],
                      "factor": system.factor_stats() if args.factor >= 0 else None}))
    system.close()


if __name__ == "__main__":
    main()
