"""Launch-shape autotuner of the step.

For one workload it times every candidate launch shape on the device and
records the fastest in a JSON table that ``bench.py`` and users read back
through ``System.tune``:

* ``pcg_blocks_per_sm``: how many 256-thread blocks of the persistent PCG
  kernel share an SM (0 = as many as occupancy allows).  Fewer blocks make
  the grid barriers cheaper; more blocks hide more load latency in the
  element-tile matvec.
* ``graph``: whether a batched elastic step is replayed from one captured CUDA
  graph (device-side substep choice) or launched kernel by kernel.
* ``row_group`` and ``batch_blocks`` (``System.tune_shape``), for the
  assembled forms: how many column slots of a matrix row have their inputs
  and blocks requested per round trip (2 or 4), and how many blocks per SM the
  batched kernels are compiled for (3 registers-richer, or 4).  They change
  only the launch shape; the results are bitwise the same.
* ``solver``: the PCG operator form (``System.set_solver``): "auto" (the
  block matrix assembled once per solve, for these workloads), for a batch
  "assembled-two-phase" (two grid barriers per iteration, fewer bytes) and
  "assembled-pipelined" (one barrier per iteration, FP64 recurrences), or
  "elementwise".  The block cap applies to the element-by-element kernels;
  the assembled ones take their own occupancy, so they are timed at 0.

Every candidate starts from the same rest state and runs the same steps, so
the candidates do the same physics; the score is device seconds per step.
The PCG tolerance and cap are those of the run the table is for (the batched
record solves every body to 1e-6 under a cap of 4000).

    python -m talus_b200.autotune --workload batch --precision mixed --tolerance 1e-6 --cap 4000
"""
from __future__ import annotations

import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def candidates(bodies: int):
    """(solver, PCG blocks per SM, graph, row group, batch blocks per SM)."""
    graphs = [True, False] if bodies > 1 else [False]
    out = [("elementwise", k, g, 0, 0) for k in (0, 1, 2, 3) for g in graphs]
    if bodies == 1:
        return out + [("auto", 0, False, rg, 0) for rg in (2, 4)]
    forms = ["assembled-two-phase", "assembled-pipelined"]
    for form in forms:
        out += [(form, 0, g, 0, 0) for g in graphs]
        out += [(form, 0, False, rg, bb) for rg in (2, 4) for bb in (3, 4) if (rg, bb) != (2, 4)]
    return out


def time_candidate(system, meshes, settings, solver, blocks, graph, row_group, batch_blocks, warmup, steps):
    import talus_b200 as tb

    system.set_solver(solver)
    system.tune(blocks, graph)
    system.tune_shape(row_group, batch_blocks)
    for i, m in enumerate(meshes):
        system.set_state(tb.rest_state(m), i)
    for _ in range(warmup):
        system.step(settings)
    seconds, iterations = 0.0, 0
    for _ in range(steps):
        reps = system.step(settings)
        seconds += reps[0].device_seconds
        iterations += sum(r.cg_iterations for r in reps)
    return seconds / steps, iterations / steps


def tune(workload: str, precision_name: str, warmup: int = 2, steps: int = 4, tolerance: float = 1e-3,
         cap: int = 64) -> dict:
    sys.path.insert(0, ROOT)
    import talus_b200 as tb
    from talus_b200.workloads import WORKLOADS, make_bodies

    spec = WORKLOADS[workload]
    meshes, mats = make_bodies(spec)
    precision = tb.FP32_MIXED if precision_name == "mixed" else tb.FP64
    law = tb.NEO_HOOKEAN if spec["law"] == "snh" else tb.COROTATED
    settings = tb.Settings(law=law, tolerance=tolerance, cg_iterations=cap)
    system = tb.System(meshes, mats, precision)
    results = []
    for solver, blocks, graph, rg, bb in candidates(len(meshes)):
        sec, its = time_candidate(system, meshes, settings, solver, blocks, graph, rg, bb, warmup, steps)
        results.append({"solver": solver, "pcg_blocks_per_sm": blocks, "graph": graph, "row_group": rg,
                        "batch_blocks": bb, "ms_per_step": sec * 1e3, "cg_iterations_per_step": its})
        print(json.dumps(results[-1]), file=sys.stderr, flush=True)
    system.close()
    best = min(results, key=lambda r: r["ms_per_step"])
    return {"solver": best["solver"], "pcg_blocks_per_sm": best["pcg_blocks_per_sm"], "graph": best["graph"],
            "row_group": best["row_group"], "batch_blocks": best["batch_blocks"],
            "ms_per_step": best["ms_per_step"], "steps": steps, "tolerance": tolerance, "cg_iterations": cap,
            "candidates": results}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="batch")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--tolerance", type=float, default=1e-3)
    ap.add_argument("--cap", type=int, default=64)
    ap.add_argument("--out", default=os.path.join(ROOT, "talus_b200", "tuning.json"))
    args = ap.parse_args()
    entry = tune(args.workload, args.precision, steps=args.steps, tolerance=args.tolerance, cap=args.cap)
    table = {}
    if os.path.exists(args.out):
        with open(args.out) as f:
            table = json.load(f)
    table[f"{args.workload}/{args.precision}"] = entry
    with open(args.out, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    print(json.dumps({k: v for k, v in entry.items() if k != "candidates"}))


if __name__ == "__main__":
    main()
