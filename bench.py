"""Benchmark of the B200 tet FEM step (element-steps/s).

Workload (N=1), WORKLOADS["plastic-block"]: a 64x32x32-cube block (393,216
tets, 70,785 nodes, 0.1 m cubes) of E=2e7 Pa, nu=0.35, rho=1000, yield 1e5 Pa,
linear hardening 2e5 Pa, bottom face pinned, top face pushed down at 0.5 m/s,
gravity 9.81, dt=1/60, FP32-mixed.  A step is one deformable::step (dt) of the full hot
path: element pass, CSR gather assembly, PCG, plastic Newton control.  Inputs
are synthetic (seeded generator of the reference's buildMesh layout).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--precision mixed|fp64] [--workload NAME]
Under torchrun (N>1) every rank steps its own replica of the block (the path
does not shard within one body; bodies are independent), no collective on
the data path; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "elem-steps/s FP32-mixed vs FP64 GPU @rel-err<=1e-5; adjoint/forward time ratio"
UNIT = "element-steps/s"

WORKLOADS = {
    # BASELINE configs[1]
    "plastic-block": dict(cells=(64, 32, 32), youngs=2e7, poisson=0.35, yield_stress=1e5, hardening=2e5,
                          push=0.5, jitter=0.0, law="corotated"),
    # BASELINE configs[0]
    "elastic-block": dict(cells=(8, 8, 8), youngs=1e6, poisson=0.3, yield_stress=float("inf"), hardening=0.0,
                          push=0.0, jitter=0.01, law="snh"),
}


def make_mesh(spec, scale_cells=None):
    import talus_b200 as tb

    cells = scale_cells or spec["cells"]
    mesh = tb.box_mesh(cells, voxel=0.1, jitter=spec["jitter"], seed=2)
    if spec["push"]:
        top = mesh.face(1, 1)
        mesh.anchored[top] = 1
        mesh.prescribed_velocity = np.zeros((mesh.nodes, 3))
        # same strain rate as the full block when the sample is shorter
        mesh.prescribed_velocity[top, 1] = -spec["push"] * cells[1] / spec["cells"][1]
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=spec["youngs"], poissons_ratio=spec["poisson"],
                              yield_stress=spec["yield_stress"], hardening_modulus=spec["hardening"])
    return mesh, mat


def sample_cells(spec):
    """Bounded CPU sample of a workload: 1/64 of the cells (1/4 per axis)."""
    return tuple(max(2, c // 4) for c in spec["cells"])


# ----------------------------------------------------------------- clocks --

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        mhz, maxmhz, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                maxmhz = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(mhz)) if mhz else None, "sm_max_mhz": maxmhz, "reasons": sorted(reasons),
                "samples": len(mhz)}


# ------------------------------------------------------------ algorithmic --

def tile_slots(mesh, tile=256):
    """Slots of the two-level assembly: distinct nodes per 256-element tile."""
    t = mesh.tet_nodes
    total = 0
    for k in range(0, t.shape[0], tile):
        total += np.unique(t[k:k + tile]).size
    return total


def pcg_bytes_per_iteration(T, V, slots, s_bytes, tangent):
    """Unique bytes one iteration of the single-body PCG (tl::kPcg1, phases A,
    B, C) must move, per the layout in talus_b200/csrc/tl_kernels.cuh:
    every array read or written once per phase.  s = 4 (FP32) or 8 (FP64)."""
    v4 = 4 * s_bytes
    # A, per element: tet 16, rotated gradients 9 s, coefficients v4, [flow normal 2 v4],
    # tile CSR codes 4 x 2 B; per slot: offset 2 B + partial write v4; per node: p, z gathered
    a = T * (16 + 9 * s_bytes + v4 + (2 * v4 if tangent else 0) + 8) + slots * (2 + v4) + V * 2 * v4
    # B, per node: p, z read, p write, slot CSR start 4 + per slot id 4 and partial v4, mass record, anchor, Ap write
    b = V * (2 * v4 + v4 + 4 + v4 + 1 + v4) + slots * (4 + v4)
    # C, per node: p, x read+write, Ap, r read+write, preconditioner (2 records), z write
    c = V * (v4 + 2 * v4 + v4 + 2 * v4 + 2 * v4 + v4)
    return a + b + c


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------- CPU side --

def cpu_sample(spec, steps_budget_s=15.0, max_steps=400):
    """The oracle (the reference's algorithm restated, FP32 like the reference)
    on a bounded sample of the workload, single-threaded like the reference
    step (Settings::stepThreads is never read, solver.h:73-74)."""
    from oracle import pyoracle as po
    from tests.helpers import oracle_material, to_oracle

    cells = sample_cells(spec)
    mesh, mat = make_mesh(spec, cells)
    om = to_oracle(mesh)
    state = po.State.rest(om)
    settings = po.Settings(law=po.LAW_SNH if spec["law"] == "snh" else po.LAW_COROTATED)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps and time.perf_counter() - t0 < steps_budget_s:
        po.step(po.F32, om, state, [oracle_material(mat)], settings, (0.0, -9.81, 0.0), 1.0 / 60.0)
        steps += 1
    secs = time.perf_counter() - t0
    return {"value": mesh.tets * steps / secs, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"oracle FP32 (reference arithmetic), {cells[0]}x{cells[1]}x{cells[2]} cells "
                      f"({mesh.tets} tets, 1/64 of the workload, same strain rate), {steps} steps from rest, "
                      f"1 thread, {secs:.1f} s"}


def cpu_info():
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return model


def run_reference(args, spec, rank, world):
    if rank != 0:
        return
    from oracle import pyoracle as po
    from tests.helpers import oracle_material, to_oracle

    cells = sample_cells(spec)
    mesh, mat = make_mesh(spec, cells)
    om = to_oracle(mesh)
    state = po.State.rest(om)
    settings = po.Settings(law=po.LAW_SNH if spec["law"] == "snh" else po.LAW_COROTATED)
    mats = [oracle_material(mat)]
    for _ in range(args.warmup):
        po.step(po.F32, om, state, mats, settings, (0.0, -9.81, 0.0), 1.0 / 60.0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        po.step(po.F32, om, state, mats, settings, (0.0, -9.81, 0.0), 1.0 / 60.0)
    secs = time.perf_counter() - t0
    value = mesh.tets * args.steps / secs
    sample = (f"oracle FP32 restatement of deformable::step (the reference cannot be built here: GLM/Eigen "
              f"fetched at configure time), {cells[0]}x{cells[1]}x{cells[2]} cells ({mesh.tets} tets, 1/64 of "
              f"{args.workload}, same strain rate), 1 thread ({cpu_info()})")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "cells": list(cells), "tets": mesh.tets, "nodes": mesh.nodes},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# --------------------------------------------------------------- GPU side --

def run_ours(args, spec, rank, world, dist):
    import torch

    import talus_b200 as tb
    from talus_b200 import _capi as capi

    device = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(device)
    precision = tb.FP32_MIXED if args.precision == "mixed" else tb.FP64
    mesh, mat = make_mesh(spec)
    law = tb.NEO_HOOKEAN if spec["law"] == "snh" else tb.COROTATED
    settings = tb.Settings(law=law, profile=True)
    context = tb.Context(device)
    system = tb.System(mesh, [mat], precision, context)
    system.set_state(tb.rest_state(mesh))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")  # > 126 MB L2
    for _ in range(args.warmup):
        system.step(settings)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing: per-step events inside the library, L2 flushed between steps
    barrier()
    totals = capi.tl_step_report()
    step_seconds = []
    with ClockSampler(device) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            rep = system.step(settings)[0]
            step_seconds.append(rep.device_seconds)
            for name, _ in rep._fields_:
                if name in ("cg_worst_relative_residual", "plastic_worst_residual", "min_volume_ratio"):
                    continue
                setattr(totals, name, getattr(totals, name) + getattr(rep, name))
        barrier()
    local = sum(step_seconds)
    if dist is not None:
        t = torch.tensor([local], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        local = float(t.item())
    total_seconds = local
    value = world * mesh.tets * args.steps / total_seconds

    # ---- end to end through the public host-state API (state in host memory every step)
    state = system.get_state()
    f32 = {k: np.ascontiguousarray(getattr(state, k), np.float32) for k in
           ("position", "velocity", "acceleration", "rotation", "plastic")}
    h2d = sum(a.nbytes for a in f32.values())
    lib = capi.lib()
    s_c = settings._c()
    g = np.asarray((0.0, -9.81, 0.0))
    rep_e2e = capi.tl_step_report()
    e2e_steps = max(3, min(args.steps, 10))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        st = lib.tl_step_host(system.handle, 0, capi.TL_DTYPE_F32, f32["position"].ctypes.data,
                              f32["velocity"].ctypes.data, f32["acceleration"].ctypes.data,
                              f32["rotation"].ctypes.data, f32["plastic"].ctypes.data, s_c, g.ctypes.data,
                              1.0 / 60.0, rep_e2e)
        if st not in (capi.TL_OK, capi.TL_ERR_NONFINITE):
            capi.check(st, context.handle)
    barrier()
    e2e_seconds = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_seconds], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_seconds = float(t.item())
    e2e_value = world * mesh.tets * e2e_steps / e2e_seconds

    # ---- roofline of the dominant kernel (persistent PCG)
    s_bytes = 4 if precision == tb.FP32_MIXED else 8
    iters = totals.cg_iterations
    tangent_iters = totals.cg_tangent_iterations
    slots = tile_slots(mesh)
    per_iter = {t: pcg_bytes_per_iteration(mesh.tets, mesh.nodes, slots, s_bytes, t) for t in (False, True)}
    pcg_bytes = per_iter[True] * tangent_iters + per_iter[False] * (iters - tangent_iters)
    launches_pcg = totals.cg_solves
    pcg_time = totals.pcg_seconds
    peak, peak_kind = peaks()
    achieved = pcg_bytes / pcg_time / 1e9 if pcg_time > 0 else 0.0
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "pcg_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr = json.load(f)
        if tr.get("workload") == args.workload and tr.get("precision") == args.precision and launches_pcg:
            # bytes per PCG iteration from one ncu capture, scaled to this run's average launch
            traffic = tr["dram_bytes_per_iteration"] * iters / launches_pcg

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_seconds * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-mixed" if precision == tb.FP32_MIXED else "f64",
        "data": "synthetic (seeded Kuhn grid in the reference buildMesh layout)",
        "config": {"workload": args.workload, "cells": list(spec["cells"]), "tets": mesh.tets, "nodes": mesh.nodes,
                   "law": spec["law"], "precision": args.precision, "dt": 1.0 / 60.0,
                   "parallelism": f"replicas{world}" if world > 1 else "single-gpu",
                   "l2": "flushed (256 MB write) between timed steps; working set > 126 MB"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                "steps": e2e_steps, "api": "tl_step_host (state in host memory, f32)"},
        "gpu_launches": int(totals.kernel_launches),
        "roofline": {"bound": "hbm", "kernel": "tl::kPcg1 (persistent block-Jacobi PCG, two-level assembly)",
                     "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "launches": launches_pcg, "iterations": iters,
                     "algorithmic_bytes_per_launch": pcg_bytes / max(1, launches_pcg),
                     "avg_launch_ms": pcg_time * 1e3 / max(1, launches_pcg)},
        "breakdown_ms_per_step": {"pcg": pcg_time * 1e3 / args.steps,
                                  "element": totals.element_seconds * 1e3 / args.steps,
                                  "assemble": totals.assemble_seconds * 1e3 / args.steps},
        "solver": {"cg_iterations_per_step": iters / args.steps,
                   "plastic_evaluations_per_step": totals.plastic_evaluations / args.steps},
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_sample(spec)
        result["cpu_baseline"]["cpu"] = cpu_info()
    if rank == 0:
        print(json.dumps(result), flush=True)
    system.close()
    context.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="plastic-block")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    spec = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as td

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td
    try:
        if args.impl == "reference":
            run_reference(args, spec, rank, world)
        else:
            run_ours(args, spec, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
