"""Benchmark of the B200 tet FEM step (element-steps/s).

Workload (N=1), WORKLOADS["plastic-block"]: a 64x32x32-cube block (393,216
tets, 70,785 nodes, 0.1 m cubes) of E=2e7 Pa, nu=0.35, rho=1000, yield 1e5 Pa,
linear hardening 2e5 Pa, bottom face pinned, top face pushed down at 0.5 m/s,
gravity 9.81, dt=1/60, FP32-mixed.  A step is one deformable::step (dt) of the
full hot path: element pass, CSR gather assembly, PCG, plastic Newton control.
Other workloads: "elastic-block" (8x8x8 neo-Hookean block) and "batch" (512
uneven bodies in one system, one graph-captured launch sequence per step).
Inputs are synthetic (seeded generator of the reference's buildMesh layout).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--precision mixed|fp64] [--workload NAME]
Under torchrun (N>1) every rank steps its own replica of the workload (the
path does not shard within one body; bodies are independent), no collective
on the data path; time = max over ranks.
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

from talus_b200.shard import aggregate  # noqa: E402
from talus_b200.workloads import WORKLOADS, make_bodies, make_mesh  # noqa: E402


def batch_sample_count(spec, budget_tets):
    """Bodies at the start of the batch that fit `budget_tets` (at least one)."""
    from talus_b200 import shard

    tets = shard.tets_of(shard.batch_dims(spec["count"], spec["seed"], spec["lo"], spec["hi"]))
    take, total = 0, 0
    while take < len(tets) and (total + tets[take] <= budget_tets or take == 0):
        total += int(tets[take])
        take += 1
    return take, total


def sample_bodies(spec, budget_tets=8000, divide=2):
    """Bounded CPU sample of a workload: a sub-block with 1/`divide` of the
    cells per axis (1/divide^3 of the workload, pushed at the same strain
    rate) of a single body; the first bodies of a batch up to `budget_tets`
    tets."""
    if spec.get("batch"):
        from talus_b200 import shard

        take, total = batch_sample_count(spec, budget_tets)
        meshes, mats = shard.batch_bodies_range(0, take, spec["count"], spec["seed"], spec["lo"], spec["hi"])
        return meshes, mats, f"the first {take} bodies of the batch ({total} tets)"
    full = 6 * spec["cells"][0] * spec["cells"][1] * spec["cells"][2]
    if full <= 50000:  # small workloads are timed whole
        mesh, mat = make_mesh(spec)
        return [mesh], [[mat]], f"the whole workload ({mesh.tets} tets)"
    cells = tuple(max(2, c // divide) for c in spec["cells"])
    mesh, mat = make_mesh(spec, cells)
    return [mesh], [[mat]], (f"{cells[0]}x{cells[1]}x{cells[2]} cells ({mesh.tets} tets, 1/{divide ** 3} of the "
                             f"workload, same strain rate)")


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


def element_bytes(T, V, s_bytes, yields, commit=False):
    """Unique bytes of one tl::kElement launch over a body (layout in
    talus_b200/csrc/tl_kernels.cuh).  Per element it reads the tet (16 B),
    Dm^-1 (9 FP64 planes, 72 B), the FP64 volume (8 B), the lane (4 B) and, for
    a yielding material, the plastic point (2 Vec4 planes); per node the
    evaluation point (base and direction records).  An evaluation writes the
    committed rotation (9 S), the matvec operator record (3 Vec4: gradients
    and coefficients) and the per-corner force/diagonal records (4 x (2 Vec4 + S));
    a commit pass writes only the plastic point."""
    v4 = 4 * s_bytes
    reads = T * (16 + 72 + 8 + 4 + (2 * v4 if yields else 0)) + V * 2 * v4
    writes = T * (2 * v4) if commit else T * (9 * s_bytes + 3 * v4 + 4 * (2 * v4 + s_bytes))
    return reads + writes


def pcg_bytes_per_iteration(T, V, slots, s_bytes, tangent):
    """Unique bytes one PCG iteration (tl::kPcg1 / kPcgBatch, phases A, B, C)
    must move for one body, per the layout in talus_b200/csrc/tl_kernels.cuh:
    every array read or written once per phase.  s = 4 (FP32) or 8 (FP64)."""
    v4 = 4 * s_bytes
    # A, per element: tet 16, operator record 3 v4 (gradients, coefficients), [flow normal 2 v4],
    # tile CSR codes 4 x 2 B; per slot: offset 2 B + partial write v4; per node: p, z gathered
    a = T * (16 + 3 * v4 + (2 * v4 if tangent else 0) + 8) + slots * (2 + v4) + V * 2 * v4
    # B, per node: p, z read, p write, slot CSR start 4 + per slot id 4 and partial v4, mass record, anchor, Ap write
    b = V * (2 * v4 + v4 + 4 + v4 + 1 + v4) + slots * (4 + v4)
    # C, per node: p, x read+write, Ap, r read+write, preconditioner (2 records), z write
    c = V * (v4 + 2 * v4 + v4 + 2 * v4 + 2 * v4 + v4)
    return a + b + c


SELL_AUTO_MIN_TETS = 32768  # smallest body TL_SOLVER_AUTO assembles (talus_b200/csrc/tl_system.cu)


def operator_blocks(mesh):
    """Nonzero 3x3 blocks of the assembled single-body operator: the ordered
    node pairs that share an element (the diagonal included)."""
    t = mesh.tet_nodes.astype(np.int64)
    pairs = (t[:, :, None] * mesh.nodes + t[:, None, :]).ravel()
    return int(np.unique(pairs).size)


def sell_bytes_per_iteration(blocks, V, s_bytes):
    """Unique bytes of one tl::kPcgSell iteration (talus_b200/csrc/tl_sell.cuh):
    every block of the matrix (9 S entries and its column index) and the
    published matvec input read once, the next input written once.  The
    iteration vectors stay in registers."""
    v4 = 4 * s_bytes
    return blocks * (9 * s_bytes + 4) + 2 * V * v4


def sell_batch_bytes_per_iteration(blocks, V, s_bytes):
    """Unique bytes of one body's iteration in tl::kPcgBatchSell: the body's
    matrix blocks (9 S entries and a column index) once; per node, the
    previous direction and z gathered, the new direction and A p written
    (phase AB), then direction, x, A p, r, the preconditioner (2 records)
    read and x, r, z written (phase C)."""
    v4 = 4 * s_bytes
    return blocks * (9 * s_bytes + 4) + V * 13 * v4


def sell_assembly_bytes(T, blocks, s_bytes, tangent):
    """Unique bytes of one tl::kSellAssemble launch: the element matvec
    operator record (3 Vec4, [2 Vec4 flow normal]) and the 16 contributor
    codes of every element read once, each block written once with its
    contributor range."""
    v4 = 4 * s_bytes
    return T * (3 * v4 + (2 * v4 if tangent else 0) + 16 * 4) + blocks * (9 * s_bytes + 4)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def tuning(workload, precision):
    path = os.path.join(ROOT, "talus_b200", "tuning.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f).get(f"{workload}/{precision}")


# --------------------------------------------------------------- CPU side --

def cpu_info():
    """Host CPU model, logical cores usable by this process and widest SIMD
    (from the /proc/cpuinfo flags; the oracle is compiled -O2 without -march,
    so it runs SSE2 code whatever the host offers)."""
    model, flags = "", set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and not model:
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = set(line.split(":", 1)[1].split())
    except OSError:
        pass
    simd = ("AVX-512 (512-bit)" if "avx512f" in flags else "AVX2 (256-bit)" if "avx2" in flags
            else "SSE2 (128-bit)" if "sse2" in flags else "unknown")
    return {"cpu": model, "nproc": host_workers(), "simd": simd, "oracle_simd": "SSE2 (128-bit, -O2, no -march)"}


def _oracle_bodies(spec, indices):
    """Oracle meshes, rest states and materials of the given batch bodies."""
    from oracle import pyoracle as po
    from talus_b200 import shard
    from tests.helpers import oracle_material, to_oracle

    out = []
    for i in indices:
        (m,), (mat,) = shard.batch_bodies_range(i, i + 1, spec["count"], spec["seed"], spec["lo"], spec["hi"])
        om = to_oracle(m)
        out.append((om, po.State.rest(om), [oracle_material(x) for x in mat]))
    return out


def _oracle_worker(conn, spec, indices):
    """A host core stepping its share of the sampled batch bodies, or its own
    copy of a single body's sample sub-block (indices None), on request."""
    from oracle import pyoracle as po
    from tests.helpers import oracle_material, to_oracle

    if indices is None:
        meshes, mats, _ = sample_bodies(spec)
        bodies = [(to_oracle(m), po.State.rest(to_oracle(m)), [oracle_material(x) for x in mat])
                  for m, mat in zip(meshes, mats)]
    else:
        bodies = _oracle_bodies(spec, indices)
    settings = po.Settings(law=po.LAW_SNH if spec["law"] == "snh" else po.LAW_COROTATED)
    conn.send("ready")
    while conn.recv() == "step":
        for om, state, mats in bodies:
            po.step(po.F32, om, state, mats, settings, (0.0, -9.81, 0.0), 1.0 / 60.0)
        conn.send("done")


class ParallelOracleRun:
    """The reference's per-body step is serial (Settings::stepThreads is never
    read, solver.h:73-74), so the host's cores are used the way a caller of
    the reference would use them: one spawned process per core, each running
    the single-threaded oracle step on independent bodies.  A batch sample is
    split round-robin over the processes; a single-body workload gives every
    process its own copy of the sample sub-block."""

    def __init__(self, spec, workers, budget_tets_per_core=8000):
        import multiprocessing as mp

        from talus_b200 import shard

        if spec.get("batch"):
            take, _ = batch_sample_count(spec, budget_tets_per_core * workers)
            take = max(take, min(spec["count"], 4 * workers))  # several bodies per process, for balance
            tets = shard.tets_of(shard.batch_dims(spec["count"], spec["seed"], spec["lo"], spec["hi"]))
            self.tets = total = int(tets[:take].sum())
            self.sample = f"the first {take} bodies of the batch ({total} tets)"
            shares = [list(range(w, take, workers)) for w in range(workers)]
        else:
            meshes, _, sample = sample_bodies(spec)
            self.tets = workers * sum(m.tets for m in meshes)
            self.sample = f"{workers} independent copies of {sample}"
            shares = [None] * workers
        ctx = mp.get_context("spawn")
        self.conns, self.procs = [], []
        for w in range(workers):
            parent, child = ctx.Pipe()
            p = ctx.Process(target=_oracle_worker, args=(child, spec, shares[w]), daemon=True)
            p.start()
            self.conns.append(parent)
            self.procs.append(p)
        for c in self.conns:
            if c.recv() != "ready":
                raise RuntimeError("oracle worker failed")

    def step(self):
        for c in self.conns:
            c.send("step")
        for c in self.conns:
            c.recv()

    def close(self):
        for c in self.conns:
            c.send("stop")
        for p in self.procs:
            p.join(timeout=30)


def host_workers():
    return max(1, min(64, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count() or 1))


class OracleRun:
    """The oracle (the reference's algorithm restated, FP32 like the
    reference), single-threaded like the reference step
    (Settings::stepThreads is never read, solver.h:73-74)."""

    def close(self):
        pass

    def __init__(self, spec, divide=2):
        from oracle import pyoracle as po
        from tests.helpers import oracle_material, to_oracle

        self.po = po
        meshes, mats, self.sample = sample_bodies(spec, divide=divide)
        self.bodies = []
        for m, mat in zip(meshes, mats):
            om = to_oracle(m)
            self.bodies.append((om, po.State.rest(om), [oracle_material(x) for x in mat]))
        self.tets = sum(m.tets for m in meshes)
        self.settings = po.Settings(law=po.LAW_SNH if spec["law"] == "snh" else po.LAW_COROTATED)

    def step(self):
        for om, state, mats in self.bodies:
            self.po.step(self.po.F32, om, state, mats, self.settings, (0.0, -9.81, 0.0), 1.0 / 60.0)


def timed_steps(run, warmup, budget_s, min_steps=3, max_steps=400):
    for _ in range(warmup):
        run.step()
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps and (steps < min_steps or time.perf_counter() - t0 < budget_s):
        run.step()
        steps += 1
    return steps, time.perf_counter() - t0


def cpu_sample(spec, budget_s=10.0):
    """The reference arithmetic (oracle FP32) on the host, after 2 warm-up
    steps from rest: one thread on the 1/8 sub-block (the reference's serial
    step), one thread on the 1/64 sub-block (a cache-resident size, to show
    what the smaller sample would inflate), and one process per host core on
    independent 1/8 sub-blocks."""
    info = cpu_info()
    run = OracleRun(spec, divide=2)
    steps, secs = timed_steps(run, 2, budget_s)
    out = {"value": run.tets * steps / secs, "unit": UNIT, "cores": 1, "kind": "port",
           "sample": f"oracle FP32 (reference arithmetic), {run.sample}, 2 warm-up and {steps} timed steps, 1 thread, "
                     f"{secs:.1f} s", **info}
    if not spec.get("batch") and 6 * int(np.prod(spec["cells"])) > 50000:
        small = OracleRun(spec, divide=4)
        s2, t2 = timed_steps(small, 2, budget_s / 2)
        out["cache_resident_sample"] = {"value": small.tets * s2 / t2, "sample": small.sample, "steps": s2}
    workers = host_workers()
    if workers > 1:
        par = ParallelOracleRun(spec, workers)
        s3, t3 = timed_steps(par, 2, budget_s)
        par.close()
        out["all_cores"] = {"value": par.tets * s3 / t3, "cores": workers, "sample": par.sample, "steps": s3,
                            "note": "one process per core, each the serial oracle step on its own bodies"}
    return out


def run_reference(args, spec, rank, world):
    if rank != 0:
        return
    workers = host_workers()
    run = ParallelOracleRun(spec, workers) if workers > 1 else OracleRun(spec)
    for _ in range(args.warmup):
        run.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        run.step()
    secs = time.perf_counter() - t0
    run.close()
    value = run.tets * args.steps / secs
    info = cpu_info()
    sample = (f"oracle FP32 restatement of deformable::step (the reference cannot be built here: GLM/Eigen "
              f"fetched at configure time), {run.sample} of {args.workload}, {workers} host "
              f"{'process' if workers == 1 else 'processes'} ({info['cpu']}, {info['simd']})")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "tets": run.tets, "sample": run.sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port", "sample": sample, **info},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# --------------------------------------------------------------- GPU side --

def run_ours(args, spec, rank, world, dist):
    import ctypes as C

    import torch

    import talus_b200 as tb
    from talus_b200 import _capi as capi

    device = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(device)
    precision = tb.FP32_MIXED if args.precision == "mixed" else tb.FP64
    meshes, mats = make_bodies(spec, rank, world)
    B = len(meshes)
    T = sum(m.tets for m in meshes)
    V = sum(m.nodes for m in meshes)
    law = tb.NEO_HOOKEAN if spec["law"] == "snh" else tb.COROTATED
    settings = tb.Settings(law=law, profile=True)
    context = tb.Context(device)
    system = tb.System(meshes, mats, precision, context)
    tune = tuning(args.workload, args.precision)
    if tune:
        system.set_solver(tune.get("solver", "auto"))
        system.tune(tune["pcg_blocks_per_sm"], tune["graph"])
        system.tune_shape(tune.get("row_group", 0), tune.get("batch_blocks", 0))
    for i, m in enumerate(meshes):
        system.set_state(tb.rest_state(m), i)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")  # > 126 MB L2
    for _ in range(args.warmup):
        system.step(settings)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident timing: per-step events inside the library, L2 flushed between steps
    barrier()
    step_seconds, launches = [], 0
    per_body = np.zeros((B, 4))  # cg iterations, tangent iterations, solves, plastic evaluations
    reps_substeps = np.zeros(B)
    totals = {"element": 0.0, "assemble": 0.0, "pcg": 0.0}
    with ClockSampler(device) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            reps = system.step(settings)
            step_seconds.append(reps[0].device_seconds)
            launches += reps[0].kernel_launches
            totals["element"] += reps[0].element_seconds
            totals["assemble"] += reps[0].assemble_seconds
            totals["pcg"] += reps[0].pcg_seconds
            for b in range(B):
                per_body[b] += (reps[b].cg_iterations, reps[b].cg_tangent_iterations, reps[b].cg_solves,
                                reps[b].plastic_evaluations)
                reps_substeps[b] += reps[b].substeps
        barrier()
    # tets stepped by all ranks (replicas: world x T; shards: the whole batch) over the slowest rank
    T_all, total_seconds = aggregate(T, sum(step_seconds), dist, f"cuda:{device}")
    value = T_all * args.steps / total_seconds
    finals = [system.get_state(i) for i in range(B)]

    # ---- end to end through the public API: the state crosses the host boundary every step
    f32 = []
    for st in finals:
        f32.append({k: np.ascontiguousarray(getattr(st, k), np.float32) for k in
                    ("position", "velocity", "acceleration", "rotation", "plastic")})
    # the rotations are outputs of a step (it writes each before reading it): uploaded by neither path
    h2d = sum(a.nbytes for d in f32 for k, a in d.items() if k != "rotation")
    d2h = sum(a.nbytes for d in f32 for a in d.values())
    lib = capi.lib()
    s_c = settings._c()
    g = np.asarray((0.0, -9.81, 0.0))
    e2e_steps = max(3, min(args.steps, 10))
    # the caller's state buffers are page-locked once (tl_host_register), as an engine that
    # steps the same bodies every frame would do: state then crosses by one DMA each way
    for d in f32:
        for arr in d.values():
            context.pin(arr)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        if B == 1:
            d = f32[0]
            st = lib.tl_step_host(system.handle, 0, capi.TL_DTYPE_F32, d["position"].ctypes.data,
                                  d["velocity"].ctypes.data, d["acceleration"].ctypes.data,
                                  d["rotation"].ctypes.data, d["plastic"].ctypes.data, s_c, g.ctypes.data,
                                  1.0 / 60.0, capi.tl_step_report())
        else:
            for i, d in enumerate(f32):
                capi.check(lib.tl_state_set(system.handle, i, capi.TL_DTYPE_F32, d["position"].ctypes.data,
                                            d["velocity"].ctypes.data, d["acceleration"].ctypes.data, None,
                                            d["plastic"].ctypes.data), context.handle)
            reps = (capi.tl_step_report * B)()
            st = lib.tl_step(system.handle, s_c, g.ctypes.data, 1.0 / 60.0, reps)
            for i, d in enumerate(f32):
                capi.check(lib.tl_state_get(system.handle, i, capi.TL_DTYPE_F32, *[d[k].ctypes.data for k in
                           ("position", "velocity", "acceleration", "rotation", "plastic")]), context.handle)
        if st not in (capi.TL_OK, capi.TL_ERR_NONFINITE):
            capi.check(st, context.handle)
    barrier()
    e2e_seconds = max_over_ranks(time.perf_counter() - t0)
    for d in f32:
        for arr in d.values():
            context.unpin(arr)
    e2e_value = T_all * e2e_steps / e2e_seconds

    # ---- roofline of the dominant kernel (persistent PCG): algorithmic bytes of every iteration run
    s_bytes = 4 if precision == tb.FP32_MIXED else 8
    pcg_bytes = 0.0
    assembly = None
    # the form the system took (TL_SOLVER_AUTO: assembled for a batch and for one body of >= 32,768 tets)
    form = tune.get("solver", "auto") if tune else "auto"
    assembled = form != "elementwise" and (B > 1 or form == "assembled" or meshes[0].tets >= SELL_AUTO_MIN_TETS)
    for b, m in enumerate(meshes):
        it, tan = per_body[b, 0], per_body[b, 1]
        if assembled:  # assembled operator (tl_sell.cuh)
            blocks = operator_blocks(m)
            per_it = (sell_bytes_per_iteration if B == 1 else sell_batch_bytes_per_iteration)(blocks, m.nodes, s_bytes)
            pcg_bytes += per_it * it
            if assembly is None:
                assembly = {"kernel": "tl::kSellAssemble (block matrix, once per solve)", "blocks": 0,
                            "algorithmic_bytes_per_launch": 0}
            assembly["blocks"] += blocks
            assembly["algorithmic_bytes_per_launch"] += sell_assembly_bytes(m.tets, blocks, s_bytes, tan > 0)
        else:
            slots = tile_slots(m)
            pcg_bytes += (pcg_bytes_per_iteration(m.tets, m.nodes, slots, s_bytes, True) * tan +
                          pcg_bytes_per_iteration(m.tets, m.nodes, slots, s_bytes, False) * (it - tan))
    launches_pcg = int(per_body[:, 2].max())
    pcg_time = totals["pcg"]
    peak, peak_kind = peaks()
    achieved = pcg_bytes / pcg_time / 1e9 if pcg_time > 0 else 0.0
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "pcg_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr = json.load(f)
        prefix = ("tl::kPcgSell" if B == 1 else "tl::kPcgBatchSell") if assembled else (
            "tl::kPcg1" if B == 1 else "tl::kPcgBatch<")
        same_kernel = tr.get("kernel", "").startswith(prefix)
        if tr.get("workload") == args.workload and tr.get("precision") == args.precision and same_kernel and launches_pcg:
            traffic = tr["dram_bytes_per_iteration"] * per_body[:, 0].sum() / launches_pcg

    if B == 1:
        kernel = ("tl::kPcgSell (persistent pipelined block-Jacobi PCG on the assembled sliced-ELL block matrix)"
                  if assembled else "tl::kPcg1 (persistent block-Jacobi PCG, element by element, two-level assembly)")
    else:
        kernel = "tl::kPcgBatchSell (persistent block-Jacobi PCG over all bodies on the assembled block matrix)"
    config = {"workload": args.workload, "bodies": B, "tets": T, "nodes": V, "law": spec["law"],
              "precision": args.precision, "dt": 1.0 / 60.0,
              "parallelism": "single-gpu" if world == 1 else (f"shards{world}" if spec.get("batch") else f"replicas{world}"),
              "l2": "flushed (256 MB write) between timed steps; working set > 126 MB"}
    if world > 1:
        config["tets_all_ranks"] = T_all
    if not spec.get("batch"):
        config["cells"] = list(spec["cells"])
    if tune:
        config["tuning"] = {"solver": tune.get("solver", "auto"), "pcg_blocks_per_sm": tune["pcg_blocks_per_sm"],
                            "graph": tune["graph"], "row_group": tune.get("row_group", 0),
                            "batch_blocks": tune.get("batch_blocks", 0),
                            "source": "talus_b200/tuning.json (talus_b200.autotune)"}
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_seconds * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-mixed" if precision == tb.FP32_MIXED else "f64",
        "data": "synthetic (seeded Kuhn grids in the reference buildMesh layout)",
        "config": config,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps,
                "api": ("tl_step_host" if B == 1 else "tl_state_set + tl_step + tl_state_get") + " (state in host memory, f32, buffers page-locked once by tl_host_register)"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic, "launches": launches_pcg,
                     "iterations": int(per_body[:, 0].max()),
                     "algorithmic_bytes_per_launch": pcg_bytes / max(1, launches_pcg),
                     "avg_launch_ms": pcg_time * 1e3 / max(1, launches_pcg)},
        "operator_assembly": assembly,
        "element_pass": element_roofline(meshes, mats, per_body, reps_substeps, s_bytes, totals["element"], peak),
        "breakdown_ms_per_step": {k: v * 1e3 / args.steps for k, v in totals.items()},
        "solver": {"cg_iterations_per_step": float(per_body[:, 0].sum() / args.steps),
                   "plastic_evaluations_per_step": float(per_body[:, 3].sum() / args.steps)},
        "clocks": clocks.summary(),
    }
    if precision == tb.FP32_MIXED:
        # the plain FP64 GPU step on the same workload, and the FP32-mixed error against it
        secs64, pos64 = run_fp64(meshes, mats, settings, args, flush, context)
        secs64 = max_over_ranks(secs64)
        worst = 0.0
        for m, st, x64 in zip(meshes, finals, pos64):
            scale = np.linalg.norm(x64 - m.rest_positions, axis=1).max()
            worst = max(worst, float(np.linalg.norm(st.position - x64, axis=1).max() / max(scale, 1e-300)))
        worst = max_over_ranks(worst)
        result["fp64"] = {"value": T_all * args.steps / secs64, "ms_per_step": secs64 * 1e3 / args.steps,
                          "mixed_speedup": secs64 / total_seconds,
                          "max_rel_displacement_error": worst,
                          "note": f"same workload and steps from rest in FP64; error = max over bodies of "
                                  f"max|x_mixed - x_fp64| / max|x_fp64 - X| after {args.warmup + args.steps} steps"}
        if not args.no_converged_check:
            result["fp64"]["converged_check"] = converged_check(meshes, mats, law, context)
    if not args.no_adjoint:
        result["adjoint"] = adjoint_ratio(precision, context)
    if not args.no_batch and not spec.get("batch") and world == 1:
        result["batch"] = batch_form(context, flush)
    yields = any(np.isfinite(m.yield_stress) and m.yield_stress > 0 for ms in mats for m in ms)
    if not args.no_hencky and not spec.get("batch") and yields:
        result["hencky"] = hencky_form(meshes[0], mats[0], settings, context)
    if not args.no_solver_state and not spec.get("batch") and world == 1:
        result["solver_state"] = solver_state_form(context)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_sample(spec)
    if rank == 0:
        print(json.dumps(result), flush=True)
    system.close()
    context.close()


def survey_element_bytes(T, V, s_bytes, yields):
    """The element pass's algorithmic bytes per evaluation in the hot-path
    byte model (tet indices 16, Dm^-1, volume and lane, the positions once
    per node, the element force and the matvec's rotation, and the plastic
    point read and written when the material yields): FP32-mixed elastic
    180 + 12 r, plastic 260 + 12 r; FP64 344 + 24 r and 424 + 24 r bytes per
    tet, r = nodes / tets."""
    r = V / T
    if s_bytes == 4:
        return T * ((260.0 if yields else 180.0) + 12.0 * r)
    return T * ((424.0 if yields else 344.0) + 24.0 * r)


def element_roofline(meshes, mats, per_body, substeps, s_bytes, seconds, peak):
    """Element pass (tl::kElement): algorithmic bytes of every launch in the
    timed steps over the summed CUDA-event time of those launches.  Elastic
    bodies take 3 evaluations per substep; yielding bodies take their Newton
    evaluations plus one commit pass per substep."""
    if seconds <= 0:
        return None
    total, survey, launches = 0.0, 0.0, 0.0
    for b, m in enumerate(meshes):
        yields = any(np.isfinite(x.yield_stress) and x.yield_stress > 0 for x in mats[b])
        evals = per_body[b, 3] if yields else 3 * substeps[b]
        total += evals * element_bytes(m.tets, m.nodes, s_bytes, yields)
        survey += evals * survey_element_bytes(m.tets, m.nodes, s_bytes, yields)
        if yields:
            total += substeps[b] * element_bytes(m.tets, m.nodes, s_bytes, yields, commit=True)
            # a commit pass reads the element data and the positions and writes the plastic point
            survey += substeps[b] * survey_element_bytes(m.tets, m.nodes, s_bytes, yields)
        launches = max(launches, evals + (substeps[b] if yields else 0))
    achieved = total / seconds / 1e9
    achieved_model = survey / seconds / 1e9
    return {"kernel": "tl::kElement", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "launches": int(launches), "avg_launch_us": seconds * 1e6 / max(1.0, launches),
            "algorithmic_bytes": total,
            "hot_path_model": {"bytes": survey, "achieved": achieved_model, "frac": achieved_model / peak,
                               "note": "bytes per tet of the hot-path byte model (FP32-mixed 180/260 + 12 r, FP64 "
                                       "344/424 + 24 r; r = nodes / tets); 'frac' above counts every byte the "
                                       "implementation moves (its per-corner diagonal records and operator record)"}}


def run_fp64(meshes, mats, settings, args, flush, context):
    import torch

    import talus_b200 as tb

    system = tb.System(meshes, mats, tb.FP64, context)
    tune = tuning(args.workload, "fp64")
    if tune:
        system.set_solver(tune.get("solver", "auto"))
        system.tune(tune["pcg_blocks_per_sm"], tune["graph"])
        system.tune_shape(tune.get("row_group", 0), tune.get("batch_blocks", 0))
    for i, m in enumerate(meshes):
        system.set_state(tb.rest_state(m), i)
    for _ in range(args.warmup):
        system.step(settings)
    secs = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        secs += system.step(settings)[0].device_seconds
    pos = [system.get_state(i).position for i in range(len(meshes))]
    system.close()
    return secs, pos


def converged_check(meshes, mats, law, context, steps=8, tolerance=1e-6, cap=3000, sample=24):
    """FP32-mixed against FP64 with every PCG solve converged (relative
    residual 1e-6): the arithmetic's own error, free of the iteration cap.
    Batches use the stiffest bodies (worst conditioned) plus evenly spaced ones."""
    import talus_b200 as tb

    idx = list(range(len(meshes)))
    if len(meshes) > sample:
        youngs = np.array([m[0].youngs_modulus for m in mats])
        stiff = list(np.argsort(-youngs)[:sample // 2])
        spread = [i for i in np.linspace(0, len(meshes) - 1, sample - len(stiff)).astype(int) if i not in stiff]
        idx = sorted(set(stiff + spread))
    M, Mt = [meshes[i] for i in idx], [mats[i] for i in idx]
    settings = tb.Settings(law=law, cg_iterations=cap, tolerance=tolerance)
    out = []
    for prec in (tb.FP32_MIXED, tb.FP64):
        s = tb.System(M, Mt, prec, context)
        for i, m in enumerate(M):
            s.set_state(tb.rest_state(m), i)
        for _ in range(steps):
            s.step(settings)
        out.append([s.get_state(i).position for i in range(len(M))])
        s.close()
    worst = max(float(np.linalg.norm(a - b, axis=1).max() / np.linalg.norm(b - m.rest_positions, axis=1).max())
                for a, b, m in zip(out[0], out[1], M))
    return {"bodies": len(M), "steps": steps, "pcg_tolerance": tolerance, "pcg_cap": cap,
            "max_rel_displacement_error": worst}


def hencky_form(mesh, mats, settings, context, warmup=3, steps=10):
    """The same body in the finite-strain plasticity mode
    (tl_system_set_plasticity(TL_PLASTICITY_HENCKY): elastic steps from each
    tet's plastic rest shape, then the flow kernel), FP32-mixed and FP64 from
    rest: throughput from the library's per-step device time, and the mixed
    error against FP64 after warmup + steps steps."""
    import talus_b200 as tb

    plain = tb.Settings(law=settings.law)
    out, finals = {}, {}
    for name, precision in (("mixed", tb.FP32_MIXED), ("fp64", tb.FP64)):
        s = tb.System(mesh, mats, precision, context)
        s.set_plasticity("hencky")
        s.set_state(tb.rest_state(mesh, hencky=True))
        seconds, flowed = 0.0, 0
        for k in range(warmup + steps):
            rep = s.step(plain)[0]
            if k >= warmup:
                seconds += rep.device_seconds
                flowed = rep.yielding
        finals[name] = s.get_state().position
        s.close()
        out[name] = {"value": mesh.tets * steps / seconds, "ms_per_step": seconds * 1e3 / steps,
                     "flowed_tets_last_step": int(flowed)}
    scale = np.linalg.norm(finals["fp64"] - mesh.rest_positions, axis=1).max()
    out["max_rel_displacement_error"] = float(np.linalg.norm(finals["mixed"] - finals["fp64"], axis=1).max() / scale)
    out["unit"] = UNIT
    out["note"] = (f"plasticity mode 'hencky' on the same body; {warmup} warm-up and {steps} timed steps from rest; "
                   f"device time per step from the step reports")
    return out


def solver_state_form(context, cells=(16, 8, 8), warmup=1, steps=4, budget=32):
    """A caller-held solver state (tl_system_use_factor: the FP64 Cholesky
    preconditioner of deformable::step's DeformableSolverState*) on a
    plastic block of the benchmark's material at reduced size, FP64, against
    the same steps with block Jacobi: device time per step from the step
    reports (the first step, which makes the factor on the host, is a warm-up
    step), PCG iterations, the factor's host time and size."""
    import talus_b200 as tb
    from talus_b200.workloads import WORKLOADS, make_bodies

    spec = dict(WORKLOADS["plastic-block"])
    spec["cells"] = tuple(cells)
    meshes, mats = make_bodies(spec)
    mesh = meshes[0]
    out = {"workload": f"plastic block {cells[0]}x{cells[1]}x{cells[2]} cells ({mesh.tets} tets), FP64",
           "factor_budget": budget}
    for name, factored in (("factor", True), ("jacobi", False)):
        s = tb.System(mesh, mats[0], tb.FP64, context)
        s.set_solver("assembled")
        if factored:
            s.use_factor(True, budget)
        s.set_state(tb.rest_state(mesh))
        seconds, iterations = 0.0, 0
        for k in range(warmup + steps):
            rep = s.step(tb.Settings())[0]
            if k >= warmup:
                seconds += rep.device_seconds
                iterations += rep.cg_iterations
        out[name] = {"ms_per_step": seconds * 1e3 / steps, "pcg_iterations_per_step": iterations / steps}
        if factored:
            st = s.factor_stats()
            out[name].update({"refactor_seconds": st["refactor_seconds"], "factor_nonzeros": st["factor_nonzeros"],
                              "refactor_count": st["refactor_count"], "retries": st["retries"]})
        s.close()
    out["note"] = ("the factored solves are latency-bound on the elimination tree's longest path "
                   "(kPcgFactor); the factor is made on the host at the first step")
    return out


def matrix_blocks(mesh):
    """Nonzero 3x3 blocks of a body's assembled operator: its nodes (the
    diagonal) plus both directions of every distinct edge of its tets."""
    t = mesh.tet_nodes.astype(np.int64)
    pairs = np.concatenate([t[:, [a, b]] for a, b in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))])
    pairs.sort(axis=1)
    edges = np.unique(pairs[:, 0] * (int(pairs.max()) + 1) + pairs[:, 1]).size
    return mesh.nodes + 2 * edges


def batch_form(context, flush, warmup=2, steps=5, tolerance=1e-6, cap=4000):
    """The batching form on its own workload: 512 uneven bodies (cells per
    axis from U{4..24}, E log-uniform in [1e5, 1e8] Pa, nu in [0.25, 0.45],
    7,907,508 tets) in one system, FP32-mixed and plain FP64, each from rest
    with every PCG solve converged (relative residual `tolerance`, the cap out
    of reach), so that the two arithmetics are compared on the same converged
    answer.  Device time per step from the step reports (CUDA events), L2
    flushed before every timed step; the error is the max over all 512 bodies
    of max|x_mixed - x_fp64| / max|x_fp64 - X| after warmup + steps steps."""
    import torch

    import talus_b200 as tb

    spec = WORKLOADS["batch"]
    meshes, mats = make_bodies(spec)
    blocks = [matrix_blocks(m) for m in meshes]
    settings = tb.Settings(cg_iterations=cap, tolerance=tolerance)
    out, finals = {}, {}
    for name, precision in (("mixed", tb.FP32_MIXED), ("fp64", tb.FP64)):
        system = tb.System(meshes, mats, precision, context)
        tune = tuning("batch", name)
        if tune:
            system.set_solver(tune.get("solver", "auto"))
            system.tune(tune["pcg_blocks_per_sm"], tune["graph"])
            system.tune_shape(tune.get("row_group", 0), tune.get("batch_blocks", 0))
        for i, m in enumerate(meshes):
            system.set_state(tb.rest_state(m), i)
        for _ in range(warmup):
            system.step(settings)
        seconds, iters, launches, capped = 0.0, [], 0, 0
        body_iters = np.zeros(len(meshes))
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            reps = system.step(settings)
            seconds += reps[0].device_seconds
            launches += reps[0].kernel_launches
            iters.append(max(r.cg_iterations for r in reps))
            body_iters += [r.cg_iterations for r in reps]
            capped += sum(r.cg_capped_solves for r in reps)
        finals[name] = [system.get_state(i).position for i in range(len(meshes))]
        # one more step with per-class device times: the batched PCG against its algorithmic bytes
        # (per body-iteration: blocks (9s + 4) for the matrix and its columns, plus the node vectors
        # each order moves: 13 (two-phase) or 19 (pipelined) four-wide vectors of s bytes)
        flush.zero_()
        torch.cuda.synchronize()
        preps = system.step(tb.Settings(cg_iterations=cap, tolerance=tolerance, profile=True))
        s_bytes = 4 if precision == tb.FP32_MIXED else 8
        form = (tune or {}).get("solver", "auto")
        piped = form == "assembled-pipelined" or (form in ("auto", "assembled") and precision == tb.FP64)
        vectors = 19 if piped else 13
        pcg_bytes = float(sum(r.cg_iterations * (blocks[i] * (9 * s_bytes + 4) + m.nodes * vectors * 4 * s_bytes)
                              for i, (r, m) in enumerate(zip(preps, meshes))))
        pcg_s = preps[0].pcg_seconds
        peak, peak_kind = peaks()
        pcg_roof = {"kernel": "tl::kPcgBatchSellPipe" if piped else "tl::kPcgBatchSell",
                    "algorithmic_bytes_per_step": pcg_bytes, "pcg_ms_per_step": pcg_s * 1e3,
                    "achieved": pcg_bytes / pcg_s / 1e9 if pcg_s > 0 else None, "peak": peak, "unit": "GB/s",
                    "frac": pcg_bytes / pcg_s / 1e9 / peak if pcg_s > 0 else None, "peak_kind": peak_kind,
                    "step_ms_with_events": preps[0].device_seconds * 1e3}
        system.close()
        tets = sum(m.tets for m in meshes)
        out[name] = {"value": tets * steps / seconds, "ms_per_step": seconds * 1e3 / steps,
                     "max_body_cg_iterations_per_step": float(np.mean(iters)), "gpu_launches": launches,
                     "body_cg_iterations_per_step": {
                         q: float(np.percentile(body_iters / steps, p)) for q, p in
                         (("min", 0), ("median", 50), ("p90", 90), ("max", 100))},
                     "capped_solves": capped, "tuning": tune, "pcg_roofline": pcg_roof}
    worst = max(float(np.linalg.norm(a - b, axis=1).max() / np.linalg.norm(b - m.rest_positions, axis=1).max())
                for a, b, m in zip(finals["mixed"], finals["fp64"], meshes))
    return {"workload": f"batch, {len(meshes)} bodies, {sum(m.tets for m in meshes)} tets", "unit": UNIT,
            "pcg_tolerance": tolerance, "pcg_cap": cap, "warmup": warmup, "steps": steps,
            "mixed": out["mixed"], "fp64": out["fp64"], "mixed_speedup": out["fp64"]["ms_per_step"] /
            out["mixed"]["ms_per_step"], "max_rel_displacement_error": worst, "bodies_checked": len(meshes),
            "l2": "flushed (256 MB write) before each timed step"}


def adjoint_ratio(precision, context, repeats=3):
    """Differentiable-rollout workload: 16^3 cubes (24,576 tets), 30 steps,
    checkpoints every 5, loss |x_T - x_target|^2; device time of the adjoint
    (checkpoint recomputation included) over that of the forward rollout."""
    import talus_b200 as tb
    from talus_b200 import gradcheck

    tol = 1e-10 if precision == tb.FP64 else 1e-6
    prob = gradcheck.make_problem(cells=16, steps=30, checkpoint_every=5, precision=precision, tolerance=tol,
                                  context=context)
    fwd, adj = [], []
    for k in range(repeats + 1):
        loss, g = prob.gradients(prob.youngs, prob.v0)
        if k:
            fwd.append(prob.roll.forward_seconds)
            adj.append(g.seconds)
    f, a = float(np.median(fwd)), float(np.median(adj))
    prob.close()
    return {"workload": "rollout 16x16x16 (24576 tets), 30 steps, checkpoints every 5, neo-Hookean",
            "forward_ms": f * 1e3, "adjoint_ms": a * 1e3, "ratio": a / f, "loss": loss,
            "precision": "fp64" if precision == tb.FP64 else "mixed", "pcg_tolerance": tol, "newton_reads": 4}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="plastic-block")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-converged-check", action="store_true")
    ap.add_argument("--no-hencky", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-solver-state", action="store_true")
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
