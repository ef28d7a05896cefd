"""Near-inversion precision stress test of the FP32-mixed step.

Workload: a 128x64x64 block of 0.1 m cubes (3,145,728 tets, 545,025 nodes),
E = 1e6 Pa, nu = 0.45, rho = 1000, yield 5e4 Pa, no hardening, gravity.  It
starts at rest; the x = 0 face is pinned and the x = max face is driven
towards it at the constant speed that shortens the block by 60 % over 90
steps of dt = 1/60; the other faces are free.  With start="homogeneous" every
node instead starts with the velocity of a uniform compression at that rate
(v_x proportional to x), which takes the impact at the driven face away.

The FP64 system steps the trajectory.  Before every step its state
(positions, velocities, accelerations, committed rotations, plastic points)
is loaded into an FP32-mixed system, both take the same step, and the runner
reports per step:
* max_rel_force_error: max over nodes |f_mixed - f_fp64| / max |f_fp64| of
  the internal forces both arithmetics evaluate (tl_evaluate) at the FP64
  step's end state;
* yield_state_differences: tets whose equivalent plastic strain grew during
  the step in one arithmetic and not in the other;
* min_volume_ratio: the smallest J the FP64 step saw.
Both systems start each step from the same state, so the numbers measure one
step of arithmetic, not the divergence of two trajectories; the divergence of
independent trajectories is reported once at the end.

    python -m talus_b200.inversion [--cells 128 64 64] [--steps 90]
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def make_block(cells=(128, 64, 64), steps=90, squeeze=0.6, dt=1.0 / 60.0):
    import talus_b200 as tb

    mesh = tb.box_mesh(cells, voxel=0.1, seed=5, anchor_axis=0, anchor_side=0)
    far = mesh.face(0, 1)
    mesh.anchored[far] = 1
    mesh.prescribed_velocity = np.zeros((mesh.nodes, 3))
    mesh.prescribed_velocity[far, 0] = -squeeze * cells[0] * 0.1 / (steps * dt)
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=1.0e6, poissons_ratio=0.45, yield_stress=5.0e4,
                              hardening_modulus=0.0)
    return mesh, mat


def initial_state(mesh, start="rest"):
    import talus_b200 as tb

    state = tb.rest_state(mesh)
    if start == "homogeneous":
        x = mesh.rest_positions[:, 0] - mesh.rest_positions[:, 0].min()
        far = mesh.face(0, 1)
        state.velocity[:, 0] = mesh.prescribed_velocity[far, 0].mean() * x / x.max()
    elif start != "rest":
        raise ValueError(start)
    return state


def run(cells=(128, 64, 64), steps=90, every=1, trajectory=True, context=None, log=None, start="rest"):
    import talus_b200 as tb

    mesh, mat = make_block(cells, steps)
    settings = tb.Settings(law=tb.COROTATED)
    ref = tb.System(mesh, [mat], tb.FP64, context)
    mix = tb.System(mesh, [mat], tb.FP32_MIXED, context)
    ref.set_state(initial_state(mesh, start))
    rows = []
    t0 = time.time()
    state = ref.get_state()
    for k in range(steps):
        check = (k + 1) % every == 0 or k + 1 == steps
        if check:
            mix.set_state(state)
            start_eq = state.plastic[:, 9].astype(np.float32).astype(np.float64)
            mix.step(settings)
            grew_mix = mix.get_state().plastic[:, 9] > start_eq
        rep = ref.step(settings)[0]
        before_eq = state.plastic[:, 9]
        state = ref.get_state()
        if not check:
            continue
        grew64 = state.plastic[:, 9] > before_eq
        mix.set_state(state)
        f64, _ = ref.evaluate(settings)
        f32, _ = mix.evaluate(settings)
        scale = np.linalg.norm(f64, axis=1).max()
        row = {"step": k + 1, "max_rel_force_error": float(np.linalg.norm(f32 - f64, axis=1).max() / scale),
               "yield_state_differences": int(np.count_nonzero(grew64 != grew_mix)),
               "yielded_fp64": int(grew64.sum()), "min_volume_ratio": rep.min_volume_ratio,
               "substeps": rep.substeps, "cg_iterations": rep.cg_iterations,
               "plastic_evaluations": rep.plastic_evaluations}
        rows.append(row)
        if log:
            print(json.dumps(row), file=log, flush=True)
    upright = [r for r in rows if r["min_volume_ratio"] > 0.0]
    first_inverted = next((r["step"] for r in rows if r["min_volume_ratio"] <= 0.0), None)
    out = {"workload": f"near-inversion {cells[0]}x{cells[1]}x{cells[2]} ({mesh.tets} tets), {steps} steps, "
                       f"start {start}",
           "tets": mesh.tets, "nodes": mesh.nodes, "rows": rows,
           "max_rel_force_error": max(r["max_rel_force_error"] for r in rows),
           "max_yield_state_differences": max(r["yield_state_differences"] for r in rows),
           "min_volume_ratio": min(r["min_volume_ratio"] for r in rows),
           "first_inverted_step": first_inverted,
           "upright": {"steps": len(upright),
                       "min_volume_ratio": min((r["min_volume_ratio"] for r in upright), default=None),
                       "max_rel_force_error": max((r["max_rel_force_error"] for r in upright), default=None),
                       "max_yield_state_differences": max((r["yield_state_differences"] for r in upright),
                                                          default=None)},
           "seconds": time.time() - t0}
    if trajectory:
        final64 = state.position
        mix.set_state(initial_state(mesh, start))
        for _ in range(steps):
            mix.step(settings)
        x = mix.get_state().position
        disp = np.linalg.norm(final64 - mesh.rest_positions, axis=1).max()
        out["trajectory_max_rel_displacement_error"] = float(np.linalg.norm(x - final64, axis=1).max() / disp)
    ref.close()
    mix.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, nargs=3, default=[128, 64, 64])
    ap.add_argument("--steps", type=int, default=90)
    ap.add_argument("--every", type=int, default=1)
    ap.add_argument("--start", choices=["rest", "homogeneous"], default="rest")
    args = ap.parse_args()
    out = run(tuple(args.cells), args.steps, args.every, log=sys.stderr, start=args.start)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
