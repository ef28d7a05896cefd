"""Named synthetic workloads of the tet FEM step.

* ``elastic-block``  8x8x8 cubes (3,072 tets, 729 nodes) of neo-Hookean
  rubber, E=1e6 Pa, nu=0.3, rest jittered +-1 % of the cell, bottom pinned.
* ``plastic-block``  64x32x32 cubes (393,216 tets) of E=2e7 Pa, nu=0.35, yield
  1e5 Pa, linear hardening 2e5 Pa, bottom pinned, top pushed down at 0.5 m/s.
* ``batch``          512 bodies with cells per axis uniform in {4..24},
  E log-uniform in [1e5, 1e8] Pa, nu uniform in [0.25, 0.45], base pinned.

All use 0.1 m cubes split into six Kuhn tets, density 1000, gravity 9.81 and
dt = 1/60 (the code that steps each workload passes those).
"""
from __future__ import annotations

import numpy as np

from .deformable import PhysicalMaterial
from .mesh import batch_bodies, box_mesh
from .shard import batch_bodies_range, batch_dims, partition, tets_of

WORKLOADS = {
    "plastic-block": dict(cells=(64, 32, 32), youngs=2e7, poisson=0.35, yield_stress=1e5, hardening=2e5,
                          push=0.5, jitter=0.0, law="corotated"),
    "elastic-block": dict(cells=(8, 8, 8), youngs=1e6, poisson=0.3, yield_stress=float("inf"), hardening=0.0,
                          push=0.0, jitter=0.01, law="snh"),
    "batch": dict(batch=True, count=512, lo=4, hi=24, seed=3, law="corotated"),
}


def make_mesh(spec, scale_cells=None):
    """One block of a single-body workload; ``scale_cells`` gives a smaller
    block pushed at the same strain rate."""
    cells = scale_cells or spec["cells"]
    mesh = box_mesh(cells, voxel=0.1, jitter=spec["jitter"], seed=2)
    if spec["push"]:
        top = mesh.face(1, 1)
        mesh.anchored[top] = 1
        mesh.prescribed_velocity = np.zeros((mesh.nodes, 3))
        mesh.prescribed_velocity[top, 1] = -spec["push"] * cells[1] / spec["cells"][1]
    mat = PhysicalMaterial(density=1000.0, youngs_modulus=spec["youngs"], poissons_ratio=spec["poisson"],
                           yield_stress=spec["yield_stress"], hardening_modulus=spec["hardening"])
    return mesh, mat


def make_bodies(spec, rank=0, world=1):
    """(meshes, per-body material lists) of a workload for one rank.  A batch
    on `world` ranks is the batch of count * world bodies, each rank taking
    its contiguous, tet-balanced share (talus_b200.shard); a single-body
    workload is the same body on every rank (replicas)."""
    if spec.get("batch"):
        if world == 1:
            return batch_bodies(spec["count"], spec["seed"], spec["lo"], spec["hi"])
        total = spec["count"] * world
        dims = batch_dims(total, spec["seed"], spec["lo"], spec["hi"])
        lo, hi = partition(tets_of(dims), world)[rank]
        return batch_bodies_range(lo, hi, total, spec["seed"], spec["lo"], spec["hi"])
    mesh, mat = make_mesh(spec)
    return [mesh], [[mat]]
