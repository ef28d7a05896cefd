"""Sharding of a batched workload over ranks (one process per GPU).

Bodies of a batch are independent, so a batch spreads over N GPUs with no
exchange on the data path: rank r steps a contiguous range of bodies, and the
ranges are balanced by tet count (the step's cost is close to linear in the
tets of a body).  The only collectives are host-side: the max over ranks of the
timed seconds and the sum of the tets stepped.

    dims = batch_dims(512 * world, seed)          # every rank draws the same sizes
    lo, hi = partition(tets_of(dims), world)[rank]
    meshes, mats = batch_bodies_range(lo, hi, seed)
"""
from __future__ import annotations

import numpy as np


def batch_dims(count: int, seed: int = 3, lo: int = 4, hi: int = 24):
    """Per-body cells per axis, Young's modulus and Poisson's ratio, drawn
    exactly as talus_b200.mesh.batch_bodies draws them."""
    rng = np.random.default_rng(seed)
    dims = rng.integers(lo, hi + 1, size=(count, 3))
    youngs = np.exp(rng.uniform(np.log(1e5), np.log(1e8), size=count))
    poisson = rng.uniform(0.25, 0.45, size=count)
    return dims, youngs, poisson


def tets_of(dims) -> np.ndarray:
    """Tets of each body: six Kuhn tets per cell."""
    d = np.asarray(dims[0] if isinstance(dims, tuple) else dims, np.int64)
    return 6 * d[:, 0] * d[:, 1] * d[:, 2]


def partition(weights, world: int):
    """Contiguous ranges [lo, hi) of the bodies, one per rank, whose weight
    sums are as even as a split at body boundaries allows: rank r ends at the
    first body where the running total reaches (r + 1) / world of the whole.
    Every body is in exactly one range; no range is empty while there are at
    least as many bodies as ranks."""
    w = np.asarray(weights, np.float64)
    n = w.size
    if world < 1:
        raise ValueError("world must be >= 1")
    if n < world:
        raise ValueError("fewer bodies than ranks")
    prefix = np.concatenate([[0.0], np.cumsum(w)])
    total = prefix[-1]
    cuts = [0]
    for r in range(1, world):
        cut = int(np.searchsorted(prefix, total * r / world, side="left"))
        # keep at least one body per remaining rank on each side
        cut = max(cut, cuts[-1] + 1)
        cut = min(cut, n - (world - r))
        cuts.append(cut)
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def aggregate(local_tets: int, local_seconds: float, dist=None, device=None):
    """(tets stepped by all ranks, max over ranks of the timed seconds): the
    two host-side collectives of a sharded or replicated run (dist is
    torch.distributed or None for one process)."""
    if dist is None:
        return int(local_tets), float(local_seconds)
    import torch

    t = torch.tensor([float(local_tets)], dtype=torch.float64, device=device)
    s = torch.tensor([float(local_seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    dist.all_reduce(s, op=dist.ReduceOp.MAX)
    return int(t.item()), float(s.item())


def batch_bodies_range(lo: int, hi: int, count: int, seed: int = 3, cells_lo: int = 4, cells_hi: int = 24,
                       voxel: float = 0.1):
    """Bodies lo..hi-1 of the count-body batch (the same bodies, seeds and
    materials talus_b200.mesh.batch_bodies(count, seed) makes)."""
    from .deformable import PhysicalMaterial
    from .mesh import box_mesh

    dims, youngs, poisson = batch_dims(count, seed, cells_lo, cells_hi)
    meshes = [box_mesh(tuple(int(c) for c in dims[i]), voxel=voxel, seed=seed + i) for i in range(lo, hi)]
    mats = [[PhysicalMaterial(density=1000.0, youngs_modulus=float(youngs[i]), poissons_ratio=float(poisson[i]))]
            for i in range(lo, hi)]
    return meshes, mats
