"""Synthetic tet meshes with the reference's buildMesh layout.

``box_mesh`` produces what talus::deformable::buildMesh
(src/talus/deformable/solver/solver.cc:2185-2418) produces for a box-shaped
lattice whose every cell is solid with fill 1:

* one node per lattice sample, numbered by first use while cells are visited
  x-fastest and each cell's corners in bit order (x = bit 0, y = bit 1,
  z = bit 2), solver.cc:2217-2250;
* six Kuhn tets per cell around the 0-7 diagonal (KUHN, solver.cc:17-24), with
  nodes 1 and 2 swapped when the rest determinant is negative
  (solver.cc:2342-2350);
* volume det/6, Dm^-1 = inverse(shape) (solver.cc:2352-2358) and lumped mass
  rho V / 4 per corner accumulated in tet order (solver.cc:2360-2364);
* anchors on one face, as a SupportVolume box around that face would give
  (solver.cc:2262-2268).

Rest positions are jittered (uniform +-jitter * voxel per coordinate, from a
counter-based splitmix64 stream) and rounded to float like the reference's
glm::vec3; Dm^-1, volumes and masses are computed in float64 from the
rounded positions.
"""
from __future__ import annotations

import numpy as np

from .deformable import PreparedMesh

KUHN = np.array([[0, 1, 3, 7], [0, 3, 2, 7], [0, 2, 6, 7], [0, 6, 4, 7], [0, 4, 5, 7], [0, 5, 1, 7]], np.int64)

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix_uniform(seed: int, count: int) -> np.ndarray:
    """Uniform [0, 1) doubles: splitmix64 (Steele, Lea & Flood 2014) of counters 1..count."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (np.arange(1, count + 1, dtype=np.uint64) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def batch_bodies(count=512, seed=3, lo=4, hi=24, voxel=0.1):
    """Uneven bodies of the batched benchmark: cell counts per axis uniform in
    {lo..hi}, Young's modulus log-uniform in [1e5, 1e8] Pa, Poisson's ratio
    uniform in [0.25, 0.45], density 1000, base (y = 0) anchored; seeded."""
    from .shard import batch_bodies_range

    return batch_bodies_range(0, count, count, seed, lo, hi, voxel)


def box_mesh(cells, voxel=0.1, origin=(0.0, 0.0, 0.0), jitter=0.0, seed=0, density=1000.0, anchor_axis=1,
             anchor_side=0, lane=0) -> PreparedMesh:
    cx, cy, cz = (int(c) for c in cells)
    if min(cx, cy, cz) < 1:
        raise ValueError("every axis needs at least one cell")
    rx, ry, rz = cx + 1, cy + 1, cz + 1
    # first cell (in x-fastest order) using each lattice sample, and the corner it is there
    i, j, k = np.meshgrid(np.arange(rx), np.arange(ry), np.arange(rz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    fx, fy, fz = np.maximum(i - 1, 0), np.maximum(j - 1, 0), np.maximum(k - 1, 0)
    corner = (i - fx) + 2 * (j - fy) + 4 * (k - fz)
    key = (fx + cx * (fy + cy * fz)) * 8 + corner
    order = np.argsort(key, kind="stable")
    V = order.size
    sample = (i + rx * (j + ry * k))[order]
    node_of = np.empty(rx * ry * rz, np.int64)
    node_of[sample] = np.arange(V)
    lattice = np.stack([i[order], j[order], k[order]], axis=1)
    u = splitmix_uniform(seed, 3 * V).reshape(V, 3)
    rest = (np.asarray(origin, np.float64) + voxel * lattice + (2.0 * u - 1.0) * jitter * voxel)
    rest = rest.astype(np.float32).astype(np.float64)
    anchored = np.zeros(V, np.uint8)
    if anchor_axis < 3:
        face = 0 if anchor_side == 0 else (cx, cy, cz)[anchor_axis]
        anchored[lattice[:, anchor_axis] == face] = 1
    # cells in x-fastest order, 8 corner nodes each
    gx, gy, gz = np.meshgrid(np.arange(cx), np.arange(cy), np.arange(cz), indexing="ij")
    cell_order = np.argsort((gx + cx * (gy + cy * gz)).ravel(), kind="stable")
    gx, gy, gz = gx.ravel()[cell_order], gy.ravel()[cell_order], gz.ravel()[cell_order]
    bits = np.arange(8)
    ci = gx[:, None] + (bits & 1)[None, :]
    cj = gy[:, None] + ((bits >> 1) & 1)[None, :]
    ck = gz[:, None] + ((bits >> 2) & 1)[None, :]
    corners = node_of[ci + rx * (cj + ry * ck)]               # [cells, 8]
    tets = corners[:, KUHN].reshape(-1, 4).copy()             # [6 cells, 4]
    def shape_of(t):
        x0 = rest[t[:, 0]]
        return np.stack([rest[t[:, 1]] - x0, rest[t[:, 2]] - x0, rest[t[:, 3]] - x0], axis=2)  # columns = edges
    shape = shape_of(tets)
    flip = np.linalg.det(shape) < 0.0
    tets[flip, 1], tets[flip, 2] = tets[flip, 2].copy(), tets[flip, 1].copy()
    shape = shape_of(tets)
    det = np.linalg.det(shape)
    keep = det / 6.0 > 0.0
    tets, shape, det = tets[keep], shape[keep], det[keep]
    volume = det / 6.0
    rest_inverse = np.linalg.inv(shape)
    mass = np.zeros(V)
    np.add.at(mass, tets.ravel(), np.repeat(density * volume * 0.25, 4))
    return PreparedMesh(
        rest_positions=rest, node_mass=mass, anchored=anchored, tet_nodes=tets.astype(np.uint32),
        rest_inverse=rest_inverse, volume=volume, material=np.full(tets.shape[0], lane, np.uint32),
        lattice=lattice.astype(np.int64), cells=(cx, cy, cz))
