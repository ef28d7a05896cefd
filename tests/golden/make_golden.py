"""Writes the golden fixtures of this directory from the oracle.

The reference cannot be compiled here (it fetches GLM, Eigen and Catch2 at
configure time, CMakeLists.txt:16-39) and none of its tests drives the tet
step, so no fixture comes from the reference itself.  These arrays are the
FP64 oracle's results (oracle/fem_oracle.cc, a restatement of
deformable/solver/solver.cc and deformable/material/material.cc), with the
oracle pinned by the law tests in tests/test_oracle_laws.py.  They freeze the
oracle against later edits (tests/test_golden.py re-runs it) and give the GPU
tests expected values that need no CPU solve (tests/test_gpu_golden.py).

Each block fixture stores how its mesh is generated (talus_b200.box_mesh) and
a checksum of the generated mesh, the positions after the first and the last
step, and the step reports the GPU path must reproduce.  hencky_block.npz is
the plastic block in the finite-strain plasticity mode (plasticflow.cc), with
its hardening variables and a sample of its plastic maps.  tet_laws.npz holds
48 disconnected tets at seeded deformations (stretched, sheared, rotated,
three inverted) with each law's element forces.

full_plastic_block.npz is the plastic benchmark block at its full size
(393,216 tets) after two FP64 oracle steps: a sample of its node positions,
sums over all nodes and the step counts.

Run from the repository root:  python -m tests.golden.make_golden [name]
"""
from __future__ import annotations

import os

import numpy as np

import talus_b200 as tb
from oracle import pyoracle as po
from tests.helpers import elastic_block, oracle_material, plastic_block, run_oracle

HERE = os.path.dirname(os.path.abspath(__file__))


def mesh_checksum(mesh: tb.PreparedMesh) -> np.ndarray:
    """Sums that change when the generator's nodes, tets or rest shapes do."""
    order = np.arange(1, mesh.tets + 1, dtype=np.float64)
    return np.array([mesh.rest_positions.sum(), np.abs(mesh.rest_positions).sum(),
                     float(mesh.tet_nodes.astype(np.float64).ravel() @ np.tile(order, 4)),
                     mesh.rest_inverse.sum(), np.abs(mesh.rest_inverse).sum(), mesh.volume.sum(),
                     float(mesh.anchored.sum())])


def material_array(m: tb.PhysicalMaterial) -> np.ndarray:
    return np.array([m.density, m.youngs_modulus, m.poissons_ratio, m.stiffness_damping, m.yield_stress,
                     m.hardening_modulus])


def material_of(a) -> tb.PhysicalMaterial:
    return tb.PhysicalMaterial(*(float(x) for x in a))


BLOCKS = {
    # name: (mesh builder, builder arguments, law, stiffness damping, steps)
    "elastic_block_corotated": ("elastic", dict(cells=(8, 8, 8), jitter=0.01, seed=1), tb.COROTATED, 0.0, 12),
    "elastic_block_snh": ("elastic", dict(cells=(8, 8, 8), jitter=0.01, seed=1), tb.NEO_HOOKEAN, 0.0, 12),
    "damped_block": ("elastic", dict(cells=(8, 8, 8), jitter=0.01, seed=1), tb.COROTATED, 0.02, 12),
    "plastic_block": ("plastic", dict(cells=(16, 8, 8), seed=2, speed=0.5), tb.COROTATED, 0.0, 10),
}


def block_case(name):
    kind, args, law, damping, steps = BLOCKS[name]
    mesh, mat = (elastic_block if kind == "elastic" else plastic_block)(**args)
    mat.stiffness_damping = damping
    return mesh, mat, tb.Settings(law=law), steps


def write_block(name):
    mesh, mat, settings, steps = block_case(name)
    record = []
    state, reports = run_oracle(po.F64, mesh, mat, settings, steps, record=record)
    record32 = []
    run_oracle(po.F32, mesh, mat, settings, steps, record=record32)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        mesh_checksum=mesh_checksum(mesh), material=material_array(mat), law=settings.law, steps=steps,
        first=record[0], last=record[-1], last_fp32=record32[-1],
        equivalent=state.plastic[:, 9],
        cg_iterations=np.array([r["cg_iterations"] for r in reports]),
        plastic_evaluations=np.array([r["plastic_evaluations"] for r in reports]))


# The plastic block in the finite-strain (Hencky) plasticity mode, P = I at rest.
HENCKY_BLOCK = dict(cells=(16, 8, 8), seed=2, speed=0.5)
HENCKY_STEPS = 8
HENCKY_SAMPLE = 16  # every 16th tet's plastic map is stored


def hencky_case():
    mesh, mat = plastic_block(**HENCKY_BLOCK)
    return mesh, mat, tb.Settings(), HENCKY_STEPS


def write_hencky_block():
    mesh, mat, settings, steps = hencky_case()
    record = []
    state, reports = run_oracle(po.F64, mesh, mat, settings, steps, record=record, plasticity=po.PLASTICITY_HENCKY)
    np.savez_compressed(
        os.path.join(HERE, "hencky_block.npz"),
        mesh_checksum=mesh_checksum(mesh), material=material_array(mat), steps=steps,
        first=record[0], last=record[-1], hardening=state.plastic[:, 9],
        plastic_map_sample=state.plastic[::HENCKY_SAMPLE, :9],
        flowed=np.array([r["yielding"] for r in reports]),
        cg_iterations=np.array([r["cg_iterations"] for r in reports]))


def single_tets(count=48, seed=11):
    """`count` tets cut from a jittered Kuhn lattice, each with its own four
    nodes, and a seeded deformation gradient per tet."""
    base = tb.box_mesh((2, 2, 2), voxel=0.1, jitter=0.01, seed=seed)
    rng = np.random.default_rng(seed)
    pick = np.arange(count) % base.tets
    corners = base.tet_nodes[pick]
    rest = base.rest_positions[corners]                          # [count,4,3]
    grads = []
    for e in range(count):
        scale = (0.001, 0.01, 0.05, 0.2)[e % 4]
        f = np.eye(3) + scale * rng.standard_normal((3, 3))
        if e % 8 == 5:                                           # a rigid turn on top
            q = np.linalg.qr(rng.standard_normal((3, 3)))[0]
            f = (q if np.linalg.det(q) > 0 else -q) @ f
        if e in (7, 23, 39):                                     # inverted: one axis flipped through zero
            f = f @ np.diag([1.0, 1.0, -0.3])
        grads.append(f)
    grads = np.array(grads)
    centroid = rest.mean(axis=1, keepdims=True)
    deformed = centroid + np.einsum("eij,ekj->eki", grads, rest - centroid)
    return rest, base.rest_inverse[pick], base.volume[pick], deformed


LAW_MATERIALS = {
    "elastic": tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3),
    "plastic": tb.PhysicalMaterial(density=1000.0, youngs_modulus=2e7, poissons_ratio=0.35, yield_stress=1e5,
                                   hardening_modulus=2e5),
}


def write_tet_laws():
    rest, rinv, volume, deformed = single_tets()
    count = rest.shape[0]
    el = oracle_material(LAW_MATERIALS["elastic"])
    pl = oracle_material(LAW_MATERIALS["plastic"])
    out = {k: np.zeros((count, 4, 3)) for k in ("corotated_force", "snh_force", "plastic_force")}
    plastic_point = np.zeros((count, 10))
    yielding = np.zeros(count, np.uint8)
    for e in range(count):
        args = (deformed[e], rest[e], rinv[e], volume[e])
        out["corotated_force"][e] = po.tet_trial(po.F64, *args, el)["force"]
        out["snh_force"][e] = po.snh_tet(po.F64, *args, el)["force"]
        p = po.tet_point_trial(po.F64, *args, pl, tangent=False)
        out["plastic_force"][e] = p["force"]
        plastic_point[e] = p["plastic"]
        yielding[e] = p["yielding"]
    np.savez_compressed(os.path.join(HERE, "tet_laws.npz"), rest=rest, rest_inverse=rinv, volume=volume,
                        deformed=deformed, elastic=material_array(LAW_MATERIALS["elastic"]),
                        plastic=material_array(LAW_MATERIALS["plastic"]), plastic_point=plastic_point,
                        yielding=yielding, **out)


# The plastic benchmark block at its full size (64x32x32 cubes, 393,216 tets,
# 70,785 nodes), two FP64 oracle steps from rest.  The oracle needs one to two
# minutes per step there (17 and 33 Newton evaluations in these first steps),
# so the result is stored instead of recomputed in the GPU test: every
# FULL_SAMPLE-th node's position, and sums over all nodes.
FULL_STEPS = 2
FULL_SAMPLE = 8


def full_block_case():
    from talus_b200.workloads import WORKLOADS, make_mesh

    mesh, mat = make_mesh(WORKLOADS["plastic-block"])
    return mesh, mat, tb.Settings(), FULL_STEPS


def position_sums(x, rest):
    """Sums over every node that a wrong node anywhere would change."""
    d = x - rest
    return np.array([d.sum(), np.abs(d).sum(), (d * d).sum(), np.linalg.norm(d, axis=1).max()])


def write_full_block():
    mesh, mat, settings, steps = full_block_case()
    record = []
    state, reports = run_oracle(po.F64, mesh, mat, settings, steps, record=record)
    np.savez_compressed(
        os.path.join(HERE, "full_plastic_block.npz"),
        mesh_checksum=mesh_checksum(mesh), material=material_array(mat), steps=steps, sample=FULL_SAMPLE,
        positions=np.array([r[::FULL_SAMPLE] for r in record]),
        sums=np.array([position_sums(r, mesh.rest_positions) for r in record]),
        equivalent_sum=float(state.plastic[:, 9].sum()),
        yielded=int((state.plastic[:, 9] > 0).sum()),
        cg_iterations=np.array([r["cg_iterations"] for r in reports]),
        plastic_evaluations=np.array([r["plastic_evaluations"] for r in reports]),
        plastic_solves=np.array([r["plastic_solves"] for r in reports]))


def main(which=None):
    for name in BLOCKS:
        if which in (None, name):
            write_block(name)
    if which in (None, "hencky_block"):
        write_hencky_block()
    if which in (None, "tet_laws"):
        write_tet_laws()
    if which in (None, "full_plastic_block"):
        write_full_block()


if __name__ == "__main__":
    import sys

    main(sys.argv[1] if len(sys.argv) > 1 else None)
