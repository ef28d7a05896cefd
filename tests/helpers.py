"""Shared fixtures: synthetic meshes of the benchmark shapes and the oracle
bridge.  The oracle (oracle/) is what the CUDA path is compared with, never the thing tested."""
from __future__ import annotations

import numpy as np

import talus_b200 as tb
from oracle import pyoracle as po

GRAVITY = (0.0, -9.81, 0.0)
DT = 1.0 / 60.0


def to_oracle(mesh: tb.PreparedMesh) -> po.Mesh:
    return po.Mesh(mesh.rest_positions, mesh.node_mass, mesh.anchored, mesh.tet_nodes, mesh.rest_inverse, mesh.volume,
                   mesh.material, element_youngs=mesh.element_youngs, prescribed=mesh.prescribed_velocity)


def oracle_material(m: tb.PhysicalMaterial) -> po.Material:
    return po.material(m.density, m.youngs_modulus, m.poissons_ratio, m.stiffness_damping, m.yield_stress,
                       m.hardening_modulus, m.crush_stress, m.crush_limit, m.plastic_max)


def oracle_settings(s: tb.Settings) -> po.Settings:
    return po.Settings(s.substeps, s.cg_iterations, s.plastic_passes, s.law, s.tolerance, s.spectral_radius,
                       s.rigid_split)


def elastic_block(cells=(8, 8, 8), jitter=0.01, seed=1):
    """The elastic benchmark block: 8x8x8 cubes of 0.1 m, E=1e6, nu=0.3, rho=1000, bottom (y=0) pinned."""
    mesh = tb.box_mesh(cells, voxel=0.1, jitter=jitter, seed=seed)
    return mesh, tb.PhysicalMaterial(density=1000.0, youngs_modulus=1e6, poissons_ratio=0.3)


def plastic_block(cells=(16, 8, 8), seed=2, speed=0.5):
    """The plastic benchmark block at reduced size: E=2e7, nu=0.35, yield 1e5, H=2e5; bottom
    pinned, top face pushed down at `speed` m/s."""
    mesh = tb.box_mesh(cells, voxel=0.1, jitter=0.0, seed=seed)
    top = mesh.face(1, 1)
    mesh.anchored[top] = 1
    mesh.prescribed_velocity = np.zeros((mesh.nodes, 3))
    mesh.prescribed_velocity[top, 1] = -speed
    mat = tb.PhysicalMaterial(density=1000.0, youngs_modulus=2e7, poissons_ratio=0.35, yield_stress=1e5,
                              hardening_modulus=2e5)
    return mesh, mat


def run_oracle(precision, mesh, mat, settings, steps, record=None, plasticity=po.PLASTICITY_SMALL_STRAIN):
    om = to_oracle(mesh)
    state = po.State.rest(om, hencky=plasticity == po.PLASTICITY_HENCKY)
    osettings = oracle_settings(settings)
    osettings.plasticity = plasticity
    reports = []
    for i in range(steps):
        rep = po.step(precision, om, state, [oracle_material(mat)], osettings, GRAVITY, DT)
        reports.append(rep.as_dict())
        if record is not None:
            record.append(state.position.copy())
    return state, reports


def run_gpu(precision, mesh, mat, settings, steps, record=None):
    system = tb.System(mesh, [mat], precision)
    system.set_state(tb.rest_state(mesh))
    reports = []
    for i in range(steps):
        rep = system.step(settings, GRAVITY, DT)[0]
        reports.append(rep.as_dict())
        if record is not None:
            record.append(system.get_state().position)
    state = system.get_state()
    system.close()
    return state, reports


def relative_error(x, ref, rest):
    """max_n |x_n - ref_n| / max_n |ref_n - X_n| (the relative displacement error the 1e-5 bar is stated in)."""
    scale = np.linalg.norm(ref - rest, axis=1).max()
    return float(np.linalg.norm(x - ref, axis=1).max() / max(scale, 1e-300))
