"""Stiffness damping in the oracle (factor.cc:755-855, solver.cc:625-902), CPU.

* The damping operator of one tet removes exactly the rigid motion fitted to
  its corners: a rigid translation or rotation about the centroid maps to zero,
  and the operator is symmetric positive semidefinite.
* In a step, damping dissipates: an oscillating block loses its kinetic energy
  far faster with stiffnessDamping > 0, and a negligible weight reproduces the
  undamped trajectory.
* The reference's FP32 arithmetic stays close to FP64 with damping on.
"""
import numpy as np

import talus_b200 as tb
from oracle import pyoracle as po
from tests.helpers import DT, GRAVITY, to_oracle


def _element():
    mesh = tb.box_mesh((1, 1, 1), voxel=0.1)
    rng = np.random.default_rng(0)
    t = mesh.tet_nodes[2]
    x = mesh.rest_positions[t] + 0.003 * rng.standard_normal((4, 3))
    rotation = po.rotation(po.F64, np.eye(3) + 0.01 * rng.standard_normal((3, 3)))
    return x, rotation, mesh.rest_inverse[2], mesh.volume[2], po.material(1000.0, 1e6, 0.3)


def _matrix(x, rotation, rinv, volume, mat):
    m = np.zeros((12, 12))
    for i in range(12):
        e = np.zeros(12)
        e[i] = 1.0
        m[:, i] = po.damping_apply(po.F64, x, rotation, rinv, volume, mat, e.reshape(4, 3)).ravel()
    return m


def test_damping_operator_removes_rigid_motion():
    x, rotation, rinv, volume, mat = _element()
    scale = np.abs(_matrix(x, rotation, rinv, volume, mat)).max()
    translation = np.tile([0.3, -0.2, 0.5], (4, 1))
    spin = np.cross(np.array([0.1, 0.4, -0.2]), x - x.mean(axis=0))
    for motion in (translation, spin):
        out = po.damping_apply(po.F64, x, rotation, rinv, volume, mat, motion)
        assert np.abs(out).max() <= 1e-12 * scale


def test_damping_operator_is_symmetric_positive_semidefinite():
    m = _matrix(*_element())
    scale = np.abs(m).max()
    assert np.abs(m - m.T).max() <= 1e-12 * scale
    assert np.linalg.eigvalsh(0.5 * (m + m.T)).min() >= -1e-12 * scale


def _run(tau, precision, steps=40):
    mesh = tb.box_mesh((6, 4, 4), voxel=0.1, jitter=0.01, seed=3)
    om = to_oracle(mesh)
    state = po.State.rest(om)
    mat = po.material(1000.0, 1e6, 0.3, tau)
    kinetic = []
    for _ in range(steps):
        kinetic.append(po.step(precision, om, state, [mat], po.Settings(), GRAVITY, DT).kinetic_energy)
    return mesh, state.position, np.array(kinetic)


def test_damping_dissipates_and_vanishes_with_its_weight():
    mesh, x0, k0 = _run(0.0, po.F64)
    _, x1, _ = _run(1e-12, po.F64)
    _, x2, k2 = _run(0.02, po.F64)
    scale = np.linalg.norm(x0 - mesh.rest_positions, axis=1).max()
    assert np.linalg.norm(x1 - x0, axis=1).max() <= 1e-8 * scale
    assert k2[-10:].mean() < 1e-6 * k0[-10:].mean()


def test_reference_precision_with_damping():
    mesh, x64, _ = _run(0.02, po.F64)
    _, x32, _ = _run(0.02, po.F32)
    scale = np.linalg.norm(x64 - mesh.rest_positions, axis=1).max()
    assert np.linalg.norm(x32 - x64, axis=1).max() <= 1e-3 * scale
