"""talus_b200 -- B200-native deformable-body (tet FEM) step for Talus.

A drop-in for talus::deformable::step's tet path: element pass, deterministic
CSR vertex gather, persistent block-Jacobi PCG, all hand-written sm_100a
kernels in libtalus_fem.so behind the C ABI of include/talus_fem.h.
"""
from . import _capi
from .deformable import (COROTATED, FP32_MIXED, FP64, NEO_HOOKEAN, Context, DeformableState, PhysicalMaterial,
                         PreparedMesh, Settings, StepReport, System, rest_state, step)
from .mesh import box_mesh
from .rollout import Gradients, Rollout

__all__ = ["COROTATED", "FP32_MIXED", "FP64", "NEO_HOOKEAN", "Context", "DeformableState", "PhysicalMaterial",
           "PreparedMesh", "Settings", "StepReport", "System", "rest_state", "step", "box_mesh", "Rollout", "Gradients"]


def library():
    """The loaded CUDA library (raises if it is missing)."""
    return _capi.lib()
