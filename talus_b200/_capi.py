"""ctypes binding of include/talus_fem.h (libtalus_fem.so, built in-tree).

The library is the product: hand-written sm_100a kernels behind a C ABI.
Loading fails loudly when the shared object is missing; there is no CPU
fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtalus_fem.so")

TL_OK = 0
TL_ERR_ARG = 1
TL_ERR_CUDA = 2
TL_ERR_NOT_CONVERGED = 3
TL_ERR_NONFINITE = 4
TL_ERR_TIMEOUT = 5
TL_ERR_UNSUPPORTED = 6
TL_ERR_NO_DEVICE = 7
TL_ERR_TOO_LARGE = 8

TL_FP64 = 0
TL_FP32_MIXED = 1
TL_LAW_COROTATED = 0
TL_LAW_SNH = 1
TL_DTYPE_F32 = 0
TL_DTYPE_F64 = 1
TL_RIGID_SPLIT_OFF = 0
TL_RIGID_SPLIT_UNPROJECTED = 1
TL_RIGID_SPLIT_PROJECTED = 2
TL_FLAG_PROFILE = 1
TL_FLAG_TRACE = 2
TL_SOLVER_AUTO = 0
TL_SOLVER_ASSEMBLED = 1
TL_SOLVER_ELEMENTWISE = 2
TL_SOLVER_ASSEMBLED_TWO_PHASE = 3
TL_SOLVER_ASSEMBLED_PIPELINED = 4
TL_SHAPE_ROW_GROUP = 0
TL_SHAPE_BATCH_BLOCKS = 1
TL_PLASTICITY_SMALL_STRAIN = 0
TL_PLASTICITY_HENCKY = 1


class tl_material(C.Structure):
    _fields_ = [
        ("density", C.c_double),
        ("youngs_modulus", C.c_double),
        ("poissons_ratio", C.c_double),
        ("stiffness_damping", C.c_double),
        ("yield_stress", C.c_double),
        ("hardening_modulus", C.c_double),
    ]


class tl_mesh_desc(C.Structure):
    _fields_ = [
        ("nodes", C.c_uint32),
        ("tets", C.c_uint32),
        ("rest_positions", C.c_void_p),
        ("node_mass", C.c_void_p),
        ("anchored", C.c_void_p),
        ("tet_nodes", C.c_void_p),
        ("rest_inverse", C.c_void_p),
        ("volume", C.c_void_p),
        ("material", C.c_void_p),
        ("materials", C.POINTER(tl_material)),
        ("lanes", C.c_uint32),
        ("element_youngs", C.c_void_p),
        ("prescribed_velocity", C.c_void_p),
    ]


class tl_settings(C.Structure):
    _fields_ = [
        ("substeps", C.c_uint32),
        ("cg_iterations", C.c_uint32),
        ("plastic_passes", C.c_uint32),
        ("rigid_split", C.c_uint32),
        ("law", C.c_uint32),
        ("flags", C.c_uint32),
        ("tolerance", C.c_double),
        ("spectral_radius", C.c_double),
    ]


class tl_step_report(C.Structure):
    _fields_ = [
        ("nodes", C.c_uint32),
        ("elements", C.c_uint32),
        ("substeps", C.c_uint32),
        ("cg_iterations", C.c_uint32),
        ("cg_capped_solves", C.c_uint32),
        ("plastic_evaluations", C.c_uint32),
        ("plastic_solves", C.c_uint32),
        ("plastic_backtracks", C.c_uint32),
        ("plastic_capped", C.c_uint32),
        ("plastic_linear_reads", C.c_uint32),
        ("plastic_handoffs", C.c_uint32),
        ("plastic_fallbacks", C.c_uint32),
        ("plastic_fallback_rejections", C.c_uint32),
        ("operator_applications", C.c_uint32),
        ("yielding", C.c_uint32),
        ("plastic_growth", C.c_uint32),
        ("non_finite", C.c_uint32),
        ("kernel_launches", C.c_uint32),
        ("cg_tangent_iterations", C.c_uint32),
        ("cg_solves", C.c_uint32),
        ("cg_worst_relative_residual", C.c_double),
        ("plastic_worst_residual", C.c_double),
        ("elastic_energy", C.c_double),
        ("kinetic_energy", C.c_double),
        ("min_volume_ratio", C.c_double),
        ("device_seconds", C.c_double),
        ("element_seconds", C.c_double),
        ("assemble_seconds", C.c_double),
        ("pcg_seconds", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class tl_factor_stats(C.Structure):
    """SolverStats (factor.h:28-38), the SystemFactor's size and the
    StepReport factor counters of a system's solver state."""
    _fields_ = [(n, C.c_uint32) for n in ("factor_age", "refactor_count", "retry_count", "substeps_since_refresh",
                                          "refresh_requested", "fresh_retry_failed")] + \
               [("mean_iterations", C.c_double), ("rows", C.c_uint32), ("ready", C.c_uint32),
                ("system_nonzeros", C.c_uint64), ("generation", C.c_uint64)] + \
               [(n, C.c_uint32) for n in ("refresh_requests", "refactors", "retries", "retries_failed",
                                          "wasted_iterations", "spent_before_refresh", "spent_after_refresh",
                                          "refreshed_at_age", "factor_applications", "reserved")] + \
               [("factor_nonzeros", C.c_uint64), ("refactor_seconds", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class tl_rollout_desc(C.Structure):
    _fields_ = [
        ("steps", C.c_uint32),
        ("checkpoint_every", C.c_uint32),
        ("newton_reads", C.c_uint32),
        ("pad", C.c_uint32),
        ("delta_time", C.c_double),
        ("gravity", C.c_double * 3),
    ]


# Every entry point of include/talus_fem.h: name -> (restype, argtypes).
SIGNATURES = {
    "tl_abi_version": (C.c_int32, []),
    "tl_status_string": (C.c_char_p, [C.c_int32]),
    "tl_ctx_create": (C.c_int32, [C.c_int32, C.POINTER(C.c_void_p)]),
    "tl_ctx_destroy": (C.c_int32, [C.c_void_p]),
    "tl_ctx_last_error": (C.c_char_p, [C.c_void_p]),
    "tl_system_create": (C.c_int32, [C.c_void_p, C.POINTER(tl_mesh_desc), C.c_uint32, C.c_int32,
                                     C.POINTER(C.c_void_p)]),
    "tl_system_destroy": (C.c_int32, [C.c_void_p]),
    "tl_system_counts": (C.c_int32, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_uint64)]),
    "tl_system_trace": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    "tl_step_substeps": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                     C.POINTER(C.c_uint32)]),
    "tl_system_tune": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "tl_system_tune_shape": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "tl_host_register": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "tl_host_unregister": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "tl_system_set_solver": (C.c_int32, [C.c_void_p, C.c_uint32]),
    "tl_system_use_factor": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "tl_system_factor_stats": (C.c_int32, [C.c_void_p, C.POINTER(tl_factor_stats)]),
    "tl_system_set_plasticity": (C.c_int32, [C.c_void_p, C.c_uint32]),
    "tl_ctx_check_wait_limit": (C.c_int32, [C.c_void_p]),
    "tl_system_expire_wait": (C.c_int32, [C.c_void_p, C.c_int32]),
    "tl_system_set_flow_limits": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_double, C.c_double,
                                              C.c_double]),
    "tl_state_set": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_int32] + [C.c_void_p] * 5),
    "tl_state_get": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_int32] + [C.c_void_p] * 5),
    "tl_step": (C.c_int32, [C.c_void_p, C.POINTER(tl_settings), C.c_void_p, C.c_double,
                            C.POINTER(tl_step_report)]),
    "tl_step_host": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_int32] + [C.c_void_p] * 5 +
                     [C.POINTER(tl_settings), C.c_void_p, C.c_double, C.POINTER(tl_step_report)]),
    "tl_settings_default": (None, [C.POINTER(tl_settings)]),
    "tl_system_set_youngs": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "tl_evaluate": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(tl_settings), C.c_void_p, C.c_void_p]),
    "tl_rollout_create": (C.c_int32, [C.c_void_p, C.POINTER(tl_rollout_desc), C.POINTER(tl_settings),
                                      C.POINTER(C.c_void_p)]),
    "tl_rollout_destroy": (C.c_int32, [C.c_void_p]),
    "tl_rollout_forward": (C.c_int32, [C.c_void_p, C.POINTER(tl_step_report), C.POINTER(C.c_double)]),
    "tl_rollout_adjoint": (C.c_int32, [C.c_void_p] + [C.c_void_p] * 5 + [C.POINTER(C.c_double)]),
    "tl_step_noalloc": (C.c_int32, [C.c_int32, C.POINTER(tl_mesh_desc), C.c_int32] + [C.c_void_p] * 5 +
                        [C.POINTER(tl_settings), C.c_void_p, C.c_double, C.POINTER(tl_step_report)]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libtalus_fem.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"talus_b200: CUDA extension missing ({LIB_PATH}); build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'`")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class TalusError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        text = lib().tl_status_string(status).decode()
        super().__init__(f"{text} ({status})" + (f": {detail}" if detail else ""))


def check(status: int, ctx=None) -> int:
    if status != TL_OK:
        detail = lib().tl_ctx_last_error(ctx).decode() if ctx else ""
        raise TalusError(status, detail)
    return status
