"""The C ABI library (CPU checks: no compute calls).

* libtalus_fem.so loads and exports every entry point include/talus_fem.h declares;
* the ctypes mirror has the same struct layout as the C header (compiled here with gcc);
* calls that need no device work, and device calls fail with a status code
  (TL_ERR_NO_DEVICE) instead of crashing when there is no GPU.
"""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from talus_b200 import _capi as capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "talus_fem.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(tl_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(capi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(capi.SIGNATURES), set(names) ^ set(capi.SIGNATURES)


def test_struct_layout_matches_the_header():
    structs = {"tl_material": capi.tl_material, "tl_mesh_desc": capi.tl_mesh_desc,
               "tl_settings": capi.tl_settings, "tl_step_report": capi.tl_step_report,
               "tl_rollout_desc": capi.tl_rollout_desc, "tl_factor_stats": capi.tl_factor_stats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines.append("  return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-o", exe, src], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    table = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for name, cls in structs.items():
        assert table[(name, "size")] == C.sizeof(cls), name
        for field, _ in cls._fields_:
            assert table[(name, field)] == getattr(cls, field).offset, (name, field)


def test_python_constants_match_the_header():
    import re

    defines = dict(re.findall(r"#define (TL_[A-Z0-9_]+) (\d+)u?\b", open(HEADER).read()))
    named = {k: v for k, v in vars(capi).items() if k.startswith("TL_") and isinstance(v, int)}
    assert named, "no TL_ constants in the binding"
    for k, v in named.items():
        assert k in defines and int(defines[k]) == v, k


def test_header_compiles_as_c_and_cpp():
    with tempfile.TemporaryDirectory() as d:
        for comp, ext in (("gcc", "c"), ("g++", "cc")):
            src = os.path.join(d, f"h.{ext}")
            open(src, "w").write(f'#include "{HEADER}"\nint main(void) {{ return tl_abi_version() == 1 ? 0 : 1; }}\n')
            subprocess.run([comp, "-Wall", "-Werror", "-c", "-o", os.path.join(d, f"h{ext}.o"), src], check=True)


def test_calls_without_device_work():
    lib = capi.lib()
    assert lib.tl_abi_version() == 1
    assert lib.tl_status_string(capi.TL_ERR_NO_DEVICE) == b"no CUDA device"
    s = capi.tl_settings()
    lib.tl_settings_default(C.byref(s))
    # deformable::Settings defaults (solver.h:51-107)
    assert (s.substeps, s.cg_iterations, s.plastic_passes) == (1, 64, 40)
    assert s.tolerance == pytest.approx(1e-3) and s.spectral_radius == pytest.approx(0.5)
    assert s.rigid_split == capi.TL_RIGID_SPLIT_PROJECTED and s.law == capi.TL_LAW_COROTATED
    # argument checks return a status, never crash
    assert lib.tl_ctx_create(0, None) == capi.TL_ERR_ARG
    assert lib.tl_step(None, None, None, 0.0, None) == capi.TL_ERR_ARG
    assert lib.tl_state_get(None, 0, 0, None, None, None, None, None) == capi.TL_ERR_ARG
    assert lib.tl_system_destroy(None) == capi.TL_ERR_ARG
    assert lib.tl_system_set_youngs(None, 0, None) == capi.TL_ERR_ARG
    assert lib.tl_rollout_create(None, None, None, None) == capi.TL_ERR_ARG
    assert lib.tl_rollout_forward(None, None, None) == capi.TL_ERR_ARG
    assert lib.tl_rollout_adjoint(None, None, None, None, None, None, None) == capi.TL_ERR_ARG
    assert lib.tl_rollout_destroy(None) == capi.TL_ERR_ARG
    assert lib.tl_system_set_plasticity(None, capi.TL_PLASTICITY_HENCKY) == capi.TL_ERR_ARG
    assert lib.tl_system_set_flow_limits(None, 0, 0, 1e3, 0.5, 1.0) == capi.TL_ERR_ARG
    assert lib.tl_ctx_check_wait_limit(None) == capi.TL_ERR_ARG


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_context_without_a_device_reports_no_device():
    handle = C.c_void_p()
    assert capi.lib().tl_ctx_create(0, C.byref(handle)) == capi.TL_ERR_NO_DEVICE
    assert not handle.value


def test_product_package_does_not_use_the_oracle():
    """The oracle is test infrastructure only: no product source links, imports or loads it."""
    banned = ("pyoracle", "fem_oracle", "from oracle", "import oracle", "libfem_oracle")
    for dirpath, _, files in os.walk(os.path.join(ROOT, "talus_b200")):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cc", ".h")):
                text = open(os.path.join(dirpath, f)).read()
                assert not any(b in text for b in banned), f
