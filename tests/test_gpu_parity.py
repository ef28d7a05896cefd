"""Parity of the CUDA step (through the C ABI) with the CPU oracle.

Bars: FP64 GPU vs FP64 oracle <= 1e-9 relative displacement error (same
algorithm, different summation order and FMA contraction); FP32-mixed GPU vs
FP64 oracle <= 1e-5 (the FP32-mixed tolerance).  Error = max over nodes of
|x - x_oracle| / max over nodes of |x_oracle - X|, per step.
"""
import numpy as np
import pytest

import talus_b200 as tb
from oracle import pyoracle as po
from tests.helpers import elastic_block, plastic_block, relative_error, run_gpu, run_oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("law", [tb.NEO_HOOKEAN, tb.COROTATED])
def test_elastic_block_fp64_matches_oracle(law):
    mesh, mat = elastic_block()
    settings = tb.Settings(law=law)
    ref, oreps = [], []
    run_oracle(po.F64, mesh, mat, settings, 12, record=ref)
    got = []
    _, greps = run_gpu(tb.FP64, mesh, mat, settings, 12, record=got)
    for step, (x, r) in enumerate(zip(got, ref)):
        err = relative_error(x, r, mesh.rest_positions)
        assert err <= 1e-9, (step, err)


@pytest.mark.parametrize("law", [tb.NEO_HOOKEAN, tb.COROTATED])
def test_elastic_block_mixed_within_tolerance(law):
    mesh, mat = elastic_block()
    settings = tb.Settings(law=law)
    ref, got = [], []
    run_oracle(po.F64, mesh, mat, settings, 60, record=ref)
    run_gpu(tb.FP32_MIXED, mesh, mat, settings, 60, record=got)
    worst = max(relative_error(x, r, mesh.rest_positions) for x, r in zip(got, ref))
    assert worst <= 1e-5, worst


def test_plastic_block_fp64_matches_oracle():
    mesh, mat = plastic_block()
    settings = tb.Settings()
    ref, got = [], []
    ostate, oreps = run_oracle(po.F64, mesh, mat, settings, 10, record=ref)
    gstate, greps = run_gpu(tb.FP64, mesh, mat, settings, 10, record=got)
    for step, (x, r) in enumerate(zip(got, ref)):
        err = relative_error(x, r, mesh.rest_positions)
        assert err <= 1e-8, (step, err)
    assert np.abs(gstate.plastic - ostate.plastic).max() <= 1e-8 * max(1.0, np.abs(ostate.plastic).max())
    assert [r["plastic_evaluations"] for r in greps] == [r["plastic_evaluations"] for r in oreps]


def test_plastic_block_mixed_within_tolerance():
    mesh, mat = plastic_block()
    settings = tb.Settings()
    ref, got = [], []
    run_oracle(po.F64, mesh, mat, settings, 10, record=ref)
    run_gpu(tb.FP32_MIXED, mesh, mat, settings, 10, record=got)
    worst = max(relative_error(x, r, mesh.rest_positions) for x, r in zip(got, ref))
    assert worst <= 1e-5, worst
