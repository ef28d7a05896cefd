"""Failure detection on the GPU without a GPU fault.

Every spin in the persistent kernels is bounded (2 s on the grid barrier);
when it runs out the kernel records TL_ERR_TIMEOUT in a status word the host
reads, and the context stays usable.  tl_ctx_check_wait_limit makes that wait
run out: one block waits at the barrier for an arrival that never comes.
Afterwards the same context steps a body normally.  The host-side failure
paths (a rank that raises, never joins) are covered with gloo ranks in
test_shard.
"""
import ctypes as C
import time

import numpy as np
import pytest

import talus_b200 as tb
from talus_b200 import _capi as capi
from tests.helpers import DT, GRAVITY, elastic_block

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_with_a_status_and_the_context_stays_usable():
    ctx = tb.Context(0)
    began = time.perf_counter()
    rc = capi.lib().tl_ctx_check_wait_limit(ctx.handle)
    waited = time.perf_counter() - began
    assert rc == capi.TL_ERR_TIMEOUT
    assert 1.5 < waited < 30.0
    assert b"bounded wait" in capi.lib().tl_ctx_last_error(ctx.handle)
    mesh, mat = elastic_block((4, 4, 4), seed=6)
    system = tb.System(mesh, [mat], tb.FP64, context=ctx)
    system.set_state(tb.rest_state(mesh))
    report = system.step(tb.Settings(), GRAVITY, DT)[0]
    assert report.cg_iterations > 0
    assert np.isfinite(system.get_state().position).all()
    system.close()
    ctx.close()


@pytest.mark.parametrize("solve", [0, 1])
def test_a_wait_that_runs_out_in_an_early_solve_is_reported_at_the_step_end(solve):
    """The elastic step runs three PCG solves.  When the barrier wait of an
    early one runs out, the later solves of the same step must not erase the
    record: the step returns TL_ERR_TIMEOUT.  The next step runs normally."""
    mesh, mat = elastic_block((4, 4, 4), seed=6)
    system = tb.System(mesh, [mat], tb.FP64)
    system.set_state(tb.rest_state(mesh))
    assert capi.lib().tl_system_expire_wait(system.handle, solve) == capi.TL_OK
    reports = (tb.StepReport * 1)()
    g = np.asarray(GRAVITY, np.float64)
    rc = capi.lib().tl_step(system.handle, C.byref(tb.Settings()._c()), g.ctypes.data, DT, reports)
    assert rc == capi.TL_ERR_TIMEOUT
    system.set_state(tb.rest_state(mesh))
    report = system.step(tb.Settings(), GRAVITY, DT)[0]
    assert report.cg_iterations > 0
    assert np.isfinite(system.get_state().position).all()
    system.close()


@pytest.mark.parametrize("solve", [0, 2])
def test_factored_solve_reports_an_expired_wait(solve):
    """The same host-armed expiry on a system with a solver state: the
    factored PCG (kPcgFactor, whose grid barriers and supernode waits are
    bounded the same way) leaves at its first barrier, the step returns
    TL_ERR_TIMEOUT, and the next step runs normally with the factor."""
    mesh, mat = elastic_block((4, 4, 4), seed=6)
    system = tb.System(mesh, [mat], tb.FP64)
    system.use_factor(True, 32)
    system.set_state(tb.rest_state(mesh))
    system.step(tb.Settings(), GRAVITY, DT)
    assert capi.lib().tl_system_expire_wait(system.handle, solve) == capi.TL_OK
    reports = (tb.StepReport * 1)()
    g = np.asarray(GRAVITY, np.float64)
    rc = capi.lib().tl_step(system.handle, C.byref(tb.Settings()._c()), g.ctypes.data, DT, reports)
    assert rc == capi.TL_ERR_TIMEOUT
    system.set_state(tb.rest_state(mesh))
    report = system.step(tb.Settings(), GRAVITY, DT)[0]
    assert report.cg_iterations > 0
    assert np.isfinite(system.get_state().position).all()
    assert system.factor_stats()["ready"] == 1
    system.close()
