"""pd_critical_time_step_static: the critical time step with no device
allocation, called through the C ABI and compared with pd_critical_time_step.

Tolerance: exact equality. Both entry points launch the same critical-dt
kernels over the same bonds; only where the block minima are kept differs, and
a minimum does not depend on reduction order.

The file is named to be collected last, so the static scratch is exercised
both in a fresh process (run alone) and after every other GPU test.
"""
import ctypes as C

import numpy as np
import pytest

from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu


def _static_dt(ctx):
    dt = C.c_double(-1.0)
    rc = ctx.L.pd_critical_time_step_static(ctx.h, C.byref(dt))
    assert rc == 0, ctx.L.pd_last_error(ctx.h).decode()
    return dt.value


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_static_matches_allocating_entry_twice(precision):
    w = workloads.notched_plate(nx=96, ny=48, nz=4, notch_cells=12)
    with Context(precision=precision) as ctx:
        workloads.setup_context(ctx, w)
        ref = ctx.critical_time_step()
        first = _static_dt(ctx)
        second = _static_dt(ctx)
    assert ref > 0.0
    assert first == ref
    assert second == ref


def test_static_shared_by_contexts_in_turn():
    """Two contexts on one device use the one static array one after the other."""
    a = workloads.notched_plate(nx=64, ny=32, nz=4, notch_cells=8)
    b = workloads.bar_wave(nx=60, ny=8, nz=8)
    with Context(precision="fp64") as ca, Context(precision="fp64") as cb:
        workloads.setup_context(ca, a)
        workloads.setup_context(cb, b)
        ra, rb = ca.critical_time_step(), cb.critical_time_step()
        assert ra != rb
        for _ in range(2):
            assert _static_dt(ca) == ra
            assert _static_dt(cb) == rb


def test_static_rejects_unset_context():
    x, vol = workloads.lattice(8, 8, 8, 1.0e-3)
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, vol)
        dt = C.c_double(-1.0)
        assert ctx.L.pd_critical_time_step_static(ctx.h, C.byref(dt)) == 5  # PD_ERR_STATE
        assert b"allocates nothing" in ctx.L.pd_last_error(ctx.h)
        assert ctx.L.pd_critical_time_step_static(ctx.h, None) == 1  # PD_ERR_ARG


def test_static_rejects_more_points_than_its_scratch_holds():
    # 1,064,960 points at 16 lanes per point need 66,560 block minima > 65,536.
    x, vol = workloads.lattice(128, 128, 65, 1.0e-3)
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, vol)
        dt = C.c_double(-1.0)
        assert ctx.L.pd_critical_time_step_static(ctx.h, C.byref(dt)) == 1  # PD_ERR_ARG
        msg = ctx.L.pd_last_error(ctx.h).decode()
        assert "65536" in msg and "pd_critical_time_step" in msg
        assert dt.value == -1.0
