"""GPU compute classes through the C ABI against direct sums of the fields:
Block_Data (Minimum / Maximum / Sum over a block, scalar and vector fields,
the reference's DBL_MIN start of Maximum), Kinetic_Energy and
Linear_Momentum (global and per point), the derived Force and Volume fields;
results bit-identical run to run. Sums to 1e-12 relative (summation order)."""
import sys

import numpy as np
import pytest

from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu


def _ctx(precision="fp64"):
    h = 1.0e-3
    x, vol = workloads.lattice(12, 9, 7, h, jitter=0.05, seed=2)
    n = len(vol)
    block = (x.reshape(-1, 3)[:, 0] > 6 * h).astype(np.int32) + (x.reshape(-1, 3)[:, 1] > 4 * h).astype(np.int32)
    rng = np.random.default_rng(4)
    vol = vol * (1.0 + 0.1 * rng.random(n))
    ctx = Context(precision=precision)
    ctx.set_points(x, vol, block)
    ctx.set_horizons([3.015 * h] * 3)
    ctx.build_bonds()
    for b, rho in enumerate((7800.0, 2700.0, 1200.0)):
        ctx.material(130.0e9, 78.0e9, rho, block=b)
    u = rng.normal(0.0, 1e-6, 3 * n)
    v = rng.normal(0.0, 1.0, 3 * n)
    ctx.set_state(u, v)
    return ctx, x, vol, block, np.array([7800.0, 2700.0, 1200.0])[block], u, v


def test_block_data_min_max_sum():
    ctx, x, vol, block, rho, u, v = _ctx()
    with ctx:
        f = ctx.compute_force(x + u)
        ctx.verlet_run(1e-9, 0)  # commit the state's force density
        fd = ctx.field("Force_Density")
        F = ctx.field("Force")
        u = ctx.field("Displacement")  # the state from y = x + u rounds u once
        assert np.allclose(F, fd * np.repeat(vol, 3), rtol=1e-15, atol=0)
        assert np.array_equal(ctx.field("Volume"), vol)
        for b in range(3):
            sel = block == b
            for field, arr in (("Velocity", v), ("Force", F), ("Displacement", u)):
                a = arr.reshape(-1, 3)[sel]
                got = ctx.block_data(field, b, "Sum")
                assert np.abs(got - a.sum(0)).max() <= 1e-12 * np.abs(a).sum()
                assert np.array_equal(ctx.block_data(field, b, "Minimum"), a.min(0))
                assert np.array_equal(ctx.block_data(field, b, "Maximum"), np.maximum(a.max(0), sys.float_info.min))
            got = ctx.block_data("Volume", b, "Sum")
            assert abs(got[0] - vol[sel].sum()) <= 1e-12 * vol[sel].sum() and got[1] == 0.0
            nn = ctx.field("Number_Of_Neighbors")
            assert ctx.block_data("Number_Of_Neighbors", b, "Maximum")[0] == nn[sel].max()
        # the reference's Maximum starts from DBL_MIN: a negative-only field reports DBL_MIN
        neg = -np.abs(v) - 1.0
        ctx.set_state(u, neg)
        assert np.all(ctx.block_data("Velocity", 0, "Maximum") == sys.float_info.min)
        with pytest.raises(Exception):
            ctx.block_data("Bond_Damage", 0, "Sum")
        with pytest.raises(Exception):
            ctx.block_data("Velocity", 7, "Sum")


def test_kinetic_energy_and_momentum():
    ctx, x, vol, block, rho, u, v = _ctx()
    with ctx:
        ke, ke_pp = ctx.kinetic_energy(per_point=True)
        lm, lm_pp = ctx.linear_momentum(per_point=True)
        ke2 = ctx.kinetic_energy()
    V = v.reshape(-1, 3)
    ref_pp = 0.5 * vol * rho * (V * V).sum(1)
    assert np.allclose(ke_pp, ref_pp, rtol=1e-15, atol=0)
    assert abs(ke - ref_pp.sum()) <= 1e-12 * ref_pp.sum()
    assert ke2 == ke  # fixed-order reductions
    mom = (rho * vol)[:, None] * V
    assert np.allclose(lm_pp.reshape(-1, 3), mom, rtol=1e-15, atol=0)
    assert np.abs(lm - mom.sum(0)).max() <= 1e-12 * np.abs(mom).sum()
