"""Prescribed-displacement functions on the explicit path against the oracle.

The oracle takes the prescribed values as a table of f(x, y, z, t0 + k dt)
computed here in Python from the same formula, and applies them with the
reference's increment rule (DirichletIncrementBC,
src/core/Peridigm_BoundaryCondition.cpp:202-241, a zero increment taking the
previous value from the displacement field, :137-142).

* A lattice bar with a cosine ramp on one end (u_x), an if/else ramp on the
  other (u_x) and a coordinate-dependent shear (u_z): 40 steps in FP64 and
  split precision, u and v against the oracle (FP64 within 1e-9 of max, split
  1e-5).
* The zero-increment rule: points given a displacement by pd_set_state and a
  prescribed value that does not change (a constant function, and the
  closed form a = 0, b = const) go to that value in the first step, as in
  the oracle.
* A function that is not finite stops the run with PD_ERR_NONFINITE; the
  implicit solve refuses contexts with functions; the quasi-static solve with
  the cube's prescribed faces as functions equals its closed-form run.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import Context, PDError, workloads

pytestmark = pytest.mark.gpu

H = 1.0e-3


def _bar():
    x, vol = workloads.lattice(16, 6, 5, H, jitter=0.05, seed=7)
    P = x.reshape(-1, 3)
    left = np.flatnonzero(P[:, 0] < 2.5 * H)
    right = np.flatnonzero(P[:, 0] > P[:, 0].max() - 2.5 * H)
    return x, vol, left, right


F_LEFT = "-2.0e-5 * 0.5*(cos(3.14159265359 + t*3.14159265359/4.0e-6) + 1.0)"
F_RIGHT = "if (t <= 2.0e-6) { value = 1.0e-5*t/2.0e-6; } else { value = 1.0e-5; }"
F_SHEAR = "0.002*y*t/1.0e-6"


def _py_left(x, y, z, t):
    return -2.0e-5 * 0.5 * (math.cos(3.14159265359 + t * 3.14159265359 / 4.0e-6) + 1.0)


def _py_right(x, y, z, t):
    return 1.0e-5 * t / 2.0e-6 if t <= 2.0e-6 else 1.0e-5


def _py_shear(x, y, z, t):
    return 0.002 * y * t / 1.0e-6


def _table(x, nsteps, dt, specs):
    """bc_mask and the (nsteps+1) x 3n table of prescribed values."""
    n = x.size // 3
    P = x.reshape(-1, 3)
    mask = np.zeros(n, np.uint8)
    vals = np.zeros((nsteps + 1, 3 * n))
    for pts, c, f in specs:
        mask[pts] |= np.uint8(1 << c)
        for k in range(nsteps + 1):
            t = 0.0 + k * dt
            vals[k, 3 * pts + c] = [f(P[i, 0], P[i, 1], P[i, 2], t) for i in pts]
    return mask, vals


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_function_bcs_match_oracle(precision):
    x, vol, left, right = _bar()
    h = 3.015 * H
    row, col = O.neighbor_search(x, h)
    nsteps = 40
    with Context(precision=precision) as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds([])
        ctx.material(130e9, 78e9, 7800.0)
        ctx.prescribed_displacement_function(left, 0, F_LEFT)
        ctx.prescribed_displacement_function(right, 0, F_RIGHT)
        ctx.prescribed_displacement_function(right, 2, F_SHEAR)
        dt = 0.7 * ctx.critical_time_step()
        ctx.verlet_run(dt, nsteps)
        u, v = ctx.field("Displacement"), ctx.field("Velocity")
    mask, vals = _table(x, nsteps, dt, [(left, 0, _py_left), (right, 0, _py_right), (right, 2, _py_shear)])
    prob = dict(x=x, vol=vol, rho=7800.0, K=130e9, mu=78e9, row=row, col=col, horizon=h, dt=dt, nsteps=nsteps,
                bc_mask=mask, bc_a=np.zeros(x.size), bc_b=np.zeros(x.size), bc_vals=vals)
    ref = O.explicit_run(prob, np.zeros_like(x), np.zeros_like(x))
    tol = 1e-9 if precision == "fp64" else 1e-5
    assert np.abs(ref["u"]).max() > 1e-6
    assert np.abs(u - ref["u"]).max() <= tol * np.abs(ref["u"]).max()
    assert np.abs(v - ref["v"]).max() <= tol * np.abs(ref["v"]).max()
    # the prescribed dofs follow the functions: u(t_n) = f(t_n) up to rounding
    t_end = nsteps * dt
    P = x.reshape(-1, 3)
    want = np.array([_py_right(*P[i], t_end) for i in right])
    assert np.abs(u[3 * right] - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("kind", ["function", "closed_form"])
def test_zero_increment_takes_the_displacement_field(kind):
    """A prescribed value that does not change over a step: the step's
    increment is taken from the displacement field, so points displaced by
    pd_set_state go to the prescribed value in the first step."""
    x, vol, left, right = _bar()
    h = 3.015 * H
    row, col = O.neighbor_search(x, h)
    n = vol.size
    rng = np.random.default_rng(3)
    u0 = np.zeros(3 * n)
    u0[3 * left + 1] = rng.uniform(-1e-6, 1e-6, left.size)
    target = 2.0e-6
    nsteps = 10
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds([])
        ctx.material(130e9, 78e9, 7800.0)
        if kind == "function":
            ctx.prescribed_displacement_function(left, 1, "2.0e-6")
        else:
            ctx.prescribed_displacement(left, 1, 0.0, target)
        ctx.set_state(u0, np.zeros(3 * n))
        dt = 0.7 * ctx.critical_time_step()
        ctx.verlet_run(dt, nsteps)
        u = ctx.field("Displacement")
    mask = np.zeros(n, np.uint8)
    mask[left] = 2
    bc_b = np.zeros(3 * n)
    bc_b[3 * left + 1] = target
    prob = dict(x=x, vol=vol, rho=7800.0, K=130e9, mu=78e9, row=row, col=col, horizon=h, dt=dt, nsteps=nsteps,
                bc_mask=mask, bc_a=np.zeros(3 * n), bc_b=bc_b)
    ref = O.explicit_run(prob, u0, np.zeros(3 * n))
    assert np.abs(ref["u"][3 * left + 1] - target).max() <= 1e-18
    assert np.abs(u - ref["u"]).max() <= 1e-9 * np.abs(ref["u"]).max()


def test_nonfinite_function_and_qs_refusal():
    x, vol, left, right = _bar()
    h = 3.015 * H
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds([])
        ctx.material(130e9, 78e9, 7800.0)
        with pytest.raises(PDError) as e:
            ctx.prescribed_displacement_function(left, 0, "value = t +")
        assert e.value.code == 1
        ctx.prescribed_displacement_function(left, 0, "sqrt(-1.0 - t)")
        dt = 0.7 * ctx.critical_time_step()
        with pytest.raises(PDError) as e:
            ctx.verlet_run(dt, 2)
        assert e.value.code == 3  # PD_ERR_NONFINITE
        assert b"BC" in ctx.L.pd_last_error(ctx.h)
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds([])
        ctx.material(130e9, 78e9, 7800.0)
        ctx.prescribed_displacement_function(left, 0, "1.0e-6*t")
        with pytest.raises(PDError) as e:
            ctx.implicit_run(1.0e-6, 1)
        assert e.value.code == 6


def test_quasi_static_functions_match_closed_forms():
    """The quasi-static cube with its prescribed faces given as functions
    (the same ramps, and a constant written as a function) equals the run with
    the closed forms, increments included."""
    w = workloads.qs_cube(n=7, h=1.0e-3, seed=3, jitter=0.05, load_steps=3)
    res = []
    for as_function in (False, True):
        with Context(precision="fp64") as ctx:
            workloads.setup_context(ctx, w)
            if as_function:
                ctx.clear_boundary_conditions()
                for b in w["bcs"]:
                    ctx.prescribed_displacement_function(b["points"], b["coordinate"], f"{b['a']!r}*t + {b['b']!r}")
            for k in range(1, len(w["times"])):
                ctx.qs_load_step(w["times"][k - 1], w["times"][k], newton_tolerance=1e-6,
                                 cg_relative_tolerance=1e-10)
            res.append(ctx.field("Displacement"))
    assert np.abs(res[1]).max() > 1e-6
    assert np.abs(res[1] - res[0]).max() <= 1e-12 * np.abs(res[0]).max()
