"""The oracle's prescribed-displacement handling (no device): the table form
(bc_vals, the prescribed values at t0 + k dt, used for functions of x, y, z,
t) against the closed form a t + b, and the zero-increment rule of
DirichletIncrementBC (src/core/Peridigm_BoundaryCondition.cpp:137-142): a
prescribed value that does not change over a step takes its previous value
from the displacement field, so a displaced point goes to the value in one
step. The same rule in the quasi-static restatement.
"""
import numpy as np

from oracle import oracle as O
from peridigm_b200 import workloads

H = 1.0e-3


def _bar():
    x, vol = workloads.lattice(10, 4, 4, H, jitter=0.05, seed=5)
    P = x.reshape(-1, 3)
    left = np.flatnonzero(P[:, 0] < 1.5 * H)
    right = np.flatnonzero(P[:, 0] > P[:, 0].max() - 1.5 * H)
    row, col = O.neighbor_search(x, 3.015 * H)
    return x, vol, left, right, row, col


def _prob(x, vol, row, col, dt, nsteps, mask, a, b, vals=None):
    return dict(x=x, vol=vol, rho=7800.0, K=130e9, mu=78e9, row=row, col=col, horizon=3.015 * H, dt=dt,
                nsteps=nsteps, bc_mask=mask, bc_a=a, bc_b=b, bc_vals=vals)


def test_table_equals_closed_form():
    x, vol, left, right, row, col = _bar()
    n = vol.size
    dt, nsteps = 1.0e-8, 25
    mask = np.zeros(n, np.uint8)
    mask[left] |= 1
    mask[right] |= 1
    a = np.zeros(3 * n)
    b = np.zeros(3 * n)
    a[3 * left] = -0.5
    a[3 * right] = 0.5
    vals = np.array([a * (0.0 + k * dt) + b for k in range(nsteps + 1)])
    u0 = np.zeros(3 * n)
    ref = O.explicit_run(_prob(x, vol, row, col, dt, nsteps, mask, a, b), u0, np.zeros(3 * n))
    tab = O.explicit_run(_prob(x, vol, row, col, dt, nsteps, mask, a, b, vals), u0, np.zeros(3 * n))
    assert np.abs(ref["u"]).max() > 0.0
    assert np.array_equal(tab["u"], ref["u"]) and np.array_equal(tab["v"], ref["v"])


def test_zero_increment_moves_to_the_value():
    x, vol, left, right, row, col = _bar()
    n = vol.size
    dt, nsteps = 1.0e-8, 5
    mask = np.zeros(n, np.uint8)
    mask[left] |= 2
    b = np.zeros(3 * n)
    b[3 * left + 1] = 3.0e-7
    u0 = np.zeros(3 * n)
    u0[3 * left + 1] = np.linspace(-1e-7, 1e-7, left.size)
    for vals in (None, np.tile(b, (nsteps + 1, 1))):
        out = O.explicit_run(_prob(x, vol, row, col, dt, nsteps, mask, np.zeros(3 * n), b, vals), u0, np.zeros(3 * n))
        assert np.abs(out["u"][3 * left + 1] - 3.0e-7).max() <= 1e-20


def test_quasi_static_constant_prescribed_value():
    x, vol, left, right, row, col = _bar()
    dofs = [(3 * int(i) + c, 0.0, 0.0) for i in left for c in range(3)] + [(3 * int(i), 0.0, 2.0e-7) for i in right]
    us = O.qs_solve(x, vol, row, col, 130e9, 78e9, 3.015 * H, dofs, [0.0, 0.5, 1.0], 1e-9)
    assert np.abs(us[1][3 * right] - 2.0e-7).max() <= 1e-20
    assert np.abs(us[2][3 * right] - 2.0e-7).max() <= 1e-20
    assert np.abs(us[1][3 * left]).max() == 0.0
