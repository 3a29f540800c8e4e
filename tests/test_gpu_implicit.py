"""Implicit dynamics on the GPU (pd_implicit_run, Peridigm::executeImplicit).

* The reference's CompressionImplicit_2x1x1 and CompressionImplicitEssentialBC_2x1x1
  gold output, step by step: displacement within the decks' .comp (1e-6
  absolute) and 1e-9 relative, velocity 1e-8 relative, Force_Density / density
  against the gold Acceleration (Compute_Acceleration) 1e-6 relative.
* A jittered 120-point lattice with a clamped face and a face moving at a
  prescribed rate, against the oracle's restatement (dense Newton solves):
  displacement, velocity and acceleration 1e-8 relative, with plain CG (the
  reference's) and block Jacobi.
Tolerances: Newton stops at ||beta dt^2 (rho a - f)|| <= tol, which bounds
the acceleration error by tol / (beta dt^2 rho); the CG solves differ from the
oracle's dense ones only within that."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")
K, MU, RHO, H, DT = 130.0e9, 78.0e9, 7800.0, 2.0, 1.0e-5


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("precond", ["none", "block_jacobi"])
@pytest.mark.parametrize("key", ["free", "essential"])
def test_implicit_gold_decks(key, precond):
    z = np.load(os.path.join(G, "compression_implicit.npz"))
    x = z[key + "_x"].ravel()
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, np.array([2.0, 2.0]))
        ctx.set_horizons([H])
        ctx.build_bonds()
        ctx.material(K, MU, RHO)
        u0 = z[key + "_Displacement"][0].ravel()
        if key == "essential":  # Prescribed Displacement 0.1 on the min-x point
            ctx.prescribed_displacement([0], 0, 0.0, 0.1)
        ctx.set_state(u0, z[key + "_Velocity"][0].ravel())
        for s in range(1, 6):
            st = ctx.implicit_run(DT, 1, t0=(s - 1) * DT, absolute_tolerance=1.0e-10, preconditioner=precond)
            assert st.newton_iterations >= 1
            u, v = ctx.field("Displacement"), ctx.field("Velocity")
            fd = ctx.field("Force_Density")
            gu = z[key + "_Displacement"][s].ravel()
            assert np.abs(u - gu).max() <= 1e-6
            assert rel(u, gu) <= 1e-9
            assert rel(v, z[key + "_Velocity"][s].ravel()) <= 1e-8
            assert rel(fd, z[key + "_Force_Density"][s].ravel()) <= 1e-6
            assert rel(fd / RHO, z[key + "_Acceleration"][s].ravel()) <= 1e-6


@pytest.mark.parametrize("precond", ["none", "block_jacobi"])
def test_implicit_lattice_matches_oracle(precond):
    h = 1.0e-3
    x, vol = workloads.lattice(6, 5, 4, h, jitter=0.05, seed=3)
    P = x.reshape(-1, 3)
    n = len(vol)
    row, col = O.neighbor_search(x, 3.015 * h)
    left = np.nonzero(P[:, 0] < P[:, 0].min() + 0.5 * h)[0]
    right = np.nonzero(P[:, 0] > P[:, 0].max() - 0.5 * h)[0]
    rate = 0.5  # m/s on the right face in x
    rng = np.random.default_rng(4)
    v0 = rng.normal(0.0, 0.05, 3 * n)
    u0 = np.zeros(3 * n)
    bc = sorted([3 * i + c for i in left for c in range(3)] + [3 * i for i in right])
    for i in left:
        v0[3 * i:3 * i + 3] = 0.0
    v0[3 * right] = rate
    dt, nsteps = 2.0e-7, 4
    ref = O.implicit_newmark(x, vol, row, col, K, MU, RHO, 3.015 * h, u0, v0, dt, nsteps, tol=1e-10, bc_dofs=bc)
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([3.015 * h])
        ctx.build_bonds()
        ctx.material(K, MU, RHO)
        for c in range(3):
            ctx.prescribed_displacement(left, c, 0.0, 0.0)
        ctx.prescribed_displacement(right, 0, rate, 0.0)
        ctx.set_state(u0, v0)
        for s in range(nsteps):
            st = ctx.implicit_run(dt, 1, t0=s * dt, absolute_tolerance=1e-10, preconditioner=precond)
            u, v, a = ctx.field("Displacement"), ctx.field("Velocity"), ctx.field("Acceleration")
            ru, rv, ra, _, _ = ref[s]
            assert rel(u, ru) <= 1e-8
            assert rel(v, rv) <= 1e-8
            assert rel(a, ra) <= 1e-8
        assert np.allclose(u[3 * right], rate * nsteps * dt, rtol=1e-12)
        assert np.all(u[[3 * i + c for i in left for c in range(3)]] == 0.0)
