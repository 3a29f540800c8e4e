"""GPU quasi-static Newton / CG against the oracle and the reference's gold file.

* matrix-free tangent (pd_jacobian_apply) vs the oracle's dense tangent
  built from its linearization: relative error <= 1e-11;
* 3x3 diagonal blocks vs the dense tangent's diagonal: <= 1e-11 of the max;
* Compression_QS_3x2x2 gold: displacement 1e-9 absolute, velocity 5e-8,
  force density 1.0 (Compression_QS_3x2x2.comp);
* a jittered cube: block-Jacobi CG, plain CG and the oracle's dense Newton
  agree on the displacement to 1e-8 relative, and block-Jacobi needs fewer
  CG iterations than plain CG.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")


def _cube_ctx(n=6, precision="fp64", seed=3):
    w = workloads.qs_cube(n=n, h=1.0e-3, seed=seed, jitter=0.05, load_steps=4)
    ctx = Context(precision=precision)
    workloads.setup_context(ctx, w)
    return w, ctx


def _bc_dofs(w):
    dofs = set()
    for bc in w["bcs"]:
        dofs |= {3 * int(p) + bc["coordinate"] for p in bc["points"]}
    return sorted(dofs)


def test_jacobian_apply_and_blocks_match_oracle():
    w, ctx = _cube_ctx(n=5)
    with ctx:
        rng = np.random.default_rng(1)
        u = rng.normal(0, 1e-6, w["x"].size)
        vec = rng.normal(0, 1.0, w["x"].size)
        kw = ctx.jacobian_apply(u, vec)
        blocks = ctx.jacobian_blocks(u)
        row, col = ctx.bonds_csr()
    dofs = _bc_dofs(w)
    T = O.tangent_dense(w["x"], w["x"] + u, w["vol"], row, col, w["K"], w["mu"], w["horizon"], dofs)
    assert np.linalg.norm(kw - T @ vec) <= 1e-11 * np.linalg.norm(T @ vec)
    n = len(w["vol"])
    D = np.stack([T[3 * i:3 * i + 3, 3 * i:3 * i + 3] for i in range(n)])
    assert np.abs(blocks - D).max() <= 1e-11 * np.abs(D).max()


@pytest.mark.parametrize("precond", ["none", "block_jacobi"])
def test_compression_qs_gold(precond):
    z = np.load(os.path.join(G, "compression_qs.npz"))
    rho, K, mu, h, t0, tf, ns, tol = z["params"]
    times = np.linspace(t0, tf, int(ns) + 1)
    with Context(precision="fp64") as ctx:
        ctx.set_points(z["x"].ravel(), z["vol"])
        ctx.set_horizons([h])
        ctx.set_bonds(z["nl"])
        ctx.material(K, mu, rho)
        for p, c, a, b in z["bc"]:
            ctx.prescribed_displacement([int(p)], int(c), a, b)
        ctx.set_state(np.zeros(36), np.zeros(36))
        for k in range(1, int(ns) + 1):
            ctx.qs_load_step(times[k - 1], times[k], newton_tolerance=tol, cg_relative_tolerance=1e-12,
                             max_newton=10, preconditioner=precond)
            u, v, f = ctx.field("Displacement"), ctx.field("Velocity"), ctx.field("Force_Density")
            for c, ax in enumerate("XYZ"):
                assert np.abs(u[c::3] - z["Displacement" + ax][k]).max() < 1e-9
                assert np.abs(v[c::3] - z["Velocity" + ax][k]).max() < 5e-8
                assert np.abs(f[c::3] - z["Force_Density" + ax][k]).max() < 1.0


def test_cube_matches_oracle_and_block_jacobi_helps():
    w = workloads.qs_cube(n=7, h=1.0e-3, seed=3, jitter=0.05, load_steps=2)
    res = {}
    for precond in ("none", "block_jacobi"):
        with Context(precision="fp64") as ctx:
            workloads.setup_context(ctx, w)
            st = None
            for k in range(1, len(w["times"])):
                st = ctx.qs_load_step(w["times"][k - 1], w["times"][k], newton_tolerance=1e-6,
                                      cg_relative_tolerance=1e-10, preconditioner=precond, stats=st)
            res[precond] = (ctx.field("Displacement"), st.cg_iterations)
            row, col = ctx.bonds_csr()
    bc = []
    for b in w["bcs"]:
        bc += [(3 * int(p) + b["coordinate"], b["a"], b["b"]) for p in b["points"]]
    us = O.qs_solve(w["x"], w["vol"], row, col, w["K"], w["mu"], w["horizon"], bc, w["times"], 1e-6)
    for precond, (u, its) in res.items():
        assert np.linalg.norm(u - us[-1]) <= 1e-8 * np.linalg.norm(us[-1]), precond
    assert res["block_jacobi"][1] < res["none"][1]


def test_constant_prescribed_displacement_is_applied():
    """A prescribed displacement that does not change between load steps
    (a = 0, b != 0): its zero increment takes the previous value from the
    displacement (Peridigm_BoundaryCondition.cpp:137-142), so the first load
    step moves the face to b, as in the oracle."""
    w = workloads.qs_cube(n=7, h=1.0e-3, seed=3, jitter=0.05, load_steps=2)
    for b in w["bcs"]:
        if b["a"] != 0.0:  # the displaced face: held at a constant instead of ramped
            b["b"], b["a"] = b["a"] * w["times"][-1], 0.0
    assert any(b["b"] != 0.0 for b in w["bcs"])
    with Context(precision="fp64") as ctx:
        workloads.setup_context(ctx, w)
        for k in range(1, len(w["times"])):
            ctx.qs_load_step(w["times"][k - 1], w["times"][k], newton_tolerance=1e-6, cg_relative_tolerance=1e-10)
        u = ctx.field("Displacement")
        row, col = ctx.bonds_csr()
    bc = []
    for b in w["bcs"]:
        bc += [(3 * int(p) + b["coordinate"], b["a"], b["b"]) for p in b["points"]]
    us = O.qs_solve(w["x"], w["vol"], row, col, w["K"], w["mu"], w["horizon"], bc, w["times"], 1e-6)
    moved = [d for d, a, bb in bc if bb != 0.0]
    assert np.abs(us[1][moved] - [bb for d, a, bb in bc if bb != 0.0]).max() <= 1e-18
    assert np.linalg.norm(u - us[-1]) <= 1e-8 * np.linalg.norm(us[-1])
