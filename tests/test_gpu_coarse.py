"""GPU aggregate coarse level of the two-level QS preconditioner against the
oracle (no reference counterpart; it preconditions the reference's CG).

* aggregates (non-empty cells of side >= 2 * horizon) identical to the
  oracle's restatement;
* the assembled Galerkin matrix P0^T K P0 equals the oracle's product with its
  dense tangent to 1e-11 of its largest entry (jittered bar, prescribed dofs);
* the Gauss-Jordan inverse: |Ac^-1 Ac - I| <= 1e-9, also over several 64-wide
  elimination steps and 128-wide update tiles with ragged edges (375 and 750
  coarse dofs);
* two-level CG solves a jittered cube to the block-Jacobi displacement (1e-8
  relative) in fewer CG iterations;
* the rigid coarse space (6 modes per aggregate): aggregates equal the
  oracle's; the assembled matrix, in the GPU's orthonormal basis, equals the
  oracle's in its QR basis up to an orthogonal 6x6 map per aggregate, so the
  Frobenius norm of every 6x6 block and the spectrum agree to 1e-9; and the
  two-level CG with rotations reaches the same displacement (1e-8) in fewer
  CG iterations than with translations only.
"""
import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu


def _bar(nx=13, ny=7, nz=7, h=1.0e-3, horizon=1.51, seed=4):
    """Jittered bar, horizon 1.51h (cells of 3.02h: 42 aggregates), left
    3 layers clamped, right 3 layers pulled in x."""
    x, vol = workloads.lattice(nx, ny, nz, h, jitter=0.05, seed=seed)
    col_id = np.arange(nx * ny * nz) % nx
    left, right = np.nonzero(col_id < 3)[0], np.nonzero(col_id >= nx - 3)[0]
    bcs = [dict(points=left, coordinate=c, a=0.0, b=0.0) for c in range(3)]
    bcs.append(dict(points=right, coordinate=0, a=1.0e-5, b=0.0))
    return dict(name="bar", x=x, vol=vol, horizon=horizon * h, K=130.0e9, mu=78.0e9, rho=7800.0, s_c=None, planes=[],
                v0=np.zeros_like(x), bcs=bcs, h=h, times=np.linspace(0.0, 1.0, 3))


def _dofs(w):
    return sorted({3 * int(p) + b["coordinate"] for b in w["bcs"] for p in b["points"]})


def test_coarse_operator_matches_oracle():
    w = _bar()
    n = len(w["vol"])
    rng = np.random.default_rng(2)
    u = rng.normal(0.0, 2e-6, 3 * n)
    with Context(precision="fp64") as ctx:
        workloads.setup_context(ctx, w)
        agg, A, Ai = ctx.coarse_operator(u)
        row, col = ctx.bonds_csr()
    oagg, side = O.coarse_aggregates(w["x"], w["horizon"])
    assert np.array_equal(agg, oagg)
    assert int(agg.max()) + 1 >= 16
    dofs = _dofs(w)
    T = O.tangent_dense(w["x"], w["x"] + u, w["vol"], row, col, w["K"], w["mu"], w["horizon"], dofs)
    Ao, _ = O.coarse_operator(T, oagg, dofs)
    assert A.shape == Ao.shape
    assert np.abs(A - Ao).max() <= 1e-11 * np.abs(Ao).max()
    assert np.abs(Ai @ A - np.eye(A.shape[0])).max() <= 1e-9


def test_two_level_cg_matches_block_jacobi():
    w = workloads.qs_cube(n=12, h=1.0e-3, seed=5, jitter=0.05, load_steps=2)
    out = {}
    for precond in ("block_jacobi", "two_level"):
        with Context(precision="fp64") as ctx:
            workloads.setup_context(ctx, w)
            st = None
            for k in range(1, len(w["times"])):
                st = ctx.qs_load_step(w["times"][k - 1], w["times"][k], newton_tolerance=-1e-8,
                                      cg_relative_tolerance=1e-8, preconditioner=precond, stats=st)
            out[precond] = (ctx.field("Displacement"), st.cg_iterations)
    ub, ib = out["block_jacobi"]
    ut, it = out["two_level"]
    print(f"CG iterations: block Jacobi {ib}, two-level {it}")
    assert np.linalg.norm(ut - ub) <= 1e-8 * np.linalg.norm(ub)
    assert it < ib


def test_rigid_coarse_operator_matches_oracle():
    w = _bar()
    n = len(w["vol"])
    u = np.random.default_rng(3).normal(0.0, 2e-6, 3 * n)
    with Context(precision="fp64") as ctx:
        workloads.setup_context(ctx, w)
        ctx.coarse_modes(6)
        agg, A, Ai = ctx.coarse_operator(u)
        row, col = ctx.bonds_csr()
    oagg, side = O.coarse_aggregates(w["x"], w["horizon"], modes=6)
    assert np.array_equal(agg, oagg)
    na = int(agg.max()) + 1
    assert A.shape == (6 * na, 6 * na)
    dofs = _dofs(w)
    T = O.tangent_dense(w["x"], w["x"] + u, w["vol"], row, col, w["K"], w["mu"], w["horizon"], dofs)
    Ao, _ = O.coarse_operator_rigid(T, w["x"], oagg, side, dofs)
    scale = np.abs(Ao).max()
    for I in range(na):
        for J in range(na):
            bg = np.linalg.norm(A[6 * I:6 * I + 6, 6 * J:6 * J + 6])
            bo = np.linalg.norm(Ao[6 * I:6 * I + 6, 6 * J:6 * J + 6])
            assert abs(bg - bo) <= 1e-9 * scale
    eg, eo = np.linalg.eigvalsh(0.5 * (A + A.T)), np.linalg.eigvalsh(0.5 * (Ao + Ao.T))
    assert np.abs(eg - eo).max() <= 1e-9 * np.abs(eo).max()
    assert np.abs(Ai @ A - np.eye(A.shape[0])).max() <= 1e-9


def test_two_level_rigid_fewer_iterations():
    w = workloads.qs_cube(n=16, h=1.0e-3, seed=5, jitter=0.05, load_steps=2)
    out = {}
    for modes in (3, 6):
        with Context(precision="fp64") as ctx:
            workloads.setup_context(ctx, w)
            ctx.coarse_modes(modes)
            st = None
            for k in range(1, len(w["times"])):
                st = ctx.qs_load_step(w["times"][k - 1], w["times"][k], newton_tolerance=-1e-8,
                                      cg_relative_tolerance=1e-8, preconditioner="two_level", stats=st)
            out[modes] = (ctx.field("Displacement"), st.cg_iterations)
    (u3, i3), (u6, i6) = out[3], out[6]
    print(f"CG iterations: translations {i3}, with rotations {i6}")
    assert np.linalg.norm(u6 - u3) <= 1e-8 * np.linalg.norm(u3)
    assert i6 < i3


@pytest.mark.parametrize("modes", [3, 6])
def test_coarse_inverse_multi_block(modes):
    """15^3 jittered lattice, cells of 3.02h: 125 aggregates, 375 or 750 coarse
    dofs (not multiples of the 64-wide steps or the 128-wide update tiles)."""
    w = _bar(nx=15, ny=15, nz=15, seed=8)
    n = len(w["vol"])
    u = np.random.default_rng(5).normal(0.0, 2e-6, 3 * n)
    with Context(precision="fp64") as ctx:
        workloads.setup_context(ctx, w)
        ctx.coarse_modes(modes)
        agg, A, Ai = ctx.coarse_operator(u)
    nc = A.shape[0]
    assert nc == modes * (int(agg.max()) + 1) == modes * 125
    assert np.abs(Ai @ A - np.eye(nc)).max() <= 1e-9
