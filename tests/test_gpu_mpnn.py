"""GPU learned CG preconditioner: gradients against the CPU oracle, training on
solver-generated pairs, and its effect inside the quasi-static CG.

* pd_mpnn_loss_grad (residual-space loss |K z - r|^2/|r|^2) vs oracle/mpnn.py
  with the oracle's dense tangent, on the same BF16 weights: loss to 1e-4
  relative, gradient to 2e-2 relative L2 (FP32 vs FP64 sums and BF16 rounding
  of stored activations);
* block-Jacobi QS solves with capture produce pairs, training lowers the loss;
* the trained preconditioner solves a held-out QS problem to the same
  displacement as block Jacobi (1e-8 relative) with fewer CG iterations.
"""
import numpy as np
import pytest

from oracle import mpnn as M
from oracle import oracle as O
from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu


def _cube(n, seed):
    w = workloads.qs_cube(n=n, h=1.0e-3, seed=seed, jitter=0.05, load_steps=4)
    ctx = Context(precision="fp64")
    workloads.setup_context(ctx, w)
    return w, ctx


def test_mpnn_gradient_matches_oracle():
    w, ctx = _cube(5, 1)
    dofs = sorted({3 * int(p) + b["coordinate"] for b in w["bcs"] for p in b["points"]})
    with ctx:
        ctx.mpnn_init(seed=3, radius=1.5e-3)
        row, col = ctx.bonds_csr()
        K = O.tangent_dense(w["x"], w["x"], w["vol"], row, col, w["K"], w["mu"], w["horizon"], dofs)
        rng = np.random.default_rng(0)
        wts = (rng.standard_normal(M.NPARAM) * 0.15).astype(np.float32)
        ctx.mpnn_set_weights(wts)
        n = len(w["vol"])
        # a residual of the cube's own tangent and a first guess of its scale
        e = rng.standard_normal(3 * n) * 1e-6
        r = (K @ e).astype(np.float32)
        a = (e * (1.0 + 0.3 * rng.standard_normal(3 * n))).astype(np.float32)
        L, g = ctx.mpnn_loss_grad(a, r)
    mrow, mcol = M.subgraph(w["x"], row, col, 1.5e-3)
    Lr, gr = M.loss_grad_residual(wts, a, r, K, dofs, mrow, mcol)
    assert abs(L - Lr) <= 1e-4 * abs(Lr)
    assert np.linalg.norm(g - gr) <= 2e-2 * np.linalg.norm(gr)


def test_mpnn_trains_and_helps_cg():
    # training pairs from block-Jacobi solves of two cubes with different moduli
    w, tr = _cube(10, 11)
    with tr:
        tr.mpnn_init(seed=7, radius=1.5e-3)
        tr.mpnn_collect(3)
        st = None
        for k in range(1, len(w["times"])):
            st = tr.qs_load_step(w["times"][k - 1], w["times"][k], newton_tolerance=-1e-8, cg_relative_tolerance=1e-8,
                                 preconditioner="block_jacobi", stats=st)
        assert tr.mpnn_num_pairs() > 20
        l1 = tr.mpnn_train(1, learning_rate=2e-3, batch=4)
        l2 = tr.mpnn_train(30, learning_rate=2e-3, batch=4)
        assert l2 < l1
        weights = tr.mpnn_weights()
    # held-out problem
    w2 = workloads.qs_cube(n=10, h=1.0e-3, seed=23, jitter=0.05, load_steps=2)
    out = {}
    for precond in ("block_jacobi", "mpnn"):
        with Context(precision="fp64") as ctx:
            workloads.setup_context(ctx, w2)
            if precond == "mpnn":
                ctx.mpnn_init(seed=0, radius=1.5e-3)
                ctx.mpnn_set_weights(weights)
            st = None
            for k in range(1, len(w2["times"])):
                st = ctx.qs_load_step(w2["times"][k - 1], w2["times"][k], newton_tolerance=-1e-8,
                                      cg_relative_tolerance=1e-8, preconditioner=precond, stats=st)
            out[precond] = (ctx.field("Displacement"), st.cg_iterations)
    ub, ib = out["block_jacobi"]
    um, im = out["mpnn"]
    print(f"CG iterations: block Jacobi {ib}, learned {im}")
    assert np.linalg.norm(um - ub) <= 1e-8 * np.linalg.norm(ub)
    assert im < ib
