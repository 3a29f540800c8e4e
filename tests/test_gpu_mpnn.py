"""GPU learned CG preconditioner: gradients against the CPU oracle, training on
solver-generated pairs, and its effect inside the quasi-static CG.

* pd_mpnn_loss_grad (residual-space loss |K z - r|^2/|r|^2) vs oracle/mpnn.py
  with the oracle's dense tangent, on the same BF16 weights: loss to 1e-4
  relative, gradient to 2e-2 relative L2 (FP32 vs FP64 sums and BF16 rounding
  of stored activations);
* block-Jacobi QS solves with capture produce pairs, training lowers the loss;
* on held-out block-Jacobi CG residuals one application of the trained
  network leaves a residual |K z - r|^2/|r|^2 at least 10 % below block
  Jacobi's (the same network with its decoder zeroed);
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


def _block_jacobi_cg_residuals(ctx, n, dofs, seed, every=3, max_it=120):
    """Residuals of a host block-Jacobi CG on the context's tangent (u = 0)."""
    u0 = np.zeros(3 * n)
    binv = np.linalg.inv(ctx.jacobian_blocks(u0))
    bj = lambda r: np.einsum("nij,nj->ni", binv, r.reshape(n, 3)).ravel()
    free = np.ones(3 * n, bool)
    free[dofs] = False
    b = np.where(free, np.random.default_rng(seed).standard_normal(3 * n), 0.0)
    x, r = np.zeros(3 * n), b.copy()
    z = bj(r)
    p, rz, out = z.copy(), r @ z, []
    for it in range(max_it):
        if np.linalg.norm(r) < 1e-6 * np.linalg.norm(b):
            break
        if it % every == 0:
            out.append(r / np.linalg.norm(r))
        q = ctx.jacobian_apply(u0, p)
        al = rz / (p @ q)
        x += al * p
        r -= al * q
        z = bj(r)
        rz, rz_old = r @ z, rz
        p = z + (rz / rz_old) * p
    return [(bj(r), r) for r in out]


def test_mpnn_trains_and_helps_cg():
    # training pairs from block-Jacobi solves of a jittered cube
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
    w2 = workloads.qs_cube(n=10, h=1.0e-3, seed=23, jitter=0.05, load_steps=2)
    n = len(w2["vol"])
    dofs = sorted({3 * int(p) + b["coordinate"] for b in w2["bcs"] for p in b["points"]})
    # what one application gains over block Jacobi (the network with its decoder
    # zeroed returns exactly z = P_bj r) on held-out block-Jacobi CG residuals
    with Context(precision="fp64") as ctx:
        workloads.setup_context(ctx, w2)
        ctx.mpnn_init(seed=0, radius=1.5e-3)
        pairs = _block_jacobi_cg_residuals(ctx, n, dofs, seed=3)
        assert len(pairs) >= 10
        zero_dec = weights.copy()
        zero_dec[M.OFF_WD:] = 0.0
        losses = {}
        for name, wts in (("block_jacobi", zero_dec), ("learned", weights)):
            ctx.mpnn_set_weights(wts)
            losses[name] = float(np.mean([ctx.mpnn_loss_grad(a.astype(np.float32), r.astype(np.float32))[0]
                                          for a, r in pairs]))
    print(f"held-out |K z - r|^2/|r|^2: block Jacobi {losses['block_jacobi']:.4f}, learned {losses['learned']:.4f}")
    assert losses["learned"] < 0.9 * losses["block_jacobi"]
    # inside the quasi-static solve (flexible CG with the block-Jacobi fallback):
    # the same displacement as block Jacobi with fewer CG iterations
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
            out[precond] = (ctx.field("Displacement"), st.cg_iterations, st.preconditioner_fallbacks)
    ub, ib, _ = out["block_jacobi"]
    um, im, fb = out["mpnn"]
    print(f"CG iterations: block Jacobi {ib}, learned {im} ({fb} fallbacks)")
    assert np.linalg.norm(um - ub) <= 1e-8 * np.linalg.norm(ub)
    assert im < ib
