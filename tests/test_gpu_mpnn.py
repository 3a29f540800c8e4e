"""GPU learned middle level of the QS CG preconditioner: gradients against the
CPU oracle, training on solver-generated pairs, and what the trained network
gains inside the quasi-static CG.

* pd_mpnn_loss_grad (1 - (r.z)^2/((z.K z)(e.r)), z = P_bj r [+ coarse] + Q S G^T G S Q^T r)
  vs oracle/mpnn.py with the oracle's dense tangent, the device's block-Jacobi
  blocks and coarse operator, on the same BF16 weights: loss to 1e-6
  relative, gradient to 1e-5 relative L2 (measured 1e-7: FP32 activations
  and sums against FP64);
* pd_mpnn_apply (one cooperative launch, grid barriers between the phases)
  vs the oracle's Q S G^T G S Q^T r, and bit-identical on a second call;
* two-level QS solves with capture produce pairs, and training lowers the loss;
* on the translation two-level base, the trained preconditioner solves a
  held-out QS problem to the two-level displacement (1e-8 relative) in fewer
  CG iterations than the same preconditioner without the network, with no
  fallback;
* on the rigid two-level base (translations and rotations, the base the
  bench uses), what training gains over the same network at its starting
  weights and over no network: measured within +-10 % of the base's CG
  iterations either way (an exact patch-level solve in place of the network
  saves at most about 12 % there, so a trained approximation has little room).
"""
import numpy as np
import pytest

from oracle import mpnn as M
from oracle import oracle as O
from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu


def _bar(nx=13, ny=7, nz=7, h=1.0e-3, horizon=1.51, seed=4):
    x, vol = workloads.lattice(nx, ny, nz, h, jitter=0.05, seed=seed)
    col_id = np.arange(nx * ny * nz) % nx
    left, right = np.nonzero(col_id < 3)[0], np.nonzero(col_id >= nx - 3)[0]
    bcs = [dict(points=left, coordinate=c, a=0.0, b=0.0) for c in range(3)]
    bcs.append(dict(points=right, coordinate=0, a=1.0e-5, b=0.0))
    return dict(name="bar", x=x, vol=vol, horizon=horizon * h, K=130.0e9, mu=78.0e9, rho=7800.0, s_c=None, planes=[],
                v0=np.zeros_like(x), bcs=bcs, h=h, times=np.linspace(0.0, 1.0, 3))


@pytest.mark.parametrize("coarse", [False, True])
def test_mpnn_gradient_matches_oracle(coarse):
    w = _bar(seed=6)
    n = len(w["vol"])
    h = w["h"]
    dofs = sorted({3 * int(p) + b["coordinate"] for b in w["bcs"] for p in b["points"]})
    with Context(precision="fp64") as ctx:
        workloads.setup_context(ctx, w)
        ctx.mpnn_init(seed=3, patch=2.0 * h)
        ctx.mpnn_coarse(0.0 if coarse else -1.0)
        row, col = ctx.bonds_csr()
        u0 = np.zeros(3 * n)
        blocks = ctx.jacobian_blocks(u0)
        agg, A, Ai = ctx.coarse_operator(u0)
        K = O.tangent_dense(w["x"], w["x"], w["vol"], row, col, w["K"], w["mu"], w["horizon"], dofs)
        rng = np.random.default_rng(0)
        wts = (rng.standard_normal(M.NPARAM) * 0.08).astype(np.float32)
        ctx.mpnn_set_weights(wts)
        e = rng.standard_normal(3 * n) * 1e-6
        e[dofs] = 0.0
        r = (K @ e).astype(np.float32)
        a = (e * (1.0 + 0.3 * rng.standard_normal(3 * n))).astype(np.float32)
        e = e.astype(np.float32)
        L, g = ctx.mpnn_loss_grad(a, r, e)
    pid, nbrs = M.patches(w["x"], 2.0 * h)
    scale = M.scales(np.linalg.inv(blocks), pid, dofs)
    z0 = None
    if coarse:
        _, P0 = O.coarse_operator(K, agg, dofs)
        z0 = P0 @ (Ai @ (P0.T @ r.astype(np.float64)))
    Lr, gr = M.loss_grad(wts, a, r, e, K, dofs, pid, nbrs, scale, z0=z0)
    assert abs(L - Lr) <= 1e-6 * abs(Lr)
    assert np.linalg.norm(g - gr) <= 1e-5 * np.linalg.norm(gr)


@pytest.mark.parametrize("seed", [6, 9])
def test_mpnn_apply_matches_oracle(seed):
    """The inference product each learned CG iteration adds (head, 3 layers,
    3 transposed layers, tail: one cooperative launch) against the oracle's
    Q S G^T G S Q^T r on the same BF16 weights (FP32 activations: 1e-5)."""
    w = _bar(seed=seed)
    n = len(w["vol"])
    h = w["h"]
    dofs = sorted({3 * int(p) + b["coordinate"] for b in w["bcs"] for p in b["points"]})
    rng = np.random.default_rng(seed)
    wts = (rng.standard_normal(M.NPARAM) * 0.08).astype(np.float32)
    r = rng.standard_normal(3 * n)
    with Context(precision="fp64") as ctx:
        workloads.setup_context(ctx, w)
        ctx.mpnn_init(seed=3, patch=2.0 * h)
        ctx.mpnn_set_weights(wts)
        blocks = ctx.jacobian_blocks(np.zeros(3 * n))
        z = ctx.mpnn_apply(r)
        z2 = ctx.mpnn_apply(r)
    pid, nbrs = M.patches(w["x"], 2.0 * h)
    npatch = int(pid.max()) + 1
    scale = M.scales(np.linalg.inv(blocks), pid, dofs)
    fixed = np.zeros(3 * n, bool)
    fixed[dofs] = True
    Am = M._mean_matrix(nbrs)
    Q = M._q(pid, fixed, npatch)
    S = np.repeat(np.asarray(scale, np.float64), 3)
    wb = M.bf16(wts).astype(np.float64)
    y, _ = M.forward(wb, (S * (Q.T @ r)).reshape(npatch, 3), Am)
    zr = Q @ (S * M.transpose(wb, y, Am).ravel())
    assert np.all(z[fixed] == 0.0)
    assert np.array_equal(z, z2)
    assert np.linalg.norm(z - zr) <= 1e-5 * np.linalg.norm(zr)


def test_mpnn_trains_and_helps_cg():
    h = 1.0e-3
    w = workloads.qs_cube(n=12, h=h, seed=11, jitter=0.05, load_steps=4)
    with Context(precision="fp64") as tr:
        workloads.setup_context(tr, w)
        tr.mpnn_init(seed=7, patch=2.0 * h)
        tr.mpnn_collect(3)
        st = None
        for k in range(1, len(w["times"])):
            st = tr.qs_load_step(w["times"][k - 1], w["times"][k], newton_tolerance=-1e-8, cg_relative_tolerance=1e-8,
                                 preconditioner="two_level", stats=st)
        assert tr.mpnn_num_pairs() >= 10
        l1 = tr.mpnn_train(1, learning_rate=2e-3, batch=4)
        l2 = tr.mpnn_train(30, learning_rate=2e-3, batch=4)
        assert l2 < l1
        weights = tr.mpnn_weights()
    w2 = workloads.qs_cube(n=12, h=h, seed=23, jitter=0.05, load_steps=2)
    out = {}
    for precond in ("two_level", "mpnn"):
        with Context(precision="fp64") as ctx:
            workloads.setup_context(ctx, w2)
            if precond == "mpnn":
                ctx.mpnn_init(seed=0, patch=2.0 * h)
                ctx.mpnn_set_weights(weights)
            st = None
            for k in range(1, len(w2["times"])):
                st = ctx.qs_load_step(w2["times"][k - 1], w2["times"][k], newton_tolerance=-1e-8,
                                      cg_relative_tolerance=1e-8, preconditioner=precond, stats=st)
            out[precond] = (ctx.field("Displacement"), st.cg_iterations, st.preconditioner_fallbacks)
    ub, ib, _ = out["two_level"]
    um, im, fb = out["mpnn"]
    print(f"CG iterations: two-level {ib}, learned {im} ({fb} fallbacks)")
    assert np.linalg.norm(um - ub) <= 1e-8 * np.linalg.norm(ub)
    assert fb == 0
    assert im < ib


def test_mpnn_training_gain_on_rigid_base():
    """Trained network against the same network at its starting weights and
    against the rigid two-level base alone, on a held-out cube: all three
    reach the same displacement with no fallback, training lowers its loss,
    and the trained network's CG iterations stay within 10 % of the base's
    (the measured gain on this base is nil)."""
    h, patch = 1.0e-3, 3.0e-3
    w = workloads.qs_cube(n=12, h=h, seed=11, jitter=0.05, load_steps=4)
    with Context(precision="fp64") as tr:
        workloads.setup_context(tr, w)
        tr.coarse_modes(6)
        tr.mpnn_init(seed=7, patch=patch)
        w0 = tr.mpnn_weights()
        tr.mpnn_collect(2)
        st = None
        for k in range(1, len(w["times"])):
            st = tr.qs_load_step(w["times"][k - 1], w["times"][k], newton_tolerance=-1e-8, cg_relative_tolerance=1e-8,
                                 preconditioner="two_level", stats=st)
        l1 = tr.mpnn_train(1, learning_rate=1e-3, batch=8)
        l2 = tr.mpnn_train(10, learning_rate=1e-3, batch=8)
        assert l2 < l1
        wt = tr.mpnn_weights()
    w2 = workloads.qs_cube(n=12, h=h, seed=23, jitter=0.05, load_steps=2)
    out = {}
    for arm, wts in (("base", None), ("init", w0), ("trained", wt)):
        with Context(precision="fp64") as ctx:
            workloads.setup_context(ctx, w2)
            ctx.coarse_modes(6)
            pre = "two_level"
            if wts is not None:
                ctx.mpnn_init(seed=0, patch=patch)
                ctx.mpnn_set_weights(wts)
                pre = "mpnn"
            st = None
            for k in range(1, len(w2["times"])):
                st = ctx.qs_load_step(w2["times"][k - 1], w2["times"][k], newton_tolerance=-1e-8,
                                      cg_relative_tolerance=1e-8, preconditioner=pre, stats=st)
            out[arm] = (ctx.field("Displacement"), st.cg_iterations, st.preconditioner_fallbacks)
    print("CG iterations on the rigid base: " + ", ".join(f"{a} {out[a][1]}" for a in out))
    ub = out["base"][0]
    for arm in ("init", "trained"):
        assert np.linalg.norm(out[arm][0] - ub) <= 1e-8 * np.linalg.norm(ub)
        assert out[arm][2] == 0
    assert abs(out["trained"][1] - out["base"][1]) <= 0.1 * out["base"][1]
