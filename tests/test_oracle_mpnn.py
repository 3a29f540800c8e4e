"""The CPU oracle of the learned preconditioner's network: analytic gradient
against central finite differences (BF16 rounding off so the loss is smooth)."""
import numpy as np

from oracle import mpnn as M
from oracle import oracle as O
from peridigm_b200 import workloads


def test_oracle_gradient_matches_finite_differences():
    x, vol = workloads.lattice(4, 3, 3, 1.0, jitter=0.05, seed=1)
    row, col = O.neighbor_search(x, 3.015)
    mrow, mcol = M.subgraph(x, row, col, 1.5)
    n = len(vol)
    rng = np.random.default_rng(0)
    w = (rng.standard_normal(M.NPARAM) * 0.2).astype(np.float32)
    a, r, e = (rng.standard_normal(3 * n).astype(np.float32) for _ in range(3))
    L, g = M.loss_grad(w, a, r, e, mrow, mcol, round_bf16=False)
    for k in list(rng.choice(M.NPARAM, 40, replace=False)) + [M.OFF_BD, M.OFF_W0, M.OFF_L + 5]:
        eps = 1e-3
        wp, wm = w.astype(np.float64).copy(), w.astype(np.float64).copy()
        wp[k] += eps
        wm[k] -= eps
        Lp, _ = M.loss_grad(wp.astype(np.float32), a, r, e, mrow, mcol, round_bf16=False)
        Lm, _ = M.loss_grad(wm.astype(np.float32), a, r, e, mrow, mcol, round_bf16=False)
        fd = (Lp - Lm) / (2 * eps)
        assert abs(fd - g[k]) <= 2e-3 * max(1.0, abs(g[k])) + 1e-3 * abs(L), (k, fd, g[k])


def test_residual_loss_gradient_matches_finite_differences():
    x, vol = workloads.lattice(3, 3, 3, 1.0, jitter=0.05, seed=2)
    row, col = O.neighbor_search(x, 3.015)
    mrow, mcol = M.subgraph(x, row, col, 1.5)
    n = len(vol)
    K = O.tangent_dense(x, x, vol, row, col, 1.0, 0.6, 3.015, bc_dofs=[0, 1, 2])
    rng = np.random.default_rng(1)
    w = (rng.standard_normal(M.NPARAM) * 0.2).astype(np.float32)
    a = (rng.standard_normal(3 * n) * 0.3).astype(np.float32)
    r = rng.standard_normal(3 * n).astype(np.float32)
    L, g = M.loss_grad_residual(w, a, r, K, [0, 1, 2], mrow, mcol, round_bf16=False)
    for k in list(rng.choice(M.NPARAM, 30, replace=False)) + [M.OFF_BD + 1, M.OFF_WD + 3]:
        eps = 1e-3
        wp, wm = w.astype(np.float64).copy(), w.astype(np.float64).copy()
        wp[k] += eps
        wm[k] -= eps
        Lp, _ = M.loss_grad_residual(wp.astype(np.float32), a, r, K, [0, 1, 2], mrow, mcol, round_bf16=False)
        Lm, _ = M.loss_grad_residual(wm.astype(np.float32), a, r, K, [0, 1, 2], mrow, mcol, round_bf16=False)
        fd = (Lp - Lm) / (2 * eps)
        assert abs(fd - g[k]) <= 2e-3 * max(1.0, abs(g[k])) + 1e-3 * abs(L), (k, fd, g[k])


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.01171875, 1.001953125, -3.1415927], np.float32)
    out = M.bf16(v)
    assert out[0] == 1.0
    assert out[1] == 1.0          # halfway, ties to even
    assert out[2] == 1.015625     # halfway, ties to even (odd -> even upward)
    assert out[3] == 1.0          # below halfway
    assert out[4] == -3.140625
