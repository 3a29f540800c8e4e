"""The CPU oracle of the learned middle level: analytic gradient against
central finite differences (BF16 rounding off so the loss is smooth), the
symmetry of the learned term, and the patch graph."""
import numpy as np

from oracle import mpnn as M
from oracle import oracle as O
from peridigm_b200 import workloads


def _problem(seed=1):
    x, vol = workloads.lattice(6, 4, 4, 1.0, jitter=0.05, seed=seed)
    row, col = O.neighbor_search(x, 1.51)
    n = len(vol)
    dofs = [0, 1, 2, 3 * 5 + 1]
    K = O.tangent_dense(x, x, vol, row, col, 1.0, 0.6, 1.51, bc_dofs=dofs)
    pid, nbrs = M.patches(x, 2.0)
    blocks = np.stack([K[3 * i:3 * i + 3, 3 * i:3 * i + 3] for i in range(n)])
    scale = M.scales(np.linalg.inv(blocks), pid, dofs)
    return x, n, dofs, K, pid, nbrs, scale


def test_patch_graph_is_symmetric_cell_adjacency():
    x, n, dofs, K, pid, nbrs, scale = _problem()
    assert int(pid.max()) + 1 == 3 * 2 * 2
    for i, js in enumerate(nbrs):
        assert i not in js
        for j in js:
            assert i in nbrs[j]
    assert np.all(scale > 0)


def test_oracle_gradient_matches_finite_differences():
    x, n, dofs, K, pid, nbrs, scale = _problem()
    rng = np.random.default_rng(0)
    w = (rng.standard_normal(M.NPARAM) * 0.1).astype(np.float32)
    e = rng.standard_normal(3 * n)
    e[dofs] = 0.0
    r = (K @ e).astype(np.float32)
    a = (e * (1.0 + 0.3 * rng.standard_normal(3 * n))).astype(np.float32)
    z0 = rng.standard_normal(3 * n) * 0.1
    e = e.astype(np.float32)
    L, g = M.loss_grad(w, a, r, e, K, dofs, pid, nbrs, scale, z0=z0, round_bf16=False)
    assert 0.0 <= L <= 1.0
    for k in list(rng.choice(M.NPARAM, 40, replace=False)) + [M.OFF_W0, M.OFF_W0 + 7, M.OFF_L + 5,
                                                               M.OFF_L + M.H * M.H + 3]:
        eps = 1e-3
        wp, wm = w.astype(np.float64).copy(), w.astype(np.float64).copy()
        wp[k] += eps
        wm[k] -= eps
        Lp, _ = M.loss_grad(wp.astype(np.float32), a, r, e, K, dofs, pid, nbrs, scale, z0=z0, round_bf16=False)
        Lm, _ = M.loss_grad(wm.astype(np.float32), a, r, e, K, dofs, pid, nbrs, scale, z0=z0, round_bf16=False)
        fd = (Lp - Lm) / (2 * eps)
        assert abs(fd - g[k]) <= 2e-3 * abs(g[k]) + 1e-6, (k, fd, g[k])


def test_learned_term_is_symmetric_positive_semidefinite():
    x, n, dofs, K, pid, nbrs, scale = _problem(2)
    rng = np.random.default_rng(3)
    w = (rng.standard_normal(M.NPARAM) * 0.1).astype(np.float32)
    wb = M.bf16(w).astype(np.float64)
    npatch = int(pid.max()) + 1
    Am = M._mean_matrix(nbrs)
    cols = []
    for k in range(3 * npatch):
        e = np.zeros(3 * npatch)
        e[k] = 1.0
        y, _ = M.forward(wb, e.reshape(npatch, 3), Am)
        cols.append(M.transpose(wb, y, Am).ravel())
    GtG = np.stack(cols, 1)
    assert np.abs(GtG - GtG.T).max() <= 1e-10 * np.abs(GtG).max()
    assert np.linalg.eigvalsh(0.5 * (GtG + GtG.T)).min() >= -1e-10 * np.abs(GtG).max()


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.01171875, 1.001953125, -3.1415927], np.float32)
    out = M.bf16(v)
    assert out[0] == 1.0
    assert out[1] == 1.0          # halfway, ties to even
    assert out[2] == 1.015625     # halfway, ties to even (odd -> even upward)
    assert out[3] == 1.0          # below halfway
    assert out[4] == -3.140625


def test_multistep_loss_gradient_matches_finite_differences():
    """The loss after k steps of preconditioned steepest descent (block Jacobi
    plus the learned term) and its adjoint gradient: central differences along
    a random weight direction, and k = 1 equal to the one-step loss."""
    x, n, dofs, K, pid, nbrs, scale = _problem(seed=3)
    rng = np.random.default_rng(2)
    w = (rng.standard_normal(M.NPARAM) * 0.1).astype(np.float32)
    e = rng.standard_normal(3 * n)
    e[dofs] = 0.0
    r = K @ e
    blocks = np.stack([K[3 * i:3 * i + 3, 3 * i:3 * i + 3] for i in range(n)])
    Mfix = np.zeros((3 * n, 3 * n))
    for i in range(n):
        Mfix[3 * i:3 * i + 3, 3 * i:3 * i + 3] = np.linalg.inv(blocks[i])
    Mfix[dofs, :] = 0.0
    Mfix[:, dofs] = 0.0
    L1, g1 = M.loss_grad_steps(w, r, e, K, Mfix, dofs, pid, nbrs, scale, 1, round_bf16=False)
    Lr, gr = M.loss_grad(w, (Mfix @ r).astype(np.float32), r.astype(np.float32), e.astype(np.float32), K, dofs, pid,
                         nbrs, scale, round_bf16=False)
    assert abs(L1 - Lr) <= 1e-6 * Lr and np.linalg.norm(g1 - gr) <= 1e-5 * np.linalg.norm(gr)
    for k in (1, 4):
        L, g = M.loss_grad_steps(w, r, e, K, Mfix, dofs, pid, nbrs, scale, k, round_bf16=False)
        d = rng.standard_normal(M.NPARAM)
        wp = (w + 1e-3 * d).astype(np.float32)
        wm = (w - 1e-3 * d).astype(np.float32)
        Lp = M.loss_grad_steps(wp, r, e, K, Mfix, dofs, pid, nbrs, scale, k, round_bf16=False)[0]
        Lm = M.loss_grad_steps(wm, r, e, K, Mfix, dofs, pid, nbrs, scale, k, round_bf16=False)[0]
        fd, an = Lp - Lm, g @ (wp.astype(np.float64) - wm.astype(np.float64))
        assert abs(fd - an) <= 1e-3 * abs(fd), (k, fd, an)
        assert 0.0 <= L <= 1.0
