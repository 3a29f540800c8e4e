"""The threaded CPU restatement of the quasi-static CG step (oracle/cpu_qs.c,
the CPU baseline of the quasi-static leg) against the oracle's dense tangent
-d(V f)/du: products 1e-11 relative, block-Jacobi blocks the inverses of the
dense diagonal blocks (1e-10), and CG solving the dense system to its
tolerance; results independent of the thread count."""
import numpy as np

from oracle import cpu_qs as Q
from oracle import oracle as O
from peridigm_b200 import workloads


def _case():
    h = 1.0e-3
    x, vol = workloads.lattice(5, 4, 4, h, jitter=0.05, seed=3)
    P = x.reshape(-1, 3)
    n = len(vol)
    rng = np.random.default_rng(1)
    u = np.zeros_like(P)
    u[:, 0] = 2e-3 * P[:, 0]
    u += rng.normal(0, 1e-4 * h, size=u.shape)
    row, col = O.neighbor_search(x, 3.015 * h)
    K = 130e9 * np.exp(0.2 * rng.normal(size=n))
    mu = 0.6 * K
    fixed = np.zeros(n, np.uint8)
    left = np.nonzero(P[:, 0] < P[:, 0].min() + 0.5 * h)[0]
    fixed[left] = 7
    fixed[np.nonzero(P[:, 0] > P[:, 0].max() - 0.5 * h)[0]] = 1
    return x, (P + u).ravel(), vol, row, col, K, mu, 3.015 * h, fixed


def test_cpu_qs_matches_dense_tangent():
    x, y, vol, row, col, K, mu, h, fixed = _case()
    n = len(vol)
    bc = [3 * i + c for i in range(n) for c in range(3) if (fixed[i] >> c) & 1]
    T = O.tangent_dense(x, y, vol, row, col, K, mu, h, bc_dofs=bc)
    p = np.random.default_rng(2).normal(size=3 * n)
    out = []
    for threads in (1, 3):
        P = Q.Problem(x, y, vol, row, col, K, mu, h, fixed=fixed, threads=threads)
        P.setup()
        q = P.apply(p)
        assert np.linalg.norm(q - T @ p) <= 1e-11 * np.linalg.norm(T @ p)
        for i in range(n):
            blk = T[3 * i:3 * i + 3, 3 * i:3 * i + 3]
            assert np.abs(P.dinv[9 * i:9 * i + 9].reshape(3, 3) - np.linalg.inv(blk)).max() <= \
                1e-10 * np.abs(np.linalg.inv(blk)).max()
        b = T @ np.random.default_rng(3).normal(size=3 * n)
        b[bc] = 0.0
        xs, r, rel = P.cg(b, 400)
        assert rel <= 1e-10
        ref = np.linalg.solve(T, b)
        assert np.linalg.norm(xs - ref) <= 1e-8 * np.linalg.norm(ref)
        out.append(q)
    assert np.array_equal(out[0], out[1])  # per-owner sums: no thread-order dependence
