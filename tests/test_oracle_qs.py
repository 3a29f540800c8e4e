"""Oracle quasi-static pieces on the CPU.

* the analytic linearization of the LPS force (oracle pdo_lps_jv) against
  central finite differences of the oracle force (the reference's own FD
  Jacobian approach, src/materials/Peridigm_Material.cpp:70-333);
* the oracle's load-step Newton solve against the Compression_QS_3x2x2 gold
  (test/regression/Compression_QS_3x2x2, Disp 1e-9 absolute).
"""
import os

import numpy as np

from oracle import oracle as O
from peridigm_b200 import workloads

G = os.path.join(os.path.dirname(__file__), "golden")


def test_linearization_matches_finite_differences():
    x, vol = workloads.lattice(5, 4, 4, 1e-3, jitter=0.05, seed=2)
    h = 3.015e-3
    row, col = O.neighbor_search(x, h)
    rng = np.random.default_rng(0)
    y = x + rng.normal(0, 2e-6, x.size)
    w = rng.normal(0, 1e-7, x.size)
    jv = O.lps_jv(x, y, vol, row, col, 130e9, 78e9, h, w)
    eps = 1e-2
    fp = O.eval_model(x, y + eps * w, vol, row, col, 130e9, 78e9, h)["force"]
    fm = O.eval_model(x, y - eps * w, vol, row, col, 130e9, 78e9, h)["force"]
    fd = (fp - fm) / (2 * eps)
    assert np.linalg.norm(jv - fd) <= 1e-8 * np.linalg.norm(fd)


def test_tangent_is_symmetric_positive_definite():
    x, vol = workloads.lattice(4, 3, 3, 1e-3, jitter=0.05, seed=5)
    h = 3.015e-3
    row, col = O.neighbor_search(x, h)
    T = O.tangent_dense(x, x, vol, row, col, 130e9, 78e9, h, bc_dofs=[0, 1, 2, 3, 4, 5, 6, 7, 8])
    assert np.abs(T - T.T).max() <= 1e-9 * np.abs(T).max()
    assert np.linalg.eigvalsh(0.5 * (T + T.T)).min() > 0


def test_compression_qs_gold():
    z = np.load(os.path.join(G, "compression_qs.npz"))
    rho, K, mu, h, t0, tf, ns, tol = z["params"]
    row, col = O.nl_to_csr(z["nl"], 12)
    bc = [(int(3 * p + c), a, b) for p, c, a, b in z["bc"]]
    us = O.qs_solve(z["x"].ravel(), z["vol"], row, col, K, mu, h, bc, np.linspace(t0, tf, int(ns) + 1), tol)
    for k in range(int(ns) + 1):
        for c, ax in enumerate("XYZ"):
            assert np.abs(us[k][c::3] - z["Displacement" + ax][k]).max() < 1e-9
