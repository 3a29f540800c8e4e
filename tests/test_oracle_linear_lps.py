"""The oracle's Linear LPS (LinearLPSPVMaterial::precompute / computeForce) and
LPS restatements against the gold output of the reference's LinearLPSBar
verification deck: bar 1 (blocks 1-3, Linear LPS Partial Volume) and bar 2
(blocks 4-6, Elastic Partial Volume = LPS) under the prescribed field
u_x = 0.1 x t at t = 0.2 .. 1.0. Tolerances are the deck's .comp: Force 1e-3,
Dilatation 1e-10, Weighted_Volume 1e-14 (absolute); the reaction sums
(Block_Data Sum of Force over the end blocks) 1e-12 relative."""
import os

import numpy as np
import pytest

from oracle import oracle as O

G = os.path.join(os.path.dirname(__file__), "golden")
K, MU, H = 160.0e10, 79.3e10, 0.1502


@pytest.mark.parametrize("bar", [0, 1])
def test_linear_lps_bar_gold(bar):
    z = np.load(os.path.join(G, "linear_lps_bar.npz"))
    x, vol, block = z["x"], z["vol"], z["block"]
    blocks = (0, 1, 2) if bar == 0 else (3, 4, 5)
    fn = O.eval_linear_lps if bar == 0 else O.eval_model
    pts = np.nonzero(np.isin(block, blocks))[0]
    xb = x[pts].ravel()
    row, col = O.neighbor_search(xb, H)
    names = list(z["global_names"])
    tag = "LLPS" if bar == 0 else "LPS"
    for s in range(1, len(z["time"])):
        u = np.zeros((len(pts), 3))
        u[:, 0] = z["displacement_x"][s][pts]
        r = fn(xb, xb + u.ravel(), vol[pts], row, col, K, MU, H)
        F = r["force"].reshape(-1, 3) * vol[pts][:, None]
        assert np.abs(F - z["force"][s][pts]).max() <= 1e-3
        assert np.abs(r["theta"] - z["dilatation"][s][pts]).max() <= 1e-10
        assert np.abs(r["m"] - z["weighted_volume"][pts]).max() <= 1e-14
        for side, b in (("Left", blocks[0]), ("Right", blocks[2])):
            sel = block[pts] == b
            g = z["globals"][s][names.index("%s_Reaction_Force_%sX" % (side, tag))]
            assert abs(F[sel, 0].sum() - g) <= 1e-12 * abs(g)
