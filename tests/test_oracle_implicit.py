"""The oracle's implicit Newmark restatement (oracle.implicit_newmark,
Peridigm::executeImplicit) against the gold output of the reference's
CompressionImplicit_2x1x1 and CompressionImplicitEssentialBC_2x1x1 decks.
The decks' .comp checks displacement at 1e-6 absolute; the restatement is held
to 1e-12 relative on displacement, velocity and force density, and its
Force_Density / density to the gold Acceleration (Compute_Acceleration)."""
import os

import numpy as np
import pytest

from oracle import oracle as O

G = os.path.join(os.path.dirname(__file__), "golden")
K, MU, RHO, H, DT = 130.0e9, 78.0e9, 7800.0, 2.0, 1.0e-5


def run_deck(key):
    z = np.load(os.path.join(G, "compression_implicit.npz"))
    x = z[key + "_x"].ravel()
    vol = np.array([2.0, 2.0])
    row, col = O.neighbor_search(x, H)
    u0 = z[key + "_Displacement"][0].ravel()
    v0 = z[key + "_Velocity"][0].ravel()
    bc = [0] if key == "essential" else []
    out = O.implicit_newmark(x, vol, row, col, K, MU, RHO, H, u0, v0, DT, 5, tol=1.0e-10, bc_dofs=bc)
    return z, out


@pytest.mark.parametrize("key", ["free", "essential"])
def test_implicit_restatement_matches_gold(key):
    z, out = run_deck(key)
    for s, (u, v, a, f, it) in enumerate(out, start=1):
        gu, gv = z[key + "_Displacement"][s].ravel(), z[key + "_Velocity"][s].ravel()
        gf = z[key + "_Force_Density"][s].ravel()
        ga = z[key + "_Acceleration"][s].ravel()
        assert np.abs(u - gu).max() <= 1e-6                      # the deck's .comp
        assert np.abs(u - gu).max() <= 1e-12 * np.abs(gu).max()
        assert np.abs(v - gv).max() <= 1e-12 * np.abs(gv).max()
        assert np.abs(f - gf).max() <= 1e-12 * np.abs(gf).max()
        assert np.abs(f / RHO - ga).max() <= 1e-12 * np.abs(ga).max()
        assert 1 <= it <= 11
