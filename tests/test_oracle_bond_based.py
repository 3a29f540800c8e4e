"""The CPU oracle of the elastic bond-based material, pinned to the reference.

* the C restatement of computeInternalForceElasticBondBased equals the
  reference's own compiled kernel (src/materials/elastic_bond_based.cxx)
  bit for bit, 3D and plane, with broken bonds;
* the ElasticBondBased3D / 2DPlaneStrain / 2DPlaneStress verification gold
  files (test/verification/ElasticBondBased, fixtures in tests/golden/):
  neighbor counts exactly, and an oracle explicit run matches Displacement
  and Velocity to 1e-9 and Force (= force density x volume) to 1e-3 absolute
  (the .comp tolerances), and the Block_Data reaction sums of block_1 and
  block_3 to 1e-3 absolute.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import workloads

G = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["bond_based_3d", "bond_based_plane_strain", "bond_based_plane_stress"]


@pytest.mark.parametrize("plane", [False, True])
def test_restatement_equals_compiled_reference(plane):
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built (the reference tree is absent)")
    x, vol = workloads.lattice(8, 5, 4, 1e-3, jitter=0.05, seed=3)
    row, col = O.neighbor_search(x, 3.015e-3)
    n = len(vol)
    rng = np.random.default_rng(0)
    y = x + rng.normal(0, 2e-6, x.size)
    dmg = (rng.random(len(col)) < 0.1).astype(float)
    nl = O.csr_to_nl(row, col)
    fr = O.ref_force_bond_based(x, y, vol, nl, n, 130e9, 3.015e-3, bond_damage=dmg, plane=plane, height=4e-3)
    fo = O.force_bond_based(x, y, vol, row, col, 130e9, 3.015e-3, bond_damage=dmg, plane=plane, height=4e-3)
    assert np.array_equal(fr, fo)


def bond_based_problem(z, row, col):
    """The gold case as an oracle.explicit_run problem: every point prescribed
    u_y = 0.001 y t / 1e-8 (u_x = 0, and u_z = 0 in 3D)."""
    rho, K, h, dt, T, plane, height = z["params"]
    n = len(z["vol"])
    x = z["x"]
    mask = np.full(n, 7 if not plane else 3, np.uint8)
    a = np.zeros(3 * n)
    a[1::3] = 0.001 * x[:, 1] / 1.0e-8
    return dict(x=x.ravel(), vol=z["vol"], rho=rho, K=K, mu=0.0, row=row, col=col, horizon=h, dt=dt,
                nsteps=int(round(T / dt)), material="bond_based", plane=bool(plane), height=height,
                bc_mask=mask, bc_a=a, bc_b=np.zeros(3 * n))


def _reaction(F, block, b):
    return np.array([F[c::3][block == b].sum() for c in range(3)])


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_bond_based_gold(case):
    z = np.load(os.path.join(G, case + ".npz"))
    h = z["params"][2]
    row, col = O.neighbor_search(z["x"].ravel(), h)
    assert np.array_equal(np.diff(row), z["nneigh"])
    prob = bond_based_problem(z, row, col)
    n = len(z["vol"])
    u, v = np.zeros(3 * n), np.zeros(3 * n)
    for k in range(1, len(z["time"])):
        p = dict(prob, nsteps=1, t0=z["time"][k - 1])
        r = O.explicit_run(p, u, v)
        u, v = r["u"], r["v"]
        F = r["force"] * np.repeat(z["vol"], 3)
        for c, ax in enumerate("XYZ"):
            assert np.abs(u[c::3] - z["Displacement" + ax][k]).max() < 1e-9
            assert np.abs(v[c::3] - z["Velocity" + ax][k]).max() < 1e-9
            assert np.abs(F[c::3] - z["Force" + ax][k]).max() < 1e-3
        for nm, b in (("Bottom_Reaction_Force", 0), ("Top_Reaction_Force", 2)):
            ref = np.array([z[nm + ax][k] for ax in "XYZ"])
            assert np.abs(_reaction(F, z["block"], b) - ref).max() < 1e-3
