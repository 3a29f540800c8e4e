"""GPU short-range contact against the reference's gold file and the oracle.

* Contact_2x1x1 gold (test/verification/Contact_2x1x1): displacement and
  velocity to 1e-13 absolute (Contact_2x1x1.comp), FP64 and split paths.
* contact search + force drop-in (pd_contact_force) vs the oracle on a
  deformed two-body configuration, with and without friction: pair lists
  identical, force relative error <= 1e-12 (FP64 arithmetic in both).
* plate + sphere explicit run with contact and damage vs the oracle explicit
  run (FP64: displacement relative error <= 1e-9, identical bond damage).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_contact_2x1x1_gold(precision):
    z = np.load(os.path.join(G, "contact_2x1x1.npz"))
    rho, K, mu, h, rs, fq, rc, ks, dt, T = z["params"]
    with Context(precision=precision) as ctx:
        ctx.set_points(z["x"].ravel(), z["vol"])
        ctx.set_horizons([h])
        ctx.set_bonds(z["nl"])
        ctx.material(K, mu, rho)
        ctx.contact(rs, int(fq), rc, ks)
        ctx.set_state(np.zeros(6), z["v0"])
        for k in range(10):
            st = ctx.verlet_run(dt, 100, t0=k * 100 * dt)
            u, v = ctx.field("Displacement"), ctx.field("Velocity")
            tol = 1e-13 if precision == "fp64" else 1e-11  # split: y = x + u rounds differently
            assert np.abs(u[0::3] - z["disp_x"][k + 1]).max() < tol
            assert np.abs(v[0::3] - z["vel_x"][k + 1]).max() < tol
        assert st["contact_pairs"] == 2


@pytest.mark.parametrize("friction", [0.0, 0.3])
def test_contact_force_dropin_matches_oracle(friction):
    # bodies a horizon apart when bonded, then the sphere pushed 0.4h into the plate
    w = workloads.plate_sphere(nx=16, ny=16, nz=4, h=1.0e-3, radius_cells=3, gap_cells=3.5)
    n = len(w["vol"])
    rng = np.random.default_rng(2)
    y = w["x"] + rng.normal(0, 0.05e-3, size=w["x"].size)
    y[2::3][w["block"] == 1] -= 3.9e-3
    v = rng.normal(0, 1.0, size=w["x"].size)
    ct = w["contact"]
    with Context(precision="fp64") as ctx:
        ctx.set_points(w["x"], w["vol"], w["block"])
        ctx.set_horizons([w["horizon"]] * 2)
        ctx.build_bonds()
        ctx.material(w["K"], w["mu"], w["rho"], block=0)
        ctx.material(w["K"], w["mu"], w["rho"], block=1)
        ctx.contact(ct["r_search"], ct["freq"], ct["r_contact"], ct["k_spring"], friction)
        fc = ctx.contact_force(y, v)
        row, col = ctx.bonds_csr()
    crow, ccol = O.contact_search(y, ct["r_search"], row, col)
    assert len(ccol) > 0
    ref = O.contact_force(y, v, w["vol"], crow, ccol, ct["r_contact"], ct["k_spring"], w["horizon"], friction)
    assert np.abs(ref).max() > 0
    assert np.linalg.norm(fc - ref) <= 1e-12 * np.linalg.norm(ref)


def test_plate_sphere_explicit_matches_oracle():
    w = workloads.plate_sphere(nx=20, ny=20, nz=4, h=1.0e-3, radius_cells=4, s_c=1e-2, speed=150.0,
                               gap_cells=3.2, freq=5)
    nsteps = 300
    with Context(precision="fp64") as ctx:
        workloads.setup_context_blocks(ctx, w)
        dt = 0.7 * ctx.critical_time_step()
        row, col = ctx.bonds_csr()
        st = ctx.verlet_run(dt, nsteps)
        u, v, bd = ctx.field("Displacement"), ctx.field("Velocity"), ctx.field("Bond_Damage")
    assert st["contact_pairs"] > 0
    ref = O.explicit_run(workloads.oracle_problem_blocks(w, row, col, dt, nsteps), np.zeros_like(w["x"]), w["v0"])
    sphere = w["block"] == 1
    assert ref["v"][2::3][sphere].mean() > -140.0, "the sphere must have been slowed by contact"
    assert ref["bond_damage"].sum() < len(col)
    assert np.array_equal(bd, ref["bond_damage"])
    assert np.abs(u - ref["u"]).max() <= 1e-9 * np.abs(ref["u"]).max()
    assert np.abs(v - ref["v"]).max() <= 1e-9 * np.abs(ref["v"]).max()
