"""Restart on the GPU, as the reference's Contact_Perforation_With_Restart
regression does (test/regression/Contact_Perforation_With_Restart): Run1
(t = 0 .. 3.5e-2, 1000 steps of 3.5e-5) writes a restart folder, Run2 reads it
into a fresh context and runs to 7.0e-2; its last state equals the full
2000-step run within the deck's .comp tolerances (displacement 1e-9,
velocity 5e-7, damage 1e-12, absolute). Deck: projectile block_1 (LPS, K 160e3,
mu 79.3e3, rho 7.7e-3) at 50 in x (nodelist_1), target block_2 (K 14.9e3,
mu 8.94e3, rho 2.2e-3, critical stretch 0.001), horizon 0.51, short-range
contact (search radius 0.6 every 50 steps, contact radius 0.2, spring 1950e3)."""
import os

import numpy as np
import pytest

from _mesh import write_exodus
from peridigm_b200 import Context
from peridigm_b200 import discretization as D
from peridigm_b200 import restart as R

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")
DT, STEPS = 3.5e-5, 1000


def _deck(tmp_path):
    z = np.load(os.path.join(G, "contact_perforation.npz"))
    blocks = [(z["mesh_conn%d" % (b + 1)], "HEX8") for b in range(len(z["mesh_blk_ids"]))]
    path = str(tmp_path / "Contact_Perforation.g")
    write_exodus(path, z["mesh_X"], blocks, z["mesh_blk_ids"], z["mesh_elem_map"], [z["mesh_ns"]])
    return D.exodus(path)


def _setup(ctx, d):
    ctx.set_points(d["x"], d["vol"], d["block"])
    ctx.set_horizons([0.51, 0.51])
    ctx.build_bonds()
    ctx.material(160.0e3, 79.3e3, 7.7e-3, block=0)
    ctx.material(14.90e3, 8.94e3, 2.2e-3, block=1)
    ctx.critical_stretch(0.001, block=1)
    ctx.contact(0.6, 50, 0.2, 1950.0e3)


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_restart_equals_full_run(precision, tmp_path):
    d = _deck(tmp_path)
    n = len(d["vol"])
    v0 = np.zeros(3 * n)
    v0[3 * d["node_sets"]["nodelist_1"]] = 50.0
    with Context(precision=precision) as full:
        _setup(full, d)
        full.set_state(np.zeros(3 * n), v0)
        full.verlet_run(DT, 2 * STEPS)
        u_f, v_f, dmg_f = full.field("Displacement"), full.field("Velocity"), full.field("Damage")
    with Context(precision=precision) as run1:
        _setup(run1, d)
        run1.set_state(np.zeros(3 * n), v0)
        run1.verlet_run(DT, STEPS)
        folder = R.write(run1, STEPS * DT, str(tmp_path), block=d["block"], block_ids=d["block_ids"],
                         horizon=[0.51, 0.51], density=[7.7e-3, 2.2e-3])
    assert os.path.basename(folder) == "restart-000001"
    with Context(precision=precision) as run2:
        _setup(run2, d)
        t = R.read(run2, path=str(tmp_path), block=d["block"])
        assert t == STEPS * DT
        run2.verlet_run(DT, STEPS, t0=t)
        u_r, v_r, dmg_r = run2.field("Displacement"), run2.field("Velocity"), run2.field("Damage")
    assert np.abs(u_f).max() > 1.0  # the projectile moved through the target
    assert dmg_f.max() > 0.0
    assert np.abs(u_r - u_f).max() <= 1.0e-9
    assert np.abs(v_r - v_f).max() <= 5.0e-7
    assert np.abs(dmg_r - dmg_f).max() <= 1.0e-12
