"""Linear LPS material on the GPU (pd_material_linear_lps).

* The reference's LinearLPSBar gold output: bar 1 (Linear LPS Partial Volume)
  and, in the same deck, bar 2 (Elastic Partial Volume = LPS) under
  u_x = 0.1 x t, t = 0.2 .. 1.0: Force within the .comp's 1e-3 absolute,
  Dilatation 1e-10, Weighted_Volume 1e-14, the Block_Data reaction sums
  1e-11 relative.
* A jittered lattice with critical-stretch damage and a smooth deformation
  against the oracle (LinearLPSPVMaterial loops): bond damage identical,
  dilatation 1e-12 and force 1e-11 relative L2.
* Five velocity-Verlet steps against the same loop driven by the oracle's
  force: displacement and velocity 1e-10 relative.
* The split-FP32 path (sliced stream, 4 lanes per point) against the same
  gold and the oracle at the split path's tolerances; other lane counts are
  refused (PD_ERR_UNSUPPORTED)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import Context, PDError, workloads

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("bar", [0, 1])
def test_linear_lps_bar_gold(bar):
    z = np.load(os.path.join(G, "linear_lps_bar.npz"))
    K, mu, h = 160.0e10, 79.3e10, 0.1502
    blocks = (0, 1, 2) if bar == 0 else (3, 4, 5)
    pts = np.nonzero(np.isin(z["block"], blocks))[0]
    x = z["x"][pts]
    vol = z["vol"][pts]
    local = z["block"][pts] - blocks[0]
    names = list(z["global_names"])
    tag = "LLPS" if bar == 0 else "LPS"
    with Context(precision="fp64") as ctx:
        ctx.set_points(x.ravel(), vol, local)
        ctx.set_horizons([h, h, h])
        ctx.build_bonds()
        for b in range(3):
            (ctx.material_linear_lps if bar == 0 else ctx.material)(K, mu, 8.05, block=b)
        assert np.abs(ctx.weighted_volume() - z["weighted_volume"][pts]).max() <= 1e-14
        for s in range(1, len(z["time"])):
            u = np.zeros_like(x)
            u[:, 0] = z["displacement_x"][s][pts]
            ctx.compute_force((x + u).ravel())
            F = ctx.field("Force").reshape(-1, 3)
            assert np.abs(F - z["force"][s][pts]).max() <= 1e-3
            assert np.abs(ctx.field("Dilatation") - z["dilatation"][s][pts]).max() <= 1e-10
            for side, b in (("Left", 0), ("Right", 2)):
                g = z["globals"][s][names.index("%s_Reaction_Force_%sX" % (side, tag))]
                assert abs(ctx.block_data("Force", b, "Sum")[0] - g) <= 1e-11 * abs(g)


def _cloud(seed=2):
    h = 1.0e-3
    x, vol = workloads.lattice(9, 8, 6, h, jitter=0.05, seed=seed)
    P = x.reshape(-1, 3)
    u = np.zeros_like(P)
    u[:, 0] = 3e-3 * P[:, 0] + 1e-3 * np.sin(P[:, 1] / (2 * h)) * h
    u[:, 1] = -1e-3 * P[:, 1] + 2e-3 * P[:, 2]
    u[:, 2] = 1e-3 * np.cos(P[:, 0] / (3 * h)) * h
    return x, vol, (P + u).ravel(), 3.015 * h


def test_linear_lps_matches_oracle_with_damage():
    x, vol, y, h = _cloud()
    K, mu, s_c = 130e9, 78e9, 2.5e-3
    row, col = O.neighbor_search(x, h)
    ref = O.eval_linear_lps(x, y, vol, row, col, K, mu, h, s_c=s_c)
    assert 0 < ref["bond_damage"].sum() < len(col)
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds()
        ctx.material_linear_lps(K, mu, 7800.0)
        ctx.critical_stretch(s_c)
        f = ctx.compute_force(y)
        assert np.array_equal(ctx.field("Bond_Damage"), ref["bond_damage"])
        assert rel_l2(ctx.field("Dilatation"), ref["theta"]) <= 1e-12
        assert rel_l2(f, ref["force"]) <= 1e-11


def test_linear_lps_verlet_matches_oracle_loop():
    x, vol, _, h = _cloud(seed=5)
    K, mu, rho = 130e9, 78e9, 7800.0
    n = len(vol)
    row, col = O.neighbor_search(x, h)
    rng = np.random.default_rng(9)
    v0 = rng.normal(0.0, 0.5, 3 * n)
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds()
        ctx.material_linear_lps(K, mu, rho)
        dt = 0.5 * ctx.critical_time_step()
        ctx.set_state(np.zeros(3 * n), v0)
        ctx.verlet_run(dt, 5)
        u_g, v_g = ctx.field("Displacement"), ctx.field("Velocity")
    u, v = np.zeros(3 * n), v0.copy()
    a = O.eval_linear_lps(x, x + u, vol, row, col, K, mu, h)["force"] / rho
    for _ in range(5):
        v = v + 0.5 * dt * a
        u = u + dt * v
        a = O.eval_linear_lps(x, x + u, vol, row, col, K, mu, h)["force"] / rho
        v = v + 0.5 * dt * a
    assert rel_l2(u_g, u) <= 1e-10
    assert rel_l2(v_g, v) <= 1e-10


@pytest.mark.parametrize("bar", [0])
def test_split_linear_lps_bar_gold(bar):
    """Split-FP32 (sliced stream, 4 lanes per point): Force within 1e-6 of the
    largest gold force, Dilatation 1e-6 of the largest, reaction sums 1e-6."""
    z = np.load(os.path.join(G, "linear_lps_bar.npz"))
    K, mu, h = 160.0e10, 79.3e10, 0.1502
    pts = np.nonzero(np.isin(z["block"], (0, 1, 2)))[0]
    x, vol, local = z["x"][pts], z["vol"][pts], z["block"][pts]
    names = list(z["global_names"])
    with Context(precision="split") as ctx:
        ctx.set_points(x.ravel(), vol, local)
        ctx.set_horizons([h, h, h])
        ctx.build_bonds()
        for b in range(3):
            ctx.material_linear_lps(K, mu, 8.05, block=b)
        for s in range(1, len(z["time"])):
            u = np.zeros_like(x)
            u[:, 0] = z["displacement_x"][s][pts]
            ctx.compute_force((x + u).ravel())
            gF = z["force"][s][pts]
            assert np.abs(ctx.field("Force").reshape(-1, 3) - gF).max() <= 1e-6 * np.abs(gF).max()
            gth = z["dilatation"][s][pts]
            assert np.abs(ctx.field("Dilatation") - gth).max() <= 1e-6 * np.abs(gth).max()
            for side, b in (("Left", 0), ("Right", 2)):
                g = z["globals"][s][names.index("%s_Reaction_Force_LLPSX" % side)]
                assert abs(ctx.block_data("Force", b, "Sum")[0] - g) <= 1e-6 * abs(g)


def test_split_linear_lps_matches_oracle():
    """Split-FP32 against the oracle: bond-break sets identical except bonds
    within 1e-6 s_c of s_c; dilatation and force 1e-6 relative L2."""
    x, vol, y, h = _cloud()
    K, mu, s_c = 130e9, 78e9, 2.5e-3
    row, col = O.neighbor_search(x, h)
    ref = O.eval_linear_lps(x, y, vol, row, col, K, mu, h, s_c=s_c)
    n = len(vol)
    owner = np.repeat(np.arange(n), np.diff(row))
    P, Y = x.reshape(-1, 3), y.reshape(-1, 3)
    zeta = np.linalg.norm(P[col] - P[owner], axis=1)
    s = (np.linalg.norm(Y[col] - Y[owner], axis=1) - zeta) / zeta
    near = np.abs(s - s_c) <= 1e-6 * s_c
    with Context(precision="split") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds()
        ctx.material_linear_lps(K, mu, 7800.0)
        ctx.critical_stretch(s_c)
        f = ctx.compute_force(y)
        bd = ctx.field("Bond_Damage")
        assert np.array_equal(bd[~near], ref["bond_damage"][~near])
        if not near.any():
            assert rel_l2(ctx.field("Dilatation"), ref["theta"]) <= 1e-6
            assert rel_l2(f, ref["force"]) <= 1e-6


def test_split_linear_lps_needs_four_lanes():
    x, vol, y, h = _cloud()
    with Context(precision="split", threads_per_point=8) as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds()
        ctx.material_linear_lps(130e9, 78e9, 7800.0)
        with pytest.raises(PDError) as e:
            ctx.compute_force(y)
        assert e.value.code == 6
