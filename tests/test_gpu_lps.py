"""GPU parity of the LPS / damage / search kernels against the CPU oracle.

Tolerances (stated per test):
* FP64 path: the reference's own unit-test tolerances on the known answers;
  relative L2 force error <= 1e-11 against the oracle on the same inputs.
* split-FP32 path: relative L2 force error <= 1e-6, per-point force error
  <= 1e-5 of max|f|, bond-break sets identical except bonds whose FP64
  stretch lies within 1e-6*s_c of s_c.
* bond families and neighbor lists: bit-exact.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import Context, PDError, plugins, workloads

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make_cloud(nx=10, ny=9, nz=7, h=1.0e-3, seed=0, strain=2e-3):
    x, vol = workloads.lattice(nx, ny, nz, h, jitter=0.05, seed=seed)
    rng = np.random.default_rng(seed + 1)
    P = x.reshape(-1, 3)
    u = np.zeros_like(P)
    u[:, 0] = strain * P[:, 0] + 0.3 * strain * np.sin(P[:, 1] / (3 * h))
    u[:, 1] = -0.3 * strain * P[:, 1] + 0.5 * strain * P[:, 2]
    u[:, 2] = 0.2 * strain * np.cos(P[:, 0] / (4 * h)) * h
    u += rng.normal(0, 1e-3 * strain * h, size=u.shape)
    return x, vol, (P + u).ravel(), 3.015 * h


@pytest.mark.parametrize("precision", ["fp64", "split"])
@pytest.mark.parametrize("case", ["two_pts", "eight_pts", "three_pts"])
def test_unit_elastic_known_answers(case, precision):
    """testTwoPts / testEightPts / testThreePts through the ElasticMaterial mirror."""
    c = json.load(open(os.path.join(G, "unit_elastic.json")))[case]
    n = len(c["vol"])
    nl = np.array(c["nl"], np.int32)
    dm = plugins.DataManager(n, len(nl) - n)
    dm.getData("Model_Coordinates")[:] = c["x"]
    dm.getData("Volume")[:] = c["vol"]
    dm.getData("Coordinates", "NP1")[:] = c["y"]
    mat = plugins.ElasticMaterial({"Density": 7800.0, "Bulk Modulus": c["K"], "Shear Modulus": c["mu"],
                                   "Horizon": c["horizon"]}, precision=precision)
    mat.initialize(1.0, n, np.arange(n), nl, dm)
    mat.computeForce(1.0, n, np.arange(n), nl, dm)
    m, th, f = dm.getData("Weighted_Volume"), dm.getData("Dilatation", "NP1"), dm.getData("Force_Density", "NP1")
    tol = (lambda t: t) if precision == "fp64" else (lambda t: max(t, 2e-6))
    np.testing.assert_allclose(m, c["m"], rtol=c["m_tol"], atol=0)
    np.testing.assert_allclose(th, c["theta"], rtol=tol(c["theta_tol"]), atol=0)
    fe = np.array(c["force"])
    big = np.abs(fe) > 1e-3 * np.abs(fe).max()
    np.testing.assert_allclose(f[big], fe[big], rtol=tol(c["force_tol"]))
    assert np.all(np.abs(f[~big]) <= 1e-3 * np.abs(fe).max())


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_eval_model_matches_oracle(precision):
    """Weighted volume, dilatation, force and damage on a jittered lattice with a
    smooth non-uniform deformation and some bonds already broken."""
    x, vol, y, h = make_cloud()
    row, col = O.neighbor_search(x, h)
    rng = np.random.default_rng(7)
    # symmetric pre-broken bonds
    bd = np.zeros(len(col))
    n = len(vol)
    owner = np.repeat(np.arange(n), np.diff(row))
    pick = rng.random(len(col)) < 0.05
    pairs = {(min(i, j), max(i, j)) for i, j, p in zip(owner, col, pick) if p}
    for b, (i, j) in enumerate(zip(owner, col)):
        if (min(i, j), max(i, j)) in pairs:
            bd[b] = 1.0
    K, mu = 130e9, 78e9
    ref = O.eval_model(x, y, vol, row, col, K, mu, h, s_c=1.5e-3, dmg_n=bd)
    with Context(precision=precision) as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds()
        r2, c2 = ctx.bonds_csr()
        assert np.array_equal(r2, row) and np.array_equal(c2, col)
        ctx.material(K, mu, 7800.0)
        ctx.critical_stretch(1.5e-3)
        ctx.set_bond_damage(bd)
        f = ctx.compute_force(y)
        m = ctx.weighted_volume()
        th = ctx.field("Dilatation")
        bdn = ctx.field("Bond_Damage")
        nd = ctx.field("Damage")
    np.testing.assert_allclose(m, ref["m"], rtol=1e-14)
    if precision == "fp64":
        assert np.array_equal(bdn, ref["bond_damage"])
        np.testing.assert_allclose(nd, ref["damage"], rtol=0, atol=1e-15)
        assert rel_l2(th, ref["theta"]) < 1e-12
        assert rel_l2(f, ref["force"]) < 1e-11
    else:
        # stretch of every bond in FP64 decides which breaks may differ
        P, Y = x.reshape(-1, 3), y.reshape(-1, 3)
        s = (np.linalg.norm(Y[col] - Y[owner], axis=1) - np.linalg.norm(P[col] - P[owner], axis=1)) / \
            np.linalg.norm(P[col] - P[owner], axis=1)
        near = np.abs(s - 1.5e-3) <= 1e-6 * 1.5e-3
        assert np.array_equal(bdn[~near], ref["bond_damage"][~near])
        # a bond within 1e-6 s_c of s_c may break on one path and not the
        # other: its endpoints' dilatation and the force of every point within
        # a family of them are left out of the comparison (none on most seeds)
        touched = np.zeros(n, bool)
        touched[owner[near]] = True
        touched[col[near]] = True
        th_ok = ~touched
        f_ok = ~np.isin(np.arange(n), np.unique(np.concatenate([owner[touched[col]], np.nonzero(touched)[0]])))
        assert f_ok.sum() > 0.8 * n
        assert rel_l2(th[th_ok], ref["theta"][th_ok]) < 1e-6
        fm, rm = f.reshape(-1, 3)[f_ok], ref["force"].reshape(-1, 3)[f_ok]
        assert rel_l2(fm, rm) < 1e-6
        assert np.abs(fm - rm).max() < 1e-5 * np.abs(ref["force"]).max()


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_half_broken_bonds_match_oracle(precision):
    """Bond damage whose two halves differ (d_ij = 1, d_ji = 0; what a
    critical stretch differing between the blocks or points of a bond leaves
    behind): each row's own half enters its dilatation and t_ij, the partner's
    half t_ji, as in the reference's scatter from both families."""
    x, vol, y, h = make_cloud(seed=11)
    row, col = O.neighbor_search(x, h)
    n = len(vol)
    owner = np.repeat(np.arange(n), np.diff(row))
    bd = (np.random.default_rng(4).random(len(col)) < 0.08).astype(float)  # rows set independently
    K = 130e9 * np.exp(0.3 * np.random.default_rng(5).standard_normal(n))
    ref = O.eval_model(x, y, vol, row, col, K, 0.6 * K, h, s_c=None, dmg_n=bd)
    with Context(precision=precision) as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds()
        ctx.material(130e9, 78e9, 7800.0)
        ctx.material_field(K, 0.6 * K)
        ctx.set_bond_damage(bd)
        f = ctx.compute_force(y)
        assert np.array_equal(ctx.field("Bond_Damage"), bd)
    assert (bd != bd[np.array([row[j] + np.searchsorted(col[row[j]:row[j + 1]], i)
                                for i, j in zip(owner, col)])]).any(), "the halves should differ"
    assert rel_l2(f, ref["force"]) < (1e-11 if precision == "fp64" else 1e-6)


@pytest.mark.parametrize("case", ["1a", "1b", "2a", "2b", "3a"])
def test_finite_plane_known_answers(case):
    d = json.load(open(os.path.join(G, "finite_plane.json")))
    c = d["cases"][case]
    with Context() as ctx:
        ctx.set_points(d["points"], np.ones(8))
        ctx.set_horizons([d["horizon"]])
        ctx.build_bonds([c])
        row, col = ctx.bonds_csr()
    for i in range(8):
        assert set(col[row[i]:row[i + 1]].tolist()) == {j for j in range(8) if not c["exclude"][i][j]}


def test_bond_family_bit_exact_with_notch():
    w = workloads.notched_plate(nx=60, ny=40, nz=4, h=0.5e-3, notch_cells=15)
    row, col = O.neighbor_search(w["x"], w["horizon"], w["planes"])
    with Context() as ctx:
        ctx.set_points(w["x"], w["vol"])
        ctx.set_horizons([w["horizon"]])
        ctx.build_bonds(w["planes"])
        r2, c2 = ctx.bonds_csr()
        nl = ctx.get_bonds()
    assert np.array_equal(r2, row) and np.array_equal(c2, col)
    assert np.array_equal(nl, O.csr_to_nl(row, col))


def test_critical_time_step_matches_oracle():
    x, vol, y, h = make_cloud()
    row, col = O.neighbor_search(x, h)
    with Context(precision="fp64") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.set_bonds(O.csr_to_nl(row, col))
        ctx.material(130e9, 78e9, 7800.0)
        dt = ctx.critical_time_step()
    assert dt == O.critical_time_step(x, vol, row, col, 130e9, 7800.0, h)


def test_device_pointer_entry():
    """pd_compute_force_device on torch-owned device buffers equals the host entry,
    with pageable and with pinned host buffers (630 points: the last chunk is not a multiple of 64)."""
    torch = pytest.importorskip("torch")
    x, vol, y, h = make_cloud(seed=4)
    with Context(precision="split") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.build_bonds()
        ctx.material(130e9, 78e9, 7800.0)
        f_host = ctx.compute_force(y)
        yd = torch.tensor(y, dtype=torch.float64, device="cuda")
        fd = torch.zeros_like(yd)
        torch.cuda.synchronize()
        ctx.compute_force_device(yd.data_ptr(), fd.data_ptr())
        assert np.array_equal(fd.cpu().numpy(), f_host)
        # pinned host buffers (the force download overlaps the chunked force pass)
        yp = torch.tensor(y, dtype=torch.float64).pin_memory()
        fp = torch.zeros(len(y), dtype=torch.float64).pin_memory()
        for _ in range(2):
            ctx._ok(ctx.L.pd_compute_force(ctx.h, C.cast(yp.data_ptr(), C.POINTER(C.c_double)),
                                           C.cast(fp.data_ptr(), C.POINTER(C.c_double))))
            assert np.array_equal(fp.numpy(), f_host)


def test_sliced_damage_mirror_follows_the_state_cycle():
    """The 4-lanes-per-point split passes read a sliced copy of the bond damage.
    Through a cycle of trial evaluations, commits, damage set from the host and
    Verlet steps, their bond damage equals the CSR split path's (8 lanes per
    point, same per-bond arithmetic) exactly, and forces agree to 1e-6."""
    x, vol, _, h = make_cloud(seed=5)
    ys = [make_cloud(seed=5, strain=s)[2] for s in (1.0e-3, 2.0e-3, 2.5e-3, 3.5e-3, 4.5e-3)]
    n = len(vol)
    ctxs = [Context(precision="split", threads_per_point=t) for t in (4, 8)]
    try:
        for c in ctxs:
            c.set_points(x, vol)
            c.set_horizons([h])
            c.build_bonds()
            c.material(130e9, 78e9, 7800.0)
            c.critical_stretch(1.5e-3)
        nb = len(ctxs[0].bonds_csr()[1])
        rng = np.random.default_rng(3)

        def both(fn):
            return [fn(c) for c in ctxs]

        def same():
            d4, d8 = both(lambda c: c.field("Bond_Damage"))
            assert np.array_equal(d4, d8)
            return d4

        seen = []
        f4, f8 = both(lambda c: c.compute_force(ys[0]))
        assert rel_l2(f4, f8) < 1e-6
        seen.append(same().sum())
        both(lambda c: c.update_state())
        f4, f8 = both(lambda c: c.compute_force(ys[2]))  # trial, not committed
        assert rel_l2(f4, f8) < 1e-6
        seen.append(same().sum())
        f4, f8 = both(lambda c: c.compute_force(ys[1]))  # trial again from the committed damage
        assert rel_l2(f4, f8) < 1e-6
        same()
        both(lambda c: c.update_state())
        bd = (rng.random(nb) < 0.02).astype(float)
        row, col = ctxs[0].bonds_csr()
        owner = np.repeat(np.arange(n), np.diff(row))
        key = {(int(i), int(j)) for i, j, b in zip(owner, col, bd) if b}
        bd = np.array([1.0 if (int(i), int(j)) in key or (int(j), int(i)) in key else 0.0 for i, j in zip(owner, col)])
        both(lambda c: c.set_bond_damage(bd))
        f4, f8 = both(lambda c: c.compute_force(ys[3]))
        assert rel_l2(f4, f8) < 1e-6
        seen.append(same().sum())
        both(lambda c: c.update_state())
        dt = 0.5 * ctxs[0].critical_time_step()
        both(lambda c: c.set_state((ys[3] - x) * 0.0, np.zeros_like(x)))
        both(lambda c: c.verlet_run(dt, 3))
        same()
        f4, f8 = both(lambda c: c.compute_force(ys[4]))
        assert rel_l2(f4, f8) < 1e-6
        seen.append(same().sum())
        assert seen[-1] > seen[0] and seen[-1] > 0  # bonds broke along the way
    finally:
        for c in ctxs:
            c.close()


def test_errors_are_reported():
    with Context() as ctx:
        y = np.zeros(3)
        rc = ctx.L.pd_compute_force(ctx.h, y.ctypes.data_as(C.POINTER(C.c_double)), None)
        assert rc == 5  # PD_ERR_STATE: no points yet
        assert b"points" in ctx.L.pd_last_error(ctx.h)
        ctx.set_points(np.zeros(6) + np.array([0, 0, 0, 1, 0, 0.0]), np.ones(2))
        with pytest.raises(PDError):
            ctx.set_bonds(np.array([1, 5, 0], np.int32))  # neighbor id out of range
        ctx.set_bonds(np.array([1, 1, 0], np.int32))  # 0->1 without 1->0: a one-sided family
        ctx.set_horizons([2.0])
        ctx.material(1.0, 1.0, 1.0)
        # both points at one place: |Y| = 0, a NaN force (the reference terminates)
        with pytest.raises(PDError) as e:
            ctx.compute_force(np.zeros(6))
        assert e.value.code == 3
        # stretched: the one-sided bond scatters t_01 to both points, as the oracle does
        x = np.array([0, 0, 0, 1, 0, 0.0])
        y = np.array([0, 0, 0, 1.001, 0.0005, 0.0])
        f = ctx.compute_force(y)
        ref = O.eval_model(x, y, np.ones(2), np.array([0, 1, 1], np.int64), np.array([1], np.int32), 1.0, 1.0, 2.0)
        assert np.abs(f - ref["force"]).max() <= 1e-6 * np.abs(ref["force"]).max()
        assert np.abs(f[:3] + f[3:]).max() <= 1e-6 * np.abs(f).max()  # equal volumes: equal and opposite


def test_split_refuses_weighted_influence_across_horizons():
    """The split passes weight both halves of a bond with the owner's
    omega(|X|, h_i); with an influence function other than "One" and blocks of
    different horizons that would differ from the neighbor's omega(|X|, h_j),
    so the split context refuses (PD_ERR_UNSUPPORTED) where FP64 runs; with
    one horizon the Gaussian split force matches the FP64 path to 1e-6."""
    x, vol, y, h = make_cloud(seed=2)
    n = len(vol)
    block = (np.arange(n) % 2).astype(np.int32)
    row, col = O.neighbor_search(x, h)
    nl = O.csr_to_nl(row, col)  # symmetric families (one search radius), given through pd_set_bonds
    f = {}
    for precision in ("fp64", "split"):
        for horizons in ([h, 1.2 * h], [h, h]):
            with Context(precision=precision, influence="Gaussian") as ctx:
                ctx.set_points(x, vol, block)
                ctx.set_horizons(horizons)
                ctx.set_bonds(nl)
                for b in (0, 1):
                    ctx.material(130e9, 78e9, 7800.0, block=b)
                if precision == "split" and horizons[1] != horizons[0]:
                    with pytest.raises(PDError) as e:
                        ctx.compute_force(y)
                    assert e.value.code == 6 and b"horizon" in ctx.L.pd_last_error(ctx.h)
                    continue
                if horizons[1] == horizons[0]:
                    f[precision] = ctx.compute_force(y)
                else:
                    ctx.compute_force(y)  # FP64 handles both horizons (omega_j with h_j)
    assert rel_l2(f["split"], f["fp64"]) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "split", "fp64_sliced"])
def test_point_without_bonds(precision):
    """A point outside every horizon has an empty family (weighted volume 0):
    the reference's loops over it leave its dilatation 0 and its force 0
    (material_utilities.cxx:235-289, elastic.cxx:55-146), and the other
    points match the oracle."""
    x, vol, y, h = make_cloud(seed=4)
    far = x.reshape(-1, 3).max(axis=0) + 10.0 * h
    x2 = np.concatenate([x, far])
    vol2 = np.concatenate([vol, vol[:1]])
    y2 = np.concatenate([y, far + 1.0e-6])
    row, col = O.neighbor_search(x2, h)
    assert row[-1] == row[-2]  # the last point has no bonds
    ev = O.eval_model(x2, y2, vol2, row, col, 130e9, 78e9, h)
    with Context(precision=precision) as ctx:
        ctx.set_points(x2, vol2)
        ctx.set_horizons([h])
        ctx.build_bonds([])
        ctx.material(130e9, 78e9, 7800.0)
        f = ctx.compute_force(y2)
        th = ctx.field("Dilatation")
    assert th[-1] == 0.0 and np.all(f[-3:] == 0.0)
    assert np.all(np.isfinite(th)) and np.all(np.isfinite(f))
    tol = 1e-6 if precision == "split" else 1e-11
    assert rel_l2(f, ev["force"]) < tol
    assert rel_l2(th, ev["theta"]) < tol
