"""The CPU oracle against the reference's own known answers and gold files.

Pins oracle/pd_oracle.c before it is trusted as the checker of the CUDA path:
* ElasticMaterial unit tests (src/materials/unit_test/utPeridigm_ElasticMaterial.cpp)
* FinitePlane filter unit tests (src/io/pdneigh/unit_test/utFinitePlaneFilter.cxx)
* BondBreakingInitialVelocity, Contact_2x1x1 (test/verification) and WaveInBar
  (test/regression) gold Exodus files, at the tolerances of their .comp files.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

G = os.path.join(os.path.dirname(__file__), "golden")


def rel_eq(a, b, tol):
    """TEST_FLOATING_EQUALITY: |a-b| / max(|a|,|b|) <= tol (zero pairs pass)."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    den = np.maximum(np.abs(a), np.abs(b))
    err = np.where(den > 0, np.abs(a - b) / np.where(den > 0, den, 1), 0.0)
    return bool(np.all(err <= tol)), float(err.max())


@pytest.mark.parametrize("case", ["two_pts", "eight_pts", "three_pts"])
def test_unit_elastic_known_answers(case):
    c = json.load(open(os.path.join(G, "unit_elastic.json")))[case]
    n = len(c["vol"])
    row, col = O.nl_to_csr(c["nl"], n)
    r = O.eval_model(c["x"], c["y"], c["vol"], row, col, c["K"], c["mu"], c["horizon"])
    assert rel_eq(r["m"], c["m"], c["m_tol"])[0]
    assert rel_eq(r["theta"], c["theta"], c["theta_tol"])[0]
    f = np.array(c["force"])
    big = np.abs(f) > 1e-3 * np.abs(f).max()
    ok, err = rel_eq(r["force"][big], f[big], c["force_tol"])
    assert ok, err
    assert np.all(np.abs(r["force"][~big]) <= 1e-3 * np.abs(f).max())


@pytest.mark.parametrize("case", ["two_pts", "eight_pts", "three_pts"])
def test_oracle_equals_compiled_reference(case):
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference tree absent when built)")
    c = json.load(open(os.path.join(G, "unit_elastic.json")))[case]
    n = len(c["vol"])
    row, col = O.nl_to_csr(c["nl"], n)
    r = O.eval_model(c["x"], c["y"], c["vol"], row, col, c["K"], c["mu"], c["horizon"])
    ref = O.ref_eval(c["x"], c["y"], c["vol"], np.array(c["nl"], np.int32), n, c["K"], c["mu"], c["horizon"])
    for k in ("m", "theta", "force"):
        assert np.array_equal(r[k], ref[k]), k


@pytest.mark.parametrize("case", ["1a", "1b", "2a", "2b", "3a"])
def test_finite_plane_known_answers(case):
    d = json.load(open(os.path.join(G, "finite_plane.json")))
    c = d["cases"][case]
    x = np.array(d["points"], float)
    row, col = O.neighbor_search(x, d["horizon"], [c])
    for i in range(8):
        kept = set(col[row[i]:row[i + 1]].tolist())
        assert kept == {j for j in range(8) if not c["exclude"][i][j]}, (case, i)


def test_bond_breaking_gold():
    """BondBreakingInitialVelocity: Disp/Vel 1e-9, Damage 1e-3 (BondBreakingInitialVelocity.comp)."""
    z = np.load(os.path.join(G, "bond_breaking.npz"))
    rho, K, mu, h, sc, dt, T = z["params"]
    row, col = O.nl_to_csr(z["nl"], 4)
    u, v, bd = np.zeros(12), z["v0"].copy(), None
    for k in range(8):
        r = O.explicit_run(dict(x=z["x"].ravel(), vol=z["vol"], rho=rho, K=K, mu=mu, row=row, col=col, horizon=h,
                                dt=dt, nsteps=1000, s_c=sc, t0=k * 1000 * dt), u, v, bd)
        u, v, bd = r["u"], r["v"], r["bond_damage"]
        assert np.abs(u[1::3] - z["disp_y"][k + 1]).max() < 1e-9
        assert np.abs(v[1::3] - z["vel_y"][k + 1]).max() < 1e-9
        assert np.abs(r["damage"] - z["damage"][k + 1]).max() < 1e-3
    assert list(r["damage"]) == [0.0, 1.0, 0.0, 1.0]


def test_contact_2x1x1_gold():
    """Contact_2x1x1: Disp/Vel 1e-13 (Contact_2x1x1.comp)."""
    z = np.load(os.path.join(G, "contact_2x1x1.npz"))
    rho, K, mu, h, rs, fq, rc, ks, dt, T = z["params"]
    row, col = O.nl_to_csr(z["nl"], 2)
    assert len(col) == 0
    u, v = np.zeros(6), z["v0"].copy()
    for k in range(10):
        r = O.explicit_run(dict(x=z["x"].ravel(), vol=z["vol"], rho=rho, K=K, mu=mu, row=row, col=col, horizon=h,
                                dt=dt, nsteps=100, t0=k * 100 * dt,
                                contact=dict(r_search=rs, freq=int(fq), r_contact=rc, k_spring=ks, horizon=h)), u, v)
        u, v = r["u"], r["v"]
        assert np.abs(u[0::3] - z["disp_x"][k + 1]).max() < 1e-13
        assert np.abs(v[0::3] - z["vel_x"][k + 1]).max() < 1e-13


def test_wave_in_bar_gold():
    """WaveInBar: Weighted_Volume 1e-15 (pins the neighbor search), Dilatation 5e-13,
    Disp 5e-14, Vel 1e-8, Force_Density 5.0 (WaveInBar.comp)."""
    z = np.load(os.path.join(G, "wave_in_bar.npz"))
    rho, K, mu, h, dt, T, fq = z["params"]
    x = z["x"].ravel().copy()
    n = len(z["vol"])
    row, col = O.neighbor_search(x, h)
    m = O.weighted_volume(x, z["vol"], row, col, h)
    assert np.abs(m - z["Weighted_Volume"][0]).max() < 1e-15
    v = np.zeros(3 * n)
    v[3 * z["initial_velocity_points"]] = -100.0
    u = np.zeros(3 * n)
    steps = [int(k) * int(fq) for k in z["keep"]]
    prev = 0
    for k, s in enumerate(steps):
        if s > prev:
            r = O.explicit_run(dict(x=x, vol=z["vol"], rho=rho, K=K, mu=mu, row=row, col=col, horizon=h, dt=dt,
                                    nsteps=s - prev, t0=prev * dt), u, v)
            u, v, f, th = r["u"], r["v"], r["force"], r["theta"]
            prev = s
        else:
            r = O.eval_model(x, x + u, z["vol"], row, col, K, mu, h)
            f, th = r["force"], r["theta"]
        for c, ax in enumerate("XYZ"):
            assert np.abs(u[c::3] - z["Displacement" + ax][k]).max() < 5e-14
            assert np.abs(v[c::3] - z["Velocity" + ax][k]).max() < 1e-8
            assert np.abs(f[c::3] - z["Force_Density" + ax][k]).max() < 5.0
        assert np.abs(th - z["Dilatation"][k]).max() < 5e-13


def test_neighbor_search_matches_brute_force():
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, size=(400, 3)).ravel()
    h = 0.17
    row, col = O.neighbor_search(x, h)
    P = x.reshape(-1, 3)
    for i in range(0, 400, 7):
        d = P - P[i]
        d2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]
        exp = np.nonzero(d2 <= h * h)[0]
        exp = exp[exp != i]
        assert np.array_equal(col[row[i]:row[i + 1]], exp)


def test_critical_time_step_formula():
    x = np.array([0, 0, 0, 1e-3, 0, 0.0])
    row, col = np.array([0, 1, 2]), np.array([1, 0], np.int32)
    dt = O.critical_time_step(x, np.array([1e-9, 1e-9]), row, col, 130e9, 7800.0, 3e-3)
    k = 18 * 130e9 / (np.pi * 3e-3 ** 4)
    assert abs(dt - np.sqrt(2 * 7800 / (1e-9 * k / 1e-3))) < 1e-20
