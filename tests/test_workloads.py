"""The synthetic inputs of the five benchmark configurations (no device).

Each generator's defaults are the configuration's stated sizes, spacings,
seeds and loads; the generated fields have the stated properties (checked on
smaller lattices where the full size is large): point order x fastest as
QuickGrid numbers points, jitter within +-0.05h, volumes h^3, horizon 3.015h;
the heterogeneous material's lognormal bulk modulus (median 130 GPa, sigma
0.3), mu = 0.6K and critical stretch uniform in [3e-4, 6e-4]; the prescribed
layers of the notched plate, the memory-scale plate and the cube; the bar's
Gaussian pulse; the dropped sphere's size and gap.
"""
import inspect

import numpy as np
import pytest

from peridigm_b200 import workloads as W


def _defaults(fn):
    return {k: p.default for k, p in inspect.signature(fn).parameters.items() if p.default is not p.empty}


def test_defaults_are_the_stated_configurations():
    assert _defaults(W.bar_wave) == dict(nx=100, ny=10, nz=10, h=1.0e-3)
    d = _defaults(W.notched_plate)
    assert (d["nx"], d["ny"], d["nz"], d["h"], d["seed"], d["s_c"], d["pull"], d["notch_cells"], d["nsteps"]) == \
        (400, 200, 4, 0.5e-3, 1, 5.0e-4, 2.0, 50, 5000)
    d = _defaults(W.plate_sphere)
    assert (d["nx"], d["ny"], d["nz"], d["h"], d["radius_cells"], d["s_c"], d["speed"], d["nsteps"]) == \
        (400, 400, 40, 0.25e-3, 25, 3.0e-4, 20.0, 2000)
    d = _defaults(W.qs_cube)
    assert (d["n"], d["h"], d["displacement"], d["load_steps"]) == (60, 1.0e-3, 1.0e-4, 20)
    d = _defaults(W.large_plate)
    assert (d["nx"], d["ny"], d["nz"], d["h"], d["seed"], d["nsteps"], d["pull"]) == (400, 400, 200, 0.5e-3, 4, 500, 1.0)
    assert d["nx"] * d["ny"] * d["nz"] == 32_000_000


def test_lattice_order_jitter_and_volume():
    h = 0.5e-3
    x0, vol = W.lattice(5, 4, 3, h)
    P = x0.reshape(-1, 3)
    assert np.allclose(P[1] - P[0], [h, 0, 0]) and np.allclose(P[5] - P[0], [0, h, 0])
    assert np.allclose(P[20] - P[0], [0, 0, h]) and np.all(vol == h ** 3)
    x1, _ = W.lattice(5, 4, 3, h, jitter=0.05, seed=1)
    assert np.abs(x1 - x0).max() <= 0.05 * h and np.abs(x1 - x0).max() > 0.04 * h
    assert np.array_equal(x1, W.lattice(5, 4, 3, h, jitter=0.05, seed=1)[0])


def test_bar_wave_pulse():
    w = W.bar_wave()
    assert w["x"].size == 3 * 10_000 and w["horizon"] == pytest.approx(3.015e-3)
    v = w["v0"].reshape(-1, 3)
    X = w["x"].reshape(-1, 3)[:, 0]
    assert np.all(v[:, 1:] == 0.0)
    assert np.allclose(v[:, 0], np.exp(-((X - 10e-3) ** 2) / (2 * (5e-3) ** 2)))
    assert v[:, 0].max() == pytest.approx(np.exp(-0.005), rel=1e-12)  # points 0.5h from the centre
    assert (w["K"], w["mu"], w["rho"], w["s_c"]) == (130.0e9, 78.0e9, 7800.0, None)


def test_notched_plate_layers_and_notch():
    w = W.notched_plate(nx=40, ny=20, nz=4, notch_cells=5)
    h = w["h"]
    P = w["x"].reshape(-1, 3)
    top, bottom = w["bcs"][0], w["bcs"][1]
    assert (top["coordinate"], top["a"], bottom["a"]) == (1, 2.0, -2.0)
    assert top["points"].size == bottom["points"].size == 3 * 40 * 4
    assert P[top["points"], 1].min() > (20 - 3) * h - 0.06 * h and P[bottom["points"], 1].max() < 3 * h + 0.06 * h
    pl = w["planes"][0]
    assert pl["normal"] == (0.0, 1.0, 0.0) and pl["lower_left"][1] == pytest.approx(10 * h)
    assert pl["bottom_length"] == pytest.approx(6 * h) and w["s_c"] == 5.0e-4


def test_large_plate_material_and_pulls():
    w = W.large_plate(nx=40, ny=40, nz=20)
    n = w["vol"].size
    lk = np.log(w["K"])
    assert np.exp(np.median(lk)) == pytest.approx(130.0e9, rel=0.01)
    assert np.std(lk) == pytest.approx(0.3, rel=0.02)
    assert np.array_equal(w["mu"], 0.6 * w["K"])
    assert w["s_c"].min() >= 3.0e-4 and w["s_c"].max() <= 6.0e-4
    assert np.mean(w["s_c"]) == pytest.approx(4.5e-4, rel=0.01)
    right, left = w["bcs"][0], w["bcs"][1]
    assert (right["coordinate"], right["a"], left["a"]) == (0, 1.0, -1.0)
    assert right["points"].size == left["points"].size == 3 * n // 40
    X = w["x"].reshape(-1, 3)[:, 0]
    assert X[left["points"]].max() < 3 * w["h"] + 0.06 * w["h"]


def test_quasi_static_cube():
    w = W.qs_cube(n=12, seed=1000)
    assert 50.0e9 <= w["K"] <= 200.0e9 and w["mu"] == 0.6 * w["K"]
    assert np.allclose(w["times"], np.linspace(0.0, 1.0, 21))
    clamped = [b for b in w["bcs"] if b["a"] == 0.0]
    pulled = [b for b in w["bcs"] if b["a"] != 0.0]
    assert sorted(b["coordinate"] for b in clamped) == [0, 1, 2]
    assert len(pulled) == 1 and pulled[0]["coordinate"] == 0 and pulled[0]["a"] == 1.0e-4
    assert pulled[0]["points"].size == 3 * 12 * 12


def test_dropped_sphere():
    w = W.plate_sphere(nx=60, ny=60, nz=6)
    blk = w["block"]
    ns = int((blk == 1).sum())
    k = np.arange(-25, 26)
    Z, Y, X = np.meshgrid(k, k, k, indexing="ij")
    assert ns == int((X ** 2 + Y ** 2 + Z ** 2 <= 625).sum())
    assert 65_000 <= ns <= 66_000  # about (4/3) pi 25^3
    P = w["x"].reshape(-1, 3)
    gap = P[blk == 1, 2].min() - P[blk == 0, 2].max()
    assert gap > w["horizon"] and gap > w["contact"]["r_contact"]
    v = w["v0"].reshape(-1, 3)
    assert np.all(v[blk == 1, 2] == -20.0) and np.all(v[blk == 0] == 0.0)
    assert w["s_c_blocks"] == [3.0e-4, -1.0]
