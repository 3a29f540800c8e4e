"""CPU-side checks of the boundary and the host logic (no kernel launches).

* libpd_b200.so loads and exports every function include/pd_b200.h declares;
* the ctypes table in peridigm_b200/_lib.py covers the header exactly;
* host helpers (elastic-constant conversions, neighbor-list formats, workload
  geometry) behave like the reference.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import _lib, plugins, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:int|const char\*|int64_t|void)\s+(pd_\w+)\s*\(", src, re.M))
    return names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(_lib.LIB_PATH)
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (pd_\w+)", out))
    declared = header_functions()
    assert declared, "no declarations parsed"
    assert declared <= exported, sorted(declared - exported)


def test_ctypes_table_matches_header():
    assert set(_lib.SIGNATURES) == header_functions()
    L = _lib.load()
    for name in _lib.SIGNATURES:
        assert getattr(L, name) is not None


def test_version_and_no_device_behaviour():
    L = _lib.load()
    assert b"sm_100a" in L.pd_version()
    h = C.c_void_p()
    cfg = _lib.Config(0, 1, 0, 0)
    rc = L.pd_create(C.byref(cfg), C.byref(h))
    if rc == 0:  # a CUDA device is present
        L.pd_destroy(h)
    else:
        assert rc == _lib.PD_ERR_CUDA
        assert not h.value
    assert L.pd_create(C.byref(_lib.Config(0, 7, 0, 0)), C.byref(h)) == _lib.PD_ERR_ARG


def test_elastic_constant_conversions():
    """Material::calculateBulkModulus/ShearModulus (Peridigm_Material.cpp:335-433)."""
    E, nu = 200e9, 0.3
    K = plugins.calculate_bulk_modulus({"Young's Modulus": E, "Poisson's Ratio": nu})
    mu = plugins.calculate_shear_modulus({"Young's Modulus": E, "Poisson's Ratio": nu})
    assert abs(K - E / (3 * (1 - 2 * nu))) < 1e-3
    assert abs(mu - E / (2 * (1 + nu))) < 1e-3
    assert abs(plugins.calculate_bulk_modulus({"Shear Modulus": mu, "Young's Modulus": E}) - K) / K < 1e-12
    with pytest.raises(ValueError):
        plugins.calculate_bulk_modulus({"Density": 1.0})


def test_neighbor_list_round_trip():
    row = np.array([0, 2, 2, 5])
    col = np.array([1, 2, 0, 1, 2], np.int32)
    nl = O.csr_to_nl(row, col)
    assert list(nl) == [2, 1, 2, 0, 3, 0, 1, 2]
    r2, c2 = O.nl_to_csr(nl, 3)
    assert np.array_equal(r2, row) and np.array_equal(c2, col)


def test_notched_plate_geometry():
    w = workloads.notched_plate(nx=40, ny=20, nz=2, h=1.0, notch_cells=5)
    x = w["x"].reshape(-1, 3)
    assert x.shape == (1600, 3)
    assert np.all(np.abs(x[:, 1] - 10.0) >= 0.45)  # no point near the notch plane
    row, col = O.neighbor_search(w["x"], w["horizon"], w["planes"])
    P = x
    cut = 0
    for i in range(len(P)):
        for j in col[row[i]:row[i + 1]]:
            assert not ((P[i, 1] - 10) * (P[j, 1] - 10) < 0 and max(P[i, 0], P[j, 0]) < 4.5)
        cut += 1
    # without the filter, bonds cross the notch
    r0, c0 = O.neighbor_search(w["x"], w["horizon"])
    assert len(c0) > len(col)
    bottom = {int(p) for p in w["bcs"][1]["points"]}
    assert all(x[p, 1] < 3.0 for p in bottom)


def test_bar_wave_initial_velocity():
    w = workloads.bar_wave()
    v = w["v0"][0::3]
    X = w["x"][0::3]
    i = np.argmax(v)
    assert abs(abs(X[i] - 10e-3) - 0.5e-3) < 1e-9  # two nearest centres straddle the pulse centre
    assert abs(v.max() - np.exp(-(0.5e-3) ** 2 / (2 * (5e-3) ** 2))) < 1e-12
