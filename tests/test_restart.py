"""Restart folders on the CPU: Matrix Market round trips, folder numbering,
the reference's file set, and write -> read through a stand-in context (the
host logic only; the GPU resume test is tests/test_gpu_restart.py)."""
import os

import numpy as np
import pytest

from peridigm_b200 import restart as R


class FakeContext:
    """The Context calls the restart module makes, on host arrays."""

    def __init__(self, n, row, rng):
        self.n = n
        self.row = row
        self.col = np.zeros(row[-1], np.int32)
        self.f = {"Model_Coordinates": rng.random(3 * n), "Displacement": rng.normal(size=3 * n),
                  "Velocity": rng.normal(size=3 * n), "Acceleration": rng.normal(size=3 * n),
                  "Force_Density": rng.normal(size=3 * n), "Contact_Force_Density": np.zeros(3 * n),
                  "Volume": rng.random(n), "Bond_Damage": (rng.random(row[-1]) < 0.3).astype(float)}
        self.f["Coordinates"] = self.f["Model_Coordinates"] + self.f["Displacement"]

    def field(self, name):
        return self.f[name].copy()

    def bonds_csr(self):
        return self.row, self.col

    def set_state(self, u, v):
        self.f["Displacement"], self.f["Velocity"] = np.array(u), np.array(v)

    def set_bond_damage(self, bd):
        self.f["Bond_Damage"] = np.array(bd)


def test_matrix_market_round_trip(tmp_path):
    v = np.array([0.1, -1e-300, 3.0, np.pi, 1e300, -0.0])
    p = str(tmp_path / "v.mat")
    R.write_matrix_market(p, v, "v")
    assert open(p).readline().startswith("%%MatrixMarket matrix array real general")
    assert np.array_equal(R.read_matrix_market(p), v)
    with open(p, "a") as fh:
        fh.write("1.0\n")
    with pytest.raises(ValueError):
        R.read_matrix_market(p)


def test_write_read_and_numbering(tmp_path):
    rng = np.random.default_rng(0)
    n = 7
    row = np.concatenate([[0], np.cumsum(rng.integers(1, 5, n))])
    a = FakeContext(n, row, rng)
    block = np.array([1, 0, 1, 1, 0, 0, 1])
    f1 = R.write(a, 0.035, str(tmp_path), block=block, block_ids=[3, 7], horizon=[0.5, 0.6], density=[1.0, 2.0])
    assert os.path.basename(f1) == "restart-000001"
    names = set(os.listdir(f1))
    for k in ("currentTime.txt", "blockIDs.mat", "horizon.mat", "volume.mat", "density.mat", "deltaTemperature.mat",
              "x.mat", "u.mat", "y.mat", "v.mat", "a.mat", "force.mat", "contactForce.mat", "externalForce.mat",
              "deltaU.mat", "scratch.mat", "BondData_block_3StateN.mat", "BondData_block_3StateNP1.mat",
              "BondData_block_7StateN.mat", "BondData_block_7StateNP1.mat"):
        assert k in names, k
    assert open(os.path.join(f1, "currentTime.txt")).read().splitlines()[0] == "Current time is "
    assert np.array_equal(R.read_matrix_market(os.path.join(f1, "horizon.mat")), np.where(block == 0, 0.5, 0.6))
    assert np.array_equal(R.read_matrix_market(os.path.join(f1, "blockIDs.mat")), np.where(block == 0, 3.0, 7.0))
    # block 7's bonds: points 0, 2, 3, 6 in order, each row in order
    sel = np.concatenate([np.arange(row[i], row[i + 1]) for i in (0, 2, 3, 6)])
    assert np.array_equal(R.read_matrix_market(os.path.join(f1, "BondData_block_7StateN.mat")),
                          a.f["Bond_Damage"][sel])
    b = FakeContext(n, row, np.random.default_rng(1))
    b.f["Model_Coordinates"], b.f["Volume"] = a.f["Model_Coordinates"], a.f["Volume"]
    t = R.read(b, path=str(tmp_path), block=block)
    assert t == 0.035
    for k in ("Displacement", "Velocity", "Bond_Damage"):
        assert np.array_equal(b.f[k], a.f[k])
    assert R.latest(str(tmp_path)) == f1
    f2 = R.write(b, 0.07, str(tmp_path), block=block, block_ids=[3, 7])
    assert os.path.basename(f2) == "restart-000002" and R.latest(str(tmp_path)) == f2
    c = FakeContext(n, row, np.random.default_rng(2))  # other points: refused
    with pytest.raises(ValueError):
        R.read(c, path=str(tmp_path), block=block)
    with pytest.raises(FileNotFoundError):
        R.read(c, path=str(tmp_path / "none"))
