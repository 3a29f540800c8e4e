"""Host-side pieces of the measurement and the Python boundary (no device):

* the algorithmic byte model of the bond passes (17 B per bond and pass for
  the split path, 29 B for the FP64 sliced path, 58 B per step for FP64; the
  per-point terms), which every roofline fraction divides by;
* the streamed-slot count of the sliced bond stream (8-owner slices padded to
  their longest row in groups of 4 bonds), which scales the ncu traffic;
* the precision names Context accepts (an unknown name is refused before any
  device is touched).
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402
from peridigm_b200 import Context  # noqa: E402


def test_algorithmic_bytes():
    nb, n = 1_000_000, 10_000
    sp = bench.algorithmic_bytes(nb, n, "split")
    assert sp == {"dilatation": 17 * nb + 80 * n, "force": 17 * nb + 193 * n, "step": 34 * nb + 176 * n}
    f6s = bench.algorithmic_bytes(nb, n, "fp64_sliced")
    assert f6s["dilatation"] == 29 * nb + 120 * n and f6s["force"] == 29 * nb + 225 * n
    assert f6s["step"] == bench.algorithmic_bytes(nb, n, "fp64")["step"] == 58 * nb + 200 * n


class _Rows:
    def __init__(self, lens):
        self.lens = np.asarray(lens, dtype=np.float64)

    def field(self, name):
        assert name == "Number_Of_Neighbors"
        return self.lens


def test_sliced_slots():
    # one slice of 8 rows, longest 9 bonds -> 3 groups of 4 -> 3 x 32 slots
    assert bench.sliced_slots(_Rows([9, 1, 2, 3, 4, 5, 6, 7])) == 96
    # two slices (the second padded with empty rows): ceil(12/4) + ceil(5/4) groups
    assert bench.sliced_slots(_Rows([12] * 8 + [5, 0, 1])) == 32 * (3 + 2)
    rng = np.random.default_rng(0)
    lens = rng.integers(80, 123, size=1000)
    pad = np.concatenate([lens, np.zeros((-lens.size) % 8, np.int64)]).reshape(-1, 8)
    assert bench.sliced_slots(_Rows(lens)) == 32 * int(((pad.max(axis=1) + 3) // 4).sum())
    assert bench.sliced_slots(_Rows(lens)) >= lens.sum()


def test_unknown_precision_is_refused():
    with pytest.raises(ValueError):
        Context(precision="fp16")
