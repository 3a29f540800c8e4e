"""The memory-scale heterogeneous plate at its stated size (400x400x200,
32,000,000 points, about 3.5e9 bonds, per-point K, mu = 0.6K and critical
stretch U[3e-4, 6e-4], +-1 m/s pulls), 10 Verlet steps from rest in each
bond-kernel precision, one context at a time (the FP64 sliced context alone
holds about 133 GB).

The oracle cannot run this size, so the check is between the paths whose
agreement with the oracle the smaller tests pin: the FP64 sliced passes
against the reference-order FP64 passes (u within 1e-12 relative L2, node
damage identical), and the split-FP32 passes against them (u within 1e-6
relative L2, at most one broken bond apart in any family). The bond
families' size (pd_num_bonds) is the same in all three.
"""
import numpy as np
import pytest

from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu

STEPS = 10


@pytest.fixture(scope="module")
def runs():
    w = workloads.large_plate()
    out = {}
    dt = None
    for precision in ("fp64", "fp64_sliced", "split"):
        with Context(precision=precision) as ctx:
            workloads.setup_context(ctx, w)
            if dt is None:
                dt = 0.7 * ctx.critical_time_step()
            ctx.verlet_run(dt, STEPS)
            out[precision] = (ctx.num_bonds(), ctx.field("Displacement"), ctx.field("Damage"),
                              ctx.field("Number_Of_Neighbors"))
    return out


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_full_size_fp64_sliced_matches_fp64(runs):
    nb, u, d, _ = runs["fp64_sliced"]
    nb0, u0, d0, _ = runs["fp64"]
    assert nb == nb0 > 3_000_000_000
    assert np.abs(u0).max() > 0.0
    assert rel_l2(u, u0) < 1e-12
    assert np.array_equal(d, d0)


def test_full_size_split_matches_fp64(runs):
    nb, u, d, nn = runs["split"]
    nb0, u0, d0, _ = runs["fp64"]
    assert nb == nb0
    assert rel_l2(u, u0) < 1e-6
    assert (np.abs(d - d0) * nn).max() <= 1.0 + 1e-9  # at most one broken bond of a family apart
