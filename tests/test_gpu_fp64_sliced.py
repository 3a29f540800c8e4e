"""FP64 passes on the sliced bond stream (PD_FP64_SLICED) against the CPU oracle.

The FP64 LPS and critical-stretch formulas on the split path's layout (the
sliced stream at 4 lanes per point, X streamed in FP64, owner constants
folded, one division per bond), so sums and products round differently from
PD_FP64 in the last bits; the break test is the reference's
(|Y| - |X|)/|X| > s_c in FP64.

* Heterogeneous plate (the memory-scale plate's per-point K, mu = 0.6K and
  s_c in [3e-4, 6e-4] on a 32x32x16 lattice, pulled at +-3 m/s): 100 Verlet
  steps, bond damage identical to the oracle's, u and v within 1e-9 of max
  (the PD_FP64 bounds).
* One evaluation at the oracle's step-60 state advanced one step, while bonds
  break: force density within 1e-12 relative L2 of the oracle's, both halves'
  bond damage identical.
* Notched plate (one s_c, plane-filtered bond families, prescribed
  velocities): 20 steps within 1e-9 of max of the oracle's displacement.
* Linear LPS, bond-based and non-"One" influence contexts are refused
  (PD_ERR_UNSUPPORTED).
"""
import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import Context, PDError, workloads

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def hetero():
    w = workloads.large_plate(nx=32, ny=32, nz=16, pull=3.0)
    row, col = O.neighbor_search(w["x"], w["horizon"], w["planes"])
    dt = 0.7 * O.critical_time_step(w["x"], w["vol"], row, col, w["K"], w["rho"], w["horizon"])
    ref60 = O.explicit_run(workloads.oracle_problem(w, row, col, dt, 60), np.zeros_like(w["x"]), w["v0"])
    ref = O.explicit_run(workloads.oracle_problem(w, row, col, dt, 100), np.zeros_like(w["x"]), w["v0"])
    return w, row, col, dt, ref60, ref


def test_hetero_run_matches_oracle(hetero):
    w, row, col, dt, _, ref = hetero
    with Context(precision="fp64_sliced") as ctx:
        workloads.setup_context(ctx, w)
        r2, c2 = ctx.bonds_csr()
        assert np.array_equal(r2, row) and np.array_equal(c2, col)
        st = ctx.verlet_run(dt, 100)
        u, v, bd = ctx.field("Displacement"), ctx.field("Velocity"), ctx.field("Bond_Damage")
        nd = ctx.field("Damage")
    assert st["broken_bonds"] > 100, "the case should break bonds"
    assert np.array_equal(bd, ref["bond_damage"])
    assert np.abs(u - ref["u"]).max() <= 1e-9 * np.abs(ref["u"]).max()
    assert np.abs(v - ref["v"]).max() <= 1e-9 * np.abs(ref["v"]).max()
    cnt = np.diff(row)
    owner = np.repeat(np.arange(len(cnt)), cnt)
    nd_ref = np.bincount(owner, weights=ref["bond_damage"], minlength=len(cnt)) / np.maximum(cnt, 1)
    assert np.abs(nd - nd_ref).max() <= 1e-15


def test_hetero_one_evaluation_matches_oracle(hetero):
    """Both halves' break decisions and the force density at a state where
    bonds break (per-point s_c: the half-bond kernels)."""
    w, row, col, dt, ref60, _ = hetero
    y = w["x"] + ref60["u"] + dt * ref60["v"]
    bd0 = ref60["bond_damage"]
    assert bd0.sum() > 0
    ev = O.eval_model(w["x"], y, w["vol"], row, col, w["K"], w["mu"], w["horizon"], s_c=w["s_c"], dmg_n=bd0)
    with Context(precision="fp64_sliced") as ctx:
        workloads.setup_context(ctx, w)
        ctx.set_bond_damage(bd0)
        f = ctx.compute_force(y)
        bd = ctx.field("Bond_Damage")
        theta = ctx.field("Dilatation")
    assert (ev["bond_damage"] != bd0).sum() > 0, "the step should break more bonds"
    assert np.array_equal(bd, ev["bond_damage"])
    assert rel_l2(f, ev["force"]) < 1e-12
    assert rel_l2(theta, ev["theta"]) < 1e-12


def test_notched_plate_matches_oracle():
    w = workloads.notched_plate(nx=24, ny=16, nz=3, h=0.5e-3, notch_cells=6, nsteps=20)
    row, col = O.neighbor_search(w["x"], w["horizon"], w["planes"])
    with Context(precision="fp64_sliced") as ctx:
        workloads.setup_context(ctx, w)
        dt = 0.7 * ctx.critical_time_step()
        ctx.verlet_run(dt, 20)
        u = ctx.field("Displacement")
    ref = O.explicit_run(workloads.oracle_problem(w, row, col, dt, 20), np.zeros_like(w["x"]), w["v0"])
    assert np.abs(u - ref["u"]).max() <= 1e-9 * np.abs(ref["u"]).max()


@pytest.mark.parametrize("kind", ["linear_lps", "bond_based", "gaussian"])
def test_refuses_other_models(kind):
    x, vol = workloads.lattice(6, 5, 4, 1.0e-3, jitter=0.05, seed=3)
    h = 3.015e-3
    row, col = O.neighbor_search(x, h)
    with Context(precision="fp64_sliced", influence="Gaussian" if kind == "gaussian" else "One") as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([h])
        ctx.set_bonds(O.csr_to_nl(row, col))
        if kind == "linear_lps":
            ctx.material_linear_lps(130e9, 78e9, 7800.0)
        elif kind == "bond_based":
            ctx.material_bond_based(130e9, 7800.0)
        else:
            ctx.material(130e9, 78e9, 7800.0)
        with pytest.raises(PDError) as e:
            ctx.compute_force(x)
        assert e.value.code == 6 and b"PD_FP64_SLICED" in ctx.L.pd_last_error(ctx.h)
