"""GPU elastic bond-based material ("Elastic Bond Based") through the C ABI.

* pd_compute_force on a jittered lattice with broken bonds vs the reference's
  own compiled computeInternalForceElasticBondBased (3D and plane): FP64
  <= 1e-11 relative (max over points), split-FP32 <= 1e-6 relative L2;
* the ElasticBondBased3D / 2DPlaneStrain / 2DPlaneStress gold files
  (tests/golden/): Number_Of_Neighbors exactly; Displacement and Velocity
  to 1e-9 and Force (force density x volume) and the Block_Data reaction
  sums (pd_block_data) to 1e-3 absolute (the .comp tolerances) on the FP64 path; the
  split path within 1e-6 of each field's largest magnitude;
* a notched plate with critical-stretch damage vs the oracle's explicit run:
  FP64 break set identical, displacement <= 1e-9 relative; two runs
  bit-identical.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from peridigm_b200 import Context, workloads

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["bond_based_3d", "bond_based_plane_strain", "bond_based_plane_stress"]


@pytest.mark.parametrize("precision", ["fp64", "split"])
@pytest.mark.parametrize("plane", [False, True])
def test_force_matches_compiled_reference(precision, plane):
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    h = 1.0e-3
    x, vol = workloads.lattice(10, 8, 6, h, jitter=0.05, seed=3)
    n = len(vol)
    rng = np.random.default_rng(1)
    y = x + rng.normal(0.0, 2e-6, x.size)
    with Context(precision=precision) as ctx:
        ctx.set_points(x, vol)
        ctx.set_horizons([3.015 * h])
        ctx.build_bonds()
        ctx.material_bond_based(130.0e9, 7800.0, plane=plane, height=4 * h)
        row, col = ctx.bonds_csr()
        dmg = (rng.random(len(col)) < 0.05).astype(float)
        # symmetric damage, as the critical-stretch law produces it
        owner = np.repeat(np.arange(n), np.diff(row))
        key = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(owner, col))}
        for k, (a, b) in enumerate(zip(owner, col)):
            if a < b:
                dmg[key[(int(b), int(a))]] = dmg[k]
        ctx.set_bond_damage(dmg)
        f = ctx.compute_force(y)
    ref = O.ref_force_bond_based(x, y, vol, O.csr_to_nl(row, col), n, 130.0e9, 3.015 * h, bond_damage=dmg,
                                 plane=plane, height=4 * h)
    if precision == "fp64":
        assert np.abs(f - ref).max() <= 1e-11 * np.abs(ref).max()
    else:
        assert np.linalg.norm(f - ref) <= 1e-6 * np.linalg.norm(ref)


def _gold_ctx(ctx, z):
    rho, K, h, dt, T, plane, height = z["params"]
    n = len(z["vol"])
    x = z["x"]
    ctx.set_points(x.ravel(), z["vol"], z["block"])
    nblk = int(z["block"].max()) + 1
    ctx.set_horizons([h] * nblk)
    ctx.build_bonds()
    for b in range(nblk):
        ctx.material_bond_based(K, rho, block=b, plane=bool(plane), height=height)
    pts = np.arange(n)
    ctx.prescribed_displacement(pts, 0, 0.0, 0.0)
    if not plane:
        ctx.prescribed_displacement(pts, 2, 0.0, 0.0)
    for yv in np.unique(x[:, 1]):  # u_y = 0.001 y t / 1e-8
        ctx.prescribed_displacement(pts[x[:, 1] == yv], 1, 0.001 * yv / 1.0e-8, 0.0)
    ctx.set_state(np.zeros(3 * n), np.zeros(3 * n))
    return dt


@pytest.mark.parametrize("precision", ["fp64", "split"])
@pytest.mark.parametrize("case", CASES)
def test_bond_based_gold(case, precision):
    z = np.load(os.path.join(G, case + ".npz"))
    with Context(precision=precision) as ctx:
        dt = _gold_ctx(ctx, z)
        assert np.array_equal(ctx.field("Number_Of_Neighbors").astype(np.int64), z["nneigh"])
        V3 = np.repeat(z["vol"], 3)
        for k in range(1, len(z["time"])):
            ctx.verlet_run(dt, 1, t0=z["time"][k - 1])
            u, v = ctx.field("Displacement"), ctx.field("Velocity")
            F = ctx.field("Force_Density") * V3
            for c, ax in enumerate("XYZ"):
                gu, gv, gf = z["Displacement" + ax][k], z["Velocity" + ax][k], z["Force" + ax][k]
                if precision == "fp64":
                    assert np.abs(u[c::3] - gu).max() < 1e-9
                    assert np.abs(v[c::3] - gv).max() < 1e-9
                    assert np.abs(F[c::3] - gf).max() < 1e-3
                else:
                    assert np.abs(u[c::3] - gu).max() <= 1e-6 * max(np.abs(gu).max(), 1e-30) + 1e-15
                    assert np.abs(v[c::3] - gv).max() <= 1e-6 * max(np.abs(gv).max(), 1e-30) + 1e-15
                    assert np.abs(F[c::3] - gf).max() <= 1e-6 * np.abs(z["ForceY"][k]).max()
            for nm, b in (("Bottom_Reaction_Force", 0), ("Top_Reaction_Force", 2)):
                ref = np.array([z[nm + ax][k] for ax in "XYZ"])
                got = ctx.block_data("Force", b, "Sum")  # the Block_Data compute class on the device
                tol = 1e-3 if precision == "fp64" else 1e-6 * np.abs(ref).max()
                assert np.abs(got - ref).max() < tol


def _plate(precision):
    w = workloads.notched_plate(nx=40, ny=24, nz=4, h=0.5e-3, notch_cells=10, s_c=2.0e-4, pull=5.0)
    ctx = Context(precision=precision)
    ctx.set_points(w["x"], w["vol"])
    ctx.set_horizons([w["horizon"]])
    ctx.build_bonds(w["planes"])
    ctx.material_bond_based(w["K"], w["rho"])
    ctx.critical_stretch(w["s_c"])
    for bc in w["bcs"]:
        ctx.prescribed_displacement(bc["points"], bc["coordinate"], bc["a"], bc["b"])
    ctx.set_state(np.zeros_like(w["x"]), w["v0"])
    return w, ctx


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_notched_plate_matches_oracle(precision):
    nsteps = 150
    w, ctx = _plate(precision)
    with ctx:
        dt = 0.7 * ctx.critical_time_step()
        row, col = ctx.bonds_csr()
        st = ctx.verlet_run(dt, nsteps)
        u, bd = ctx.field("Displacement"), ctx.field("Bond_Damage")
    prob = dict(workloads.oracle_problem(w, row, col, dt, nsteps), material="bond_based")
    ref = O.explicit_run(prob, np.zeros_like(w["x"]), w["v0"])
    assert st["broken_bonds"] > 0, "the case should break bonds"
    if precision == "fp64":
        assert np.array_equal(bd, ref["bond_damage"])
        assert np.abs(u - ref["u"]).max() <= 1e-9 * np.abs(ref["u"]).max()
    else:
        assert np.sum(bd != ref["bond_damage"]) <= 0.01 * max(st["broken_bonds"], 1)
        assert np.abs(u - ref["u"]).max() <= 2e-3 * np.abs(ref["u"]).max()


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_deterministic(precision):
    out = []
    for _ in range(2):
        w, ctx = _plate(precision)
        with ctx:
            dt = 0.7 * ctx.critical_time_step()
            ctx.verlet_run(dt, 100)
            out.append((ctx.field("Displacement"), ctx.field("Bond_Damage")))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_quasi_static_rejects_bond_based():
    w, ctx = _plate("fp64")
    with ctx:
        with pytest.raises(Exception, match="LPS"):
            ctx.qs_load_step(0.0, 1.0, newton_tolerance=-1e-8)


def test_bond_based_output_file(tmp_path):
    """The 3D case written by peridigm_b200.output as the reference's deck asks
    (Volume, Displacement, Velocity, Force, Number_Of_Neighbors, the two
    Block_Data reaction forces, every step): the same variable names as the
    gold file and its values within the .comp tolerances."""
    from scipy.io import netcdf_file

    from peridigm_b200 import output

    z = np.load(os.path.join(G, "bond_based_3d.npz"))
    path = str(tmp_path / "ElasticBondBased3D.e")
    sums = {"Top_Reaction_Force": ("Force", 2, "Sum"), "Bottom_Reaction_Force": ("Force", 0, "Sum")}
    with Context(precision="fp64") as ctx:
        dt = _gold_ctx(ctx, z)
        with output.ExodusWriter(path, z["x"].ravel(), z["block"], vector_fields=["Displacement", "Velocity", "Force"],
                                 scalar_fields=["Volume", "Number_Of_Neighbors"], global_fields=list(sums)) as w:
            output.write_context_step(w, ctx, 0.0, sums)
            for k in range(1, len(z["time"])):
                ctx.verlet_run(dt, 1, t0=z["time"][k - 1])
                output.write_context_step(w, ctx, z["time"][k], sums)
    nc = netcdf_file(path, "r", mmap=False)
    try:
        names = lambda key: [b"".join(r).decode().strip("\x00 ") for r in nc.variables[key][:]]
        assert names("name_nod_var") == list(z["gold_nod_vars"])
        assert names("name_elem_var") == list(z["gold_elem_vars"])
        assert names("name_glo_var") == list(z["gold_glo_vars"])
        assert np.abs(nc.variables["time_whole"][:] - z["time"]).max() < 1e-14
        nod = names("name_nod_var")
        for j, nm in enumerate(nod):
            tol = 1e-3 if nm.startswith("Force") else 1e-9
            assert np.abs(nc.variables["vals_nod_var%d" % (j + 1)][:] - z[nm]).max() < tol
        glo = nc.variables["vals_glo_var"][:]
        for j, nm in enumerate(names("name_glo_var")):
            assert np.abs(glo[:, j] - z[nm]).max() < 1e-3
        for b in range(3):
            sel = z["block"] == b
            assert np.array_equal(nc.variables["vals_elem_var1eb%d" % (b + 1)][0], z["vol"][sel])
            assert np.array_equal(nc.variables["vals_elem_var2eb%d" % (b + 1)][0], z["nneigh"][sel].astype(float))
    finally:
        nc.close()
