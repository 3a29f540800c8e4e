"""Generate the golden fixtures in tests/golden/ from the reference tree.

Run in a container that holds the reference source tree (default
/root/reference, override with PERIDIGM_REF):

    python tests/golden/make_golden.py

It reads the reference's unit-test known answers and the gold Exodus (netCDF
classic) files of its verification/regression tests, and writes small .npz /
.json fixtures. Nothing at test time reads the reference tree; the fixtures
are committed.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np
from scipy.io import netcdf_file

REF = os.environ.get("PERIDIGM_REF", "/root/reference")
OUT = os.path.dirname(os.path.abspath(__file__))


def _names(nc, key):
    if key not in nc.variables:
        return []
    return [b"".join(r).decode().strip() for r in nc.variables[key][:]]


def read_exodus_results(path):
    nc = netcdf_file(path, "r", mmap=False)
    res = {"time": np.array(nc.variables["time_whole"][:], dtype=np.float64)}
    res["x"] = np.stack([nc.variables["coordx"][:], nc.variables["coordy"][:], nc.variables["coordz"][:]], 1)
    for k, nm in enumerate(_names(nc, "name_nod_var")):
        res[nm] = np.array(nc.variables["vals_nod_var%d" % (k + 1)][:], dtype=np.float64)
    for k, nm in enumerate(_names(nc, "name_elem_var")):
        res[nm] = np.array(nc.variables["vals_elem_var%deb1" % (k + 1)][:], dtype=np.float64)
    nc.close()
    return res


# ---------------------------------------------------------------------------
# 1. ElasticMaterial unit tests (src/materials/unit_test/utPeridigm_ElasticMaterial.cpp)
# ---------------------------------------------------------------------------
def unit_elastic():
    cases = {}
    # testTwoPts :78-187
    cases["two_pts"] = {
        "x": [0.0, 0.0, 0.0, 1.0, 0.0, 0.0],
        "y": [0.0, 0.0, 0.0, 2.0, 0.0, 0.0],
        "vol": [1.0, 1.0],
        "nl": [1, 1, 1, 0],
        "K": 130.0e9, "mu": 78.0e9, "horizon": 10.0,
        "m": [1.0, 1.0], "m_tol": 1e-15,
        "theta": [3.0, 3.0], "theta_tol": 1e-15,
        "force": [2.34e12, 0, 0, -2.34e12, 0, 0], "force_tol": 1e-2,
    }
    # testEightPts :189-454: unit cube corners, z compressed to 0.98.
    x8 = [0, 0, 0, 0, 0, 1, 0, 1, 0, 0, 1, 1, 1, 0, 0, 1, 0, 1, 1, 1, 0, 1, 1, 1]
    y8 = [0, 0, 0, 0, 0, .98, 0, 1, 0, 0, 1, .98, 1, 0, 0, 1, 0, .98, 1, 1, 0, 1, 1, .98]
    nl8 = []
    for i in range(8):
        nl8.append(7)
        nl8.extend(j for j in range(8) if j != i)
    # hand solution on cell 0 (:355-405): t = (|y|-|x|)*9.75e10, factor 2
    f = [0.0, 0.0, 0.0]
    for (t, uvec) in [
        ((0.98 - 1.0) * 9.75e10, (0.0, 0.0, 1.0)),
        ((math.sqrt(1.0 + 0.98 * 0.98) - math.sqrt(2.0)) * 9.75e10,
         (0.0, 1.0 / math.sqrt(1.0 + 0.98 * 0.98), 0.98 / math.sqrt(1.0 + 0.98 * 0.98))),
        ((math.sqrt(1.0 + 0.98 * 0.98) - math.sqrt(2.0)) * 9.75e10,
         (1.0 / math.sqrt(1.0 + 0.98 * 0.98), 0.0, 0.98 / math.sqrt(1.0 + 0.98 * 0.98))),
        ((math.sqrt(2.0 + 0.98 * 0.98) - math.sqrt(3.0)) * 9.75e10,
         (1.0 / math.sqrt(2.0 + 0.98 * 0.98), 1.0 / math.sqrt(2.0 + 0.98 * 0.98),
          0.98 / math.sqrt(2.0 + 0.98 * 0.98))),
    ]:
        for k in range(3):
            f[k] += 2.0 * uvec[k] * t
    # signs per cell (:409-449)
    signs = [(1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1)]
    f8 = []
    for s in signs:
        f8.extend(s[k] * f[k] for k in range(3))
    cases["eight_pts"] = {
        "x": x8, "y": y8, "vol": [1.0] * 8, "nl": nl8,
        "K": 130.0e9, "mu": 78.0e9, "horizon": 10.0,
        "m": [12.0] * 8, "m_tol": 1e-12,
        "theta": [-0.01991593994643333] * 8, "theta_tol": 1e-12,
        "force": f8, "force_tol": 1e-11,
    }
    # testThreePts :456-664
    V = [0.9, 1.1, 0.8]
    t01 = (-2753550531.144094, -1510011581.595148, -621769474.7744727)
    t10 = (3398655528.6806289, 1863778838.308732, 767438345.18594845)
    t02 = (7736514797.0571524, 15402697641.41379, -11956431959.088315)
    t20 = (-8687228655.850972, -17295482505.73966, 13425717013.587864)
    t12 = (5110873051.7924152, -1252163897.689138, 6133047662.15088)
    t21 = (-4649613866.523322, 1139155397.2982139, -5579536639.827986)
    f3 = []
    f3 += [t01[k] * V[1] - t10[k] * V[1] + t02[k] * V[2] - t20[k] * V[2] for k in range(3)]
    f3 += [t10[k] * V[0] - t01[k] * V[0] + t12[k] * V[2] - t21[k] * V[2] for k in range(3)]
    f3 += [t20[k] * V[0] - t02[k] * V[0] + t21[k] * V[1] - t12[k] * V[1] for k in range(3)]
    cases["three_pts"] = {
        "x": [1.1, 2.6, -0.1, -2.0, 0.9, -0.3, 0.0, 0.01, 1.8],
        "y": [1.2, 2.4, -0.1, -1.9, 0.7, -0.8, 0.1, 0.21, 1.6],
        "vol": V, "nl": [2, 1, 2, 2, 0, 2, 2, 0, 1],
        "K": 130.0e9, "mu": 78.0e9, "horizon": 10.0,
        "m": [23.016479999999931, 18.64767999999997, 20.497599999999963], "m_tol": 1e-12,
        "theta": [-0.114127034572639, 0.08257537372985, -0.12166177890553], "theta_tol": 1e-11,
        "force": f3, "force_tol": 1e-10,
    }
    with open(os.path.join(OUT, "unit_elastic.json"), "w") as fh:
        json.dump(cases, fh, indent=1)


# ---------------------------------------------------------------------------
# 2. QuickGrid decks (PdQuickGrid discretization, QuickGrid.cxx:160-169,394-409,596-611)
# ---------------------------------------------------------------------------
def _cell_nbhd(cell, horizon, ncells):
    d = horizon / cell
    n = int(d)
    if abs(d - n) >= 0.5:
        n += 1
    return min(n, ncells)


def quickgrid(origin, length, npts, horizon, spherical):
    """Cell centres, cell volumes and the neighbor list of a PdQuickGrid
    tensor-product mesh: box neighborhood (NoOpNormFunction) by default,
    strict d^2 < r^2 for "Spherical"."""
    cells = [length[k] / npts[k] for k in range(3)]
    axes = [[origin[k] + cells[k] / 2 + i * cells[k] for i in range(npts[k])] for k in range(3)]
    nC = [_cell_nbhd(cells[k], horizon, npts[k]) for k in range(3)]
    nx, ny, nz = npts
    x, nl = [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                x.append((axes[0][i], axes[1][j], axes[2][k]))
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                nb = []
                p = (axes[0][i], axes[1][j], axes[2][k])
                for kk in range(max(0, k - nC[2]), min(nz, k + nC[2] + 1)):
                    for jj in range(max(0, j - nC[1]), min(ny, j + nC[1] + 1)):
                        for ii in range(max(0, i - nC[0]), min(nx, i + nC[0] + 1)):
                            if (ii, jj, kk) == (i, j, k):
                                continue
                            q = (axes[0][ii], axes[1][jj], axes[2][kk])
                            if spherical:
                                dx, dy, dz = q[0] - p[0], q[1] - p[1], q[2] - p[2]
                                if not (dx * dx + dy * dy + dz * dz - horizon * horizon < 0.0):
                                    continue
                            nb.append(ii + jj * nx + kk * nx * ny)
                nl.append(len(nb))
                nl.extend(nb)
    vol = cells[0] * cells[1] * cells[2]
    return np.array(x), np.full(len(x), vol), np.array(nl, dtype=np.int32)


def bond_breaking():
    d = os.path.join(REF, "test/verification/BondBreakingInitialVelocity")
    g = read_exodus_results(os.path.join(d, "BondBreakingInitialVelocity_gold.e"))
    x, vol, nl = quickgrid((0.0, 0.0, 0.0), (2.1, 2.0, 1.0), (2, 2, 1), 0.51, spherical=False)
    assert np.allclose(x, g["x"])
    v0 = np.zeros(12)
    # Node Set k = "k+1" (1-based point ids); y velocities from the deck.
    for pid, val in [(0, -244.939), (1, -244.959), (2, 244.939), (3, 244.959)]:
        v0[3 * pid + 1] = val
    np.savez_compressed(
        os.path.join(OUT, "bond_breaking.npz"), x=x, vol=vol, nl=nl, v0=v0,
        params=np.array([7800.0, 130.0e9, 60.0e9, 0.51, 0.02, 1.0e-8, 8.0e-5]),
        time=g["time"], disp_y=g["DisplacementY"], vel_y=g["VelocityY"], damage=g["Damage"],
        weighted_volume=g["Weighted_Volume"], dilatation=g["Dilatation"])


def contact_2x1x1():
    d = os.path.join(REF, "test/verification/Contact_2x1x1")
    g = read_exodus_results(os.path.join(d, "Contact_2x1x1_gold.e"))
    x, vol, nl = quickgrid((-2.0, -0.5, -0.5), (4.0, 1.0, 1.0), (2, 1, 1), 1.0, spherical=True)
    assert np.allclose(x, g["x"])
    v0 = np.array([1.0, 0, 0, -1.0, 0, 0])
    np.savez_compressed(
        os.path.join(OUT, "contact_2x1x1.npz"), x=x, vol=vol, nl=nl, v0=v0,
        # density, K, mu, horizon, search radius, freq, contact radius, spring, dt, final time
        params=np.array([7.8e-3, 130.0e3, 78.0e3, 1.0, 5.0, 100, 2.0, 1950.0e3, 4.150386640644e-8,
                         4.150386640644e-5]),
        time=g["time"], disp_x=g["DisplacementX"], vel_x=g["VelocityX"])


# ---------------------------------------------------------------------------
# 3. WaveInBar (Exodus hex mesh -> centroid/volume points, Peridigm_GeometryUtils.cpp:69-)
# ---------------------------------------------------------------------------
def _tet_volume(a, b, c, d):
    return abs(np.dot(b - a, np.cross(c - a, d - a))) / 6.0


def hex_volume(P):
    """Volume of a hexahedron from 24 tetrahedra on face barycentres and the
    body barycentre (the decomposition Peridigm_GeometryUtils.cpp:69-380 uses)."""
    faces = [(0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (0, 4, 7, 3), (0, 3, 2, 1), (4, 5, 6, 7)]
    fc = [P[list(f)].mean(0) for f in faces]
    c = 0.5 * (fc[4] + fc[5])
    v = 0.0
    for f, cf in zip(faces, fc):
        for k in range(4):
            v += _tet_volume(P[f[k]], P[f[(k + 1) % 4]], cf, c)
    return v


def wave_in_bar():
    d = os.path.join(REF, "test/regression/WaveInBar")
    g = netcdf_file(os.path.join(d, "WaveInBar.g"), "r", mmap=False)
    X = np.stack([g.variables["coordx"][:], g.variables["coordy"][:], g.variables["coordz"][:]], 1).astype(np.float64)
    conn = np.array(g.variables["connect1"][:]) - 1
    ns = np.array(g.variables["node_ns1"][:]) - 1
    g.close()
    vol = np.array([hex_volume(X[c]) for c in conn])
    in_set = set(ns.tolist())
    # Exodus node sets become the elements that contain one of their nodes
    # (Peridigm_ExodusDiscretization.cpp:557-566).
    elems = np.array([e for e, c in enumerate(conn) if any(int(k) in in_set for k in c)], dtype=np.int32)
    r = read_exodus_results(os.path.join(d, "WaveInBar_gold.e"))
    keep = [0, 1, 6, 11]
    out = dict(x=r["x"], vol=vol, initial_velocity_points=elems,
               # density, K, mu, horizon, dt, final time, output frequency
               params=np.array([2200.0, 14.90e9, 8.94e9, 0.00601, 9.0659e-08, 0.00002, 20]),
               time=r["time"][keep], keep=np.array(keep))
    for nm in ["DisplacementX", "DisplacementY", "DisplacementZ", "VelocityX", "VelocityY", "VelocityZ",
               "Force_DensityX", "Force_DensityY", "Force_DensityZ", "Dilatation", "Weighted_Volume"]:
        out[nm] = r[nm][keep]
    np.savez_compressed(os.path.join(OUT, "wave_in_bar.npz"), **out)


# ---------------------------------------------------------------------------
# 4. FinitePlane filter known answers (src/io/pdneigh/unit_test/utFinitePlaneFilter.cxx)
# ---------------------------------------------------------------------------
def finite_plane():
    """Planes of getCase_1a..3a (:118-161) and the expected exclusion flags of
    each point over the 8 corner points of a unit cube (:200-209, :310-319,
    :420-429, :528-537, :638-647), parsed from the reference test file."""
    import re

    path = os.path.join(REF, "src/io/pdneigh/unit_test/utFinitePlaneFilter.cxx")
    src = open(path).read()
    s2 = math.sqrt(2.0)
    env = {"sqrt2": s2, "sqrt": math.sqrt}
    cases = {}
    for name in ["1a", "1b", "2a", "2b", "3a"]:
        body = re.search(r"FinitePlane getCase_%s\(\)\{(.*?)\n\}" % name, src, re.S).group(1)
        vals = {}
        for var in ["n", "r0", "ub"]:
            comps = []
            for k in range(3):
                expr = re.search(r"%s\[%d\]\s*=\s*([^;]+);" % (var, k), body).group(1)
                comps.append(eval(expr, {}, env))
            vals[var] = comps
        for var in ["a", "b"]:
            vals[var] = eval(re.search(r"\b%s\s*=\s*([^,;]+)[,;]" % var, body).group(1), {}, env)
        test = src[src.index("FinitePlane plane = getCase_%s();" % name):]
        flags = []
        for k in range(8):
            arr = re.search(r"bool n%d\[\]\s*=\s*\{([^}]*)\}" % k, test).group(1)
            flags.append([int(t) for t in arr.split(",")])
        cases[name] = {"normal": vals["n"], "lower_left": vals["r0"], "bottom_unit": vals["ub"],
                       "bottom_length": vals["b"], "side_length": vals["a"], "exclude": flags}
    pts = [0, 0, 0, 1, 0, 0, 0, 1, 0, 1, 1, 0, 0, 0, 1, 1, 0, 1, 0, 1, 1, 1, 1, 1]
    with open(os.path.join(OUT, "finite_plane.json"), "w") as fh:
        json.dump({"points": pts, "horizon": 1.1 * math.sqrt(3.0), "cases": cases}, fh, indent=1)


def compression_qs():
    """Compression_QS_3x2x2 (test/regression/Compression_QS_3x2x2): 12-point
    PdQuickGrid, spherical neighborhood, 20 quasi-static load steps."""
    d = os.path.join(REF, "test/regression/Compression_QS_3x2x2")
    g = read_exodus_results(os.path.join(d, "Compression_QS_3x2x2_gold.e"))
    x, vol, nl = quickgrid((-1.5, -1.0, -1.0), (3.0, 2.0, 2.0), (3, 2, 2), 1.75, spherical=True)
    assert np.allclose(x, g["x"])
    # node sets (1-based ids in the deck) -> (points, coordinate, a, b) with u(t) = a t + b
    bcs = [([0, 3, 6, 9], 0, 0.0, 0.0), ([2, 5, 8, 11], 0, -0.1 / 0.00005, 0.0), ([0, 3], 2, 0.0, 0.0),
           ([0, 6], 1, 0.0, 0.0)]
    bc = np.array([(p, c, a, b) for pts, c, a, b in bcs for p in pts], dtype=np.float64)
    out = dict(x=x, vol=vol, nl=nl, bc=bc, params=np.array([7800.0, 130.0e9, 78.0e9, 1.75, 0.0, 0.00005, 20, 1.0e-2]),
               time=g["time"])
    for nm in ["DisplacementX", "DisplacementY", "DisplacementZ", "VelocityX", "VelocityY", "VelocityZ",
               "Force_DensityX", "Force_DensityY", "Force_DensityZ", "Weighted_Volume", "Dilatation"]:
        out[nm] = g[nm]
    np.savez_compressed(os.path.join(OUT, "compression_qs.npz"), **out)


# ---------------------------------------------------------------------------
# 7. ElasticBondBased verification tests (3D, plane strain, plane stress):
#    Exodus hex mesh (points = element centroids, Volume from the gold file),
#    every point prescribed u_y = 0.001*y*t/1e-8 (and u_x = 0, u_z = 0 in 3D),
#    Block_Data sums of Force over block_1 (bottom) and block_3 (top).
# ---------------------------------------------------------------------------
def _bond_based_case(sub, stem, gold, plane, height, mesh):
    d = os.path.join(REF, "test/verification/ElasticBondBased", sub)
    # the genesis mesh itself, for the discretization reader's tests
    g = netcdf_file(os.path.join(d, mesh), "r", mmap=False)
    mesh_out = dict(mesh_X=np.stack([g.variables["coord" + a][:] for a in "xyz"], 1).astype(np.float64),
                    mesh_blk_ids=np.array(g.variables["eb_prop1"][:], np.int64),
                    mesh_elem_map=np.array(g.variables["elem_num_map"][:], np.int64),
                    mesh_ns=np.array(g.variables["node_ns1"][:], np.int64))
    for b in range(g.dimensions["num_el_blk"]):
        mesh_out["mesh_conn%d" % (b + 1)] = np.array(g.variables["connect%d" % (b + 1)][:], np.int64)
    g.close()
    nc = netcdf_file(os.path.join(d, gold), "r", mmap=False)
    x = np.stack([nc.variables["coordx"][:], nc.variables["coordy"][:], nc.variables["coordz"][:]], 1).astype(np.float64)
    nblk = nc.dimensions["num_el_blk"]
    ev = _names(nc, "name_elem_var")
    n = x.shape[0]
    vol, nn, block = np.zeros(n), np.zeros(n, np.int64), np.full(n, -1, np.int32)
    for b in range(nblk):
        pts = np.array(nc.variables["connect%d" % (b + 1)][:, 0], np.int64) - 1  # element -> output point
        vol[pts] = nc.variables["vals_elem_var%deb%d" % (ev.index("Volume") + 1, b + 1)][0]
        nn[pts] = nc.variables["vals_elem_var%deb%d" % (ev.index("Number_Of_Neighbors") + 1, b + 1)][0]
        block[pts] = b
    assert (block >= 0).all()
    nv = _names(nc, "name_nod_var")
    gv = _names(nc, "name_glo_var")
    out = dict(x=x, vol=vol, block=block, nneigh=nn,
               time=np.array(nc.variables["time_whole"][:], np.float64),
               # density, bulk modulus, horizon, dt, final time, plane, height
               params=np.array([7800.0, 200.0e9, 0.751, 2.0e-9, 1.0e-8, float(plane), height]))
    for nm in ["DisplacementX", "DisplacementY", "DisplacementZ", "VelocityX", "VelocityY", "VelocityZ",
               "ForceX", "ForceY", "ForceZ"]:
        out[nm] = np.array(nc.variables["vals_nod_var%d" % (nv.index(nm) + 1)][:], np.float64)
    out.update(gold_nod_vars=np.array(nv), gold_elem_vars=np.array(ev), gold_glo_vars=np.array(gv))
    glo = np.array(nc.variables["vals_glo_var"][:], np.float64)
    for k, nm in enumerate(gv):
        out[nm] = glo[:, k]
    nc.close()
    out.update(mesh_out)
    np.savez_compressed(os.path.join(OUT, stem + ".npz"), **out)


def elastic_bond_based():
    _bond_based_case("ElasticBondBased3D", "bond_based_3d", "ElasticBondBased3D_gold.e", False, 0.0,
                     "ElasticBondBased3D.g")
    _bond_based_case("ElasticBondBased2DPlaneStrain", "bond_based_plane_strain",
                     "ElasticBondBased2DPlaneStrain_gold.e", True, 0.25, "ElasticBondBased2D.g")
    _bond_based_case("ElasticBondBased2DPlaneStress", "bond_based_plane_stress",
                     "ElasticBondBased2DPlaneStress_gold.e", True, 0.25, "ElasticBondBased2D.g")


def contact_perforation():
    """The genesis mesh of the restart regression deck (projectile block_1 and
    target block_2, HEX8, node set nodelist_1 = the projectile's nodes) for
    the restart test, which checks Run1 + restart + Run2 against the full run
    as the deck's driver does (its gold output is not in the tree)."""
    d = os.path.join(REF, "test/regression/Contact_Perforation_With_Restart")
    g = netcdf_file(os.path.join(d, "Contact_Perforation.g"), "r", mmap=False)
    ne = g.dimensions["num_elem"]
    emap = g.variables["elem_num_map"][:] if "elem_num_map" in g.variables else np.arange(1, ne + 1)
    out = dict(mesh_X=np.stack([g.variables["coord" + a][:] for a in "xyz"], 1).astype(np.float64),
               mesh_blk_ids=np.array(g.variables["eb_prop1"][:], np.int64),
               mesh_elem_map=np.array(emap, np.int64),
               mesh_ns=np.array(g.variables["node_ns1"][:], np.int64))
    for b in range(g.dimensions["num_el_blk"]):
        out["mesh_conn%d" % (b + 1)] = np.array(g.variables["connect%d" % (b + 1)][:], np.int64)
    g.close()
    np.savez_compressed(os.path.join(OUT, "contact_perforation.npz"), **out)


def compression_implicit():
    """Gold output of the two implicit-dynamics verification decks (two points
    at x = -1, 1, volume 2 each, horizon 2, K 130e9, mu 78e9, rho 7800,
    Newmark beta 0.25, gamma 0.5, dt 1e-5, five steps, absolute tolerance 1e-10):
    CompressionImplicit_2x1x1 (initial velocities +-1 in x) and
    CompressionImplicitEssentialBC_2x1x1 (point 0 held at u_x = 0.1, point 1
    at v_x = -1). Acceleration in the output is Compute_Acceleration
    (Force_Density / density)."""
    out = {}
    for stem in ("CompressionImplicit_2x1x1", "CompressionImplicitEssentialBC_2x1x1"):
        nc = netcdf_file(os.path.join(REF, "test/verification", stem, stem + "_gold.e"), "r", mmap=False)
        nv = _names(nc, "name_nod_var")
        key = "essential" if "Essential" in stem else "free"
        out[key + "_time"] = np.array(nc.variables["time_whole"][:], np.float64)
        out[key + "_x"] = np.stack([nc.variables["coord" + a][:] for a in "xyz"], 1).astype(np.float64)
        for nm in ("Displacement", "Velocity", "Force", "Force_Density", "Acceleration"):
            out[key + "_" + nm] = np.stack([np.array(nc.variables["vals_nod_var%d" % (nv.index(nm + c) + 1)][:],
                                                     np.float64) for c in "XYZ"], 2)
        nc.close()
    np.savez_compressed(os.path.join(OUT, "compression_implicit.npz"), **out)


def linear_lps_bar():
    """LinearLPSBar (test/verification/LinearLPSBar): two separate bars of 500
    points, blocks 1-3 Linear LPS Partial Volume and blocks 4-6 Elastic Partial
    Volume (LPS), K 160e10, mu 79.3e10, horizon 0.1502, every dof prescribed
    (u_x = 0.1 x t, u_y = u_z = 0), five quasi-static load steps to t = 1.
    Stores the points, volumes, blocks, the gold displacement (x only; y and
    z are zero), Force, Dilatation, Weighted_Volume and the reaction sums."""
    d = os.path.join(REF, "test/verification/LinearLPSBar")
    nc = netcdf_file(os.path.join(d, "LinearLPSBar_gold.e"), "r", mmap=False)
    x = np.stack([nc.variables["coord" + a][:] for a in "xyz"], 1).astype(np.float64)
    n = x.shape[0]
    nv, ev, gv = _names(nc, "name_nod_var"), _names(nc, "name_elem_var"), _names(nc, "name_glo_var")
    vol, wv = np.zeros(n), np.zeros(n)
    block = np.full(n, -1, np.int32)
    nt = nc.variables["time_whole"].shape[0]
    th = np.zeros((nt, n))
    for b in range(nc.dimensions["num_el_blk"]):
        pts = np.array(nc.variables["connect%d" % (b + 1)][:, 0], np.int64) - 1
        block[pts] = b
        vol[pts] = nc.variables["vals_elem_var%deb%d" % (ev.index("Volume") + 1, b + 1)][0]
        wv[pts] = nc.variables["vals_elem_var%deb%d" % (ev.index("Weighted_Volume") + 1, b + 1)][0]
        th[:, pts] = nc.variables["vals_elem_var%deb%d" % (ev.index("Dilatation") + 1, b + 1)][:]
    var = lambda nm: np.array(nc.variables["vals_nod_var%d" % (nv.index(nm) + 1)][:], np.float64)
    for c in "YZ":
        assert not var("Displacement" + c).any()
    out = dict(x=x, vol=vol, block=block, weighted_volume=wv, dilatation=th,
               time=np.array(nc.variables["time_whole"][:], np.float64), displacement_x=var("DisplacementX"),
               force=np.stack([var("Force" + c) for c in "XYZ"], 2),
               globals=np.array(nc.variables["vals_glo_var"][:], np.float64), global_names=np.array(gv))
    nc.close()
    np.savez_compressed(os.path.join(OUT, "linear_lps_bar.npz"), **out)


def main():
    linear_lps_bar()
    compression_implicit()
    contact_perforation()
    elastic_bond_based()
    unit_elastic()
    finite_plane()
    compression_qs()
    bond_breaking()
    contact_2x1x1()
    wave_in_bar()
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
