"""Exodus II output writer (peridigm_b200.output), on the CPU: the file's
layout is the reference's (names, dimensions, SPHERE element blocks of
points, per-block element variables, global variables), and the values read
back are the values written."""
import numpy as np
from scipy.io import netcdf_file

from peridigm_b200 import output


def _names(nc, key):
    return [b"".join(r).decode().strip("\x00 ") for r in nc.variables[key][:]]


def test_round_trip_layout(tmp_path):
    rng = np.random.default_rng(0)
    n = 30
    x = rng.random(3 * n)
    block = np.repeat([0, 1, 2], 10)
    rng.shuffle(block)
    path = str(tmp_path / "out.e")
    steps = []
    with output.ExodusWriter(path, x, block, block_ids=[1, 2, 3], node_sets={"nodelist_1": np.arange(0, n, 2)},
                             vector_fields=["Displacement", "Force"], scalar_fields=["Volume", "Damage"],
                             global_fields=["Top_Reaction_Force", "Kinetic_Energy"],
                             scalar_globals=["Kinetic_Energy"]) as w:
        for k in range(3):
            rec = dict(vectors={"Displacement": rng.random(3 * n), "Force": rng.random(3 * n)},
                       scalars={"Volume": rng.random(n), "Damage": rng.random(n)},
                       globals_={"Top_Reaction_Force": rng.random(3), "Kinetic_Energy": rng.random()})
            w.write_step(1e-9 * k, **rec)
            steps.append(rec)
    nc = netcdf_file(path, "r", mmap=False)
    try:
        assert _names(nc, "name_nod_var") == [f + a for f in ("Displacement", "Force") for a in "XYZ"]
        assert _names(nc, "name_elem_var") == ["Volume", "Damage"]
        assert _names(nc, "name_glo_var") == ["Top_Reaction_ForceX", "Top_Reaction_ForceY", "Top_Reaction_ForceZ",
                                             "Kinetic_Energy"]
        assert _names(nc, "eb_names") == ["block_1", "block_2", "block_3"]
        assert nc.dimensions["num_nodes"] == n and nc.dimensions["num_elem"] == n
        assert np.array_equal(nc.variables["time_whole"][:], [0.0, 1e-9, 2e-9])
        assert np.array_equal(np.stack([nc.variables["coord" + a][:] for a in "xyz"], 1), x.reshape(-1, 3))
        assert np.array_equal(nc.variables["node_ns1"][:], np.arange(0, n, 2) + 1)
        for b in range(3):
            conn = nc.variables["connect%d" % (b + 1)]
            assert conn._attributes["elem_type"] == b"SPHERE"
            assert np.array_equal(conn[:, 0] - 1, np.nonzero(block == b)[0])
        for k, rec in enumerate(steps):
            for j, f in enumerate(("Displacement", "Force")):
                for c in range(3):
                    assert np.array_equal(nc.variables["vals_nod_var%d" % (3 * j + c + 1)][k], rec["vectors"][f][c::3])
            for v, f in enumerate(("Volume", "Damage")):
                for b in range(3):
                    got = nc.variables["vals_elem_var%deb%d" % (v + 1, b + 1)][k]
                    assert np.array_equal(got, rec["scalars"][f][block == b])
            g = nc.variables["vals_glo_var"][k]
            assert np.array_equal(g[:3], rec["globals_"]["Top_Reaction_Force"]) and g[3] == rec["globals_"]["Kinetic_Energy"]
    finally:
        nc.close()
