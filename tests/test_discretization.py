"""Discretizations (peridigm_b200.discretization) against the reference.

* element centroid and volume of hexahedra and tetrahedra equal the
  reference's compiled hexCentroidAndVolume / tetCentroidAndVolume
  (src/io/discretization/Peridigm_GeometryUtils.cpp) bit for bit;
* the ElasticBondBased genesis meshes (3D: 384 hexes in 3 blocks; 2D: one
  layer, block ids 2, 3, 1 in file order), written back to Exodus files from
  the fixtures and read: the points, volumes and blocks equal the reference's
  own output (its gold file) and the node set covers every point;
* a mixed hex + tet mesh with a permuted element id map: points in file
  element order with their global ids, node sets mapped to the elements
  that contain their nodes;
* text-file discretization: comments and blank lines skipped, block ids
  mapped in ascending order, a bad line rejected.
"""
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

from _mesh import write_exodus

from oracle import oracle as O
from peridigm_b200 import discretization as D

G = os.path.join(os.path.dirname(__file__), "golden")


def _unit_hex(rng, m):
    base = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    return base[None] * rng.uniform(0.5, 2.0, (m, 1, 3)) + rng.normal(0, 0.05, (m, 8, 3)) + rng.normal(0, 3, (m, 1, 3))


def test_element_geometry_equals_compiled_reference():
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built (the reference tree is absent)")
    rng = np.random.default_rng(0)
    H = _unit_hex(rng, 50)
    c, v = D.hex_centroid_volume(H)
    for k in range(len(H)):
        rc, rv = O.ref_element_point(H[k])
        assert np.array_equal(c[k], rc) and v[k] == rv
    T = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)[None] + rng.normal(0, 0.1, (40, 4, 3))
    c, v = D.tet_centroid_volume(T)
    for k in range(len(T)):
        rc, rv = O.ref_element_point(T[k])
        assert np.array_equal(c[k], rc) and v[k] == rv


@pytest.mark.parametrize("case", ["bond_based_3d", "bond_based_plane_strain"])
def test_genesis_mesh_matches_reference_output(case, tmp_path):
    z = np.load(os.path.join(G, case + ".npz"))
    nblk = len(z["mesh_blk_ids"])
    blocks = [(z["mesh_conn%d" % (b + 1)], "HEX8") for b in range(nblk)]
    path = str(tmp_path / "mesh.g")
    write_exodus(path, z["mesh_X"], blocks, z["mesh_blk_ids"], z["mesh_elem_map"], [z["mesh_ns"]])
    d = D.exodus(path)
    x = d["x"].reshape(-1, 3)
    assert np.abs(x - z["x"]).max() <= 1e-12          # .comp COORDINATES absolute 1e-12
    assert np.abs(d["vol"] - z["vol"]).max() <= 1e-15 * z["vol"].max() + 1e-18
    assert np.array_equal(d["block"], z["block"])
    assert d["block_names"] == ["block_%d" % i for i in sorted(z["mesh_blk_ids"])]
    assert np.array_equal(d["node_sets"]["nodelist_1"], np.arange(len(z["vol"])))


def test_mixed_mesh_and_node_sets(tmp_path):
    rng = np.random.default_rng(2)
    # two hexes sharing a face, then two tets on top of the second hex
    X = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1],
                  [2, 0, 0], [2, 1, 0], [2, 0, 1], [2, 1, 1], [1.5, 0.5, 2.0]], float)
    X += rng.normal(0, 0.02, X.shape)
    hexes = np.array([[1, 2, 3, 4, 5, 6, 7, 8], [2, 9, 10, 3, 6, 11, 12, 7]])
    tets = np.array([[6, 11, 7, 13], [11, 12, 7, 13]])
    elem_map = np.array([3, 1, 4, 2])  # global ids of the file's elements
    write_exodus(str(tmp_path / "m.g"), X, [(hexes, "HEX8"), (tets, "TETRA")], [5, 2], elem_map,
                  [np.array([13]), np.array([1, 4])])
    d = D.exodus(str(tmp_path / "m.g"))
    hc, hv = D.hex_centroid_volume(X[hexes - 1])
    tc, tv = D.tet_centroid_volume(X[tets - 1])
    cen = np.concatenate([hc, tc])
    vol = np.concatenate([hv, tv])
    assert np.array_equal(d["x"].reshape(-1, 3), cen) and np.array_equal(d["vol"], vol)
    assert np.array_equal(d["global_id"], elem_map - 1)
    # block ids 5 (hexes) and 2 (tets): ascending ids -> indices 1 and 0
    assert list(d["block"]) == [1, 1, 0, 0]
    assert list(d["node_sets"]["nodelist_1"]) == [2, 3]   # node 13: both tets
    assert list(d["node_sets"]["nodelist_2"]) == [0]      # nodes 1, 4: the first hex


def test_text_file(tmp_path):
    p = tmp_path / "pts.txt"
    p.write_text("# x y z block volume\n\n0.0 0.0 0.0 3 1.0e-9\n/ comment\n1.0e-3 0 0 1 2.0e-9\n"
                 "* another\n2.0e-3 0 0 3 1.0e-9\n")
    d = D.text_file(str(p))
    assert np.array_equal(d["x"], [0, 0, 0, 1e-3, 0, 0, 2e-3, 0, 0])
    assert np.array_equal(d["vol"], [1e-9, 2e-9, 1e-9])
    assert list(d["block"]) == [1, 0, 1] and list(d["block_ids"]) == [1, 3]
    p.write_text("0 0 0 1\n")
    with pytest.raises(ValueError, match="invalid line"):
        D.text_file(str(p))
