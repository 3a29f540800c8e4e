"""Discretizations: the reference's mesh inputs turned into points.

Host-side ingest for the two file-based discretizations of the reference, so
its input decks' meshes feed this library's points (`Context.set_points`),
blocks and node sets (prescribed displacements, initial velocities):

* text file (PeridigmNS::TextFileDiscretization::getDecomp,
  src/io/discretization/Peridigm_TextFileDiscretization.cpp:128-300): one
  point per line "x y z block_id volume"; lines starting with '#', '/' or '*'
  and empty lines are skipped; any other line without exactly five numbers is
  an error;
* Exodus II genesis mesh (PeridigmNS::ExodusDiscretization::loadData,
  src/io/discretization/Peridigm_ExodusDiscretization.cpp:250-570): one point
  per element, at the element's centroid with its volume
  (Peridigm_GeometryUtils.cpp: hexCentroidAndVolume :69-339 for HEX/HEX8/HEX20
  with the side nodes of HEX20 dropped, tetCentroidAndVolume :52-67 for
  TET/TETRA/TET4/TET10, the node and the second attribute for SPHERE);
  points are in the file's element order, block by block as stored (the
  order the reference keeps and writes them in; the element id map gives
  their global ids, returned as `global_id`); a node set becomes the points
  of the elements that contain any of its nodes (:557-566); blocks are named
  "block_<id>" unless the file names them.

Blocks map to this library's 0-based block indices in ascending block id
order (block_1 -> 0, ...), the order the reference writes them out in.
Exodus files are netCDF classic; they are read with scipy.io.netcdf_file.
The arithmetic of the centroid and volume follows the reference's operation
order, so both come out bit for bit as the reference computes them.
"""
from __future__ import annotations

import numpy as np

# Hexahedron faces by their barycentres (GeometryUtils.cpp:82-101), and the
# 24 tetrahedra (node, node, face barycentre, hex barycentre) in the
# reference's order (:110-332); 8, 9, .. index the face barycentres f0..f5.
_HEX_FACES = [(0, 1, 4, 5), (1, 2, 5, 6), (2, 3, 6, 7), (0, 3, 4, 7), (0, 1, 2, 3), (4, 5, 6, 7)]
_HEX_TETS = [(1, 0, 8), (5, 1, 8), (4, 5, 8), (0, 4, 8),
             (2, 1, 9), (6, 2, 9), (5, 6, 9), (1, 5, 9),
             (3, 2, 10), (7, 3, 10), (6, 7, 10), (2, 6, 10),
             (0, 3, 11), (3, 7, 11), (7, 4, 11), (4, 0, 11),
             (0, 1, 12), (1, 2, 12), (2, 3, 12), (3, 0, 12),
             (5, 4, 13), (4, 7, 13), (7, 6, 13), (6, 5, 13)]


def _tet_volume(p0, p1, p2, p3):
    """|a.(b x c)|/6 with a, b, c relative to p0, in the reference's order
    (GeometryUtils.cpp:375-391, scalarTripleProduct :911-919); arrays [..., 3]."""
    a, b, c = p1 - p0, p2 - p0, p3 - p0
    t = (a[..., 0] * (b[..., 1] * c[..., 2] - b[..., 2] * c[..., 1])
         + a[..., 1] * (b[..., 2] * c[..., 0] - b[..., 0] * c[..., 2])
         + a[..., 2] * (b[..., 0] * c[..., 1] - b[..., 1] * c[..., 0]))
    v = t / 6.0
    if np.any(v < 0.0):
        raise ValueError("tetVolume() computed negative volume, possible element inversion or incorrect node numbering")
    return v


def _tet_centroid(p0, p1, p2, p3):
    return (((p0 + p1) + p2) + p3) * 0.25


def tet_centroid_volume(nodes):
    """Centroids [m, 3] and volumes [m] of 4-node tetrahedra, nodes [m, 4, 3]."""
    P = np.asarray(nodes, np.float64)
    return _tet_centroid(P[:, 0], P[:, 1], P[:, 2], P[:, 3]), _tet_volume(P[:, 0], P[:, 1], P[:, 2], P[:, 3])


def hex_centroid_volume(nodes):
    """Centroids [m, 3] and volumes [m] of 8-node hexahedra, nodes [m, 8, 3]:
    24 tetrahedra on the face barycentres and the body barycentre, the
    centroid their volume-weighted mean."""
    P = np.asarray(nodes, np.float64)
    pts = [P[:, k] for k in range(8)]
    for f in _HEX_FACES:
        pts.append(0.25 * (((P[:, f[0]] + P[:, f[1]]) + P[:, f[2]]) + P[:, f[3]]))
    c = 0.5 * (pts[12] + pts[13])
    vol = np.zeros(P.shape[0])
    cen = np.zeros((P.shape[0], 3))
    for a, b, f in _HEX_TETS:
        tv = _tet_volume(pts[a], pts[b], pts[f], c)
        vol = vol + tv
        cen = cen + _tet_centroid(pts[a], pts[b], pts[f], c) * tv[:, None]
    return cen / vol[:, None], vol


def text_file(path):
    """Points of a text-file discretization: dict(x [3n], vol [n], block [n]
    0-based indices, block_ids [nblocks] original ids in index order)."""
    rows = []
    with open(path) as fh:
        for raw in fh:
            s = raw.strip()
            if not s or s[0] in "#/*":
                continue
            vals = s.split()
            try:
                data = [float(v) for v in vals]
            except ValueError:
                data = []
            if len(data) != 5:
                raise ValueError("**** Error parsing text file, invalid line: " + s)
            rows.append(data)
    if not rows:
        raise ValueError("**** Error reading discretization text file, no data found.")
    a = np.array(rows, np.float64)
    ids = a[:, 3].astype(np.int64)
    uniq = np.unique(ids)
    return dict(x=np.ascontiguousarray(a[:, :3].ravel()), vol=a[:, 4].copy(),
                block=np.searchsorted(uniq, ids).astype(np.int32), block_ids=uniq)


def _names(nc, key, count, prefix):
    out = []
    if key in nc.variables:
        for r in nc.variables[key][:]:
            out.append(b"".join(r).decode(errors="ignore").strip("\x00 ").strip())
    while len(out) < count:
        out.append("")
    return out


def exodus(path):
    """Points of an Exodus II genesis mesh: dict(x, vol, block (0-based, by
    ascending block id), block_ids, block_names, node_sets {name: sorted
    point indices}, global_id (element id map minus one), element_type per
    block id)."""
    from scipy.io import netcdf_file

    nc = netcdf_file(path, "r", mmap=False)
    try:
        X = np.stack([np.asarray(nc.variables["coord" + a][:], np.float64) for a in "xyz"], 1)
        nblk = nc.dimensions["num_el_blk"]
        blk_ids = np.asarray(nc.variables["eb_prop1"][:], np.int64)
        blk_names = _names(nc, "eb_names", nblk, "block_")
        blk_names = [nm if nm else "block_%d" % bid for nm, bid in zip(blk_names, blk_ids)]
        nelem = nc.dimensions["num_elem"]
        if "elem_num_map" in nc.variables:
            gid = np.asarray(nc.variables["elem_num_map"][:], np.int64) - 1
        else:
            gid = np.arange(nelem)
        cen = np.zeros((nelem, 3))
        vol = np.zeros(nelem)
        bid = np.zeros(nelem, np.int64)
        conn_all = []
        etypes = {}
        k0 = 0
        for b in range(nblk):
            var = nc.variables["connect%d" % (b + 1)]
            conn = np.asarray(var[:], np.int64) - 1
            et = var._attributes.get("elem_type", b"").decode().upper()
            etypes[int(blk_ids[b])] = et
            m = conn.shape[0]
            sl = slice(k0, k0 + m)
            if et == "SPHERE":
                attr = np.asarray(nc.variables["attrib%d" % (b + 1)][:], np.float64)
                cen[sl] = X[conn[:, 0]]
                vol[sl] = attr[:, 1]
            elif et in ("TET", "TETRA", "TET4", "TET10"):
                cen[sl], vol[sl] = tet_centroid_volume(X[conn[:, :4]])
            elif et in ("HEX", "HEX8", "HEX20"):
                cen[sl], vol[sl] = hex_centroid_volume(X[conn[:, :8]])
            else:
                raise ValueError("unknown element type " + et)
            bid[sl] = blk_ids[b]
            conn_all.append(conn)
            k0 += m
        if not np.array_equal(np.sort(gid), np.arange(nelem)):
            raise ValueError("the element id map is not a permutation of 1..num_elem")
        uniq = np.unique(blk_ids)
        node_sets = {}
        nns = nc.dimensions.get("num_node_sets", 0) or 0
        if nns:
            ns_ids = np.asarray(nc.variables["ns_prop1"][:], np.int64)
            ns_names = _names(nc, "ns_names", nns, "nodelist_")
            # elements that contain each node
            elem_of_node = [[] for _ in range(X.shape[0])]
            e = 0
            for conn in conn_all:
                for row in conn:
                    for nd in row:
                        elem_of_node[nd].append(e)
                    e += 1
            for s in range(nns):
                nodes = np.asarray(nc.variables["node_ns%d" % (s + 1)][:], np.int64) - 1
                pts = sorted({int(el) for nd in nodes for el in elem_of_node[nd]})
                name = ns_names[s] if ns_names[s] else "nodelist_%d" % ns_ids[s]
                node_sets[name] = np.array(pts, np.int64)
        return dict(x=np.ascontiguousarray(cen.ravel()), vol=vol,
                    block=np.searchsorted(uniq, bid).astype(np.int32), block_ids=uniq,
                    block_names=[blk_names[list(blk_ids).index(u)] for u in uniq], node_sets=node_sets,
                    global_id=gid, element_type=etypes)
    finally:
        nc.close()
