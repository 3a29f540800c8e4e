"""Test helper: a minimal Exodus II genesis writer (netCDF classic)."""
import numpy as np
from scipy.io import netcdf_file


def write_exodus(path, X, blocks, blk_ids, elem_map, node_sets):
    """A minimal Exodus II genesis file: coordinates, element blocks
    (connectivity 1-based, elem_type), element id map, node sets."""
    nc = netcdf_file(path, "w", version=2)
    nc.createDimension("num_nodes", X.shape[0])
    nc.createDimension("num_dim", 3)
    nc.createDimension("num_elem", sum(len(c) for c, _ in blocks))
    nc.createDimension("num_el_blk", len(blocks))
    nc.createDimension("num_node_sets", len(node_sets))
    for a, k in zip("xyz", range(3)):
        nc.createVariable("coord" + a, "d", ("num_nodes",))[:] = X[:, k]
    nc.createVariable("eb_prop1", "i", ("num_el_blk",))[:] = blk_ids
    for b, (conn, et) in enumerate(blocks):
        nc.createDimension("num_el_in_blk%d" % (b + 1), conn.shape[0])
        nc.createDimension("num_nod_per_el%d" % (b + 1), conn.shape[1])
        v = nc.createVariable("connect%d" % (b + 1), "i", ("num_el_in_blk%d" % (b + 1), "num_nod_per_el%d" % (b + 1)))
        v[:] = conn
        v.elem_type = et
    nc.createVariable("elem_num_map", "i", ("num_elem",))[:] = elem_map
    nc.createVariable("ns_prop1", "i", ("num_node_sets",))[:] = np.arange(1, len(node_sets) + 1)
    for s, nodes in enumerate(node_sets):
        nc.createDimension("num_nod_ns%d" % (s + 1), len(nodes))
        nc.createVariable("node_ns%d" % (s + 1), "i", ("num_nod_ns%d" % (s + 1),))[:] = nodes
    nc.close()
