"""Exodus II output of a run (host side), in the reference's layout.

PeridigmNS::OutputManager_ExodusII (src/io/Peridigm_OutputManager_ExodusII.cpp)
writes each point as a node and as a one-node SPHERE element of its block:

* coordinates coordx/y/z (the model coordinates), element blocks
  connect<b> (1-based point ids, elem_type SPHERE) with ids eb_prop1 and
  names "block_<id>", node sets node_ns<s> (1-based point ids),
  node_num_map / elem_num_map (global ids + 1);
* vector fields as node variables "<Name>X", "<Name>Y", "<Name>Z";
* scalar fields as element variables, per block (vals_elem_var<v>eb<b>);
* compute-class results as global variables (vectors as X/Y/Z entries);
* one record per output step on the unlimited time_step dimension
  (time_whole).

Files are netCDF classic (64-bit offset), written with scipy.io.netcdf_file,
and read back by Exodus tools and by peridigm_b200.discretization. Field
values come from `Context.field` and the compute classes; `write_context_step`
gathers the usual ones.
"""
from __future__ import annotations

import numpy as np

LEN_NAME = 256


def _chars(names, width=LEN_NAME):
    a = np.zeros((len(names), width), dtype="S1")
    for k, nm in enumerate(names):
        b = nm.encode()[:width]
        a[k, :len(b)] = np.frombuffer(b, dtype="S1")
    return a


class ExodusWriter:
    """Writer of one output file.

    x [3n] model coordinates; block [n] 0-based block index per point;
    block_ids the Exodus id of each block index (default 1, 2, ...);
    node_sets {name: point indices}; vector_fields / scalar_fields / global
    fields: the names written every step (global entries are vectors unless
    listed in scalar_globals).
    """

    def __init__(self, path, x, block, block_ids=None, node_sets=None, vector_fields=(), scalar_fields=(),
                 global_fields=(), scalar_globals=(), global_id=None, title="Peridigm"):
        from scipy.io import netcdf_file

        x = np.asarray(x, np.float64).reshape(-1, 3)
        n = x.shape[0]
        block = np.asarray(block, np.int64)
        nblk = int(block.max()) + 1 if n else 0
        block_ids = np.arange(1, nblk + 1) if block_ids is None else np.asarray(block_ids, np.int64)
        self.points_of_block = [np.nonzero(block == b)[0] for b in range(nblk)]
        self.vector_fields = list(vector_fields)
        self.scalar_fields = list(scalar_fields)
        self.global_fields = list(global_fields)
        self.scalar_globals = set(scalar_globals)
        self.n = n
        self.step = 0
        nc = netcdf_file(path, "w", version=2)
        self.nc = nc
        nc.api_version = np.float32(8.06)
        nc.version = np.float32(8.06)
        nc.floating_point_word_size = np.int32(8)
        nc.file_size = np.int32(1)
        nc.maximum_name_length = np.int32(32)
        nc.int64_status = np.int32(0)
        nc.title = title
        nc.createDimension("time_step", None)  # the unlimited dimension comes first in this writer
        nc.createDimension("len_name", LEN_NAME)
        nc.createDimension("num_dim", 3)
        nc.createDimension("num_nodes", n)
        nc.createDimension("num_elem", n)
        nc.createDimension("num_el_blk", nblk)
        node_sets = dict(node_sets or {})
        if node_sets:
            nc.createDimension("num_node_sets", len(node_sets))
        nc.createVariable("time_whole", "d", ("time_step",))
        nc.createVariable("eb_status", "i", ("num_el_blk",))[:] = 1
        v = nc.createVariable("eb_prop1", "i", ("num_el_blk",))
        v[:] = block_ids
        v.name = "ID"
        for a, k in zip("xyz", range(3)):
            nc.createVariable("coord" + a, "d", ("num_nodes",))[:] = x[:, k]
        nc.createVariable("eb_names", "c", ("num_el_blk", "len_name"))[:] = _chars(
            ["block_%d" % i for i in block_ids])
        nc.createVariable("coor_names", "c", ("num_dim", "len_name"))[:] = _chars(["x", "y", "z"])
        for b, pts in enumerate(self.points_of_block):
            nc.createDimension("num_el_in_blk%d" % (b + 1), len(pts))
            nc.createDimension("num_nod_per_el%d" % (b + 1), 1)
            c = nc.createVariable("connect%d" % (b + 1), "i", ("num_el_in_blk%d" % (b + 1), "num_nod_per_el%d" % (b + 1)))
            c[:] = (pts + 1).reshape(-1, 1)
            c.elem_type = "SPHERE"
        if node_sets:
            nc.createVariable("ns_status", "i", ("num_node_sets",))[:] = 1
            v = nc.createVariable("ns_prop1", "i", ("num_node_sets",))
            v[:] = np.arange(1, len(node_sets) + 1)
            v.name = "ID"
            nc.createVariable("ns_names", "c", ("num_node_sets", "len_name"))[:] = _chars(list(node_sets))
            for s, (nm, pts) in enumerate(node_sets.items()):
                nc.createDimension("num_nod_ns%d" % (s + 1), len(pts))
                nc.createVariable("node_ns%d" % (s + 1), "i", ("num_nod_ns%d" % (s + 1),))[:] = np.asarray(pts) + 1
        gid = np.arange(n) if global_id is None else np.asarray(global_id, np.int64)
        nc.createVariable("node_num_map", "i", ("num_nodes",))[:] = gid + 1
        nc.createVariable("elem_num_map", "i", ("num_elem",))[:] = gid + 1
        gnames = []
        for g in self.global_fields:
            gnames += [g] if g in self.scalar_globals else [g + "X", g + "Y", g + "Z"]
        self.global_names = gnames
        if gnames:
            nc.createDimension("num_glo_var", len(gnames))
            nc.createVariable("name_glo_var", "c", ("num_glo_var", "len_name"))[:] = _chars(gnames)
            nc.createVariable("vals_glo_var", "d", ("time_step", "num_glo_var"))
        nnames = [f + ax for f in self.vector_fields for ax in "XYZ"]
        self.nod_names = nnames
        if nnames:
            nc.createDimension("num_nod_var", len(nnames))
            nc.createVariable("name_nod_var", "c", ("num_nod_var", "len_name"))[:] = _chars(nnames)
            for k in range(len(nnames)):
                nc.createVariable("vals_nod_var%d" % (k + 1), "d", ("time_step", "num_nodes"))
        if self.scalar_fields:
            nc.createDimension("num_elem_var", len(self.scalar_fields))
            nc.createVariable("name_elem_var", "c", ("num_elem_var", "len_name"))[:] = _chars(self.scalar_fields)
            for v in range(len(self.scalar_fields)):
                for b in range(nblk):
                    nc.createVariable("vals_elem_var%deb%d" % (v + 1, b + 1), "d",
                                      ("time_step", "num_el_in_blk%d" % (b + 1)))
            nc.createVariable("elem_var_tab", "i", ("num_el_blk", "num_elem_var"))[:] = 1

    def write_step(self, time, vectors=None, scalars=None, globals_=None):
        """Appends one record: vectors {name: [3n]}, scalars {name: [n]},
        globals_ {name: scalar or 3-vector}; every declared field is needed."""
        nc, k = self.nc, self.step
        nc.variables["time_whole"][k] = time
        vectors, scalars, globals_ = vectors or {}, scalars or {}, globals_ or {}
        for j, f in enumerate(self.vector_fields):
            a = np.asarray(vectors[f], np.float64).reshape(-1, 3)
            for c in range(3):
                nc.variables["vals_nod_var%d" % (3 * j + c + 1)][k] = a[:, c]
        for v, f in enumerate(self.scalar_fields):
            a = np.asarray(scalars[f], np.float64)
            for b, pts in enumerate(self.points_of_block):
                nc.variables["vals_elem_var%deb%d" % (v + 1, b + 1)][k] = a[pts]
        if self.global_names:
            row = []
            for g in self.global_fields:
                val = np.atleast_1d(np.asarray(globals_[g], np.float64))
                row += [float(val[0])] if g in self.scalar_globals else [float(t) for t in val[:3]]
            nc.variables["vals_glo_var"][k] = np.array(row)
        self.step += 1
        nc.flush()

    def close(self):
        if self.nc is not None:
            self.nc.close()
            self.nc = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def write_context_step(writer, ctx, time, block_sums=None):
    """One record from a Context: the writer's vector and scalar fields by
    name (Context.field), and globals from the Block_Data compute class:
    block_sums {label: (field, block index, calculation)}."""
    vec = {f: ctx.field(f) for f in writer.vector_fields}
    sca = {f: ctx.field(f) for f in writer.scalar_fields}
    glo = {}
    for label, (field, block, calc) in (block_sums or {}).items():
        glo[label] = ctx.block_data(field, block, calc)
    writer.write_step(time, vec, sca, glo)
