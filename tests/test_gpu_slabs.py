"""Slab decomposition through the C ABI on one GPU: the stepping form and the
ghost-state pack/unpack entry points.

* pd_verlet_begin + pd_verlet_step(n - 1) + pd_verlet_finish gives the state
  of pd_verlet_run(n), bit for bit;
* three slab contexts of a notched plate with damage, stepped in turn with
  their ghost state swapped once per step (host-ordered: no kernel waits on
  another), reproduce the one-context run bit for bit on every owned point
  (displacement, velocity, node damage), on both precisions;
* an index outside the context is reported as PD_ERR_ARG, not accessed.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from peridigm_b200 import Context, slabs, workloads

pytestmark = pytest.mark.gpu


def _plate():
    return workloads.notched_plate(nx=90, ny=30, nz=3, notch_cells=20, pull=40.0, s_c=2.0e-4)


@pytest.mark.parametrize("precision", ["split", "fp64"])
def test_stepping_equals_run(precision):
    w = _plate()
    out = []
    for stepping in (False, True):
        with Context(precision=precision) as ctx:
            workloads.setup_context(ctx, w)
            dt = 0.7 * ctx.critical_time_step()
            if stepping:
                ctx.verlet_begin(dt)
                ctx.verlet_step(14)
                st = ctx.verlet_finish()
            else:
                st = ctx.verlet_run(dt, 15)
            out.append((ctx.field("Displacement"), ctx.field("Velocity"), ctx.field("Damage"), st["broken_bonds"]))
    assert out[0][3] > 0
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("precision", ["split", "fp64"])
def test_three_slabs_match_one_context(precision):
    w = _plate()
    nsteps = 20
    with Context(precision=precision) as full:
        workloads.setup_context(full, w)
        dt = 0.7 * full.critical_time_step()
        full.verlet_run(dt, nsteps)
        ref = (full.field("Displacement").reshape(-1, 3), full.field("Velocity").reshape(-1, 3),
               full.field("Damage"))
    plans = slabs.slab_plans(w["x"], w["horizon"], 3)
    ctxs = [Context(precision=precision) for _ in plans]
    try:
        for c, p in zip(ctxs, plans):
            workloads.setup_context(c, slabs.local_workload(w, p))
        dev = torch.device("cuda:0")
        links = [(r, q) for r, p in enumerate(plans) for q in p.send]
        sidx = {(r, q): torch.as_tensor(plans[r].send[q], device=dev) for r, q in links}
        ridx = {(r, q): torch.as_tensor(plans[q].recv[r], device=dev) for r, q in links}
        bufs = {k: torch.zeros((len(v), 6), dtype=torch.float64, device=dev) for k, v in sidx.items()}

        def swap():
            for (r, q) in links:
                ctxs[r].pack_state(sidx[(r, q)], bufs[(r, q)])
            for (r, q) in links:
                ctxs[q].unpack_state(ridx[(r, q)], bufs[(r, q)])

        for c in ctxs:
            c.verlet_begin(dt)
        swap()
        for _ in range(nsteps - 1):
            for c in ctxs:
                c.verlet_step(1)
            swap()
        for c in ctxs:
            c.verlet_finish()
        seen = np.zeros(len(w["vol"]), dtype=int)
        for c, p in zip(ctxs, plans):
            own = p.owned_local
            assert np.array_equal(c.field("Displacement").reshape(-1, 3)[own], ref[0][p.owned])
            assert np.array_equal(c.field("Velocity").reshape(-1, 3)[own], ref[1][p.owned])
            assert np.array_equal(c.field("Damage")[own], ref[2][p.owned])
            seen[p.owned] += 1
        assert (seen == 1).all()
        assert ref[2].max() > 0
    finally:
        for c in ctxs:
            c.close()


def test_pack_rejects_out_of_range_index():
    w = workloads.notched_plate(nx=20, ny=10, nz=3, notch_cells=4)
    with Context(precision="split") as ctx:
        workloads.setup_context(ctx, w)
        ctx.verlet_begin(0.7 * ctx.critical_time_step())
        n = len(w["vol"])
        idx = torch.tensor([0, n, 3], dtype=torch.int32, device="cuda:0")
        out = torch.zeros((3, 6), dtype=torch.float64, device="cuda:0")
        rc = ctx.L.pd_pack_state_device(ctx.h, 3, C.c_void_p(idx.data_ptr()), C.c_void_p(out.data_ptr()))
        assert rc == 1
        ctx.verlet_finish()
