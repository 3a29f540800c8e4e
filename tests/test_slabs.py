"""Slab domain decomposition and the multi-rank paths on CPU (gloo).

* slab plans: owned sets partition the points, ghost layers cover every point
  within two horizons of an owned point, send and receive lists mirror;
* two gloo ranks, each stepping its slab of a notched plate with critical
  stretch damage (oracle engine) and exchanging ghost state once per step,
  reproduce the one-domain run bit for bit on every owned point
  (displacement, velocity, bond damage count);
* the bench's max-over-ranks reduction over two gloo ranks.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
from peridigm_b200 import slabs, workloads

from slab_engine_cpu import OracleEngine


def _plate():
    return workloads.notched_plate(nx=48, ny=20, nz=3, notch_cells=12, pull=40.0, s_c=2.0e-4)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slab_plans_cover_and_mirror():
    w = _plate()
    P = w["x"].reshape(-1, 3)
    plans = slabs.slab_plans(w["x"], w["horizon"], 3)
    owned = np.concatenate([p.owned for p in plans])
    assert np.array_equal(np.sort(owned), np.arange(len(P)))
    for p in plans:
        d = np.sqrt(((P[:, None, :] - P[None, p.owned, :]) ** 2).sum(-1)).min(1)
        need = np.nonzero(d <= 2.0 * w["horizon"])[0]
        assert np.isin(need, p.local).all()
        assert np.array_equal(p.local[p.owned_local], p.owned)
        for q, idx in p.send.items():
            assert np.array_equal(p.local[idx], plans[q].local[plans[q].recv[p.rank]])


def _rank_main(rank, world, port, outdir, nsteps, dt):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        w = _plate()
        plan = slabs.slab_plans(w["x"], w["horizon"], world)[rank]
        eng = OracleEngine(slabs.local_workload(w, plan))
        halo = slabs.HaloExchange(plan, "cpu", dist)
        slabs.run_slab(eng, halo, dt, nsteps)
        own = plan.owned_local
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), owned=plan.owned, u=eng.u.reshape(-1, 3)[own],
                 v=eng.v.reshape(-1, 3)[own])
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        np.save(os.path.join(outdir, f"max{rank}.npy"), t.numpy())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_one_domain(tmp_path):
    w = _plate()
    row, col = O.neighbor_search(w["x"], w["horizon"], w["planes"])
    dt = 0.7 * O.critical_time_step(w["x"], w["vol"], row, col, w["K"], w["rho"], w["horizon"])
    nsteps = 25
    ref = OracleEngine(w)
    slabs.run_slab(ref, slabs.HaloExchange(slabs.slab_plans(w["x"], w["horizon"], 1)[0], "cpu"), dt, nsteps)
    assert ref.dmg.sum() > 0  # the pull breaks bonds within the run
    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path), nsteps, dt), nprocs=2, join=True,
                       start_method="spawn")
    u = np.zeros_like(ref.u).reshape(-1, 3)
    v = np.zeros_like(ref.v).reshape(-1, 3)
    seen = np.zeros(len(w["vol"]), dtype=int)
    for r in range(2):
        z = np.load(tmp_path / f"rank{r}.npz")
        u[z["owned"]] = z["u"]
        v[z["owned"]] = z["v"]
        seen[z["owned"]] += 1
        assert float(np.load(tmp_path / f"max{r}.npy")[0]) == 2.0
    assert (seen == 1).all()
    assert np.array_equal(u.ravel(), ref.u)
    assert np.array_equal(v.ravel(), ref.v)


def test_single_rank_plan_equals_the_full_plans():
    """slab_plan (one rank, vectorised) gives each rank exactly its entry of slab_plans."""
    w = _plate()
    for nr in (2, 3, 4):
        full = slabs.slab_plans(w["x"], w["horizon"], nr)
        for r in range(nr):
            one = slabs.slab_plan(w["x"], w["horizon"], nr, r)
            assert one.axis == full[r].axis
            assert np.array_equal(one.owned, full[r].owned) and np.array_equal(one.local, full[r].local)
            assert np.array_equal(one.owned_local, full[r].owned_local)
            assert set(one.send) == set(full[r].send) and set(one.recv) == set(full[r].recv)
            for q in one.send:
                assert np.array_equal(one.send[q], full[r].send[q])
            for q in one.recv:
                assert np.array_equal(one.recv[q], full[r].recv[q])
