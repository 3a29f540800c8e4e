"""Slab domain decomposition of one body over ranks (one GPU each).

The reference partitions points with Zoltan RCB (src/io/pdneigh/PdZoltan.cxx)
and brings ghost data in with Epetra imports inside the step loop
(src/core/Peridigm.cpp:1497-1546). Here each rank owns a slab of points along
the body's longest axis (equal point counts) and holds a ghost layer `depth`
horizons deep. With the force in gather form, an owned point's force reads
the dilatation of neighbors up to one horizon away, and their dilatation
reads displacements up to two horizons away, so with depth 2 one exchange of
ghost state per step makes every owned point's damage, dilatation, force and
update identical to a one-domain run: the local bond families of owned
points equal the global ones, and local points keep the global order, so
every sum runs in the same order.

The exchange moves 6 doubles per ghost point (displacement and current
coordinates, as the owner holds them for the next evaluation) with
torch.distributed point-to-point operations: NCCL between GPUs, gloo on CPU.
Contact is not part of the slab path (it would also need ghost velocities).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class SlabPlan:
    rank: int
    nranks: int
    axis: int
    owned: np.ndarray          # global ids owned by this rank, ascending
    local: np.ndarray          # global ids held locally (owned + ghosts), ascending
    owned_local: np.ndarray    # positions of the owned points in `local`
    send: dict = field(default_factory=dict)  # peer -> local indices of owned points that are ghosts there
    recv: dict = field(default_factory=dict)  # peer -> local indices of ghosts owned by that peer


def slab_owner(x, nranks, axis=None):
    """Owner rank of every point: equal-count slabs along `axis` (default the
    longest extent), ties broken by point id."""
    P = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    if axis is None:
        axis = int(np.argmax(P.max(0) - P.min(0)))
    order = np.lexsort((np.arange(len(P)), P[:, axis]))
    owner = np.empty(len(P), dtype=np.int32)
    for r, chunk in enumerate(np.array_split(order, nranks)):
        owner[chunk] = r
    return owner, axis


def slab_plans(x, horizon, nranks, depth=2.0, axis=None):
    """Plans of all ranks (every rank can compute them from the same inputs).

    Ghosts of rank r: points of other ranks whose slab coordinate lies within
    depth * max(horizon) of r's owned coordinate range (a superset of the
    points within that distance of an owned point)."""
    P = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    owner, axis = slab_owner(P, nranks, axis)
    h = float(np.max(horizon))
    c = P[:, axis]
    owned = [np.nonzero(owner == r)[0] for r in range(nranks)]
    local = []
    for r in range(nranks):
        if len(owned[r]) == 0:
            local.append(owned[r])
            continue
        lo, hi = c[owned[r]].min() - depth * h, c[owned[r]].max() + depth * h
        near = np.nonzero((c >= lo) & (c <= hi))[0]
        local.append(np.union1d(owned[r], near))
    plans = []
    for r in range(nranks):
        plan = SlabPlan(rank=r, nranks=nranks, axis=axis, owned=owned[r], local=local[r],
                        owned_local=np.searchsorted(local[r], owned[r]))
        for p in range(nranks):
            if p == r:
                continue
            out = np.intersect1d(owned[r], local[p], assume_unique=True)
            inc = np.intersect1d(owned[p], local[r], assume_unique=True)
            if len(out):
                plan.send[p] = np.searchsorted(local[r], out).astype(np.int32)
            if len(inc):
                plan.recv[p] = np.searchsorted(local[r], inc).astype(np.int32)
        plans.append(plan)
    return plans


def slab_plan(x, horizon, nranks, rank, depth=2.0, axis=None):
    """This rank's plan alone, equal to slab_plans(...)[rank], from vectorised
    passes over the points (what a rank of a large body computes)."""
    P = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    owner, axis = slab_owner(P, nranks, axis)
    h = float(np.max(horizon))
    c = P[:, axis]
    lo = np.full(nranks, np.inf)
    hi = np.full(nranks, -np.inf)
    np.minimum.at(lo, owner, c)
    np.maximum.at(hi, owner, c)

    def within(r):  # coordinates inside rank r's owned range widened by depth horizons
        return (c >= lo[r] - depth * h) & (c <= hi[r] + depth * h)

    mine = owner == rank
    local = np.nonzero(mine | within(rank))[0] if mine.any() else np.zeros(0, np.int64)
    owned = np.nonzero(mine)[0]
    plan = SlabPlan(rank=rank, nranks=nranks, axis=axis, owned=owned, local=local,
                    owned_local=np.searchsorted(local, owned))
    here = np.zeros(len(c), bool)
    here[local] = True
    for p in range(nranks):
        if p == rank or not np.isfinite(lo[p]):
            continue
        out = np.nonzero(mine & within(p))[0]
        inc = np.nonzero((owner == p) & here)[0]
        if len(out):
            plan.send[p] = np.searchsorted(local, out).astype(np.int32)
        if len(inc):
            plan.recv[p] = np.searchsorted(local, inc).astype(np.int32)
    return plan


def local_workload(w, plan):
    """The workload restricted to a rank's local points (same keys as the
    workload dicts of peridigm_b200.workloads)."""
    ids = plan.local
    g2l = np.full(len(w["vol"]), -1, dtype=np.int64)
    g2l[ids] = np.arange(len(ids))
    x = np.asarray(w["x"]).reshape(-1, 3)[ids].ravel()
    out = dict(w)
    out["x"] = np.ascontiguousarray(x)
    out["vol"] = np.asarray(w["vol"])[ids]
    out["v0"] = np.asarray(w["v0"]).reshape(-1, 3)[ids].ravel()
    for key in ("K", "mu", "s_c"):
        if w.get(key) is not None and np.ndim(w[key]) > 0:
            out[key] = np.asarray(w[key])[ids]
    if w.get("block") is not None:
        out["block"] = np.asarray(w["block"])[ids]
    bcs = []
    for bc in w.get("bcs", []):
        pts = g2l[np.asarray(bc["points"], dtype=np.int64)]
        bcs.append(dict(bc, points=pts[pts >= 0]))
    out["bcs"] = bcs
    out["name"] = f"{w.get('name', 'workload')}[slab {plan.rank}/{plan.nranks}]"
    return out


class HaloExchange:
    """Per-step ghost exchange of one rank: pack the owned points the peers hold
    as ghosts, swap with batched point-to-point sends and receives, unpack."""

    def __init__(self, plan, device, dist=None):
        import torch

        self.dist = dist
        self.peers = sorted(set(plan.send) | set(plan.recv))
        self.sidx = {p: torch.as_tensor(plan.send.get(p, np.zeros(0, np.int32)), device=device) for p in self.peers}
        self.ridx = {p: torch.as_tensor(plan.recv.get(p, np.zeros(0, np.int32)), device=device) for p in self.peers}
        self.sbuf = {p: torch.zeros((len(self.sidx[p]), 6), dtype=torch.float64, device=device) for p in self.peers}
        self.rbuf = {p: torch.zeros((len(self.ridx[p]), 6), dtype=torch.float64, device=device) for p in self.peers}

    def exchange(self, engine):
        if not self.peers:
            return
        for p in self.peers:
            if len(self.sidx[p]):
                engine.pack(self.sidx[p], self.sbuf[p])
        ops = []
        for p in self.peers:
            if len(self.ridx[p]):
                ops.append(self.dist.P2POp(self.dist.irecv, self.rbuf[p], p))
            if len(self.sidx[p]):
                ops.append(self.dist.P2POp(self.dist.isend, self.sbuf[p], p))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        for p in self.peers:
            if len(self.ridx[p]):
                engine.unpack(self.ridx[p], self.rbuf[p])


def run_slab(engine, halo, dt, nsteps, t0=0.0):
    """Velocity-Verlet over nsteps >= 1 steps with one ghost exchange per step:
    begin (initial evaluation, first half of step 1), then exchange -> step."""
    if nsteps < 1:
        raise ValueError("run_slab needs at least one step")
    engine.begin(dt, t0)
    halo.exchange(engine)
    for _ in range(nsteps - 1):
        engine.step(1)
        halo.exchange(engine)
    return engine.finish()


class ContextEngine:
    """The slab engine over a peridigm_b200.Context (device tensors)."""

    def __init__(self, ctx):
        self.ctx = ctx

    def begin(self, dt, t0):
        self.ctx.verlet_begin(dt, t0)

    def step(self, k):
        self.ctx.verlet_step(k)

    def finish(self):
        return self.ctx.verlet_finish()

    def pack(self, idx, out):
        self.ctx.pack_state(idx, out)

    def unpack(self, idx, vals):
        self.ctx.unpack_state(idx, vals)
