"""Restart snapshots (host side) in the reference's folder layout.

PeridigmNS::Peridigm::writeRestart / readRestart (src/core/Peridigm.cpp:4449-4620,
names from setRestartNames :1009-1080, folder discovery InitializeRestart
:969-1007) write, per restart, a folder `restart-NNNNNN` (six digits, one more
than the folder the run started from; the first run starts from
`restart-000000`) holding

* `currentTime.txt`: the line "Current time is " and the time (:4464-4468);
* one Matrix Market array file per global vector (EpetraExt
  VectorToMatrixMarketFile): blockIDs, horizon, volume, density,
  deltaTemperature (scalar per point) and x, u, y, v, a, force, contactForce,
  externalForce, deltaU, scratch (three per point, interleaved xyz);
* per block, its two-step state: `BondData_<block>State{N,NP1}.mat` with the
  bond fields in the block's bond order (the owned points of the block in
  order, each point's bonds in neighbor-list order; here the one stateful bond
  field, Bond_Damage), State::writeStateData (src/core/Peridigm_State.cpp:153-185).

Reading restores what the next run needs: displacement, velocity and the
committed bond damage (the N state); the time is returned, and a run resumed
from it starts with the reference's initial evaluation, which recomputes the
acceleration and forces from that state (Peridigm.cpp:1393-1423). The model
coordinates and volumes in the folder must equal the context's. As in the
reference, a resumed run must start at the snapshot's time.
"""
from __future__ import annotations

import glob
import os
import re

import numpy as np

_SCALARS = ("blockIDs", "horizon", "volume", "density", "deltaTemperature")
_VECTORS = ("x", "u", "y", "v", "a", "force", "contactForce", "externalForce", "deltaU", "scratch")


def write_matrix_market(path, values, name=""):
    """A dense column vector as a Matrix Market array file."""
    values = np.asarray(values, np.float64).ravel()
    with open(path, "w") as fh:
        fh.write("%%MatrixMarket matrix array real general\n")
        fh.write("%% %s\n" % name)
        fh.write("%d 1\n" % values.size)
        for v in values:
            fh.write("%.17g\n" % v)


def read_matrix_market(path):
    """The values of a Matrix Market array file (column-major), as a flat array."""
    with open(path) as fh:
        head = fh.readline()
        if not head.startswith("%%MatrixMarket") or "array" not in head:
            raise ValueError(path + ": not a Matrix Market array file")
        line = fh.readline()
        while line.startswith("%"):
            line = fh.readline()
        m, k = (int(t) for t in line.split()[:2])
        data = np.array(fh.read().split(), np.float64)
    if data.size != m * k:
        raise ValueError(path + ": expected %d values, found %d" % (m * k, data.size))
    return data


def _number(folder):
    m = re.search(r"restart-(\d+)$", os.path.basename(os.path.normpath(folder)))
    return int(m.group(1)) if m else -1


def latest(path="."):
    """The restart folder with the highest number under `path`, or None."""
    folders = [f for f in glob.glob(os.path.join(path, "restart-*")) if os.path.isdir(f) and _number(f) >= 0]
    return max(folders, key=_number) if folders else None


def write(ctx, time, path=".", block=None, block_ids=None, block_names=None, horizon=None, density=None,
          previous=None):
    """Writes the next restart folder under `path` and returns it.

    ctx: a Context after a run (its committed state is written); time: the
    time the state belongs to; block [n] 0-based block index per point,
    block_ids (Exodus ids, default 1, 2, ...), block_names (default
    "block_<id>"), horizon and density per block (written per point, as the
    reference does). previous: the folder the run started from (default the
    latest under `path`; none means restart-000000)."""
    n = ctx.n
    block = np.zeros(n, np.int64) if block is None else np.asarray(block, np.int64)
    nblk = int(block.max()) + 1 if n else 1
    block_ids = np.arange(1, nblk + 1) if block_ids is None else np.asarray(block_ids, np.int64)
    block_names = ["block_%d" % i for i in block_ids] if block_names is None else list(block_names)
    prev = previous if previous is not None else latest(path)
    number = (_number(prev) if prev else 0) + 1
    folder = os.path.join(path, "restart-%06d" % number)
    os.makedirs(folder, exist_ok=False)
    with open(os.path.join(folder, "currentTime.txt"), "w") as fh:
        fh.write("Current time is \n%.17g\n" % time)
    x = ctx.field("Model_Coordinates")
    u = ctx.field("Displacement")
    per_block = lambda vals: np.asarray(vals, np.float64)[block] if vals is not None else np.zeros(n)
    scalars = dict(blockIDs=block_ids[block].astype(np.float64), horizon=per_block(horizon), volume=ctx.field("Volume"),
                   density=per_block(density), deltaTemperature=np.zeros(n))
    vectors = dict(x=x, u=u, y=x + u, v=ctx.field("Velocity"), a=ctx.field("Acceleration"),
                   force=ctx.field("Force_Density"), contactForce=ctx.field("Contact_Force_Density"),
                   externalForce=np.zeros(3 * n), deltaU=np.zeros(3 * n), scratch=np.zeros(3 * n))
    for k in _SCALARS:
        write_matrix_market(os.path.join(folder, k + ".mat"), scalars[k], k)
    for k in _VECTORS:
        write_matrix_market(os.path.join(folder, k + ".mat"), vectors[k], k)
    row, _ = ctx.bonds_csr()
    bd = ctx.field("Bond_Damage")
    for b in range(nblk):
        pts = np.nonzero(block == b)[0]
        sel = np.concatenate([np.arange(row[i], row[i + 1]) for i in pts]) if len(pts) else np.zeros(0, np.int64)
        for state in ("StateN", "StateNP1"):
            nm = block_names[b] + state
            write_matrix_market(os.path.join(folder, "BondData_%s.mat" % nm), bd[sel], nm)
    return folder


def read(ctx, folder=None, path=".", block=None, block_names=None, tolerance=0.0):
    """Restores displacement, velocity and committed bond damage from a
    restart folder (default the latest under `path`) into ctx and returns the
    snapshot's time. The folder's model coordinates and volumes must equal
    the context's to `tolerance` (absolute)."""
    folder = folder or latest(path)
    if folder is None:
        raise FileNotFoundError("no restart folder under " + os.path.abspath(path))
    with open(os.path.join(folder, "currentTime.txt")) as fh:
        fh.readline()
        time = float(fh.readline())
    n = ctx.n
    x = read_matrix_market(os.path.join(folder, "x.mat"))
    vol = read_matrix_market(os.path.join(folder, "volume.mat"))
    x_ctx = ctx.field("Model_Coordinates")
    if x.size != 3 * n or np.abs(x - x_ctx).max(initial=0.0) > tolerance or \
            np.abs(vol - ctx.field("Volume")).max(initial=0.0) > tolerance:
        raise ValueError("restart folder %s does not hold this context's points" % folder)
    u = read_matrix_market(os.path.join(folder, "u.mat"))
    v = read_matrix_market(os.path.join(folder, "v.mat"))
    block = np.zeros(n, np.int64) if block is None else np.asarray(block, np.int64)
    nblk = int(block.max()) + 1 if n else 1
    if block_names is None:
        ids = read_matrix_market(os.path.join(folder, "blockIDs.mat")).astype(np.int64)
        first = {int(b): int(ids[np.argmax(block == b)]) for b in range(nblk)}
        block_names = ["block_%d" % first[b] for b in range(nblk)]
    row, _ = ctx.bonds_csr()
    bd = np.zeros(int(row[-1]))
    for b in range(nblk):
        pts = np.nonzero(block == b)[0]
        if not len(pts):
            continue
        sel = np.concatenate([np.arange(row[i], row[i + 1]) for i in pts])
        vals = read_matrix_market(os.path.join(folder, "BondData_%sStateN.mat" % block_names[b]))
        if vals.size != sel.size:
            raise ValueError("restart bond data of %s holds %d bonds, the context %d" %
                             (block_names[b], vals.size, sel.size))
        bd[sel] = vals
    ctx.set_state(u, v)
    ctx.set_bond_damage(bd)
    return time
