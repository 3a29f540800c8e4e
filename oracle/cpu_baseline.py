"""CPU baseline of the explicit LPS + damage step on the host cores.

TEST / MEASUREMENT INFRASTRUCTURE ONLY (used by bench.py's cpu_baseline leg
and its ``--impl reference`` arm). It times the reference's own compiled
kernels (oracle/_ref/libpdref.so: computeDilatation and
computeInternalForceLinearElastic built from the reference sources) when that
library exists, else the oracle's C restatement; damage is the oracle's
restatement of CriticalStretchDamageModel::computeDamage and the Verlet update
is a numpy restatement of Peridigm::executeExplicit's vector loops.

Decomposition mirrors the reference's MPI layout: P worker processes, each
owning a slab of points along x with a one-horizon ghost layer, points in the
owned-first overlap order Peridigm uses (owned ids first, ghosts after), the
force pass scattering into ghost entries as elastic.cxx:128-130 does. The
export of ghost forces and the halo import are not performed, so the baseline
is optimistic for the CPU. Workers start with the ``spawn`` method.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np


def _slab_problem(x, vol, row, col, lo, hi):
    n = vol.size
    X = x.reshape(-1, 3)[:, 0]
    owned = np.nonzero((X >= lo) & (X < hi))[0]
    if owned.size == 0:
        return None
    nbr = np.concatenate([col[row[i]:row[i + 1]] for i in owned]) if owned.size else np.zeros(0, np.int32)
    ghosts = np.setdiff1d(np.unique(nbr), owned)
    overlap = np.concatenate([owned, ghosts])
    g2l = -np.ones(n, np.int64)
    g2l[overlap] = np.arange(overlap.size)
    counts = np.diff(row)[owned]
    lrow = np.zeros(owned.size + 1, np.int64)
    np.cumsum(counts, out=lrow[1:])
    lcol = g2l[nbr].astype(np.int32)
    xo = x.reshape(-1, 3)[overlap].ravel().copy()
    return dict(n_owned=owned.size, x=xo, vol=vol[overlap].copy(), row=lrow, col=lcol, owned=owned)


def _worker(args):
    """Runs `steps` explicit steps on one slab; returns (seconds, owned bonds)."""
    prob, K, mu, rho, s_c, horizon, steps, use_ref, dt, warmup = args
    from oracle import oracle as O

    n_own = prob["n_owned"]
    x, vol, row, col = prob["x"], prob["vol"], prob["row"], prob["col"]
    n_ov = vol.size
    nl = O.csr_to_nl(row, col)
    m = np.zeros(n_ov)
    L = O.lib()
    R = O.ref_lib() if use_ref else None
    _d = O._d
    # weighted volume of owned points (ElasticMaterial::initialize)
    if R is not None:
        R.pdref_weighted_volume(_d(x), _d(vol), _d(m), n_own, O._i32(nl), horizon)
    else:
        L.pdo_weighted_volume(n_own, _d(x), _d(vol), O._i64(row), O._i32(col), 0, horizon, _d(m))
    u = np.zeros(3 * n_ov)
    v = np.zeros(3 * n_ov)
    a = np.zeros(3 * n_ov)
    y = x.copy()
    f = np.zeros(3 * n_ov)
    th = np.zeros(n_ov)
    nb = int(row[-1])
    dn = np.zeros(max(nb, 1))
    dnp1 = np.zeros(max(nb, 1))
    nd = np.zeros(n_ov)
    scp = np.full(n_ov, s_c if s_c is not None else 1e300)
    Kp, mup = np.full(n_ov, K), np.full(n_ov, mu)
    dt2 = dt / 2.0

    def step():
        nonlocal dn, dnp1
        v[:] = v + dt2 * a
        y[:] = x + u + dt * v
        u[:] = u + dt * v
        L.pdo_damage_critical_stretch(n_own, _d(x), _d(y), O._i64(row), O._i32(col), _d(scp), _d(dn), _d(dnp1),
                                      _d(nd))
        f[:] = 0.0
        if R is not None:
            R.pdref_dilatation(_d(x), _d(y), _d(m), _d(vol), _d(dnp1), _d(th), O._i32(nl), n_own, horizon)
            R.pdref_force_linear_elastic(_d(x), _d(y), _d(m), _d(vol), _d(th), _d(dnp1), _d(f), O._i32(nl), n_own,
                                         K, mu, horizon)
        else:
            L.pdo_dilatation(n_own, _d(x), _d(y), _d(m), _d(vol), _d(dnp1), O._i64(row), O._i32(col), 0, horizon,
                             _d(th))
            L.pdo_force_lps(n_own, _d(x), _d(y), _d(m), _d(vol), _d(th), _d(dnp1), O._i64(row), O._i32(col), _d(Kp),
                            _d(mup), 0, horizon, _d(f))
        a[:] = f / rho
        v[:] = v + dt2 * a
        dn, dnp1 = dnp1, dn

    for _ in range(max(1, warmup)):
        step()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    return time.perf_counter() - t0, nb


def run(w, row, col, steps, processes=None, dt=None, warmup=1):
    """Time `steps` explicit steps of workload dict `w` (bond family row/col) on
    `processes` host processes. Returns a dict with the rate in bond evals/s."""
    from oracle import oracle as O

    P = processes or os.cpu_count() or 1
    x, vol = w["x"], w["vol"]
    X = x.reshape(-1, 3)[:, 0]
    edges = np.quantile(X, np.linspace(0, 1, P + 1))
    edges[-1] = np.nextafter(edges[-1], np.inf)
    probs = [_slab_problem(x, vol, row, col, edges[k], edges[k + 1]) for k in range(P)]
    probs = [p for p in probs if p is not None]
    use_ref = O.ref_lib() is not None
    K = float(np.median(w["K"])) if np.ndim(w["K"]) else float(w["K"])
    mu = float(np.median(w["mu"])) if np.ndim(w["mu"]) else float(w["mu"])
    s_c = w.get("s_c")
    if s_c is not None and np.ndim(s_c):
        s_c = float(np.median(s_c))
    if dt is None:
        dt = 0.7 * O.critical_time_step(x, vol, row, col, K, w["rho"], w["horizon"])
    args = [(p, K, mu, float(w["rho"]), s_c, float(w["horizon"]), steps, use_ref, dt, warmup) for p in probs]
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(args)) as pool:
        res = pool.map(_worker, args)
    tmax = max(r[0] for r in res)
    nb = sum(r[1] for r in res)
    return {"value": nb * steps / tmax, "seconds": tmax, "bonds": nb, "steps": steps, "cores": len(args),
            "kind": "reference" if use_ref else "port"}
