"""Python side of oracle/cpu_qs.c: the threaded CPU restatement of the
quasi-static block-Jacobi CG step.

TEST / MEASUREMENT INFRASTRUCTURE ONLY: tests/test_cpu_qs.py checks it against
the oracle's dense tangent, and bench.py's quasi-static leg times it on the
host cores as the CPU baseline (seconds per CG iteration and per Newton
set-up, scaled by the block-Jacobi solve's counts)."""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from oracle import oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
_L = None
_dp = C.POINTER(C.c_double)
_u8 = C.POINTER(C.c_uint8)


def lib():
    global _L
    if _L is None:
        path = os.path.join(_HERE, "libpdqs.so")
        if not os.path.exists(path):
            O.build()
        L = C.CDLL(path)
        common = [C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        L.pdq_set_threads.argtypes = [C.c_int]
        L.pdq_bond_geom.argtypes = common + [_u8, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.pdq_block_jacobi.argtypes = common + [_dp, _dp, _dp, _dp, _dp, _dp, _u8, _dp]
        L.pdq_tangent.argtypes = common + [_dp, _dp, _dp, _dp, _dp, _dp, _u8, _dp, _dp, _dp]
        L.pdq_bj_cg.restype = C.c_double
        L.pdq_bj_cg.argtypes = common + [_dp, _dp, _dp, _dp, _dp, _dp, _u8, _dp, _dp, _dp, C.c_int, _dp]
        _L = L
    return _L


def _d(a):
    return a.ctypes.data_as(_dp)


class Problem:
    """The state the CG step needs: geometry at y, weighted volume, dilatation,
    moduli per point, prescribed-dof mask and block-Jacobi inverse blocks."""

    def __init__(self, x, y, vol, row, col, K, mu, horizon, fixed=None, bond_damage=None, threads=1):
        n = len(vol)
        self.n = n
        self.x, self.y, self.vol = (np.ascontiguousarray(a, np.float64) for a in (x, y, vol))
        self.row, self.col = np.ascontiguousarray(row, np.int64), np.ascontiguousarray(col, np.int32)
        nb = len(col)
        self.dmg = np.zeros(nb, np.uint8) if bond_damage is None else np.asarray(bond_damage, np.uint8)
        self.K = np.ascontiguousarray(np.broadcast_to(np.asarray(K, np.float64), (n,)))
        self.mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu, np.float64), (n,)))
        self.fixed = np.zeros(n, np.uint8) if fixed is None else np.ascontiguousarray(fixed, np.uint8)
        self.m = O.weighted_volume(self.x, self.vol, row, col, horizon)
        self.theta = O.dilatation(self.x, self.y, self.m, self.vol, self.dmg.astype(np.float64), row, col, horizon)
        self.g = np.zeros(4 * nb)
        self.gc = np.zeros(2 * nb)
        self.dinv = np.zeros(9 * n)
        lib().pdq_set_threads(int(threads))

    def _rc(self):
        return self.n, self.row.ctypes.data_as(C.POINTER(C.c_int64)), self.col.ctypes.data_as(C.POINTER(C.c_int32))

    def setup(self):
        """Per-bond geometry and block-Jacobi blocks (once per Newton iteration)."""
        L = lib()
        L.pdq_bond_geom(*self._rc(), self.dmg.ctypes.data_as(_u8), _d(self.x), _d(self.y), _d(self.vol), _d(self.m),
                        _d(self.theta), _d(self.K), _d(self.mu), _d(self.g), _d(self.gc))
        L.pdq_block_jacobi(*self._rc(), _d(self.g), _d(self.gc), _d(self.vol), _d(self.m), _d(self.K), _d(self.mu),
                           self.fixed.ctypes.data_as(_u8), _d(self.dinv))

    def apply(self, p):
        p = np.ascontiguousarray(p, np.float64)
        q, dth = np.zeros(3 * self.n), np.zeros(4 * self.n)  # dilatation increments + masked direction
        lib().pdq_tangent(*self._rc(), _d(self.g), _d(self.gc), _d(self.vol), _d(self.m), _d(self.K), _d(self.mu),
                          self.fixed.ctypes.data_as(_u8), _d(p), _d(dth), _d(q))
        return q

    def cg(self, b, iters):
        r = np.ascontiguousarray(b, np.float64).copy()
        x = np.zeros(3 * self.n)
        work = np.zeros(13 * self.n)
        rel = lib().pdq_bj_cg(*self._rc(), _d(self.g), _d(self.gc), _d(self.vol), _d(self.m), _d(self.K), _d(self.mu),
                              self.fixed.ctypes.data_as(_u8), _d(self.dinv), _d(r), _d(x), int(iters), _d(work))
        return x, r, rel


def sample(x, y, vol, row, col, K, mu, horizon, fixed, threads, cg_iters=20, seed=0):
    """Seconds of one Newton set-up (force evaluation, geometry, blocks) and
    of one block-Jacobi CG iteration on `threads` host threads, from a run of
    `cg_iters` iterations on a random right-hand side."""
    t0 = time.perf_counter()
    P = Problem(x, y, vol, row, col, K, mu, horizon, fixed=fixed, threads=threads)
    t_eval = time.perf_counter() - t0  # weighted volume + dilatation of the oracle (the force pass is alike)
    t1 = time.perf_counter()
    P.setup()
    t_setup = time.perf_counter() - t1
    b = np.random.default_rng(seed).normal(size=3 * len(vol))
    b[np.repeat(fixed, 3).astype(bool) & (np.tile([1, 2, 4], len(vol)) & np.repeat(fixed, 3)).astype(bool)] = 0.0
    t2 = time.perf_counter()
    P.cg(b, cg_iters)
    t_cg = (time.perf_counter() - t2) / cg_iters
    return {"seconds_per_cg_iteration": t_cg, "seconds_per_newton_setup": t_setup + t_eval, "threads": threads,
            "cg_iterations_sampled": cg_iters}
