"""CPU oracle: Python bindings over the C restatement (``oracle/libpdoracle.so``)
and over the reference's own LPS kernels compiled from its sources
(``oracle/_ref/libpdref.so``).

TEST INFRASTRUCTURE ONLY. tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it as the checker; the product package
``peridigm_b200`` never imports it.

Parity of the restatement is pinned by tests/test_oracle_golden.py (known
answers of src/materials/unit_test/utPeridigm_ElasticMaterial.cpp, the gold
Exodus files of the reference's verification/regression tests kept as
fixtures in tests/golden/) and by tests/test_oracle_vs_ref.py (the compiled
reference kernels).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpdoracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libpdref.so")

INFLUENCE = {"One": 0, "Parabolic Decay": 1, "Gaussian": 2}

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


class Plane(C.Structure):
    """Rectangular_Plane bond filter (Peridigm_Discretization.cpp:158-175)."""

    _fields_ = [
        ("normal", C.c_double * 3),
        ("lower_left", C.c_double * 3),
        ("bottom_unit", C.c_double * 3),
        ("bottom_length", C.c_double),
        ("side_length", C.c_double),
    ]


class Explicit(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("x", _dp),
        ("vol", _dp),
        ("rho", _dp),
        ("K", _dp),
        ("mu", _dp),
        ("row", _i64p),
        ("col", _i32p),
        ("influence", C.c_int),
        ("horizon", C.c_double),
        ("damage_on", C.c_int),
        ("s_c", _dp),
        ("contact_on", C.c_int),
        ("r_search", C.c_double),
        ("search_freq", C.c_int),
        ("r_contact", C.c_double),
        ("k_spring", C.c_double),
        ("friction", C.c_double),
        ("contact_horizon", _dp),
        ("bc_mask", _u8p),
        ("bc_a", _dp),
        ("bc_b", _dp),
        ("bc_vals", _dp),
        ("dt", C.c_double),
        ("t0", C.c_double),
        ("nsteps", C.c_int),
        ("material", C.c_int),
        ("plane", C.c_int),
        ("height", C.c_double),
    ]


_lib = None
_ref = None


def build(quiet: bool = True) -> None:
    """Compile the oracle (and oracle/_ref when the reference tree exists)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.pdo_influence.restype = C.c_double
        L.pdo_influence.argtypes = [C.c_int, C.c_double, C.c_double]
        L.pdo_plane_cuts_bond.argtypes = [C.POINTER(Plane), _dp, _dp]
        L.pdo_neighbor_count.restype = C.c_int64
        L.pdo_neighbor_count.argtypes = [C.c_int64, _dp, _dp, C.POINTER(Plane), C.c_int, _i32p]
        L.pdo_neighbor_fill.argtypes = [C.c_int64, _dp, _dp, C.POINTER(Plane), C.c_int, _i64p, _i32p]
        L.pdo_weighted_volume.argtypes = [C.c_int64, _dp, _dp, _i64p, _i32p, C.c_int, C.c_double, _dp]
        L.pdo_damage_critical_stretch.argtypes = [C.c_int64, _dp, _dp, _i64p, _i32p, _dp, _dp, _dp, _dp]
        L.pdo_dilatation.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _dp, _i64p, _i32p, C.c_int, C.c_double, _dp]
        L.pdo_force_lps.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _dp, _dp, _i64p, _i32p, _dp, _dp,
                                    C.c_int, C.c_double, _dp]
        L.pdo_force_bond_based.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _i64p, _i32p, _dp, C.c_double, C.c_int,
                                           C.c_double, _dp]
        L.pdo_dilatation_linear_lps.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _dp, _i64p, _i32p, C.c_int,
                                                C.c_double, _dp]
        L.pdo_force_linear_lps.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _dp, _dp, _i64p, _i32p, _dp, _dp,
                                           C.c_int, C.c_double, _dp]
        L.pdo_critical_time_step.restype = C.c_double
        L.pdo_critical_time_step.argtypes = [C.c_int64, _dp, _dp, _i64p, _i32p, _dp, _dp, C.c_double]
        L.pdo_contact_count.restype = C.c_int64
        L.pdo_contact_count.argtypes = [C.c_int64, _dp, C.c_double, _i64p, _i32p, _i32p]
        L.pdo_contact_fill.argtypes = [C.c_int64, _dp, C.c_double, _i64p, _i32p, _i64p, _i32p]
        L.pdo_contact_force.argtypes = [C.c_int64, _dp, _dp, _dp, _i64p, _i32p, C.c_double, C.c_double,
                                        C.c_double, _dp, _dp]
        L.pdo_lps_jv.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, _dp, _dp, _i64p, _i32p, _dp, _dp, C.c_int, C.c_double,
                                 _dp, _dp]
        L.pdo_explicit_run.argtypes = [C.POINTER(Explicit), _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own compiled LPS kernels, or None when not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH):
            return None
        L = C.CDLL(REF_PATH)
        L.pdref_set_influence.argtypes = [C.c_char_p]
        L.pdref_weighted_volume.argtypes = [_dp, _dp, _dp, C.c_int, _i32p, C.c_double]
        L.pdref_dilatation.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _i32p, C.c_int, C.c_double]
        L.pdref_force_linear_elastic.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _dp, _i32p, C.c_int,
                                                 C.c_double, C.c_double, C.c_double]
        L.pdref_hex_centroid_volume.argtypes = [_dp, _dp, _dp]
        L.pdref_tet_centroid_volume.argtypes = [_dp, _dp, _dp]
        L.pdref_force_bond_based.argtypes = [_dp, _dp, _dp, _dp, _dp, _i32p, C.c_int, C.c_double, C.c_double,
                                             C.c_int, C.c_double]
        _ref = L
    return _ref


def _d(a):
    return a.ctypes.data_as(_dp)


def _i64(a):
    return a.ctypes.data_as(_i64p)


def _i32(a):
    return a.ctypes.data_as(_i32p)


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None:
        assert a.size == n, (a.size, n)
    return a


def _per_point(v, n):
    a = np.asarray(v, dtype=np.float64)
    if a.ndim == 0:
        a = np.full(n, float(a))
    return np.ascontiguousarray(a)


# ---------------------------------------------------------------------------
# Neighbor-list formats
# ---------------------------------------------------------------------------
def csr_to_nl(row, col):
    """CSR -> Peridigm's flattened list [n_0, j.., n_1, j..] (NeighborhoodData.hpp:56)."""
    n = len(row) - 1
    counts = np.diff(row)
    out = np.empty(n + len(col), dtype=np.int32)
    pos = np.arange(n) + row[:-1]
    out[pos] = counts
    mask = np.ones(len(out), dtype=bool)
    mask[pos] = False
    out[mask] = col
    return out


def nl_to_csr(nl, n):
    nl = np.asarray(nl, dtype=np.int64)
    row = np.zeros(n + 1, dtype=np.int64)
    cols = []
    k = 0
    for i in range(n):
        c = int(nl[k])
        cols.append(nl[k + 1:k + 1 + c])
        row[i + 1] = row[i] + c
        k += c + 1
    col = np.concatenate(cols).astype(np.int32) if cols else np.zeros(0, np.int32)
    return row, col


def planes_array(planes):
    if not planes:
        return None, 0
    arr = (Plane * len(planes))()
    for k, p in enumerate(planes):
        arr[k].normal[:] = list(p["normal"])
        arr[k].lower_left[:] = list(p["lower_left"])
        arr[k].bottom_unit[:] = list(p["bottom_unit"])
        arr[k].bottom_length = float(p["bottom_length"])
        arr[k].side_length = float(p["side_length"])
    return arr, len(planes)


# ---------------------------------------------------------------------------
# Wrappers
# ---------------------------------------------------------------------------
def neighbor_search(x, horizon, planes=None):
    x = _f64(x)
    n = x.size // 3
    h = _per_point(horizon, n)
    parr, npl = planes_array(planes)
    counts = np.zeros(n, dtype=np.int32)
    L = lib()
    L.pdo_neighbor_count(n, _d(x), _d(h), parr, npl, _i32(counts))
    row = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=row[1:])
    col = np.zeros(int(row[-1]), dtype=np.int32)
    L.pdo_neighbor_fill(n, _d(x), _d(h), parr, npl, _i64(row), _i32(col))
    return row, col


def weighted_volume(x, vol, row, col, horizon, influence=0):
    x, vol = _f64(x), _f64(vol)
    n = vol.size
    m = np.zeros(n)
    lib().pdo_weighted_volume(n, _d(x), _d(vol), _i64(row), _i32(col), influence, horizon, _d(m))
    return m


def damage_critical_stretch(x, y, row, col, s_c, dmg_n):
    x, y = _f64(x), _f64(y)
    n = x.size // 3
    sc = _per_point(s_c, n)
    dn = _f64(dmg_n)
    dnp1 = dn.copy()
    nd = np.zeros(n)
    lib().pdo_damage_critical_stretch(n, _d(x), _d(y), _i64(row), _i32(col), _d(sc), _d(dn), _d(dnp1), _d(nd))
    return dnp1, nd


def dilatation(x, y, m, vol, dmg, row, col, horizon, influence=0):
    x, y, m, vol, dmg = _f64(x), _f64(y), _f64(m), _f64(vol), _f64(dmg)
    n = vol.size
    th = np.zeros(n)
    lib().pdo_dilatation(n, _d(x), _d(y), _d(m), _d(vol), _d(dmg), _i64(row), _i32(col), influence, horizon, _d(th))
    return th


def force_lps(x, y, m, vol, theta, dmg, row, col, K, mu, horizon, influence=0):
    x, y, m, vol, theta, dmg = map(_f64, (x, y, m, vol, theta, dmg))
    n = vol.size
    Kp, mup = _per_point(K, n), _per_point(mu, n)
    f = np.zeros(3 * n)
    lib().pdo_force_lps(n, _d(x), _d(y), _d(m), _d(vol), _d(theta), _d(dmg), _i64(row), _i32(col),
                        _d(Kp), _d(mup), influence, horizon, _d(f))
    return f


def eval_linear_lps(x, y, vol, row, col, K, mu, horizon, s_c=None, dmg_n=None, influence=0):
    """The Linear LPS material's evaluation (LinearLPSPVMaterial::precompute +
    computeForce, Peridigm_LinearLPSPVMaterial.cpp:231-394) after the damage
    model, in evalModel order: weighted volume, dilatation, force density."""
    x, y, vol = _f64(x), _f64(y), _f64(vol)
    n = vol.size
    m = weighted_volume(x, vol, row, col, horizon, influence)
    if dmg_n is None:
        dmg_n = np.zeros(len(col))
    if s_c is not None:
        dmg, nd = damage_critical_stretch(x, y, row, col, s_c, dmg_n)
    else:
        dmg, nd = np.asarray(dmg_n, dtype=np.float64).copy(), None
    th = np.zeros(n)
    lib().pdo_dilatation_linear_lps(n, _d(x), _d(y), _d(m), _d(vol), _d(dmg), _i64(row), _i32(col), influence,
                                    horizon, _d(th))
    f = np.zeros(3 * n)
    lib().pdo_force_linear_lps(n, _d(x), _d(y), _d(m), _d(vol), _d(th), _d(dmg), _i64(row), _i32(col),
                               _d(_per_point(K, n)), _d(_per_point(mu, n)), influence, horizon, _d(f))
    return {"m": m, "theta": th, "force": f, "bond_damage": dmg, "damage": nd}


def eval_model(x, y, vol, row, col, K, mu, horizon, s_c=None, dmg_n=None, influence=0, m=None):
    """ModelEvaluator::evalModel order (Peridigm_ModelEvaluator.cpp:57-131): damage -> dilatation -> force."""
    n = len(vol)
    if m is None:
        m = weighted_volume(x, vol, row, col, horizon, influence)
    if dmg_n is None:
        dmg_n = np.zeros(len(col))
    if s_c is not None:
        dmg, nd = damage_critical_stretch(x, y, row, col, s_c, dmg_n)
    else:
        dmg, nd = np.asarray(dmg_n, dtype=np.float64).copy(), None
    th = dilatation(x, y, m, vol, dmg, row, col, horizon, influence)
    f = force_lps(x, y, m, vol, th, dmg, row, col, K, mu, horizon, influence)
    return {"m": m, "theta": th, "force": f, "bond_damage": dmg, "damage": nd}


def lps_jv(x, y, vol, row, col, K, mu, horizon, w, bond_damage=None, influence=0):
    """(d f / d u) w at configuration y (force density linearization)."""
    x, y, vol, w = map(_f64, (x, y, vol, w))
    n = vol.size
    dmg = np.zeros(len(col)) if bond_damage is None else _f64(bond_damage)
    m = weighted_volume(x, vol, row, col, horizon, influence)
    th = dilatation(x, y, m, vol, dmg, row, col, horizon, influence)
    df = np.zeros(3 * n)
    lib().pdo_lps_jv(n, _d(x), _d(y), _d(m), _d(vol), _d(th), _d(dmg), _i64(row), _i32(col),
                     _d(_per_point(K, n)), _d(_per_point(mu, n)), influence, horizon, _d(w), _d(df))
    return df


def tangent_dense(x, y, vol, row, col, K, mu, horizon, bc_dofs=(), bond_damage=None):
    """Dense quasi-static tangent -d(V f)/du (Peridigm.cpp:2793-2800: V-weighted
    Jacobian, Scale(-1)), BC rows/columns replaced by identity (small n only)."""
    n = len(vol)
    T = np.zeros((3 * n, 3 * n))
    for k in range(3 * n):
        e = np.zeros(3 * n)
        e[k] = 1.0
        T[:, k] = -np.repeat(np.asarray(vol, float), 3) * lps_jv(x, y, vol, row, col, K, mu, horizon, e, bond_damage)
    for k in bc_dofs:
        T[k, :] = 0.0
        T[:, k] = 0.0
        T[k, k] = 1.0
    return T


def qs_residual(x, u, vol, row, col, K, mu, horizon, bc_dofs=(), bond_damage=None):
    """Peridigm::computeQuasiStaticResidual (Peridigm.cpp:4176-4317): r = V (f_int + f_ext),
    BC rows zeroed; returns (r, ||r||_2 + 20 ||r||_inf)."""
    y = _f64(x) + _f64(u)
    f = eval_model(x, y, vol, row, col, K, mu, horizon, dmg_n=bond_damage)["force"]
    r = np.repeat(np.asarray(vol, float), 3) * f
    r[list(bc_dofs)] = 0.0
    return r, float(np.linalg.norm(r) + 20.0 * np.abs(r).max())


def qs_solve(x, vol, row, col, K, mu, horizon, bc, times, tol, max_iter=50, u0=None):
    """Quasi-static load steps restated from Peridigm::executeQuasiStatic
    (Peridigm.cpp:2651-3043) with a dense linear solve in place of Belos CG and
    full Newton steps: per step, prescribed increments on the BC dofs, then
    Newton on the free dofs until ||r||_2 + 20||r||_inf <= tol.
    bc: list of (dof, a, b) with u_dof(t) = a t + b; a zero increment takes
    the previous value from u (Peridigm_BoundaryCondition.cpp:137-142).
    Returns u per time."""
    n = len(vol)
    u = np.zeros(3 * n) if u0 is None else _f64(u0).copy()
    dofs = [d for d, a, b in bc]
    out = [u.copy()]
    for s in range(1, len(times)):
        tp, tc = times[s - 1], times[s]
        for d, a, b in bc:
            inc = (a * tc + b) - (a * tp + b)
            # a zero increment takes the previous value from the displacement
            # (Peridigm_BoundaryCondition.cpp:137-142)
            u[d] += inc if inc != 0.0 else (a * tc + b) - u[d]
        r, nrm = qs_residual(x, u, vol, row, col, K, mu, horizon, dofs)
        it = 0
        while nrm > tol and it < max_iter:
            T = tangent_dense(x, _f64(x) + u, vol, row, col, K, mu, horizon, dofs)
            du = np.linalg.solve(T, r)
            du[dofs] = 0.0
            u += du
            r, nrm = qs_residual(x, u, vol, row, col, K, mu, horizon, dofs)
            it += 1
        out.append(u.copy())
    return out


def implicit_newmark(x, vol, row, col, K, mu, rho, horizon, u0, v0, dt, nsteps, beta=0.25, gamma=0.5,
                     tol=1.0e-6, max_iter=10, bc_dofs=()):
    """Implicit dynamics restated from Peridigm::executeImplicit
    (Peridigm.cpp:3620-4016) with a dense linear solve in place of Belos CG.
    Per step: u2 = un + dt vn + 0.5 dt^2 (1 - 2 beta) an, v2 = vn + dt (1 -
    gamma) an (:3726-3730); u = u2, a = (u - u2)/(beta dt^2), v = v2 + dt
    gamma a (:3752-3759); R = beta dt^2 (rho a - f) with the prescribed rows
    zeroed (:3803-3810); while ||R||_2 > tol and at most max_iter + 1 times
    (:3815): J = rho I + beta dt^2 K with K = -d(V f)/du
    (computeImplicitJacobian :4319-4338), prescribed rows and columns zeroed
    with a unit diagonal, J du = -R, u += du, a and v updated, R recomputed.
    Prescribed dofs keep the predictor (the solve leaves them alone). rho per
    point or scalar. Returns per step (u, v, a, f, Newton iterations)."""
    n = len(vol)
    rho3 = np.repeat(_per_point(rho, n), 3)
    bc = list(bc_dofs)
    u, v, a = _f64(u0).copy(), _f64(v0).copy(), np.zeros(3 * n)
    bdt2 = beta * (dt * dt)
    out = []
    for _ in range(nsteps):
        un, vn, an = u.copy(), v.copy(), a.copy()
        u2 = (un + dt * vn) + (0.5 * (dt * dt) * (1.0 - 2.0 * beta)) * an
        v2 = vn + (dt * (1.0 - gamma)) * an
        u = u2.copy()
        a = (u - u2) * (1.0 / bdt2)
        v = v2 + (dt * gamma) * a

        def resid(u, a):
            f = eval_model(x, _f64(x) + u, vol, row, col, K, mu, horizon)["force"]
            R = bdt2 * (rho3 * a - f)
            R[bc] = 0.0
            return f, R

        f, R = resid(u, a)
        it = 0
        while np.linalg.norm(R) > tol and it <= max_iter:
            J = bdt2 * tangent_dense(x, _f64(x) + u, vol, row, col, K, mu, horizon) + np.diag(rho3)
            for d in bc:
                J[d, :] = 0.0
                J[:, d] = 0.0
                J[d, d] = 1.0
            du = np.linalg.solve(J, -R)
            du[bc] = 0.0
            u = u + du
            a = (u - u2) * (1.0 / bdt2)
            v = v2 + (dt * gamma) * a
            f, R = resid(u, a)
            it += 1
        out.append((u.copy(), v.copy(), a.copy(), f.copy(), it))
    return out


def coarse_aggregates(x, horizon_max, cell=0.0, max_coarse=6144, modes=3):
    """Aggregates of the two-level preconditioner (no reference counterpart):
    the non-empty cells, numbered in cell order (x fastest), of a grid of side
    max(cell, 2 * max horizon * (1 + 1e-6)) from the coordinate minimum, dims =
    floor(extent / side) + 1 per axis, the side grown 1.25x until there are at
    most max_coarse / modes aggregates. Returns (aggregate of each point, side)."""
    x = _f64(x).reshape(-1, 3)
    lo, hi = x.min(axis=0), x.max(axis=0)
    side = max(float(cell), 2.0 * float(horizon_max) * (1.0 + 1.0e-6))
    while True:
        dims = np.floor((hi - lo) / side).astype(np.int64) + 1
        if 3 * min(int(np.prod(dims)), x.shape[0]) > 64 * max_coarse:  # far too fine: grow before binning
            side *= 1.25
            continue
        c = np.clip(np.floor((x - lo) / side).astype(np.int64), 0, dims - 1)
        cid = (c[:, 2] * dims[1] + c[:, 1]) * dims[0] + c[:, 0]
        cells = np.unique(cid)
        if modes * cells.size <= max_coarse:
            return np.searchsorted(cells, cid).astype(np.int32), side
        side *= 1.25


def coarse_operator(T, agg, fixed_dofs=()):
    """Galerkin coarse matrix P0^T T P0 of the two-level preconditioner: P0 maps
    coarse dof 3I + c to component c of the free dofs of the points of aggregate
    I (piecewise-constant translations, prescribed dofs excluded); a coarse dof
    with no free fine dof gets a unit diagonal. Returns (Ac, P0)."""
    agg = np.asarray(agg, np.int64)
    n = agg.size
    nc = 3 * (int(agg.max()) + 1)
    P = np.zeros((3 * n, nc))
    for i in range(n):
        for c in range(3):
            P[3 * i + c, 3 * agg[i] + c] = 1.0
    P[list(fixed_dofs), :] = 0.0
    A = P.T @ T @ P
    for k in range(nc):
        if A[k, k] == 0.0:
            A[k, k] = 1.0
    return A, P


def gauss_jordan_blocked(A, bk=64):
    """In-place blocked Gauss-Jordan inverse without pivoting of an SPD matrix
    with every entry updated, in numpy: the step structure that
    gauss_jordan_sym_blocked (the form peridigm_b200/csrc/k_coarse.cu runs)
    restricts to the tiles on and above the diagonal. For each block k of
    width bk (the last one ragged):

      P  = A_kk^-1                      (pivot block)
      R  = P A_k*, with P itself in R's block-k columns   (row panel)
      Ct = A_*k^T                       (old block column, transposed)
      rows i of block k:   A_i* = R_(i-k0)*
      other rows i:        A_ij = [j outside block k] A_ij - (Ct_*i . R_*j)

    which is A_ij -= C_i R_j, A_kj = R_j, A_ik = -C_i P and A_kk = P. Returns the
    inverse (a new array)."""
    A = np.array(A, dtype=np.float64, copy=True)
    nc = A.shape[0]
    for k0 in range(0, nc, bk):
        k1 = min(nc, k0 + bk)
        P = np.linalg.inv(A[k0:k1, k0:k1])
        R = P @ A[k0:k1, :]
        R[:, k0:k1] = P
        Ct = A[:, k0:k1].T.copy()
        upd = Ct.T @ R
        keep = np.ones(nc, bool)
        keep[k0:k1] = False
        A[:, ~keep] = 0.0
        A -= upd
        A[k0:k1, :] = R
    return A


def gauss_jordan_sym_blocked(A, bk=64, tile=128):
    """The symmetric form of gauss_jordan_blocked that k_coarse.cu runs
    (k_gj_pivot, k_gj_panel_sym, k_gj_update on the tiles on and above the
    diagonal, k_gj_mirror), in numpy. Sweeping pivot blocks of a symmetric
    matrix keeps it sign-symmetric: M_ba = -M_ab when exactly one of a, b lies
    in a block already swept, M_ba = M_ab otherwise (the inverse, all blocks
    swept, is symmetric). So only the entries of tiles (I, J), I <= J (tile
    side `tile`, a multiple of bk), are kept; for block k (rows k0..k1):

      P  = A_kk^-1                   (the diagonal tile holds every entry)
      W  = the true block row M_k*:  A[k, j] where tile(j) >= tile(k0),
                                     -A[j, k] where tile(j) < tile(k0)
      R  = P W, with P in R's block-k columns
      Ct = s W, s_j = -1 for j < k0  (the true block column, transposed)
      kept entries (i, j): rows of block k take R, the others
                           [j outside block k] A_ij - (Ct_*i . R_*j)

    and at the end every entry below the diagonal is the transpose of the one
    above (inside the diagonal tiles too, where both halves were kept and
    round apart): the inverse is exactly symmetric. Returns it (a new array)."""
    A = np.array(A, dtype=np.float64, copy=True)
    nc = A.shape[0]
    tid = np.arange(nc) // tile
    kept = tid[:, None] <= tid[None, :]
    A[~kept] = np.nan  # never read
    for k0 in range(0, nc, bk):
        k1 = min(nc, k0 + bk)
        tk = k0 // tile
        P = np.linalg.inv(A[k0:k1, k0:k1])
        W = np.where((tid >= tk)[None, :], A[k0:k1, :], -A[:, k0:k1].T)
        Ct = W * np.where(np.arange(nc) < k0, -1.0, 1.0)[None, :]
        R = P @ W
        R[:, k0:k1] = P
        outside = np.ones(nc, bool)
        outside[k0:k1] = False
        new = np.where(outside[None, :], A, 0.0) - Ct.T @ R
        new[k0:k1, :] = R
        A = np.where(kept, new, A)
    low = np.tril(np.ones((nc, nc), bool), -1)
    A[low] = A.T[low]
    return A


def coarse_operator_rigid(T, x, agg, side, fixed_dofs=()):
    """Galerkin coarse matrix of the rigid coarse space (6 modes per aggregate,
    no reference counterpart): per aggregate the translations and the
    rotations about its center (mean of its points), scaled by 1/side,
    prescribed dofs masked, orthonormalised by QR with the columns whose
    |R_kk| falls below 1e-4 of the largest dropped (1e-8 of the Gram
    pivots, as the GPU's Cholesky does); dropped coarse dofs get a unit
    diagonal. The basis differs from the GPU's by an orthogonal 6x6 map per
    aggregate, so compare basis-free quantities. Returns (Ac, P)."""
    x = _f64(x).reshape(-1, 3)
    agg = np.asarray(agg, np.int64)
    n = agg.size
    na = int(agg.max()) + 1
    P = np.zeros((3 * n, 6 * na))
    fixed = np.zeros(3 * n, bool)
    fixed[list(fixed_dofs)] = True
    for a in range(na):
        pts = np.nonzero(agg == a)[0]
        c = x[pts].mean(axis=0)
        d = (x[pts] - c) / side
        B = np.zeros((3 * pts.size, 6))
        for k in range(3):
            B[k::3, k] = 1.0
        B[0::3, 3], B[1::3, 3] = -d[:, 1], d[:, 0]
        B[1::3, 4], B[2::3, 4] = -d[:, 2], d[:, 1]
        B[2::3, 5], B[0::3, 5] = -d[:, 0], d[:, 2]
        rows = (3 * pts[:, None] + np.arange(3)).ravel()
        B[fixed[rows]] = 0.0
        Q, Rm = np.linalg.qr(B)
        dg = np.abs(np.diag(Rm))
        keep = dg > 1e-4 * dg.max() if dg.max() > 0 else np.zeros(6, bool)
        P[np.ix_(rows, 6 * a + np.nonzero(keep)[0])] = Q[:, keep]
    A = P.T @ T @ P
    for k in range(6 * na):
        if A[k, k] == 0.0:
            A[k, k] = 1.0
    return A, P


def critical_time_step(x, vol, row, col, K, rho, horizon):
    x, vol = _f64(x), _f64(vol)
    n = vol.size
    return lib().pdo_critical_time_step(n, _d(x), _d(vol), _i64(row), _i32(col), _d(_per_point(K, n)),
                                        _d(_per_point(rho, n)), horizon)


def contact_search(y, r_search, brow, bcol):
    y = _f64(y)
    n = y.size // 3
    counts = np.zeros(n, dtype=np.int32)
    L = lib()
    L.pdo_contact_count(n, _d(y), r_search, _i64(brow), _i32(bcol), _i32(counts))
    crow = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=crow[1:])
    ccol = np.zeros(int(crow[-1]), dtype=np.int32)
    L.pdo_contact_fill(n, _d(y), r_search, _i64(brow), _i32(bcol), _i64(crow), _i32(ccol))
    return crow, ccol


def contact_force(y, v, vol, crow, ccol, r_contact, k_spring, horizon, friction=0.0):
    y, v, vol = _f64(y), _f64(v), _f64(vol)
    n = vol.size
    fc = np.zeros(3 * n)
    lib().pdo_contact_force(n, _d(y), _d(v), _d(vol), _i64(crow), _i32(ccol), r_contact, k_spring, friction,
                            _d(_per_point(horizon, n)), _d(fc))
    return fc


def explicit_run(prob, u, v, bond_damage=None):
    """Peridigm::executeExplicit restated (Peridigm.cpp:1290-1593).

    ``prob`` keys: x, vol, rho, K, mu, row, col, horizon, dt, nsteps; optional
    influence, s_c (enables damage), contact dict {r_search, freq, r_contact,
    k_spring, friction, horizon}, bc_mask/bc_a/bc_b (or bc_vals, the prescribed
    values at t0 + k dt, k = 0..nsteps, for non-linear prescribed functions),
    t0, material ("lps" or "bond_based") with plane/height for the bond-based
    constant.
    """
    x = _f64(prob["x"])
    n = x.size // 3
    keep = []

    def arr(a):
        a = np.ascontiguousarray(a)
        keep.append(a)
        return a

    vol = arr(_f64(prob["vol"]))
    row = arr(np.asarray(prob["row"], np.int64))
    col = arr(np.asarray(prob["col"], np.int32))
    P = Explicit()
    P.n = n
    P.x = _d(arr(x))
    P.vol = _d(vol)
    P.rho = _d(arr(_per_point(prob["rho"], n)))
    P.K = _d(arr(_per_point(prob["K"], n)))
    P.mu = _d(arr(_per_point(prob["mu"], n)))
    P.row = _i64(row)
    P.col = _i32(col)
    P.influence = int(prob.get("influence", 0))
    P.horizon = float(prob["horizon"])
    P.material = 1 if prob.get("material", "lps") == "bond_based" else 0
    P.plane = 1 if prob.get("plane", False) else 0
    P.height = float(prob.get("height", 0.0))
    sc = prob.get("s_c")
    P.damage_on = 1 if sc is not None else 0
    P.s_c = _d(arr(_per_point(sc if sc is not None else 0.0, n)))
    ct = prob.get("contact")
    P.contact_on = 1 if ct else 0
    if ct:
        P.r_search = ct["r_search"]
        P.search_freq = int(ct["freq"])
        P.r_contact = ct["r_contact"]
        P.k_spring = ct["k_spring"]
        P.friction = ct.get("friction", 0.0)
        P.contact_horizon = _d(arr(_per_point(ct["horizon"], n)))
    if prob.get("bc_mask") is not None:
        P.bc_mask = arr(np.asarray(prob["bc_mask"], np.uint8)).ctypes.data_as(_u8p)
        P.bc_a = _d(arr(_f64(prob["bc_a"])))
        P.bc_b = _d(arr(_f64(prob["bc_b"])))
        if prob.get("bc_vals") is not None:  # [(nsteps+1) x 3n] prescribed values at t0 + k dt
            bv = arr(_f64(prob["bc_vals"]))
            assert bv.size == (int(prob["nsteps"]) + 1) * 3 * n
            P.bc_vals = _d(bv)
    P.dt = float(prob["dt"])
    P.t0 = float(prob.get("t0", 0.0))
    P.nsteps = int(prob["nsteps"])
    u = _f64(u).copy()
    v = _f64(v).copy()
    a = np.zeros(3 * n)
    f = np.zeros(3 * n)
    fc = np.zeros(3 * n)
    th = np.zeros(n)
    nd = np.zeros(n)
    bd = np.zeros(len(col)) if bond_damage is None else _f64(bond_damage).copy()
    lib().pdo_explicit_run(C.byref(P), _d(u), _d(v), _d(a), _d(f), _d(fc), _d(th), _d(nd), _d(bd))
    return {"u": u, "v": v, "a": a, "force": f, "contact_force": fc, "theta": th, "damage": nd,
            "bond_damage": bd}


# ---------------------------------------------------------------------------
# Reference kernels (compiled from the reference's sources)
# ---------------------------------------------------------------------------
def force_bond_based(x, y, vol, row, col, K, horizon, bond_damage=None, plane=False, height=0.0):
    """Restated computeInternalForceElasticBondBased (elastic_bond_based.cxx:55-124)."""
    x, y, vol = _f64(x), _f64(y), _f64(vol)
    n = vol.size
    row = np.asarray(row, np.int64)
    dmg = np.zeros(int(row[-1])) if bond_damage is None else _f64(bond_damage)
    f = np.zeros(3 * n)
    lib().pdo_force_bond_based(n, _d(x), _d(y), _d(vol), _d(dmg), _i64(row), _i32(col),
                               _d(_per_point(K, n)), float(horizon), 1 if plane else 0, float(height), _d(f))
    return f


def ref_force_bond_based(x, y, vol, nl, n, K, horizon, bond_damage=None, plane=False, height=0.0):
    """The reference's own computeInternalForceElasticBondBased<double>, compiled
    from src/materials/elastic_bond_based.cxx, on a zeroed force vector."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libpdref.so is not built")
    x, y, vol = _f64(x), _f64(y), _f64(vol)
    nl = np.ascontiguousarray(nl, dtype=np.int32)
    nb = len(nl) - n
    dmg = np.zeros(nb) if bond_damage is None else _f64(bond_damage)
    f = np.zeros(3 * n)
    L.pdref_force_bond_based(_d(x), _d(y), _d(vol), _d(dmg), _d(f), _i32(nl), n, float(K), float(horizon),
                             1 if plane else 0, float(height))
    return f


def ref_element_point(nodes):
    """(centroid, volume) of one hex (8x3) or tet (4x3) element by the
    reference's compiled hexCentroidAndVolume / tetCentroidAndVolume."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libpdref.so is not built")
    P = np.ascontiguousarray(nodes, np.float64).ravel()
    c = np.zeros(3)
    v = np.zeros(1)
    (L.pdref_hex_centroid_volume if P.size == 24 else L.pdref_tet_centroid_volume)(_d(P), _d(c), _d(v))
    return c, v[0]


def ref_eval(x, y, vol, nl, n, K, mu, horizon, bond_damage=None):
    """computeWeightedVolume + computeDilatation + computeInternalForceLinearElastic
    exactly as ElasticMaterial::initialize/computeForce call them
    (Peridigm_ElasticMaterial.cpp:137, :170-171)."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libpdref.so is not built")
    x, y, vol = _f64(x), _f64(y), _f64(vol)
    nl = np.ascontiguousarray(nl, dtype=np.int32)
    nb = len(nl) - n
    dmg = np.zeros(nb) if bond_damage is None else _f64(bond_damage)
    m = np.zeros(n)
    th = np.zeros(n)
    f = np.zeros(3 * n)
    L.pdref_weighted_volume(_d(x), _d(vol), _d(m), n, _i32(nl), horizon)
    L.pdref_dilatation(_d(x), _d(y), _d(m), _d(vol), _d(dmg), _d(th), _i32(nl), n, horizon)
    L.pdref_force_linear_elastic(_d(x), _d(y), _d(m), _d(vol), _d(th), _d(dmg), _d(f), _i32(nl), n, K, mu,
                                 horizon)
    return {"m": m, "theta": th, "force": f}
