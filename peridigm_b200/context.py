"""Thin Python owner of one ``pd_ctx`` (include/pd_b200.h).

Every method maps to one C entry point, converts numpy arrays to pointers and
raises :class:`PDError` on a non-zero status, the way the reference raises
(TEUCHOS_TEST_FOR_EXCEPT) or terminates (TEUCHOS_TEST_FOR_TERMINATION).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import PDError

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


def _d(a):
    return a.ctypes.data_as(_dp)


def _f64(a, size=None, name="array"):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if size is not None and a.size != size:
        raise ValueError(f"{name}: expected {size} values, got {a.size}")
    return a


def expr_eval(function, x=0.0, y=0.0, z=0.0, t=0.0):
    """A prescribed-displacement "Value" string evaluated once on the host
    (pd_expr_eval; no device needed): the value the explicit path prescribes
    at model coordinates (x, y, z) and time t."""
    L = _lib.load()
    out = C.c_double()
    rc = L.pd_expr_eval(function.encode(), float(x), float(y), float(z), float(t), C.byref(out))
    if rc != 0:
        raise PDError(rc, f"boundary-condition function {function!r} does not compile")
    return out.value


class Context:
    """One device-resident discretization (points, bond family, material, state)."""

    def __init__(self, device=0, precision="split", influence="One", threads_per_point=0):
        self.L = _lib.load()
        cfg = _lib.Config()
        cfg.device = int(device)
        names = {"fp64": _lib.PD_FP64, "split": _lib.PD_SPLIT_FP32, "split_fp32": _lib.PD_SPLIT_FP32,
                 "fp64_sliced": _lib.PD_FP64_SLICED}
        if precision in names:
            cfg.precision = names[precision]
        elif precision in names.values():
            cfg.precision = int(precision)
        else:
            raise ValueError(f"precision {precision!r}: one of {sorted(names)}")
        cfg.influence = {"One": 0, "Parabolic Decay": 1, "Gaussian": 2}[influence]
        cfg.threads_per_point = int(threads_per_point)
        h = C.c_void_p()
        rc = self.L.pd_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise PDError(rc, "pd_create failed (no CUDA device or bad configuration)")
        self.h = h
        self.precision = cfg.precision
        self.n = 0

    # -- plumbing -----------------------------------------------------------
    def _ok(self, rc):
        if rc != 0:
            raise PDError(rc, self.L.pd_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.pd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- discretization -----------------------------------------------------
    def set_points(self, x, vol, block=None):
        vol = _f64(vol, name="vol")
        n = vol.size
        x = _f64(x, 3 * n, "x")
        self._keep_x = x
        blk = None
        if block is not None:
            blk = np.ascontiguousarray(block, dtype=np.int32)
            if blk.size != n:
                raise ValueError("block: one id per point")
        self._ok(self.L.pd_set_points(self.h, n, _d(x), _d(vol), blk.ctypes.data_as(_i32p) if blk is not None else None))
        self.n = n

    def set_horizons(self, horizons):
        h = _f64(np.atleast_1d(horizons))
        self._ok(self.L.pd_set_block_horizons(self.h, h.size, _d(h)))

    def build_bonds(self, planes=()):
        arr = None
        if planes:
            arr = (_lib.PlaneFilter * len(planes))()
            for k, p in enumerate(planes):
                arr[k].normal[:] = [float(v) for v in p["normal"]]
                arr[k].lower_left[:] = [float(v) for v in p["lower_left"]]
                arr[k].bottom_unit[:] = [float(v) for v in p["bottom_unit"]]
                arr[k].bottom_length = float(p["bottom_length"])
                arr[k].side_length = float(p["side_length"])
        self._ok(self.L.pd_build_bonds(self.h, arr, len(planes)))

    def set_bonds(self, neighborhood_list):
        nl = np.ascontiguousarray(neighborhood_list, dtype=np.int32)
        self._ok(self.L.pd_set_bonds(self.h, nl.ctypes.data_as(_i32p), nl.size))

    def num_bonds(self):
        nb = C.c_int64()
        self._ok(self.L.pd_num_bonds(self.h, C.byref(nb)))
        return nb.value

    def get_bonds(self):
        ln = C.c_int64()
        self._ok(self.L.pd_get_bonds(self.h, None, 0, C.byref(ln)))
        out = np.zeros(ln.value, dtype=np.int32)
        self._ok(self.L.pd_get_bonds(self.h, out.ctypes.data_as(_i32p), out.size, C.byref(ln)))
        return out

    def bonds_csr(self):
        nl = self.get_bonds()
        n = self.n
        counts = np.zeros(n, dtype=np.int64)
        k = 0
        keep = np.ones(nl.size, dtype=bool)
        for i in range(n):
            c = int(nl[k])
            counts[i] = c
            keep[k] = False
            k += c + 1
        row = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(counts, out=row[1:])
        return row, nl[keep].astype(np.int32)

    # -- material / damage --------------------------------------------------
    def material(self, K, mu, rho, block=0):
        self._ok(self.L.pd_material_lps(self.h, int(block), float(K), float(mu), float(rho)))

    def material_bond_based(self, K, rho, block=0, plane=False, height=0.0):
        """Elastic bond-based material ("Elastic Bond Based"): 3D, or plane strain/stress with the height."""
        self._ok(self.L.pd_material_bond_based(self.h, int(block), float(K), float(rho), 1 if plane else 0,
                                               float(height)))

    def material_linear_lps(self, K, mu, rho, block=0):
        """Linear LPS material ("Linear LPS Partial Volume" without partial volumes); FP64 contexts only."""
        self._ok(self.L.pd_material_linear_lps(self.h, int(block), float(K), float(mu), float(rho)))

    def material_field(self, K, mu):
        K, mu = _f64(K, self.n, "K"), _f64(mu, self.n, "mu")
        self._ok(self.L.pd_material_lps_field(self.h, _d(K), _d(mu)))

    def critical_stretch(self, s_c, block=0):
        self._ok(self.L.pd_damage_critical_stretch(self.h, int(block), float(s_c)))

    def critical_stretch_field(self, s_c):
        s = _f64(s_c, self.n, "s_c")
        self._ok(self.L.pd_damage_critical_stretch_field(self.h, _d(s)))

    def weighted_volume(self):
        m = np.zeros(self.n)
        self._ok(self.L.pd_weighted_volume(self.h, _d(m)))
        return m

    # -- evaluation -----------------------------------------------------------
    def compute_force(self, y):
        y = _f64(y, 3 * self.n, "y")
        f = np.zeros(3 * self.n)
        self._ok(self.L.pd_compute_force(self.h, _d(y), _d(f)))
        return f

    def compute_force_device(self, y_ptr, f_ptr):
        self._ok(self.L.pd_compute_force_device(self.h, C.c_void_p(y_ptr), C.c_void_p(f_ptr)))

    def compute_damage(self, y):
        y = _f64(y, 3 * self.n, "y")
        self._ok(self.L.pd_compute_damage(self.h, _d(y)))

    def update_state(self):
        self._ok(self.L.pd_update_state(self.h))

    def set_bond_damage(self, bd):
        bd = _f64(bd, self.num_bonds(), "bond damage")
        self._ok(self.L.pd_set_bond_damage(self.h, _d(bd)))

    # -- contact ---------------------------------------------------------------
    def contact(self, search_radius, search_frequency, contact_radius, spring_constant, friction=0.0):
        self._ok(self.L.pd_contact_short_range(self.h, float(search_radius), int(search_frequency),
                                               float(contact_radius), float(spring_constant), float(friction)))

    def contact_force(self, y, v):
        y, v = _f64(y, 3 * self.n, "y"), _f64(v, 3 * self.n, "v")
        fc = np.zeros(3 * self.n)
        self._ok(self.L.pd_contact_force(self.h, _d(y), _d(v), _d(fc)))
        return fc

    # -- integration ----------------------------------------------------------
    def critical_time_step(self):
        dt = C.c_double()
        self._ok(self.L.pd_critical_time_step(self.h, C.byref(dt)))
        return dt.value

    def set_state(self, u=None, v=None):
        uu = _f64(u, 3 * self.n, "u") if u is not None else None
        vv = _f64(v, 3 * self.n, "v") if v is not None else None
        self._ok(self.L.pd_set_state(self.h, _d(uu) if uu is not None else None, _d(vv) if vv is not None else None))

    def prescribed_displacement(self, points, coordinate, a, b=0.0):
        p = np.ascontiguousarray(points, dtype=np.int64)
        self._ok(self.L.pd_add_prescribed_displacement(self.h, p.size, p.ctypes.data_as(_i64p), int(coordinate),
                                                       float(a), float(b)))

    def prescribed_displacement_function(self, points, coordinate, function):
        """u_c = f(x, y, z, t) from a reference "Value" string (pd_add_prescribed_displacement_function)."""
        p = np.ascontiguousarray(points, dtype=np.int64)
        self._ok(self.L.pd_add_prescribed_displacement_function(self.h, p.size, p.ctypes.data_as(_i64p),
                                                                int(coordinate), function.encode()))

    def clear_boundary_conditions(self):
        self._ok(self.L.pd_clear_boundary_conditions(self.h))

    def verlet_run(self, dt, nsteps, t0=0.0):
        st = _lib.Stats()
        self._ok(self.L.pd_verlet_run(self.h, float(dt), float(t0), int(nsteps), C.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.Stats._fields_}

    def verlet_begin(self, dt, t0=0.0):
        """Stepping form of verlet_run: begin + step(n - 1) + finish == verlet_run(n)."""
        self._ok(self.L.pd_verlet_begin(self.h, float(dt), float(t0)))

    def verlet_step(self, nsteps=1):
        self._ok(self.L.pd_verlet_step(self.h, int(nsteps)))

    def verlet_finish(self):
        st = _lib.Stats()
        self._ok(self.L.pd_verlet_finish(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.Stats._fields_}

    def pack_state(self, idx, out):
        """out[k] = (u, y) of point idx[k]; idx int32 and out float64 [len(idx), 6]
        torch tensors on this context's device."""
        import torch

        torch.cuda.current_stream(idx.device).synchronize()
        self._ok(self.L.pd_pack_state_device(self.h, int(idx.numel()), C.c_void_p(idx.data_ptr()),
                                             C.c_void_p(out.data_ptr())))

    def unpack_state(self, idx, vals):
        import torch

        torch.cuda.current_stream(idx.device).synchronize()
        self._ok(self.L.pd_unpack_state_device(self.h, int(idx.numel()), C.c_void_p(idx.data_ptr()),
                                               C.c_void_p(vals.data_ptr())))

    # -- quasi-static --------------------------------------------------------
    def qs_load_step(self, t_prev, t_cur, newton_tolerance, cg_relative_tolerance=1e-8, max_newton=20,
                     max_cg=20000, preconditioner="block_jacobi", use_predictor=True, stats=None, coarse_cell=0.0):
        """One load step; preconditioner "none", "block_jacobi", "two_level" (block Jacobi + aggregate
        coarse correction, cells of side max(coarse_cell, 2 * max horizon)) or "mpnn" (the learned
        correction on the base set by mpnn_coarse)."""
        o = _lib.QsOptions()
        o.newton_tolerance = float(newton_tolerance)
        o.cg_relative_tolerance = float(cg_relative_tolerance)
        o.max_newton_iterations = int(max_newton)
        o.max_cg_iterations = int(max_cg)
        o.preconditioner = {"none": _lib.PD_PRECOND_NONE, "block_jacobi": _lib.PD_PRECOND_BLOCK_JACOBI,
                            "mpnn": _lib.PD_PRECOND_MPNN, "two_level": _lib.PD_PRECOND_TWO_LEVEL}[preconditioner]
        o.use_predictor = 1 if use_predictor else 0
        o.coarse_cell = float(coarse_cell)
        st = stats if stats is not None else _lib.Stats()
        self._ok(self.L.pd_qs_load_step(self.h, float(t_prev), float(t_cur), C.cast(C.byref(o), C.c_void_p),
                                        C.byref(st)))
        return st

    def implicit_run(self, dt, nsteps, t0=0.0, beta=0.25, gamma=0.5, absolute_tolerance=1.0e-6,
                     cg_relative_tolerance=1.0e-10, max_newton=10, max_cg=None, preconditioner="block_jacobi",
                     stats=None):
        """nsteps implicit Newmark-beta steps (Peridigm::executeImplicit); preconditioner "none" (the
        reference's plain CG) or "block_jacobi"."""
        o = _lib.ImplicitOptions()
        o.beta, o.gamma = float(beta), float(gamma)
        o.absolute_tolerance = float(absolute_tolerance)
        o.cg_relative_tolerance = float(cg_relative_tolerance)
        o.max_newton_iterations = int(max_newton)
        o.max_cg_iterations = int(max_cg if max_cg is not None else max(3 * self.n, 100))
        o.preconditioner = {"none": _lib.PD_PRECOND_NONE, "block_jacobi": _lib.PD_PRECOND_BLOCK_JACOBI}[preconditioner]
        st = stats if stats is not None else _lib.Stats()
        self._ok(self.L.pd_implicit_run(self.h, float(dt), float(t0), int(nsteps), C.cast(C.byref(o), C.c_void_p),
                                        C.byref(st)))
        return st

    def coarse_modes(self, modes):
        """Coarse dofs per aggregate of the two-level preconditioner: 3 (translations) or 6 (with rotations)."""
        self._ok(self.L.pd_qs_coarse_modes(self.h, int(modes)))

    def jacobian_apply(self, u, w):
        u, w = _f64(u, 3 * self.n, "u"), _f64(w, 3 * self.n, "w")
        kw = np.zeros(3 * self.n)
        self._ok(self.L.pd_jacobian_apply(self.h, _d(u), _d(w), _d(kw)))
        return kw

    def jacobian_blocks(self, u):
        u = _f64(u, 3 * self.n, "u")
        b = np.zeros(9 * self.n)
        self._ok(self.L.pd_jacobian_block_diagonal(self.h, _d(u), _d(b)))
        return b.reshape(self.n, 3, 3)

    def coarse_operator(self, u, cell=0.0):
        """(aggregate of each point, assembled P0^T K P0, its inverse) of the two-level preconditioner
        at displacement u."""
        u = _f64(u, 3 * self.n, "u")
        nc = C.c_int64(0)
        self._ok(self.L.pd_qs_coarse_operator(self.h, _d(u), float(cell), C.byref(nc), None, None, None))
        agg = np.zeros(self.n, dtype=np.int32)
        A = np.zeros((nc.value, nc.value))
        Ai = np.zeros((nc.value, nc.value))
        self._ok(self.L.pd_qs_coarse_operator(self.h, _d(u), float(cell), C.byref(nc),
                                              agg.ctypes.data_as(C.POINTER(C.c_int32)), _d(A), _d(Ai)))
        return agg, A, Ai

    # -- learned preconditioner ----------------------------------------------
    def mpnn_coarse(self, cell=0.0):
        """cell >= 0: the network corrects the two-level preconditioner; < 0: block Jacobi alone."""
        self._ok(self.L.pd_mpnn_coarse(self.h, float(cell)))

    def mpnn_init(self, seed=0, patch=None):
        """Initialise the learned middle level on patches (grid cells) of side `patch`."""
        self._ok(self.L.pd_mpnn_init(self.h, int(seed), float(patch)))

    def mpnn_collect(self, every):
        self._ok(self.L.pd_mpnn_collect(self.h, int(every)))

    def mpnn_num_pairs(self):
        k = C.c_int64()
        self._ok(self.L.pd_mpnn_num_pairs(self.h, C.byref(k)))
        return k.value

    def mpnn_train(self, epochs, learning_rate=1e-3, batch=8):
        loss = C.c_double()
        self._ok(self.L.pd_mpnn_train(self.h, int(epochs), float(learning_rate), int(batch), C.byref(loss)))
        return loss.value

    @staticmethod
    def mpnn_num_params():
        k = C.c_int64()
        _lib.load().pd_mpnn_num_params(C.byref(k))
        return k.value

    def mpnn_weights(self):
        w = np.zeros(self.mpnn_num_params(), dtype=np.float32)
        self._ok(self.L.pd_mpnn_get_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float))))
        return w

    def mpnn_set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._ok(self.L.pd_mpnn_set_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float))))

    def mpnn_loss_grad(self, a, r, e):
        """Loss and weight gradient for one pair (a = P_bj r, r = K e, e)."""
        pair = np.ascontiguousarray(np.concatenate([a, r, e]), dtype=np.float32)
        loss = C.c_double()
        g = np.zeros(self.mpnn_num_params(), dtype=np.float32)
        self._ok(self.L.pd_mpnn_loss_grad(self.h, pair.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss),
                                          g.ctypes.data_as(C.POINTER(C.c_float))))
        return loss.value, g

    def mpnn_apply(self, r):
        """Middle level of the learned preconditioner alone: Q S G^T G S Q^T r."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros(3 * self.n)
        self._ok(self.L.pd_mpnn_apply(self.h, _d(r), _d(z)))
        return z

    # -- compute classes --------------------------------------------------------
    def block_data(self, field, block, calculation="Sum"):
        """Block_Data compute class: "Minimum", "Maximum" or "Sum" of a field over a block (3 values)."""
        calc = {"Minimum": 0, "Maximum": 1, "Sum": 2}[calculation]
        out = np.zeros(3)
        self._ok(self.L.pd_block_data(self.h, _lib.FIELDS[field], int(block), calc, _d(out)))
        return out

    def kinetic_energy(self, per_point=False):
        g = np.zeros(1)
        pp = np.zeros(self.n) if per_point else None
        self._ok(self.L.pd_kinetic_energy(self.h, _d(g), _d(pp) if per_point else None))
        return (g[0], pp) if per_point else g[0]

    def linear_momentum(self, per_point=False):
        g = np.zeros(3)
        pp = np.zeros(3 * self.n) if per_point else None
        self._ok(self.L.pd_linear_momentum(self.h, _d(g), _d(pp) if per_point else None))
        return (g, pp) if per_point else g

    def kernel_timing(self, enable=True):
        self._ok(self.L.pd_set_kernel_timing(self.h, 1 if enable else 0))

    def kernel_times(self):
        ms = np.zeros(2)
        cnt = C.c_int64()
        self._ok(self.L.pd_get_kernel_timing(self.h, _d(ms), C.byref(cnt)))
        return {"dilatation_ms": ms[0], "force_ms": ms[1], "evaluations": cnt.value}

    def field(self, name):
        fid = _lib.FIELDS[name]
        size = {0: 3, 1: 3, 2: 3, 3: 3, 4: 3, 9: 3, 11: 3, 13: 3}.get(fid, 1) * self.n
        if fid == _lib.FIELDS["Bond_Damage"]:
            size = self.num_bonds()
        out = np.zeros(size)
        self._ok(self.L.pd_get_field(self.h, fid, _d(out)))
        return out
