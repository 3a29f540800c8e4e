"""Seeded synthetic discretizations with the shapes of the benchmark configurations.

The reference measures on no public dataset; these lattices stand in for the
inputs its decks would build (PdQuickGrid-style tensor-product point sets).
Points sit at cell centres (i + 1/2) h, volume h^3, optional uniform jitter of
each coordinate by +-j*h from a numpy default_rng seed.
"""
from __future__ import annotations

import math

import numpy as np


def lattice(nx, ny, nz, h, origin=(0.0, 0.0, 0.0), jitter=0.0, seed=None):
    i = (np.arange(nx) + 0.5) * h + origin[0]
    j = (np.arange(ny) + 0.5) * h + origin[1]
    k = (np.arange(nz) + 0.5) * h + origin[2]
    Z, Y, X = np.meshgrid(k, j, i, indexing="ij")  # x fastest, like QuickGrid ids i + j*nx + k*nx*ny
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    if jitter:
        rng = np.random.default_rng(seed)
        x = x + rng.uniform(-jitter * h, jitter * h, size=x.shape)
    vol = np.full(x.shape[0], h ** 3)
    return np.ascontiguousarray(x.ravel()), vol


def bar_wave(nx=100, ny=10, nz=10, h=1.0e-3):
    """Elastic wave in a bar: Gaussian x-velocity pulse (amplitude 1 m/s, width 5h,
    centred 10h from the left end), LPS K=130 GPa, mu=78 GPa, rho=7800, delta=3.015h."""
    x, vol = lattice(nx, ny, nz, h)
    X = x[0::3]
    v = np.zeros_like(x)
    v[0::3] = 1.0 * np.exp(-((X - 10 * h) ** 2) / (2.0 * (5 * h) ** 2))
    return dict(name=f"bar_wave_{nx}x{ny}x{nz}", x=x, vol=vol, horizon=3.015 * h, K=130.0e9, mu=78.0e9,
                rho=7800.0, s_c=None, planes=[], v0=v, bcs=[], safety=0.7, nsteps=1000, h=h)


def notched_plate(nx=400, ny=200, nz=4, h=0.5e-3, seed=1, s_c=5.0e-4, pull=2.0, notch_cells=50, nsteps=5000):
    """LPS + critical stretch on a notched plate in tension.

    Jitter +-0.05h (seed), delta = 3.015h, K=130 GPa, mu=78 GPa, rho=7800.
    Notch: every bond crossing the plane y = ny*h/2 for x in [x_min - h, x_min + notch_cells*h]
    (a Rectangular_Plane filter spanning the thickness). Top and bottom 3-point
    layers: prescribed displacement u_y = +-pull * t."""
    x, vol = lattice(nx, ny, nz, h, jitter=0.05, seed=seed)
    ymid = ny * h / 2.0
    plane = dict(normal=(0.0, 1.0, 0.0), lower_left=(-h, ymid, -h), bottom_unit=(1.0, 0.0, 0.0),
                 bottom_length=(notch_cells + 1) * h, side_length=nz * h + 2 * h)
    row_id = np.arange(nx * ny * nz) // nx % ny
    bottom = np.nonzero(row_id < 3)[0]
    top = np.nonzero(row_id >= ny - 3)[0]
    bcs = [dict(points=top, coordinate=1, a=pull, b=0.0), dict(points=bottom, coordinate=1, a=-pull, b=0.0)]
    return dict(name=f"notched_plate_{nx}x{ny}x{nz}", x=x, vol=vol, horizon=3.015 * h, K=130.0e9, mu=78.0e9,
                rho=7800.0, s_c=s_c, planes=[plane], v0=np.zeros_like(x), bcs=bcs, safety=0.7, nsteps=nsteps, h=h)


def large_plate(nx=400, ny=400, nz=200, h=0.5e-3, seed=4, nsteps=500, pull=1.0):
    """Memory-scale heterogeneous plate: per-point K lognormal (median 130 GPa, sigma 0.3,
    seed 5), mu = 0.6K, critical stretch uniform in [3e-4, 6e-4] (seed 6), +-pull m/s
    prescribed on the x faces (3 layers; 1 m/s in the benchmark)."""
    x, vol = lattice(nx, ny, nz, h, jitter=0.05, seed=seed)
    n = vol.size
    K = 130.0e9 * np.exp(0.3 * np.random.default_rng(5).standard_normal(n))
    s_c = np.random.default_rng(6).uniform(3.0e-4, 6.0e-4, n)
    col_id = np.arange(n) % nx
    left = np.nonzero(col_id < 3)[0]
    right = np.nonzero(col_id >= nx - 3)[0]
    bcs = [dict(points=right, coordinate=0, a=pull, b=0.0), dict(points=left, coordinate=0, a=-pull, b=0.0)]
    return dict(name=f"large_plate_{nx}x{ny}x{nz}", x=x, vol=vol, horizon=3.015 * h, K=K, mu=0.6 * K, rho=7800.0,
                s_c=s_c, planes=[], v0=np.zeros_like(x), bcs=bcs, safety=0.7, nsteps=nsteps, h=h)


def setup_context(ctx, w):
    """Load a workload dict into a Context (points, horizon, bonds, material, damage, BCs, v0)."""
    ctx.set_points(w["x"], w["vol"])
    ctx.set_horizons([w["horizon"]])
    ctx.build_bonds(w["planes"])
    K, mu = w["K"], w["mu"]
    if np.ndim(K) == 0:
        ctx.material(K, mu, w["rho"])
    else:
        ctx.material(float(np.median(K)), float(np.median(mu)), w["rho"])
        ctx.material_field(K, mu)
    if w.get("s_c") is not None:
        if np.ndim(w["s_c"]) == 0:
            ctx.critical_stretch(w["s_c"])
        else:
            ctx.critical_stretch(0.0)
            ctx.critical_stretch_field(w["s_c"])
    for bc in w["bcs"]:
        ctx.prescribed_displacement(bc["points"], bc["coordinate"], bc["a"], bc["b"])
    ctx.set_state(np.zeros_like(w["x"]), w["v0"])
    return ctx


def oracle_problem(w, row, col, dt, nsteps):
    """The same workload as an oracle.explicit_run problem dict (test helper)."""
    n = w["vol"].size
    bc_mask = np.zeros(n, np.uint8)
    bc_a = np.zeros(3 * n)
    bc_b = np.zeros(3 * n)
    for bc in w["bcs"]:
        p = np.asarray(bc["points"])
        c = bc["coordinate"]
        bc_mask[p] |= np.uint8(1 << c)
        bc_a[3 * p + c] = bc["a"]
        bc_b[3 * p + c] = bc["b"]
    return dict(x=w["x"], vol=w["vol"], rho=w["rho"], K=w["K"], mu=w["mu"], row=row, col=col,
                horizon=w["horizon"], dt=dt, nsteps=nsteps, s_c=w.get("s_c"), bc_mask=bc_mask, bc_a=bc_a, bc_b=bc_b)


def bonds_per_point_estimate(horizon_over_h):
    r = horizon_over_h
    return 4.0 / 3.0 * math.pi * r ** 3


def plate_sphere(nx=400, ny=400, nz=40, h=0.25e-3, radius_cells=25, s_c=3.0e-4, speed=20.0, gap_cells=3.5,
                 search_extra=0.6, freq=100, nsteps=2000):
    """Brittle plate (block 0, critical stretch s_c) and a dropped sphere (block 1,
    elastic only) on the same lattice spacing, short-range contact.

    Sphere: lattice points within radius_cells*h of its centre, centred above the
    plate middle, its lowest point gap_cells*h above the plate's top layer (more
    than a horizon, so no bond joins the bodies); initial velocity -speed in z.
    Contact radius 0.9h, spring constant = plate bulk modulus, search radius
    0.9h + search_extra*h (a pair outside it at a search cannot close the extra
    gap within freq steps at these speeds), search frequency freq."""
    xp, vp = lattice(nx, ny, nz, h)
    r = radius_cells
    k = np.arange(-r, r + 1)
    Z, Y, X = np.meshgrid(k, k, k, indexing="ij")
    keep = X ** 2 + Y ** 2 + Z ** 2 <= r * r
    c = np.array([nx * h / 2.0, ny * h / 2.0, nz * h - 0.5 * h + (r + gap_cells) * h])
    xs = (np.stack([X[keep], Y[keep], Z[keep]], 1) * h + c).ravel()
    x = np.concatenate([xp, xs])
    vol = np.full(x.size // 3, h ** 3)
    block = np.concatenate([np.zeros(xp.size // 3, np.int32), np.ones(xs.size // 3, np.int32)])
    v0 = np.zeros_like(x)
    v0[xp.size + 2::3] = -speed
    return dict(name=f"plate_sphere_{nx}x{ny}x{nz}_r{r}", x=x, vol=vol, block=block, horizon=3.015 * h,
                K=130.0e9, mu=78.0e9, rho=7800.0, s_c=s_c, s_c_blocks=[s_c, -1.0], planes=[], v0=v0, bcs=[],
                safety=0.7, nsteps=nsteps, h=h,
                contact=dict(r_search=0.9 * h + search_extra * h, freq=freq, r_contact=0.9 * h, k_spring=130.0e9,
                             friction=0.0))


def setup_context_blocks(ctx, w):
    """Multi-block variant of setup_context (one material, per-block damage, contact)."""
    ctx.set_points(w["x"], w["vol"], w.get("block"))
    nblk = int(np.max(w["block"])) + 1 if w.get("block") is not None else 1
    ctx.set_horizons([w["horizon"]] * nblk)
    ctx.build_bonds(w["planes"])
    for b in range(nblk):
        ctx.material(w["K"], w["mu"], w["rho"], block=b)
        ctx.critical_stretch(w["s_c_blocks"][b], block=b)
    ct = w.get("contact")
    if ct:
        ctx.contact(ct["r_search"], ct["freq"], ct["r_contact"], ct["k_spring"], ct.get("friction", 0.0))
    for bc in w["bcs"]:
        ctx.prescribed_displacement(bc["points"], bc["coordinate"], bc["a"], bc["b"])
    ctx.set_state(np.zeros_like(w["x"]), w["v0"])
    return ctx


def oracle_problem_blocks(w, row, col, dt, nsteps):
    p = oracle_problem(w, row, col, dt, nsteps)
    blk = w["block"]
    p["s_c"] = np.where(np.asarray(w["s_c_blocks"])[blk] >= 0, np.asarray(w["s_c_blocks"])[blk], 1e300)
    ct = w.get("contact")
    if ct:
        p["contact"] = dict(r_search=ct["r_search"], freq=ct["freq"], r_contact=ct["r_contact"],
                            k_spring=ct["k_spring"], friction=ct.get("friction", 0.0),
                            horizon=np.full(len(w["vol"]), w["horizon"]))
    return p


def qs_cube(n=60, h=1.0e-3, seed=0, displacement=1.0e-4, load_steps=20, jitter=0.0):
    """Quasi-static tensile cube: n^3 lattice, delta = 3.015h, bulk modulus drawn
    log-uniform in [50, 200] GPa from the seed, shear modulus 0.6K; the x = min
    face (3 layers) clamped in all components, the x = max face (3 layers)
    displaced u_x = displacement * t for load parameter t in [0, 1], reached in
    load_steps equal steps."""
    x, vol = lattice(n, n, n, h, jitter=jitter, seed=seed)
    rng = np.random.default_rng(seed)
    K = float(np.exp(rng.uniform(np.log(50.0e9), np.log(200.0e9))))
    col_id = np.arange(n ** 3) % n
    left = np.nonzero(col_id < 3)[0]
    right = np.nonzero(col_id >= n - 3)[0]
    bcs = [dict(points=left, coordinate=c, a=0.0, b=0.0) for c in range(3)]
    bcs.append(dict(points=right, coordinate=0, a=displacement, b=0.0))
    return dict(name=f"qs_cube_{n}", x=x, vol=vol, horizon=3.015 * h, K=K, mu=0.6 * K, rho=7800.0, s_c=None,
                planes=[], v0=np.zeros_like(x), bcs=bcs, h=h, times=np.linspace(0.0, 1.0, load_steps + 1))
