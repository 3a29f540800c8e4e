"""Benchmark: bond evaluations per second of the explicit LPS + critical-stretch
step, split-FP32 against FP64, on one B200; quasi-static time to 1e-8.

Headline workload (default): the memory-scale heterogeneous plate,
400x400x200 = 32,000,000 points, h = 0.5 mm, jitter +-0.05h (seed 4),
delta = 3.015h, per-point bulk modulus lognormal (median 130 GPa, sigma 0.3,
seed 5), mu = 0.6K, critical stretch uniform in [3e-4, 6e-4] (seed 6),
+-1 m/s prescribed pulls on the x faces (3 layers). --workload picks another:
notched_plate (400x200x4, 320,000 points, s_c = 5e-4, +-2 m/s pulls),
plate_sphere (400x400x40 plate + dropped sphere, contact) or bar_wave
(100x10x10 bar, Gaussian velocity pulse, no damage).

One bench step = one velocity-Verlet step: damage + dilatation pass, force
pass with the Verlet epilogue, over every bond. value = bonds x steps /
device time (CUDA events on the library's stream). With N > 1 GPUs the body
is split into N slabs with ghost layers and one NCCL exchange per step
(strong scaling; bonds of owned points, max over ranks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload W]

Prints one JSON line on rank 0. Two further modes print one JSON line per
run for profilers (no timing claims beyond the device time they print):

    python bench.py --profile [--workload W] [--nx --ny --nz] [--precision split|fp64|both]
                    [--material lps|bond_based|linear_lps] [--profile-steps 3]
        a few explicit steps; with --precision both, the split and FP64 runs
        and the relative L2 difference of their displacements
    python bench.py --qs-profile block_jacobi|two_level|mpnn [--qs-n 60] [--qs-tol 1e-4]
                    [--coarse-modes 3|6] [--coarse-build-only]
        one load step of the quasi-static cube (the learned level at its
        starting weights), or, with --coarse-build-only, the two-level coarse
        operator built once at zero displacement
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "bond evals/s per explicit step, split-FP32 vs FP64 (1 B200); QS time to 1e-8 res"
UNIT = "bond evals/s"


def algorithmic_bytes(nb, n, precision="split"):
    """Bytes an explicit step must move at minimum (every per-point record
    counted once: ideal reuse of gathered neighbors), per pass and per step.

    Split-FP32, per bond and pass: neighbor id 4 + bond damage 1 + reference
    bond vector X in FP32 12 = 17 B; per step 34 B.
    Per point, dilatation pass: row 8, owner terms 16, displacement record 32,
    writes A/B 8, theta 8, node damage 8 -> 80 B.
    Per point, force pass: row 8, displacement record 32, rho 8, v read+write
    48, acceleration 24, u read+write 48, next displacement record 24, BC mask
    1 -> 193 B.
    Per step (both passes, per-point terms counted once): 34 nb + 176 n.
    FP64 paths per step: X in FP64 (24 B) instead of FP32, 58 nb + 200 n.
    FP64 sliced passes: 29 B per bond and pass; per point, dilatation: row 8,
    m/K/mu 24, s_c 8, own (y, V) 32, writes (A, B, theta) 32, theta 8, node
    damage 8 -> 120 B; force: own (y, V) 32 and (A, B) 16, x 24, rho 8, v
    read+write 48, acceleration 24, u read+write 48, next y 24, BC mask 1 ->
    225 B."""
    if precision == "split":
        return {"dilatation": 17 * nb + 80 * n, "force": 17 * nb + 193 * n, "step": 34 * nb + 176 * n}
    if precision == "fp64_sliced":
        return {"dilatation": 29 * nb + 120 * n, "force": 29 * nb + 225 * n, "step": 58 * nb + 200 * n}
    return {"step": 58 * nb + 200 * n}


# DRAM bytes (read + write) per launch of the split bond passes from one ncu
# capture (--set full) of step 1 of the heterogeneous plate at 160x160x40
# (1,024,000 points, 108,999,624 bonds, half-bond variants), with the
# streamed slots of that run. Launches of other sizes are scaled by their slot
# counts (the per-slot traffic, not the per-point share, dominates).
NCU_TRAFFIC = {"workload": "large_plate_160x160x40", "slots": 114618496, "dilatation": 2.0402e9, "force": 2.1889e9}

WORKLOADS = ("large_plate", "notched_plate", "plate_sphere", "bar_wave")


def make_workload(name, dims=None):
    from peridigm_b200 import workloads

    kw = {k: v for k, v in zip(("nx", "ny", "nz"), dims or ()) if v}
    if name == "large_plate":
        return workloads.large_plate(**kw), False
    if name == "notched_plate":
        return workloads.notched_plate(**kw), False
    if name == "plate_sphere":
        return workloads.plate_sphere(**kw), True
    if name == "bar_wave":
        return workloads.bar_wave(**kw), False
    raise ValueError(name)


def setup(ctx, w, blocks):
    from peridigm_b200 import workloads

    (workloads.setup_context_blocks if blocks else workloads.setup_context)(ctx, w)
    return ctx


def sliced_slots(ctx):
    """Streamed slots of the 4-lanes-per-point split passes: each 8-owner
    slice holds 32 slots per group of 4 bonds of its longest row."""
    lens = ctx.field("Number_Of_Neighbors").astype(np.int64)
    pad = (-lens.size) % 8
    lens = np.concatenate([lens, np.zeros(pad, np.int64)]).reshape(-1, 8)
    return int(32 * ((lens.max(axis=1) + 3) // 4).sum())


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [q.strip() for q in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


T_START = time.perf_counter()


def log(msg):
    """Progress of the run on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.perf_counter() - T_START:7.1f}s] {msg}", file=sys.stderr, flush=True)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peak_hbm():
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# CPU sample of the heterogeneous plate: a 128x128x64 block of the same
# lattice spacing, jitter, material statistics and pulls (1,048,576 points).
CPU_SAMPLE_DIMS = {"large_plate": (128, 128, 64), "notched_plate": (100, 200, 4), "plate_sphere": None,
                   "bar_wave": (100, 10, 10)}


def cpu_sample(name):
    """The bounded CPU sample of a workload: the reference's compiled kernels
    run with block constants (the reference has per-block K, mu and s_c; the
    heterogeneous plate's medians are used, which costs the same)."""
    dims = CPU_SAMPLE_DIMS.get(name)
    if dims is None:
        dims = (100, 200, 4)
        name = "notched_plate"
    w, _ = make_workload(name, dims)
    return w, name, dims


def reference_arm(args, world, rank):
    """The reference's own CPU implementation of the step (oracle/_ref: its
    computeDilatation + computeInternalForceLinearElastic compiled from source,
    with the restated critical-stretch damage and Verlet loops) on all host
    cores, over a bounded sample of the workload (cpu_sample)."""
    if rank != 0:
        return
    from oracle import cpu_baseline
    from oracle import oracle as O

    O.build()
    w, sname, dims = cpu_sample(args.workload)
    row, col = O.neighbor_search(w["x"], w["horizon"], w["planes"])
    r = cpu_baseline.run(w, row, col, steps=args.steps, warmup=args.warmup)
    value = r["value"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"] / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{workload_name(args.workload)} (sample: {sname}_{dims[0]}x{dims[1]}x{dims[2]})",
                       "points": int(len(w["vol"])), "bonds": int(len(col)), "precision": "fp64"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": f"{args.steps} explicit steps of {sname}_{dims[0]}x{dims[1]}x{dims[2]} "
                                       f"({len(col)} bonds), {r['cores']} processes"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_name(name):
    w = {"large_plate": "large_plate_400x400x200", "notched_plate": "notched_plate_400x200x4",
         "plate_sphere": "plate_sphere_400x400x40_r25", "bar_wave": "bar_wave_100x10x10"}
    return w[name]


def qs_leg(local, load_steps, cpu_threads=0, learned_modes=6):
    """Quasi-static time to 1e-8: the 60^3 tensile cube (216,000 points, h = 1 mm,
    delta = 3.015h, K log-uniform in [50, 200] GPa from seed 1000, mu = 0.6K, x = 0
    face clamped, x = max face pulled to 1e-4 m) over `load_steps` equal load
    steps; Newton to 1e-8 of each load increment's residual, CG to 1e-8 relative.
    Four preconditioners: block Jacobi (the reference's "Block 3x3"), two-level
    (block Jacobi + exact Galerkin coarse correction on aggregate cells of two
    horizons, translations), two-level rigid (the coarse space with the three
    rotations per aggregate as well) and learned (the learned middle level on
    3 mm patches over the two-level base with `learned_modes` coarse modes,
    trained here on about 2000 (residual, error) pairs that two-level solves
    of a 12^3 cube generate, every CG iterate, over twelve moduli and load
    paths drawn from seeds 100-111; the weights kept are the checkpoint, every
    5 epochs from epoch 0, with the fewest CG iterations on a held-out 12^3
    solve; the last epoch's weights are reported too). Times are device time
    of the Newton loops (CUDA events); each arm first runs one untimed load
    step in a throwaway context of the same cube.
    With cpu_threads > 0 the block-Jacobi arm also gets a CPU baseline: the
    same CG step restated in C (oracle/cpu_qs.c) on that many host threads,
    timed on a sample and scaled by the solve's Newton and CG counts."""
    from peridigm_b200 import Context, workloads

    patch = 3.0e-3
    t0 = time.perf_counter()
    w = workloads.qs_cube(n=12, h=1.0e-3, seed=11, jitter=0.05, load_steps=4)
    with Context(device=local, precision="fp64") as tr:
        workloads.setup_context(tr, w)
        tr.coarse_modes(learned_modes)
        tr.mpnn_init(seed=7, patch=patch)
        init_weights = tr.mpnn_weights()
        tr.mpnn_collect(1)
        for seed in range(100, 112):
            rng = np.random.default_rng(seed)
            K = float(np.exp(rng.uniform(np.log(50e9), np.log(200e9))))
            tr.material(K, 0.6 * K, 7800.0)
            tr.clear_boundary_conditions()
            for bc in w["bcs"][:3]:
                tr.prescribed_displacement(bc["points"], bc["coordinate"], 0.0, 0.0)
            right = w["bcs"][3]["points"]
            tr.prescribed_displacement(right, 0, float(rng.uniform(0.5e-4, 1.5e-4)), 0.0)
            tr.prescribed_displacement(right, 1, float(rng.uniform(-0.5e-4, 0.5e-4)), 0.0)
            tr.set_state(np.zeros_like(w["x"]), np.zeros_like(w["x"]))
            st = None
            for k in range(1, len(w["times"])):
                st = tr.qs_load_step(w["times"][k - 1], w["times"][k], newton_tolerance=-1e-8,
                                     cg_relative_tolerance=1e-8, preconditioner="two_level", stats=st)
        pairs = tr.mpnn_num_pairs()
        # model selection: checkpoints every 5 epochs (epoch 0 = the starting
        # weights), each scored by the CG iterations of a held-out 12^3 solve
        wv = workloads.qs_cube(n=12, h=1.0e-3, seed=12, jitter=0.05, load_steps=2)

        def validate(wts):
            with Context(device=local, precision="fp64") as vc:
                workloads.setup_context(vc, wv)
                vc.coarse_modes(learned_modes)
                vc.mpnn_init(seed=0, patch=patch)
                vc.mpnn_set_weights(wts)
                sv = None
                for k in range(1, len(wv["times"])):
                    sv = vc.qs_load_step(wv["times"][k - 1], wv["times"][k], newton_tolerance=-1e-8,
                                         cg_relative_tolerance=1e-8, preconditioner="mpnn", stats=sv)
                return int(sv.cg_iterations)

        checkpoints = {0: (validate(init_weights), init_weights)}
        loss = None
        for epoch in (5, 10, 15, 20):
            loss = tr.mpnn_train(5, learning_rate=1e-3, batch=8)
            wts = tr.mpnn_weights()
            checkpoints[epoch] = (validate(wts), wts)
        last_weights = checkpoints[20][1]
        best_epoch = min(checkpoints, key=lambda e: (checkpoints[e][0], e))
        weights = checkpoints[best_epoch][1]
    train_s = time.perf_counter() - t0
    w2 = workloads.qs_cube(n=60, h=1.0e-3, seed=1000, load_steps=load_steps)
    out = {"workload": f"qs_cube_60x60x60 (seed 1000, {load_steps} load steps)", "points": int(len(w2["vol"])),
           "tolerance": 1e-8, "training": {"pairs": pairs, "epochs": 20, "final_loss": loss, "seconds": train_s,
                                           "patch_m": patch, "coarse_modes": learned_modes,
                                           "validation_cg_iterations": {e: v[0] for e, v in checkpoints.items()},
                                           "selected_epoch": best_epoch}}

    def arm_context(arm, precond):
        ctx = Context(device=local, precision="fp64")
        workloads.setup_context(ctx, w2)
        if arm == "two_level_rigid":
            ctx.coarse_modes(6)
        if precond == "mpnn":
            ctx.coarse_modes(learned_modes)
            ctx.mpnn_init(seed=0, patch=patch)
            ctx.mpnn_set_weights(weights if arm == "mpnn" else last_weights)
        return ctx

    for arm in ("block_jacobi", "two_level", "two_level_rigid", "mpnn", "mpnn_last_epoch"):
        precond = {"two_level_rigid": "two_level", "mpnn_last_epoch": "mpnn"}.get(arm, arm)
        # warm-up: one untimed load step in a throwaway context of the same
        # cube (first-use costs of kernels and of the full-size buffers)
        with arm_context(arm, precond) as warm:
            warm.qs_load_step(w2["times"][0], w2["times"][1], newton_tolerance=-1e-8, cg_relative_tolerance=1e-8,
                              preconditioner=precond)
        with arm_context(arm, precond) as ctx:
            out["_bonds"] = ctx.num_bonds()
            st = None
            clocks = ClockSampler(local)
            clocks.start()
            for k in range(1, len(w2["times"])):
                st = ctx.qs_load_step(w2["times"][k - 1], w2["times"][k], newton_tolerance=-1e-8,
                                      cg_relative_tolerance=1e-8, preconditioner=precond, stats=st)
            clk = clocks.stop()
            out[arm] = {"seconds": st.device_ms / 1e3, "cg_iterations": st.cg_iterations,
                        "newton_iterations": st.newton_iterations, "fallbacks": st.preconditioner_fallbacks,
                        "coarse_builds": st.coarse_builds, "sm_mhz": clk["sm_mhz"], "clock_reasons": clk["reasons"]}
            if arm == "block_jacobi" and cpu_threads:
                # CPU baseline: the same block-Jacobi CG step restated in C on the
                # host threads, timed on a sample at the solved state and scaled
                # by this solve's Newton and CG counts
                from oracle import cpu_qs

                row, col = ctx.bonds_csr()
                y = w2["x"] + ctx.field("Displacement")
                fixed = np.zeros(len(w2["vol"]), np.uint8)
                for bc in w2["bcs"]:
                    fixed[bc["points"]] |= np.uint8(1 << bc["coordinate"])
                smp = cpu_qs.sample(w2["x"], y, w2["vol"], row, col, w2["K"], w2["mu"], w2["horizon"], fixed,
                                    threads=cpu_threads, cg_iters=20)
                est = st.newton_iterations * smp["seconds_per_newton_setup"] + \
                    st.cg_iterations * smp["seconds_per_cg_iteration"]
                out["cpu_baseline"] = dict(smp, seconds=est, kind="port",
                                           sample="block-Jacobi CG restated in C on %d host threads: 20 CG "
                                                  "iterations and one Newton set-up at the solved state, scaled by "
                                                  "the GPU solve's Newton and CG counts" % cpu_threads)
    # Roofline of the CG iterations: bytes one iteration must move at least,
    # over the solve's device time per iteration (Newton set-up included, so
    # the fractions are lower bounds). Tangent apply: pass 1 streams the bond
    # geometry (32 B) and neighbor id (4 B), pass 2 the geometry, the
    # coefficient pair (16 B) and the id: 88 B per bond; per point the
    # gathered vector, dilatation increments and output (about 64 B) and about
    # ten FP64 3-vectors of CG and block Jacobi (240 B). The coarse arms also
    # read the dense FP64 coarse inverse (modes x aggregates squared x 8 B;
    # aggregates: the non-empty cells of side two horizons).
    nb2 = out.pop("_bonds")
    n2 = len(w2["vol"])
    side = 2.0 * w2["horizon"] * (1.0 + 1.0e-6)
    P2 = w2["x"].reshape(-1, 3)
    cells = np.floor((P2 - P2.min(0)) / side).astype(np.int64)
    naggr = len(np.unique(cells @ np.array([1, 1 << 20, 1 << 40], np.int64)))
    hbm, peak_src = peak_hbm()
    it_bytes = 88 * nb2 + 304 * n2
    roof = {"bytes_per_cg_iteration": it_bytes, "aggregates": naggr, "peak_gbs": hbm, "peak_source": peak_src}
    for arm, modes in (("block_jacobi", 0), ("two_level", 3), ("two_level_rigid", 6)):
        b = it_bytes + 8 * (modes * naggr) ** 2
        ach = b * out[arm]["cg_iterations"] / out[arm]["seconds"] / 1e9
        roof[arm] = {"bytes_per_cg_iteration": b, "achieved_gbs": ach, "frac": ach / hbm}
    out["roofline"] = roof
    bj = out["block_jacobi"]["seconds"]
    for arm in ("two_level", "two_level_rigid", "mpnn", "mpnn_last_epoch"):
        out[f"{arm}_speedup_over_block_jacobi"] = bj / out[arm]["seconds"]
    if "cpu_baseline" in out:
        out["block_jacobi_speedup_over_cpu"] = out["cpu_baseline"]["seconds"] / bj
    return out


def explicit_leg(w, blocks, local, steps, warmup, precision, world, max_over_ranks, barrier, timed_clocks=False):
    """W untimed + K timed Verlet steps from rest of workload w; returns the
    context (still open) and the timing."""
    from peridigm_b200 import Context

    import torch

    ctx = Context(device=local, precision=precision)
    setup(ctx, w, blocks)
    nb = ctx.num_bonds()
    free_b, total_b = torch.cuda.mem_get_info(local)
    dt = w.get("safety", 0.7) * ctx.critical_time_step()
    ctx.verlet_run(dt, warmup)
    barrier()
    clocks = ClockSampler(local) if timed_clocks else None
    if clocks:
        clocks.start()
    st = ctx.verlet_run(dt, steps, t0=warmup * dt)
    barrier()
    clk = clocks.stop() if clocks else None
    ms = max_over_ranks(st["device_ms"])
    return ctx, {"nb": nb, "dt": dt, "ms": ms, "value": world * nb * steps / (ms / 1e3), "t_done": (warmup + steps) * dt,
                 "clocks": clk, "broken_bonds": st["broken_bonds"], "device_gb": (total_b - free_b) / 1e9}


def kernel_roofline(ctx, dt, t0, ksteps, nb, n, hbm, peak_src, slots, precision="split"):
    """Per-launch CUDA-event durations of the two bond passes (split, or the
    FP64 sliced passes) over ksteps steps and the dominant pass's roofline on
    the algorithmic bytes."""
    ctx.kernel_timing(True)
    ctx.verlet_run(dt, ksteps, t0=t0)
    kt = ctx.kernel_times()
    ctx.kernel_timing(False)
    per = {"dilatation": kt["dilatation_ms"] / kt["evaluations"], "force": kt["force_ms"] / kt["evaluations"]}
    algo = algorithmic_bytes(nb, n, precision)
    dom = max(per, key=per.get)
    achieved = algo[dom] / (per[dom] / 1e3) / 1e9
    traffic = None
    if precision == "split" and NCU_TRAFFIC.get("slots") and NCU_TRAFFIC.get(dom):
        traffic = NCU_TRAFFIC[dom] * slots / NCU_TRAFFIC["slots"]
    kname = f"k_{dom}_split" if precision == "split" else f"k_{dom}_f64s"
    return {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_source": peak_src, "traffic": traffic, "algorithmic_bytes": algo[dom],
            "launch_ms": per[dom], "per_kernel_ms": per, "steps_timed": ksteps,
            "per_kernel_frac": {k: algo[k] / (per[k] / 1e3) / 1e9 / hbm for k in per},
            "streamed_slots": slots, "bonds": nb}


def e2e_leg(ctx, n, nb, esteps, ranks, max_over_ranks, barrier):
    """The drop-in computeForce call with host buffers: each step the H2D of the
    current coordinates from pinned memory, damage + dilatation + force on the
    device, D2H of the force density, then the state update that commits the
    step's bond damage (the reference's evalModel + updateState cycle,
    Peridigm.cpp:1536, 1589)."""
    import ctypes as C

    import torch

    y = torch.from_numpy(ctx.field("Coordinates")).pin_memory()
    f = torch.zeros(3 * n, dtype=torch.float64).pin_memory()
    yp = C.cast(y.data_ptr(), C.POINTER(C.c_double))
    fp = C.cast(f.data_ptr(), C.POINTER(C.c_double))
    for _ in range(3):
        ctx._ok(ctx.L.pd_compute_force(ctx.h, yp, fp))
        ctx._ok(ctx.L.pd_update_state(ctx.h))
    barrier()
    t0 = time.perf_counter()
    for _ in range(esteps):
        ctx._ok(ctx.L.pd_compute_force(ctx.h, yp, fp))
        ctx._ok(ctx.L.pd_update_state(ctx.h))
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    # nb: the bonds evaluated per step over all ranks; n: this rank's points
    # (ranks of about equal size copy about ranks x 24 n bytes each way)
    return {"value": nb * esteps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 24 * n * ranks,
            "d2h_bytes_per_step": 24 * n * ranks, "steps": esteps,
            "api": "pd_compute_force (host y in, host force out) + pd_update_state"}


def slab_leg(args, world, rank, local, max_over_ranks, barrier, hbm, peak_src):
    """N > 1: one body split over the ranks (peridigm_b200.slabs: equal-count
    slabs along the longest axis, a ghost layer two horizons deep, one NCCL
    point-to-point exchange of ghost state per step), strong scaling. value =
    bond evaluations of all ranks' owned points per second over the device
    time of the step loop (library stream events, exchanges included), max
    over ranks."""
    import torch
    import torch.distributed as dist

    from peridigm_b200 import Context, slabs

    w, blocks = make_workload(args.workload)
    n = int(len(w["vol"]))
    plan = slabs.slab_plan(w["x"], w["horizon"], world, rank)
    lw = slabs.local_workload(w, plan)
    log(f"rank {rank}: {len(plan.owned)} owned of {n} points, {len(plan.local) - len(plan.owned)} ghosts, "
        f"peers {sorted(set(plan.send) | set(plan.recv))}")
    ctx = Context(device=local, precision="split")
    setup(ctx, lw, blocks)
    dt_t = torch.tensor([w.get("safety", 0.7) * ctx.critical_time_step()], dtype=torch.float64, device="cuda")
    dist.all_reduce(dt_t, op=dist.ReduceOp.MIN)  # ghosts' truncated families only over-estimate theirs
    dt = float(dt_t.item())
    owned_bonds = int(ctx.field("Number_Of_Neighbors")[plan.owned_local].sum())
    tot = torch.tensor([owned_bonds], dtype=torch.float64, device="cuda")
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    nb = int(tot.item())
    engine = slabs.ContextEngine(ctx)
    halo = slabs.HaloExchange(plan, torch.device("cuda", local), dist)
    slabs.run_slab(engine, halo, dt, args.warmup)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    st = slabs.run_slab(engine, halo, dt, args.steps, t0=args.warmup * dt)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(st["device_ms"])
    value = nb * args.steps / (ms / 1e3)
    ghost_bytes = 48 * sum(len(v) for v in plan.recv.values())
    # e2e: the drop-in computeForce on every rank's slab with host buffers (the
    # ghost layer makes the owned points' forces exact without an exchange)
    e2e = e2e_leg(ctx, len(plan.local), nb, args.e2e_steps, world, max_over_ranks, barrier)
    ctx.close()
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "split-f32 (f64 state)", "data": "synthetic",
            "config": {"workload": workload_name(args.workload), "points": n, "bonds": nb, "horizon_over_h": 3.015,
                       "dt": dt, "precision": "split_fp32", "l2": "inputs larger than L2",
                       "parallelism": f"slabs x{world} (ghost layer 2 horizons, NCCL point-to-point exchange "
                                      f"per step, {ghost_bytes} bytes received by rank 0)"},
            "roofline": {"bound": "hbm", "kernel": "split passes (slab of rank 0)", "achieved": None, "peak": hbm,
                         "unit": "GB/s", "frac": None, "peak_source": peak_src, "traffic": None},
            "cpu_baseline": None, "e2e": e2e, "clocks": clk,
            "gpu_launches": (2 + 2 * len(halo.peers)) * args.steps}
    if rank == 0:
        print(json.dumps(line), flush=True)


def profile_mode(args):
    """A few explicit steps for a profiler (replaces a separate driver)."""
    from peridigm_b200 import Context

    w, blocks = make_workload(args.workload, (args.nx, args.ny, args.nz))
    precisions = ["split", "fp64"] if args.precision == "both" else [args.precision]
    res = {}
    for p in precisions:
        with Context(precision=p, threads_per_point=args.tpo) as ctx:
            setup(ctx, w, blocks)
            nblk = int(np.max(w["block"])) + 1 if blocks else 1
            for b in range(nblk):
                if args.material == "bond_based":
                    ctx.material_bond_based(float(np.median(w["K"])), w["rho"], block=b)
                elif args.material == "linear_lps":
                    ctx.material_linear_lps(float(np.median(w["K"])), float(np.median(w["mu"])), w["rho"], block=b)
            dt = w.get("safety", 0.7) * ctx.critical_time_step()
            st = ctx.verlet_run(dt, args.profile_steps)
            nb = ctx.num_bonds()
            line = {"workload": w["name"], "material": args.material, "precision": p, "points": int(len(w["vol"])),
                    "bonds": int(nb), "steps": args.profile_steps, "device_ms": st["device_ms"],
                    "ms_per_step": st["device_ms"] / max(args.profile_steps, 1),
                    "bond_evals_per_s": nb * args.profile_steps / (st["device_ms"] / 1e3) if st["device_ms"] else 0.0,
                    "broken_bonds": st["broken_bonds"]}
            if p == "split" and args.tpo in (0, 4):
                line["streamed_slots"] = sliced_slots(ctx)
            print(json.dumps(line), flush=True)
            res[p] = (ctx.field("Displacement"), ctx.field("Damage"))
    if len(res) == 2:
        (us, ds), (u6, d6) = res["split"], res["fp64"]
        print(json.dumps({"split_vs_fp64_u_rel_l2": float(np.linalg.norm(us - u6) / max(np.linalg.norm(u6), 1e-300)),
                          "max_node_damage_diff": float(np.max(np.abs(ds - d6)))}), flush=True)


def qs_profile_mode(args):
    """One quasi-static load step of the cube with a chosen preconditioner, or
    the two-level coarse operator alone (replaces a separate driver)."""
    from peridigm_b200 import Context, workloads

    w = workloads.qs_cube(n=args.qs_n, h=1.0e-3, seed=1000, load_steps=20)
    with Context(precision="fp64") as ctx:
        workloads.setup_context(ctx, w)
        ctx.coarse_modes(args.coarse_modes)
        if args.coarse_build_only:
            _, A, Ai = ctx.coarse_operator(np.zeros(3 * len(w["vol"])))
            m = min(256, A.shape[0])
            err = float(np.abs(Ai[:m] @ A - np.eye(A.shape[0])[:m]).max())
            print(json.dumps({"coarse_dofs": int(A.shape[0]), "max_abs_inverse_error": err}))
            return
        if args.qs_profile == "mpnn":
            ctx.mpnn_init(seed=0, patch=args.patch)
        st = ctx.qs_load_step(w["times"][0], w["times"][1], newton_tolerance=-1e-3, cg_relative_tolerance=args.qs_tol,
                              preconditioner=args.qs_profile)
        print(json.dumps({"precond": args.qs_profile, "points": int(len(w["vol"])), "cg_iterations": st.cg_iterations,
                          "newton_iterations": st.newton_iterations, "device_ms": st.device_ms}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="large_plate", choices=WORKLOADS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-qs", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the notched-plate extra line")
    ap.add_argument("--qs-load-steps", type=int, default=20)
    ap.add_argument("--kernel-steps", type=int, default=50, help="steps of the per-kernel event timing")
    ap.add_argument("--e2e-steps", type=int, default=200, help="steps of the host-buffer e2e leg")
    ap.add_argument("--fp64-steps", type=int, default=20, help="timed steps of the FP64 leg")
    ap.add_argument("--slabs", action="store_true", help="the slab path (the default for N > 1) also at N = 1")
    # profiling modes
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--precision", default="split", choices=["split", "fp64", "fp64_sliced", "both"])
    ap.add_argument("--material", default="lps", choices=["lps", "bond_based", "linear_lps"])
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--nx", type=int, default=0)
    ap.add_argument("--ny", type=int, default=0)
    ap.add_argument("--nz", type=int, default=0)
    ap.add_argument("--tpo", type=int, default=0)
    ap.add_argument("--qs-profile", default=None, choices=["block_jacobi", "two_level", "mpnn"])
    ap.add_argument("--qs-n", type=int, default=60)
    ap.add_argument("--qs-tol", type=float, default=1e-4)
    ap.add_argument("--patch", type=float, default=3.0e-3)
    ap.add_argument("--coarse-modes", type=int, default=3, choices=[3, 6])
    ap.add_argument("--coarse-build-only", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup()

    if args.impl == "reference":
        reference_arm(args, world, rank)
        return
    if args.profile:
        profile_mode(args)
        return
    if args.qs_profile or args.coarse_build_only:
        args.qs_profile = args.qs_profile or "two_level"
        qs_profile_mode(args)
        return

    # CPU baseline processes are spawned before any CUDA call in this process.
    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1 or args.slabs:
        import datetime

        import torch.distributed as dist

        if "MASTER_ADDR" not in os.environ:  # one process outside torchrun
            import socket

            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(sk.getsockname()[1]), RANK="0",
                                  WORLD_SIZE="1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    def max_over_ranks(v):
        if pg is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()

    hbm, peak_src = peak_hbm()
    if world > 1 or args.slabs:
        slab_leg(args, world, rank, local, max_over_ranks, barrier, hbm, peak_src)
        pg.destroy_process_group()
        return
    w, blocks = make_workload(args.workload)
    n = int(len(w["vol"]))
    log(f"workload {w['name']}: {n} points")

    # ---- value: split-FP32 explicit steps, state resident in HBM -----------
    ctx, sp = explicit_leg(w, blocks, local, args.steps, args.warmup, "split", world, max_over_ranks, barrier,
                           timed_clocks=True)
    nb, dt = sp["nb"], sp["dt"]
    log(f"split: {nb} bonds, {sp['ms'] / args.steps:.3f} ms/step")
    u_split = ctx.field("Displacement")
    d_split = ctx.field("Damage")
    slots = sliced_slots(ctx)
    step_bytes = algorithmic_bytes(nb, n, "split")["step"]

    # ---- per-kernel launch durations (CUDA events around each launch) -------
    roofline = kernel_roofline(ctx, dt, sp["t_done"], args.kernel_steps, nb, n, hbm, peak_src, slots)
    roofline["step_frac"] = step_bytes / (sp["ms"] / args.steps / 1e3) / 1e9 / hbm

    log(f"per-kernel ms {roofline['per_kernel_ms']}")
    # ---- e2e: the drop-in computeForce call with host buffers ---------------
    e2e = e2e_leg(ctx, n, nb, args.e2e_steps, 1, max_over_ranks, barrier)
    ctx.close()
    log(f"e2e {e2e['value']:.3e}")

    # ---- plain FP64 path, same workload, same steps from rest ----------------
    fp64 = None
    if not args.no_fp64:
        c64, s64 = explicit_leg(w, blocks, local, args.fp64_steps if args.fp64_steps else args.steps, args.warmup,
                                "fp64", world, max_over_ranks, barrier)
        k64 = args.fp64_steps if args.fp64_steps else args.steps
        fp64 = {"value": s64["value"], "split_over_fp64": sp["value"] / s64["value"], "ms_per_step": s64["ms"] / k64,
                "steps": k64,
                "step_frac": algorithmic_bytes(nb, n, "fp64")["step"] / (s64["ms"] / k64 / 1e3) / 1e9 / hbm,
                "split_step_frac": roofline["step_frac"]}
        u64, d64 = c64.field("Displacement"), c64.field("Damage")
        if k64 == args.steps:  # same step count from rest: the two paths' states compare
            fp64["split_vs_fp64_after_steps"] = args.warmup + args.steps
            fp64["u_rel_l2"] = float(np.linalg.norm(u_split - u64) / max(np.linalg.norm(u64), 1e-300))
            fp64["node_damage_max_diff"] = float(np.max(np.abs(d_split - d64)))
        c64.close()
        log(f"fp64 {fp64['value']:.3e}, split/fp64 {fp64['split_over_fp64']:.2f}")

        # the same FP64 formulas on the split passes' layout (sliced stream at
        # 4 lanes per point, X streamed in FP64): the ratio on equal engineering
        c6, s6 = explicit_leg(w, blocks, local, k64, args.warmup, "fp64_sliced", world, max_over_ranks, barrier)
        u6s, d6s = c6.field("Displacement"), c6.field("Damage")  # after the same steps as the FP64 leg
        r6 = kernel_roofline(c6, s6["dt"], s6["t_done"], min(k64, args.kernel_steps), nb, n, hbm, peak_src, slots,
                             precision="fp64_sliced")
        c6.close()
        fp64["sliced"] = {
            "value": s6["value"], "split_over_fp64_sliced": sp["value"] / s6["value"], "ms_per_step": s6["ms"] / k64,
            "step_frac": algorithmic_bytes(nb, n, "fp64")["step"] / (s6["ms"] / k64 / 1e3) / 1e9 / hbm,
            "per_kernel_ms": r6["per_kernel_ms"], "per_kernel_frac": r6["per_kernel_frac"],
            "u_rel_l2_vs_fp64": float(np.linalg.norm(u6s - u64) / max(np.linalg.norm(u64), 1e-300)),
            "node_damage_max_diff_vs_fp64": float(np.max(np.abs(d6s - d64)))}
        log(f"fp64 sliced {s6['value']:.3e}, split/fp64_sliced {fp64['sliced']['split_over_fp64_sliced']:.2f}")

    # ---- the notched plate (the split/FP64 comparison case) as an extra ------
    extra = None
    if not args.no_extra and args.workload != "notched_plate":
        wp, _ = make_workload("notched_plate")
        cp, spn = explicit_leg(wp, False, local, max(args.steps, 200), args.warmup, "split", world, max_over_ranks,
                               barrier)
        nbp, npt = spn["nb"], int(len(wp["vol"]))
        rp = kernel_roofline(cp, spn["dt"], spn["t_done"], max(args.kernel_steps, 200), nbp, npt, hbm, peak_src,
                             sliced_slots(cp))
        extra = {"workload": "notched_plate_400x200x4", "value": spn["value"],
                 "ms_per_step": spn["ms"] / max(args.steps, 200), "bonds": nbp,
                 "force_frac": rp["per_kernel_frac"]["force"], "dilatation_frac": rp["per_kernel_frac"]["dilatation"],
                 "per_kernel_ms": rp["per_kernel_ms"]}
        cp.close()

    # ---- quasi-static time to 1e-8 (rank 0 only) -----------------------------
    qs = None
    log("qs leg")
    if rank == 0 and not args.no_qs:
        qs = qs_leg(local, args.qs_load_steps, cpu_threads=0 if args.no_cpu_baseline else (os.cpu_count() or 1))

    # ---- CPU baseline (rank 0, N = 1 only) ----------------------------------
    cpu = None
    log("cpu baseline")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import cpu_baseline
        from oracle import oracle as O

        O.build()
        ws, sname, dims = cpu_sample(args.workload)
        row, col = O.neighbor_search(ws["x"], ws["horizon"], ws["planes"])
        r = cpu_baseline.run(ws, row, col, steps=40)
        cpu = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
               "sample": f"{r['steps']} explicit steps of {sname}_{dims[0]}x{dims[1]}x{dims[2]} ({len(col)} bonds) "
                         f"on {r['cores']} processes (slabs with ghost layers, reference LPS kernels compiled from "
                         f"source, block constants)"}

    # the compact comparison keys first (fp64, e2e, roofline), the long QS object last
    line = {"metric": METRIC, "value": sp["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sp["ms"] / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "split-f32 (f64 state)", "data": "synthetic", "fp64": fp64, "e2e": e2e,
            "roofline": roofline,
            "config": {"workload": workload_name(args.workload), "points": n, "bonds": nb, "horizon_over_h": 3.015,
                       "dt": dt, "precision": "split_fp32", "device_gb_in_use": round(sp["device_gb"], 1),
                       "l2": "inputs larger than L2 (%.1f GB of algorithmic bytes per step vs 126 MB L2)"
                             % (step_bytes / 1e9),
                       "parallelism": "one GPU"},
            "cpu_baseline": cpu, "clocks": sp["clocks"], "gpu_launches": 2 * args.steps, "notched_plate": extra,
            "qs": qs}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
