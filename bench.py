"""Benchmark: bond evaluations per second of the explicit LPS + critical-stretch
step on the notched-plate workload (400x200x4 = 320,000 points, h = 0.5 mm,
jitter +-0.05h seed 1, delta = 3.015h, s_c = 5e-4, +-2 m/s prescribed pulls).

One bench step = one velocity-Verlet step: damage + dilatation pass, force
pass with the Verlet epilogue, over every bond. value = bonds x steps /
device time (CUDA events on the library's stream, max over ranks, summed over
ranks for N > 1: each rank runs its own plate, weak scaling).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line on rank 0.
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
    """Bytes each bond pass must move at minimum with this layout (one launch),
    every per-point record counted once (ideal reuse of gathered neighbors).

    Split-FP32, per bond, both passes: col 4 + bond damage 1 + bond vector
    record (X in FP32, omega*V_j) 16 = 21 B.
    Per point, dilatation pass: row 8, owner terms 16, displacement record 32,
    writes A/B 8, theta 8, node damage 8 -> 80 B.
    Per point, force pass: row 8, displacement record 32, rho 8, v read+write 48,
    acceleration 24, u read+write 48, next displacement record 24, BC mask 1 -> 193 B.
    FP64 path (no bond records): per bond col 4 + damage 1; per point the
    gathered FP64 coordinates, material and owner terms (144 B / 217 B)."""
    if precision == "split":
        return {"dilatation": 21 * nb + 80 * n, "force": 21 * nb + 193 * n}
    return {"dilatation": 5 * nb + 144 * n, "force": 5 * nb + 217 * n}


# DRAM bytes (read + write) per launch of the split bond passes on this
# workload, from one ncu capture (--set full, step 1 of the notched plate,
# sliced bond stream, 128-thread blocks): k_dilatation_split<4> 586.0 MB read
# + 7.7 MB written, k_force_split<4> 605.8 MB read + 8.0 MB written. The excess over the
# algorithmic bytes is the slices' padding records (6.3 % of the slots).
NCU_TRAFFIC = {"dilatation": 593.7e6, "force": 613.9e6}


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


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reference_arm(args, world, rank):
    """The reference's own CPU implementation of the step (oracle/_ref: its
    computeDilatation + computeInternalForceLinearElastic compiled from source,
    with the restated critical-stretch damage and Verlet loops) on all host
    cores, over a bounded sample of the workload: the left 100 columns of the
    notched plate (80,000 points, the notch included)."""
    if rank != 0:
        return
    from oracle import cpu_baseline
    from oracle import oracle as O
    from peridigm_b200 import workloads

    O.build()
    w = workloads.notched_plate(nx=100)
    row, col = O.neighbor_search(w["x"], w["horizon"], w["planes"])
    r = cpu_baseline.run(w, row, col, steps=args.steps, warmup=args.warmup)
    value = r["value"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "notched_plate_100x200x4 (sample of notched_plate_400x200x4)",
                       "points": int(len(w["vol"])), "bonds": int(len(col)), "precision": "fp64"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": f"{args.steps} explicit steps of a 100x200x4 slab of the plate "
                                       f"({len(col)} bonds), {r['cores']} processes"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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
    trained here on such two-level solves of a 12^3 cube over six random
    moduli and load paths; the weights kept are the checkpoint, every 10
    epochs from epoch 0, with the fewest CG iterations on a held-out 12^3
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
        tr.mpnn_collect(4)
        rng = np.random.default_rng(5)
        for _ in range(6):
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
        # model selection: checkpoints every 10 epochs (epoch 0 = the starting
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
        for epoch in (10, 20, 30, 40):
            loss = tr.mpnn_train(10, learning_rate=1e-3, batch=8)
            wts = tr.mpnn_weights()
            checkpoints[epoch] = (validate(wts), wts)
        last_weights = checkpoints[40][1]
        best_epoch = min(checkpoints, key=lambda e: (checkpoints[e][0], e))
        weights = checkpoints[best_epoch][1]
    train_s = time.perf_counter() - t0
    w2 = workloads.qs_cube(n=60, h=1.0e-3, seed=1000, load_steps=load_steps)
    out = {"workload": f"qs_cube_60x60x60 (seed 1000, {load_steps} load steps)", "points": int(len(w2["vol"])),
           "tolerance": 1e-8, "training": {"pairs": pairs, "epochs": 40, "final_loss": loss, "seconds": train_s,
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
            st = None
            clocks = ClockSampler(local)
            clocks.start()
            t1 = time.perf_counter()
            for k in range(1, len(w2["times"])):
                st = ctx.qs_load_step(w2["times"][k - 1], w2["times"][k], newton_tolerance=-1e-8,
                                      cg_relative_tolerance=1e-8, preconditioner=precond, stats=st)
            wall = time.perf_counter() - t1
            clk = clocks.stop()
            out[arm] = {"seconds": st.device_ms / 1e3, "wall_seconds": wall, "cg_iterations": st.cg_iterations,
                            "newton_iterations": st.newton_iterations, "final_cg_residual": st.final_residual,
                            "fallbacks": st.preconditioner_fallbacks, "coarse_builds": st.coarse_builds,
                            "sm_mhz": clk["sm_mhz"],
                            "clock_reasons": clk["reasons"]}
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
                                           sample="block-Jacobi CG restated in C (matrix-free LPS tangent, "
                                                  "3x3 block inverses) on %d host threads: 20 CG iterations and one "
                                                  "Newton set-up at the solved state, scaled by the GPU solve's %d "
                                                  "Newton and %d CG iterations" % (cpu_threads, st.newton_iterations,
                                                                                  st.cg_iterations))
    bj = out["block_jacobi"]["seconds"]
    out["two_level_speedup_over_block_jacobi"] = bj / out["two_level"]["seconds"]
    out["two_level_rigid_speedup_over_block_jacobi"] = bj / out["two_level_rigid"]["seconds"]
    out["mpnn_speedup_over_block_jacobi"] = bj / out["mpnn"]["seconds"]
    out["mpnn_last_epoch_speedup_over_block_jacobi"] = bj / out["mpnn_last_epoch"]["seconds"]
    if "cpu_baseline" in out:
        out["block_jacobi_speedup_over_cpu"] = out["cpu_baseline"]["seconds"] / bj
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-qs", action="store_true")
    ap.add_argument("--qs-load-steps", type=int, default=20)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup(args.gpus)

    if args.impl == "reference":
        reference_arm(args, world, rank)
        return

    # CPU baseline processes are spawned before any CUDA call in this process.
    from peridigm_b200 import Context, workloads

    w = workloads.notched_plate()
    n = int(len(w["vol"]))

    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

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

    ctx = Context(device=local, precision="split")
    workloads.setup_context(ctx, w)
    nb = ctx.num_bonds()
    dt = 0.7 * ctx.critical_time_step()

    # ---- value: split-FP32 explicit steps, state resident in HBM -----------
    ctx.verlet_run(dt, args.warmup)
    t_done = args.warmup * dt
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    st = ctx.verlet_run(dt, args.steps, t0=t_done)
    barrier()
    clk = clocks.stop()
    t_done += args.steps * dt
    ms = max_over_ranks(st["device_ms"])
    value = world * nb * args.steps / (ms / 1e3)

    # ---- per-kernel launch durations (CUDA events around each launch) -------
    ksteps = min(args.steps, 500)
    ctx.kernel_timing(True)
    ctx.verlet_run(dt, ksteps, t0=t_done)
    kt = ctx.kernel_times()
    ctx.kernel_timing(False)
    t_done += ksteps * dt
    per = {"dilatation": kt["dilatation_ms"] / kt["evaluations"], "force": kt["force_ms"] / kt["evaluations"]}
    dom = max(per, key=per.get)
    algo = algorithmic_bytes(nb, n, "split")
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        hbm, peak_src = float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        hbm, peak_src = 6650.0, "fallback"
    achieved = algo[dom] / (per[dom] / 1e3) / 1e9
    traffic = NCU_TRAFFIC[dom]
    roofline = {"bound": "hbm", "kernel": f"k_{dom}_split", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": peak_src, "traffic": traffic,
                "algorithmic_bytes": algo[dom], "launch_ms": per[dom],
                "per_kernel_ms": per}

    # ---- plain FP64 path, same workload --------------------------------------
    fsteps = min(args.steps, 1000)
    c64 = Context(device=local, precision="fp64")
    workloads.setup_context(c64, w)
    c64.verlet_run(dt, args.warmup)
    barrier()
    st64 = c64.verlet_run(dt, fsteps, t0=args.warmup * dt)
    barrier()
    ms64 = max_over_ranks(st64["device_ms"])
    value64 = world * nb * fsteps / (ms64 / 1e3)
    c64.close()

    # ---- e2e: the drop-in computeForce call with host buffers ---------------
    # Each step: H2D of the current coordinates from pinned memory, damage +
    # dilatation + force on the device, D2H of the force density, then the
    # state update that commits the step's bond damage (the reference's
    # evalModel + updateState cycle, Peridigm.cpp:1536, 1589).
    esteps = min(args.steps, 500)
    y = torch.from_numpy(ctx.field("Coordinates")).pin_memory()
    f = torch.zeros(3 * n, dtype=torch.float64).pin_memory()
    import ctypes as C

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
    e2e = {"value": world * nb * esteps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 24 * n,
           "d2h_bytes_per_step": 24 * n, "steps": esteps, "api": "pd_compute_force (host y in, host force out) + pd_update_state"}

    # ---- quasi-static time to 1e-8 (rank 0 only) -----------------------------
    qs = None
    if rank == 0 and not args.no_qs:
        qs = qs_leg(local, args.qs_load_steps, cpu_threads=0 if args.no_cpu_baseline else (os.cpu_count() or 1))

    # ---- CPU baseline (rank 0, N = 1 only) ----------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import cpu_baseline
        from oracle import oracle as O

        row, col = ctx.bonds_csr()
        O.build()
        r = cpu_baseline.run(w, row, col, steps=40, dt=dt)
        cpu = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
               "sample": f"{r['steps']} explicit steps of the full 400x200x4 plate on {r['cores']} processes "
                         f"(slabs with ghost layers, reference LPS kernels compiled from source)"}
    ctx.close()

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "split-f32 (f64 state)", "data": "synthetic",
            "config": {"workload": "notched_plate_400x200x4", "points": n, "bonds": nb, "horizon_over_h": 3.015,
                       "critical_stretch": 5e-4, "dt": dt, "precision": "split_fp32",
                       "l2": "inputs larger than L2 (about 1.2 GB read per step vs 126 MB L2)",
                       "parallelism": f"replicas x{world}"},
            "fp64": {"value": value64, "unit": UNIT, "steps": fsteps, "ms_per_step": ms64 / fsteps,
                     "split_over_fp64": value / value64},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "qs": qs, "clocks": clk,
            "gpu_launches": 2 * args.steps}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
