"""Small driver for profiling and for throughput at other sizes: sets up a
workload and runs a few velocity-Verlet steps, so a profiler sees a short list
of launches.

    python -m peridigm_b200.profile_run [--precision split|fp64] [--nx 400 --ny 200 --nz 4] [--steps 3]
    python -m peridigm_b200.profile_run --workload large_plate --steps 20 --compare
    python -m peridigm_b200.profile_run --material bond_based --steps 200 --compare

--workload picks the notched plate (default, sized by --nx/--ny/--nz), the
32M-point heterogeneous plate (large_plate, 400x400x200) or the plate with a
dropped sphere and contact (plate_sphere, 400x400x40 + sphere). --compare runs
the split-FP32 and the FP64 path one after the other on the same workload and
prints both throughputs and the relative L2 difference of the displacements.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import Context, workloads


def _run(w, precision, steps, tpo, blocks, material="lps"):
    with Context(precision=precision, threads_per_point=tpo) as ctx:
        (workloads.setup_context_blocks if blocks else workloads.setup_context)(ctx, w)
        if material == "bond_based":  # same bulk modulus and density, elastic bond-based model
            for b in range(int(np.max(w["block"])) + 1 if blocks else 1):
                ctx.material_bond_based(float(np.median(w["K"])), w["rho"], block=b)
        if material == "linear_lps":  # same moduli and density, the LPS model linearised
            for b in range(int(np.max(w["block"])) + 1 if blocks else 1):
                ctx.material_linear_lps(float(np.median(w["K"])), float(np.median(w["mu"])), w["rho"], block=b)
        dt = w.get("safety", 0.7) * ctx.critical_time_step()
        st = ctx.verlet_run(dt, steps)
        nb = ctx.num_bonds()
        line = {"workload": w["name"], "material": material, "precision": precision, "points": int(len(w["vol"])), "bonds": int(nb),
                "steps": steps, "device_ms": st["device_ms"], "ms_per_step": st["device_ms"] / max(steps, 1),
                "bond_evals_per_s": nb * steps / (st["device_ms"] / 1e3) if st["device_ms"] > 0 else 0.0,
                "broken_bonds": st["broken_bonds"]}
        return line, ctx.field("Displacement"), ctx.field("Damage")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    ap.add_argument("--workload", default="notched_plate", choices=["notched_plate", "large_plate", "plate_sphere"])
    ap.add_argument("--nx", type=int, default=400)
    ap.add_argument("--ny", type=int, default=200)
    ap.add_argument("--nz", type=int, default=4)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--tpo", type=int, default=0)
    ap.add_argument("--compare", action="store_true")
    ap.add_argument("--material", default="lps", choices=["lps", "bond_based", "linear_lps"])
    a = ap.parse_args()
    blocks = False
    if a.workload == "large_plate":
        w = workloads.large_plate()
    elif a.workload == "plate_sphere":
        w, blocks = workloads.plate_sphere(), True
    else:
        w = workloads.notched_plate(nx=a.nx, ny=a.ny, nz=a.nz)
    precisions = ["split", "fp64"] if a.compare else [a.precision]
    res = {}
    for p in precisions:
        line, u, d = _run(w, p, a.steps, a.tpo, blocks, a.material)
        res[p] = (u, d)
        print(json.dumps(line), flush=True)
    if a.compare:
        (us, ds), (u6, d6) = res["split"], res["fp64"]
        print(json.dumps({"split_vs_fp64_u_rel_l2": float(np.linalg.norm(us - u6) / max(np.linalg.norm(u6), 1e-300)),
                          "max_node_damage_diff": float(np.max(np.abs(ds - d6)))}), flush=True)


if __name__ == "__main__":
    main()
