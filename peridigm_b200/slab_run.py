"""One body over several GPUs: slab decomposition with a per-step ghost exchange.

    python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 \\
        -m peridigm_b200.slab_run [--workload notched_plate|large_plate] [--steps 100] [--precision split|fp64]

Each rank builds the workload, takes its slab (peridigm_b200.slabs), steps it
with the library's stepping entry points and swaps ghost state with its
neighbors over NCCL once per step. The stable time step is the minimum over
ranks of the local estimates (ghost points with truncated families only
over-estimate theirs, so the minimum is the one-domain value). Rank 0 prints
one JSON line: bond evaluations of owned points per second over all ranks
(strong scaling: the body is fixed, the ranks share it).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="notched_plate", choices=["notched_plate", "large_plate"])
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    a = ap.parse_args()

    import torch
    import torch.distributed as dist

    from . import Context, slabs, workloads

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        w = workloads.large_plate() if a.workload == "large_plate" else workloads.notched_plate()
        plan = slabs.slab_plans(w["x"], w["horizon"], world)[rank]
        with Context(device=local, precision=a.precision) as ctx:
            workloads.setup_context(ctx, slabs.local_workload(w, plan))
            dt_local = torch.tensor([0.7 * ctx.critical_time_step()], dtype=torch.float64, device="cuda")
            dist.all_reduce(dt_local, op=dist.ReduceOp.MIN)
            dt = float(dt_local.item())
            owned_bonds = int(ctx.field("Number_Of_Neighbors")[plan.owned_local].sum())
            halo = slabs.HaloExchange(plan, torch.device("cuda", local), dist)
            dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            slabs.run_slab(slabs.ContextEngine(ctx), halo, dt, a.steps)
            torch.cuda.synchronize()
            dist.barrier()
            sec = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
            dist.all_reduce(sec, op=dist.ReduceOp.MAX)
            bonds = torch.tensor([owned_bonds], dtype=torch.float64, device="cuda")
            dist.all_reduce(bonds, op=dist.ReduceOp.SUM)
        if rank == 0:
            print(json.dumps({"workload": w["name"], "ranks": world, "precision": a.precision, "steps": a.steps,
                              "bonds": int(bonds.item()), "seconds": float(sec.item()),
                              "bond_evals_per_s": float(bonds.item()) * a.steps / float(sec.item()),
                              "scaling": "strong"}), flush=True)
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
