"""Small driver for profiling the explicit step: sets up a notched plate and
runs a few velocity-Verlet steps, so a profiler sees a short list of launches.

    python -m peridigm_b200.profile_run [--precision split|fp64] [--nx 400 --ny 200 --nz 4] [--steps 3]
"""
from __future__ import annotations

import argparse

from . import Context, workloads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    ap.add_argument("--nx", type=int, default=400)
    ap.add_argument("--ny", type=int, default=200)
    ap.add_argument("--nz", type=int, default=4)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--tpo", type=int, default=0)
    a = ap.parse_args()
    w = workloads.notched_plate(nx=a.nx, ny=a.ny, nz=a.nz)
    with Context(precision=a.precision, threads_per_point=a.tpo) as ctx:
        workloads.setup_context(ctx, w)
        dt = 0.7 * ctx.critical_time_step()
        st = ctx.verlet_run(dt, a.steps)
        print(f"points={len(w['vol'])} bonds={ctx.num_bonds()} steps={a.steps} device_ms={st['device_ms']:.3f}")


if __name__ == "__main__":
    main()
