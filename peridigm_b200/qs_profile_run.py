"""Small driver for profiling the quasi-static path: one load step of the
60^3 tensile cube (216,000 points) with a chosen preconditioner, so a
profiler sees the tangent, preconditioner and reduction launches of a short
CG solve.

    python -m peridigm_b200.qs_profile_run [--precond block_jacobi|two_level|mpnn] [--n 60] [--tol 1e-4]
        [--coarse-modes 3|6] [--coarse-build-only]

With --precond mpnn the learned middle level runs untrained (its starting
weights): the launch sequence and its cost are those of a trained one. With
--coarse-build-only no load step runs: the two-level coarse operator is built
at zero displacement (pd_qs_coarse_operator: one call for its size, one for
its contents, each a full build) and |Ac^-1 Ac - I| over its first 256 rows
is printed.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import Context, workloads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--precond", default="two_level", choices=["block_jacobi", "two_level", "mpnn"])
    ap.add_argument("--n", type=int, default=60)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--patch", type=float, default=3.0e-3)
    ap.add_argument("--coarse-modes", type=int, default=3, choices=[3, 6])
    ap.add_argument("--coarse-build-only", action="store_true")
    a = ap.parse_args()
    w = workloads.qs_cube(n=a.n, h=1.0e-3, seed=1000, load_steps=20)
    with Context(precision="fp64") as ctx:
        workloads.setup_context(ctx, w)
        ctx.coarse_modes(a.coarse_modes)
        if a.coarse_build_only:
            _, A, Ai = ctx.coarse_operator(np.zeros(3 * len(w["vol"])))
            m = min(256, A.shape[0])
            err = float(np.abs(Ai[:m] @ A - np.eye(A.shape[0])[:m]).max())
            print(json.dumps({"coarse_dofs": int(A.shape[0]), "max_abs_inverse_error": err}))
            return
        if a.precond == "mpnn":
            ctx.mpnn_init(seed=0, patch=a.patch)
        st = ctx.qs_load_step(w["times"][0], w["times"][1], newton_tolerance=-1e-3, cg_relative_tolerance=a.tol,
                              preconditioner=a.precond)
        print(json.dumps({"precond": a.precond, "points": int(len(w["vol"])), "cg_iterations": st.cg_iterations,
                          "newton_iterations": st.newton_iterations, "device_ms": st.device_ms}))


if __name__ == "__main__":
    main()
