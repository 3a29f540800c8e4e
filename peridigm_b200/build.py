"""In-tree build of the CUDA library (sm_100a) and of the CPU oracle."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build(verbose: bool = False) -> None:
    """nvcc -gencode arch=compute_100a,code=sm_100a for every .cu in csrc/ into
    peridigm_b200/libpd_b200.so, then the oracle (test infrastructure)."""
    jobs = str(min(8, os.cpu_count() or 2))
    for d in (os.path.join(HERE, "csrc"), os.path.join(ROOT, "oracle")):
        r = subprocess.run(["make", "-j", jobs, "-C", d], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"build failed in {d}:\n{r.stdout[-4000:]}\n{r.stderr[-4000:]}")
        if verbose:
            print(r.stdout)


if __name__ == "__main__":
    build(verbose=True)
