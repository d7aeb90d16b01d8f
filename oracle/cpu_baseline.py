"""Timed CPU baseline of the force path -- TEST INFRASTRUCTURE ONLY.

Runs the oracle's restatement of the reference's Morton-tree path on this
host's cores: ``morton_tree_type%init`` (keys, merge sort, level-by-level node
build, quadrupole upward pass; fortran/morton/morton_octree.f90:73-111,
328-625) followed by ``forces_par`` (the per-target barnes_hut walk of every
body under OpenMP; :150-180, 627-766), one full force evaluation per run.  The
library is the oracle source built with the reference's optimisation flags
(-O3 -march=native -fopenmp) for this host, not the parity build.

The benchmark starts this module in a child process so that the OpenMP
environment (OMP_NUM_THREADS = the usable cores, OMP_PROC_BIND = close) is set
before the OpenMP runtime starts, and so that no CUDA context is shared with
the timing.  Prints one JSON line per timed run and a summary line.

  python -m oracle.cpu_baseline --n 1048576 --runs 3 --warmup 1 --order 4 --seed 1000
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def usable_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def child_env(cores: int) -> dict:
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(cores)
    env["OMP_PROC_BIND"] = "close"
    env["OMP_PLACES"] = "cores" if cores > 1 else "threads"
    env["CUDA_VISIBLE_DEVICES"] = ""
    return env


def run(n: int, runs: int, warmup: int, order: int, seed: int, theta: float, eps: float) -> dict:
    import numpy as np

    import oracle
    from hierarquicos_b200.initial_values import generate_initial_values

    so = oracle.use_native_build()
    m, q, _ = generate_initial_values(n, 100.0, -1.0, True, False, "hernquist", (1.0, 1.0),
                                      seed=seed, velocities=False)
    x, y, z = (np.ascontiguousarray(q[:, k]) for k in range(3))
    quad = order >= 4
    rows = []
    for i in range(warmup + runs):
        t0 = time.perf_counter()
        tree = oracle.MortonTree(m, x, y, z, L=21, ssa=1.2, use_quadrupole=quad, fma_mode=1)
        t1 = time.perf_counter()
        tree.forces_par(1.0, eps * eps, theta * theta, quad)
        t2 = time.perf_counter()
        del tree
        if i >= warmup:
            row = {"run": i - warmup, "build_s": t1 - t0, "walk_s": t2 - t1, "total_s": t2 - t0}
            rows.append(row)
            print(json.dumps(row), flush=True)
    tot = [r["total_s"] for r in rows]
    return {"n": n, "runs": runs, "warmup": warmup, "threads": oracle.num_threads(),
            "library": os.path.relpath(so, ROOT), "median_total_s": statistics.median(tot),
            "mean_total_s": statistics.mean(tot),
            "median_build_s": statistics.median(r["build_s"] for r in rows),
            "median_walk_s": statistics.median(r["walk_s"] for r in rows),
            "per_run_s": tot}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--runs", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--order", type=int, default=4)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--theta", type=float, default=0.5)
    ap.add_argument("--eps", type=float, default=0.01)
    a = ap.parse_args()
    summary = run(a.n, a.runs, a.warmup, a.order, a.seed, a.theta, a.eps)
    print(json.dumps({"summary": summary}), flush=True)


if __name__ == "__main__":
    main()
