"""Generates the committed fixtures in this folder.

1. recorded_errors.json -- the force-error statistics the reference recorded
   in benchmarks/forces_time_and_error/out/aarseth/test_{monopole,quadrupole,
   octupole}.txt (produced by benchmarks/forces_time_and_error/
   forces_time_and_error.f90:66-111 and :204-308: Plummer spheres, size 10,
   b = 0.58, eps = 0, N = 1024 and 4096, 21 draws per N, methods 10/11/12),
   and for Dehnen's method in benchmarks/dehnen/out/direct_vs_bh_vs_dehnen/
   dehnen_{monopole,quadrupole}.txt (benchmarks/dehnen/forces_dehnen.f90:
   13-153, the same spheres, N = 5000 and 10000, 6 draws, methods 20/21).
   For each (order, N, theta) the median and the 10th/90th percentiles of the
   recorded normalised RMS error are stored.  Needs a checkout of the
   reference, named by the REFERENCE_ROOT environment variable; without it
   this part is skipped.

2. oracle_small.npz -- keys, permutation and forces of the CPU oracle on small
   seeded inputs, so that a change to the oracle is caught even without the
   reference.

Usage: REFERENCE_ROOT=<checkout of the reference> python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

REFERENCE_ROOT = os.environ.get("REFERENCE_ROOT")


def recorded_errors():
    base = os.path.join(REFERENCE_ROOT, "benchmarks", "forces_time_and_error", "out", "aarseth")
    out = {}
    for order, name in ((1, "monopole"), (4, "quadrupole"), (8, "octupole")):
        rows = np.loadtxt(os.path.join(base, f"test_{name}.txt"))
        rows = rows[rows[:, 1] > 0]  # drop the direct-sum rows (theta = -1)
        for n in np.unique(rows[:, 0]).astype(int):
            for th in np.unique(rows[:, 1]):
                sel = rows[(rows[:, 0] == n) & (rows[:, 1] == th)]
                e = sel[:, 4]
                out[f"{order}/{n}/{th:.1f}"] = dict(
                    order=order, n=int(n), theta=float(round(th, 1)), count=int(e.size),
                    median=float(np.median(e)), p10=float(np.percentile(e, 10)),
                    p90=float(np.percentile(e, 90)))
    # Dehnen's method (methods 20/21): benchmarks/dehnen/forces_dehnen.f90:13-153
    # (Plummer, size 10, b = 0.58, eps = 0, 6 draws per N), keys "dehnen<order>/N/theta"
    base = os.path.join(REFERENCE_ROOT, "benchmarks", "dehnen", "out", "direct_vs_bh_vs_dehnen")
    for order, name in ((1, "dehnen_monopole"), (4, "dehnen_quadrupole")):
        rows = np.loadtxt(os.path.join(base, f"{name}.txt"))
        rows = rows[rows[:, 1] > 0]
        for n in (5000, 10000):
            for th in np.unique(rows[:, 1]):
                sel = rows[(rows[:, 0] == n) & (rows[:, 1] == th)]
                e, e2 = sel[:, 4], sel[:, 6]
                out[f"dehnen{order}/{n}/{th:.1f}"] = dict(
                    order=order, n=int(n), theta=float(round(th, 1)), count=int(e.size),
                    median=float(np.median(e)), p10=float(np.percentile(e, 10)),
                    p90=float(np.percentile(e, 90)), median_rel_l2=float(np.median(e2)))
    with open(os.path.join(HERE, "recorded_errors.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote recorded_errors.json", len(out))


def oracle_small():
    import oracle
    from conftest import plummer, xyz

    pts = np.array([[0.45931272, 0.22315240], [0.40157369, 0.21211072], [0.70372114, 0.64428738],
                    [0.20444018, 0.68014233], [0.73388286, 0.59264995], [0.68856885, 0.48249009],
                    [0.48843330, 0.28037004], [0.15927911, 0.69084037], [0.30486200, 0.50604824],
                    [0.59676033, 0.80020091]])
    m10 = np.ones(10)
    x10, y10, z10 = pts[:, 0].copy(), pts[:, 1].copy(), np.zeros(10)
    t10 = oracle.MortonTree(m10, x10, y10, z10, L=0, ssa=1.2, use_quadrupole=True, fma_mode=1)
    k10, p10 = t10.sorted()
    f10 = t10.forces_par(1.0, 0.01 ** 2, 0.1 ** 2, True)
    m, q = plummer(256, seed=0)
    x, y, z = xyz(q)
    t = oracle.MortonTree(m, x, y, z, L=21, ssa=1.2, use_quadrupole=True, fma_mode=1)
    k, p = t.sorted()
    f = t.forces_par(1.0, 0.01 ** 2, 0.5 ** 2, True)
    fo = oracle.Octree(m, 12).init(x, y, z).forces(0.5 ** 2, 1.0, 0.01 ** 2)
    fg = oracle.Octree(m, 31).init(x, y, z).forces(0.5 ** 2, 1.0, 0.01 ** 2)
    fd = oracle.direct_forces(m, x, y, z, 1.0, 0.01 ** 2)
    fdh = oracle.Octree(m, 21).init(x, y, z).forces(0.5 ** 2, 1.0, 0.01 ** 2)
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), m10=m10, x10=x10, y10=y10,
                        z10=z10, L10=t10.L, keys10=k10, perm10=p10, forces10=f10, m=m, x=x, y=y,
                        z=z, keys=k, perm=p, forces_morton_quad=f, forces_octupole=fo,
                        forces_grouped_quad=fg, forces_direct=fd, forces_dehnen_quad=fdh)
    print("wrote oracle_small.npz")


if __name__ == "__main__":
    if REFERENCE_ROOT and os.path.isdir(REFERENCE_ROOT):
        recorded_errors()
    else:
        print("REFERENCE_ROOT not set: recorded_errors.json left as it is")
    oracle_small()
