"""Builds tests/golden/ambiguous_keys.npz: an input on which the device's
parallel centre-of-mass sum and the reference's sequential sum give different
Morton keys for one body, so the strict-key repair path must run.

The device sums sum(m), sum(m q) with a fixed order (separately rounded
products, com_mode 0): 296 blocks x 256 threads, each thread summing a
grid-stride slice, a tree reduction per block, then per quantity 32 lanes
summing blocks b = lane, lane + 32, ... and a butterfly (see
hierarquicos_b200/csrc/bh_keys.cu).  This script emulates that order in
float64, moves one body onto a 2^-21 cell edge of the normalised box and
nudges it by ulps until the two centres of mass disagree on its key (checked
with the CPU oracle's keys for the sequential sum).

Usage: python tests/golden/make_ambiguous.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

BLOCKS, THREADS = 296, 256


def parallel_sums(vals):
    """Sum with the device's order; vals: 1-D float64."""
    n = vals.size
    G = BLOCKS * THREADS
    acc = np.zeros(G)
    for start in range(0, n, G):
        chunk = vals[start:start + G]
        acc[:chunk.size] = acc[:chunk.size] + chunk
    blocks = acc.reshape(BLOCKS, THREADS).copy()
    w = THREADS // 2
    while w > 0:
        blocks[:, :w] = blocks[:, :w] + blocks[:, w:2 * w]
        w //= 2
    part = blocks[:, 0]
    lanes = np.zeros(32)
    for b in range(BLOCKS):
        lanes[b % 32] = lanes[b % 32] + part[b]
    o = 16
    while o > 0:
        lanes = lanes + lanes[np.arange(32) ^ o]
        o //= 2
    return lanes[0]


def device_com(m, x, y, z):
    sm = parallel_sums(m)
    return np.array([parallel_sums(m * a) / sm for a in (x, y, z)])


def xn_of(a_vals, a_all_min, a_all_max, c, ssa):
    """x_n of morton_octree.f90:373-384 with every operation rounded."""
    v = (a_vals - c) / ssa
    vc = 0.5 * ((a_all_min - c) / ssa + (a_all_max - c) / ssa)
    return (v + 0.5) - vc


def main():
    import oracle
    from conftest import plummer, xyz

    rng = np.random.default_rng(5)
    m, q = plummer(20000, seed=0)
    m = rng.random(20000) + 0.5
    m /= m.sum()
    x, y, z = [a.copy() + off for a, off in zip(xyz(q), (1000.123, -77.7, 3.3))]
    p = 123
    m[p] = 1e-40   # a massless-in-practice probe: moving it leaves both sums unchanged
    _, _, c_seq4, ssa = oracle.morton_keys(m, x, y, z, 21, 1.2, 0)
    c_seq = c_seq4[:3]
    c_par = device_com(m, x, y, z)
    print("com seq", c_seq, "com par", c_par, "diff", c_par - c_seq)
    for axis in np.argsort(-np.abs(c_par - c_seq)):
        a = (x, y, z)[axis]
        if c_par[axis] == c_seq[axis]:
            continue
        lo, hi = np.sort(a)[1], np.sort(a)[-2]
        for frac in np.linspace(0.2, 0.8, 61):
            cell = np.floor(frac * 2 ** 21)
            target = 0.5 * (a.min() + a.max()) + (cell / 2 ** 21 - 0.5) * ssa
            cand = target + np.arange(-20000, 20000) * np.spacing(target)
            cand = cand[(cand > lo) & (cand < hi)]
            kp = np.floor(xn_of(cand, a.min(), a.max(), c_par[axis], ssa) * 2 ** 21)
            ks = np.floor(xn_of(cand, a.min(), a.max(), c_seq[axis], ssa) * 2 ** 21)
            hit = np.nonzero(kp != ks)[0]
            if hit.size:
                a[p] = cand[hit[0]]
                k_seq, _, c2, _ = oracle.morton_keys(m, x, y, z, 21, 1.2, 0)
                assert np.array_equal(c2[:3], c_seq) and np.array_equal(device_com(m, x, y, z), c_par)
                np.savez_compressed(os.path.join(HERE, "ambiguous_keys.npz"), m=m, x=x, y=y, z=z,
                                    body=p, axis=axis, keys_seq=k_seq)
                print("found: axis", axis, "frac", frac, "x", repr(a[p]))
                return
    raise SystemExit("no ambiguous configuration found")


if __name__ == "__main__":
    main()
