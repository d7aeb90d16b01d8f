"""Helpers that turn the oracle's reference-layout tree (one node per key
prefix per level, morton_octree.f90:420-493) into the compact octree the
device builds: one node per particle range with >= 2 particles, at the deepest
level of its chain (the link that splits, nchild != 1, or a level-L leaf)."""
from __future__ import annotations

import numpy as np


def compact_from_reference(nodes: dict):
    """(ref_ids, meta (M,4), children (M,8), nchildren (M,)) of the compact
    tree.  meta = first, count, level, nchild.  A child is the compact index of
    the deepest link of its chain, or ~first for a lone particle; entries at or
    beyond nchildren are 0.  Vectorised over the levels (nodes are stored level
    by level, children after parents), so it runs on 10^7-node trees."""
    level, first, last = nodes["level"], nodes["first"], nodes["last"]
    nchild, child = nodes["nchild"], nodes["child"]
    nn = level.size
    multi = last > first
    is_compact = multi & (nchild != 1)
    ref_ids = np.nonzero(is_compact)[0]            # already in (level, first) order
    cidx = np.full(nn, -1, np.int64)
    cidx[ref_ids] = np.arange(ref_ids.size)
    # deepest link of every chain, from the deepest level up
    deep = np.arange(nn, dtype=np.int64)
    chain = multi & (nchild == 1)
    top = int(level.max()) if nn else 0
    bounds = np.searchsorted(level, np.arange(top + 2), side="left")
    for lv in range(top, -1, -1):
        a, b = bounds[lv], bounds[lv + 1]
        r = a + np.nonzero(chain[a:b])[0]
        deep[r] = deep[child[r, 0]]
    nch = np.where(nchild[ref_ids] == 0, 0, nchild[ref_ids]).astype(np.int64)
    meta = np.stack([first[ref_ids], last[ref_ids] - first[ref_ids] + 1, level[ref_ids], nch],
                    axis=1).astype(np.int64)
    used = np.arange(8)[None, :] < nch[:, None]
    ch = np.where(used, child[ref_ids], 0)
    val = np.where(multi[ch], cidx[deep[ch]], ~first[ch].astype(np.int64))
    children = np.where(used, val, 0)
    return ref_ids, meta, children, nch


def exact_octupole(spos_m, spos_x, meta, com):
    """Raw third moments (octree_default.f90 layout, 14 entries) of every
    compact node about the given centres of mass, summed in FP64 with numpy."""
    M = meta.shape[0]
    out = np.zeros((M, 14))
    for j in range(M):
        f, c = meta[j, 0], meta[j, 1]
        m = spos_m[f:f + c]
        d = spos_x[f:f + c] - com[j, :3]
        dx, dy, dz = d[:, 0], d[:, 1], d[:, 2]
        o = [np.sum(m * dx * dx * dx), np.sum(m * dx * dy * dy), np.sum(m * dx * dz * dz),
             np.sum(m * dy * dx * dx), np.sum(m * dy * dy * dy), np.sum(m * dy * dz * dz),
             np.sum(m * dz * dx * dx), np.sum(m * dz * dy * dy), np.sum(m * dz * dz * dz),
             np.sum(m * dx * dy * dz)]
        out[j, :10] = o
        out[j, 10] = sum(o)
        out[j, 11] = o[0] + o[1] + o[2]
        out[j, 12] = o[3] + o[4] + o[5]
        out[j, 13] = o[6] + o[7] + o[8]
    return out
