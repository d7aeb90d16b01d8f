"""Autotuner for the walk's decomposition parameters.

The accuracy of a walk is fixed by theta and the order (the MAC is the
reference's); its speed depends on how targets are grouped and how deep cells
are opened: ``group_size`` (32 or 64 targets per warp), ``group_span``
(consecutive small subtrees packed into one group) and ``leaf_cap`` (cells of
at most this many bodies that fail the MAC are summed body by body).  The
tuner times every candidate on the caller's own batch (a full build + walk,
CUDA events, best of ``reps``), rejects candidates whose error against the
FP64 direct sum on sampled targets exceeds ``max_rms`` (or grows by more than
``slack`` over the default's), and returns the fastest.  Results are cached
in memory and in a JSON file keyed by the workload's shape, so a later run
with the same shape reuses them.
"""
from __future__ import annotations

import itertools
import json
import math
import os
import time

import numpy as np
import torch

from ._lib import BHParams, default_params
from .system import BHSystem, direct_targets

CACHE_PATH = os.path.join(os.path.expanduser("~"), ".cache", "hierarquicos_b200", "autotune.json")
_memory: dict = {}

GROUP_SIZES = (32, 64)
SPAN_FACTORS = (1, 2, 4)
LEAF_CAPS = (4, 8, 16)


def signature(n_total: int, nsys: int, p: BHParams) -> str:
    """Workload shape: log2 buckets of the body and system counts plus the
    parameters that change the work (theta, order, precision, softening)."""
    return (f"n{int(math.log2(max(n_total, 1)))}-s{int(math.log2(max(nsys, 1)))}-t{p.theta:.3f}"
            f"-o{p.order}-p{p.precision}-e{int(p.eps > 0)}")


def _load() -> dict:
    try:
        with open(CACHE_PATH) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(key: str, val: dict) -> None:
    data = _load()
    data[key] = val
    try:
        os.makedirs(os.path.dirname(CACHE_PATH), exist_ok=True)
        tmp = CACHE_PATH + f".{os.getpid()}"
        with open(tmp, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
        os.replace(tmp, CACHE_PATH)
    except OSError:
        pass


def _time_config(sysm: BHSystem, m, x, y, z, off, p: BHParams, out, reps: int) -> float:
    stream = torch.cuda.current_stream()
    best = float("inf")
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sysm.forces_batch(m, x, y, z, off, p, out=out)
        b.record(stream)
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def _errors(out, fd, tg, off) -> float:
    # forces of sampled targets from the per-system blocks
    f = out.view(-1)
    rows = []
    for g in tg.tolist():
        s = int(np.searchsorted(off, g, side="right") - 1)
        a, b = int(off[s]), int(off[s + 1])
        i = g - a
        rows.append([3 * a + i, 3 * a + (b - a) + i, 3 * a + 2 * (b - a) + i])
    idx = torch.as_tensor(np.array(rows), device=out.device)
    fb = f[idx]
    d = torch.linalg.norm(fb - fd, dim=1) / torch.linalg.norm(fd, dim=1)
    return float(torch.sqrt(torch.mean(d * d)))


def tune(m, x, y, z, offsets, params: BHParams | None = None, reps: int = 2,
         max_rms: float = 1e-3, slack: float = 1.5, n_err_targets: int = 2048,
         use_cache: bool = True, verbose: bool = False, **kw) -> tuple[BHParams, dict]:
    """Tunes group_size, group_span and leaf_cap for this batch (CUDA tensors
    or arrays; offsets as for ``BHSystem.forces_batch``).  Returns the tuned
    parameters and a report."""
    p0 = params if params is not None else default_params(**kw)
    dev = torch.device("cuda", torch.cuda.current_device())
    t = [a if isinstance(a, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(a), device=dev)
         for a in (m, x, y, z)]
    m, x, y, z = (a.to(dev, torch.float64).contiguous() for a in t)
    off = np.ascontiguousarray(offsets, np.int64)
    key = signature(int(off[-1]), off.size - 1, p0)
    if use_cache:
        hit = _memory.get(key) or _load().get(key)
        if hit:
            p = default_params()
            for f, _ in BHParams._fields_:
                setattr(p, f, getattr(p0, f))
            p.group_size, p.group_span, p.leaf_cap = hit["group_size"], hit["group_span"], hit["leaf_cap"]
            _memory[key] = hit
            return p, dict(hit, cached=True)
    n = int(off[-1])
    rng = np.random.default_rng(1)
    tg = np.sort(rng.choice(n, min(n_err_targets, n), replace=False))
    # direct sums of the sampled targets within their own systems
    fd_rows = []
    for s in range(off.size - 1):
        a, b = int(off[s]), int(off[s + 1])
        sel = tg[(tg >= a) & (tg < b)]
        if sel.size:
            loc = torch.as_tensor(sel - a, device=dev)
            fd_rows.append(direct_targets(m[a:b], x[a:b], y[a:b], z[a:b], loc, p0.G, p0.eps).T)
    fd = torch.cat(fd_rows)
    sysm = BHSystem()
    out = torch.empty(3 * n, dtype=torch.float64, device=dev)
    results = []
    base_err = None
    cands = [(g, g * f, lc) for g, f, lc in itertools.product(GROUP_SIZES, SPAN_FACTORS, LEAF_CAPS)]
    cands.sort(key=lambda c: (c[0] != p0.group_size, c))
    for g, span, lc in cands:
        p = default_params()
        for f, _ in BHParams._fields_:
            setattr(p, f, getattr(p0, f))
        p.group_size, p.group_span, p.leaf_cap = g, span, lc
        sysm.forces_batch(m, x, y, z, off, p, out=out)  # warm-up (and growth)
        ms = _time_config(sysm, m, x, y, z, off, p, out, reps)
        err = _errors(out, fd, tg, off)
        if g == p0.group_size and lc == p0.leaf_cap and span == (p0.group_span or 2 * g):
            base_err = err
        results.append(dict(group_size=g, group_span=span, leaf_cap=lc, ms=ms, rms=err))
        if verbose:
            print(f"  G={g:2d} span={span:3d} leaf={lc:2d}: {ms:8.3f} ms  rms {err:.3e}", flush=True)
    limit = max_rms if base_err is None else min(max_rms, slack * base_err)
    ok = [r for r in results if r["rms"] <= limit] or results
    best = min(ok, key=lambda r: r["ms"])
    rep = dict(best, candidates=results, key=key, cached=False, when=time.time())
    _memory[key] = rep
    if use_cache:
        _store(key, {k: rep[k] for k in ("group_size", "group_span", "leaf_cap", "ms", "rms", "key")})
    p = default_params()
    for f, _ in BHParams._fields_:
        setattr(p, f, getattr(p0, f))
    p.group_size, p.group_span, p.leaf_cap = best["group_size"], best["group_span"], best["leaf_cap"]
    return p, rep
