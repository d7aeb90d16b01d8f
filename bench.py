#!/usr/bin/env python
"""Benchmark of the Barnes-Hut force path on B200.

Workload (one step = one full force evaluation: keys -> radix sort -> octree
-> multipoles -> groups -> walk): Hernquist sphere, N = 1,048,576, a = 1,
truncated at 100 a, equal masses, seeded; theta = 0.5, quadrupole, softening
0.01, FP32 Kahan-compensated group walk.  The metric is forces/s; the error
of every run against the FP64 direct sum is measured on 16,384 seeded targets.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1): every rank evaluates its own
independent system (weak scaling, no collective on the data path); times are
the max over ranks.  ``--impl reference`` times the CPU restatement of the
reference's Fortran (the reference cannot be compiled here: no Fortran
compiler) on this host's cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

N_DEFAULT = 1 << 20
THETA, EPS, ORDER = 0.5, 0.01, 4
N_ERR_TARGETS = 16384
FLOPS_PP = 20          # body-body (GPU Gems 3 convention), morton_octree.f90:676-686
FLOPS_PC = {1: 20, 4: 60, 8: 140}  # cell terms, octree_default.f90:1993-2083
METRIC = "forces/s (N=1M, theta=0.5, err<=1e-3 vs FP64)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--order", type=int, default=ORDER)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--group-size", type=int, default=64)
    ap.add_argument("--leaf-cap", type=int, default=8)
    ap.add_argument("--no-extras", action="store_true",
                    help="timed steps only (no error check, e2e, probe or CPU baseline)")
    return ap.parse_args()


def workload(n, seed):
    from hierarquicos_b200.initial_values import generate_initial_values

    m, q, _ = generate_initial_values(n, 100.0, -1.0, True, False, "hernquist", (1.0, 1.0),
                                      seed=seed, velocities=False)
    return m, q


def config(args, world):
    return {"workload": f"hernquist N={args.n} a=1 r<=100a equal masses seeded",
            "n_per_gpu": args.n, "theta": THETA, "eps": EPS, "order": args.order,
            "walk": {0: "fp32-kahan group walk", 1: "fp64 group walk", 2: "fp64 per-target"}[args.precision],
            "group_size": args.group_size, "leaf_cap": args.leaf_cap, "keys": "63-bit, strict",
            "l2": "flushed (256 MiB write) before every timed step", "parallelism": f"independent systems x{world}"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def gpu_launches_per_step(n, order, strict=True):
    """Kernel launches of one build + walk (counted from the pipeline)."""
    sort_tiles = (n + 4095) // 4096
    scan = 3
    particle_sort = 8 * (1 + scan + 1)          # 8 passes: upsweep, scan x3, downsweep
    first_bits = int(np.ceil(np.log2(n + 1))) + 1
    node_sort = ((first_bits + 5 + 7) // 8) * (1 + scan + 1)
    keys = 3 + (1 if strict else 0)             # reduce, finalize, keys (+ sequential COM)
    tree = 2 + scan + 1 + 1 + node_sort + 1 + 1 + 1   # karras, mark, scan, count, keys, sort, bin2cn, records, levels
    upward = 22
    groups = 1 + scan + 1 + 1                   # flags, scan, count, first
    walk = 1 + (1 if strict else 0)             # walk (+ key verification)
    del sort_tiles
    return keys + particle_sort + 1 + tree + upward + groups + walk


def run_ours(args):
    import torch
    import torch.distributed as dist

    from hierarquicos_b200 import _lib
    from hierarquicos_b200.metrics import error_stats
    from hierarquicos_b200.system import BHSystem, direct_targets

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    n = args.n
    m, q = workload(n, seed=1000 + rank)
    tm = torch.as_tensor(m, device=dev)
    tx, ty, tz = (torch.as_tensor(np.ascontiguousarray(q[:, k]), device=dev) for k in range(3))
    out = torch.empty(3 * n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    p = _lib.default_params(theta=THETA, eps=EPS, order=args.order, precision=args.precision,
                            group_size=args.group_size, leaf_cap=args.leaf_cap)
    sysm = BHSystem(local)
    stream = torch.cuda.current_stream()

    def step():
        sysm.build(tm, tx, ty, tz, p)
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record(stream)
        sysm.walk(p, out)
        return e1

    for _ in range(args.warmup):
        step()
        sysm.sync()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t_total, t_build, t_walk = [], [], []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e2 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            e1 = step()
            e2.record(stream)
            sysm.sync()
            t_total.append(e0.elapsed_time(e2))
            t_build.append(e0.elapsed_time(e1))
            t_walk.append(e1.elapsed_time(e2))
        torch.cuda.synchronize()
    sum_ms = float(sum(t_total))
    if world > 1:
        tt = torch.tensor([sum_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        sum_ms = float(tt.item())
        dist.barrier()
    ms_per_step = sum_ms / args.steps
    value = world * n * args.steps / (sum_ms * 1e-3)

    line = {"metric": METRIC, "value": value, "unit": "forces/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 walk (Kahan), f64 keys/moments", "data": "synthetic (seeded Hernquist ICs)",
            "config": config(args, world), "clocks": clocks.summary(),
            "phases_ms": {"build": statistics.mean(t_build), "walk": statistics.mean(t_walk)},
            "gpu_launches": gpu_launches_per_step(n, args.order) * args.steps}

    if not args.no_extras:
        # accuracy against the FP64 direct sum on seeded targets
        rng = np.random.default_rng(12345 + rank)
        tg = np.sort(rng.choice(n, N_ERR_TARGETS, replace=False))
        ttg = torch.as_tensor(tg, device=dev)
        fd = direct_targets(tm, tx, ty, tz, ttg, 1.0, EPS).T.cpu().numpy()
        f = out.view(3, n).T[ttg].cpu().numpy()
        err = error_stats(f, fd, m[tg], q[tg])
        # reference-semantics interaction counts on the same targets
        fr, cnt = sysm.reference_targets(tg, p, counts=True)
        err_ref = error_stats(fr, fd)
        mean_pp, mean_pc = cnt.mean(axis=0)
        line["accuracy"] = {"targets": N_ERR_TARGETS, "rms_rel": err["rms_rel"],
                            "max_rel": err["max_rel"], "normalised_rms": err.get("normalised_rms"),
                            "reference_walk_rms_rel": err_ref["rms_rel"],
                            "meets_1e-3": err["rms_rel"] <= 1e-3}
        # executed interactions of the group walk
        p.count_stats = 1
        sysm.walk(p, out)
        sysm.sync()
        st = sysm.stats()
        p.count_stats = 0
        peak = np.zeros(2)
        _lib.check(_lib.lib().bh_probe_fma_peak(local, peak.ctypes.data_as(__import__("ctypes").c_void_p)))
        alg_flops = n * (mean_pp * FLOPS_PP + mean_pc * FLOPS_PC[args.order])
        exe_flops = float(st[0]) * FLOPS_PP + float(st[1]) * FLOPS_PC[args.order]
        t_w = statistics.mean(t_walk) * 1e-3
        achieved = alg_flops / t_w / 1e12
        traffic = None
        tf = os.path.join(ROOT, "profiles", "walk_dram_traffic.json")
        if os.path.exists(tf):
            with open(tf) as fh:
                tj = json.load(fh)
            traffic = tj.get("bytes_per_launch_scaled")
        line["roofline"] = {"bound": "fp32", "kernel": "group_walk_kernel", "achieved": achieved,
                            "peak": peak[0] / 1e3, "unit": "TFLOP/s", "frac": achieved / (peak[0] / 1e3),
                            "traffic": traffic,
                            "peak_source": "measured FP32 FMA probe in this run (MEASURED_PEAKS.json has no FP32 figure)",
                            "algorithmic_flops_per_launch": alg_flops,
                            "executed_flops_per_launch": exe_flops,
                            "reference_interactions_per_target": {"body_body": float(mean_pp), "body_cell": float(mean_pc)},
                            "executed_interactions_per_target": {"body_body": float(st[0]) / n, "body_cell": float(st[1]) / n},
                            "walk_ms": t_w * 1e3, "fp64_peak_tflops": peak[1] / 1e3}
        # end to end through the public host API, pinned host buffers
        hm = torch.empty(n, dtype=torch.float64, pin_memory=True)
        hx = torch.empty_like(hm)
        hy = torch.empty_like(hm)
        hz = torch.empty_like(hm)
        hout = torch.empty(3 * n, dtype=torch.float64, pin_memory=True)
        hm.numpy()[:] = m
        hx.numpy()[:] = q[:, 0]
        hy.numpy()[:] = q[:, 1]
        hz.numpy()[:] = q[:, 2]
        import ctypes as C

        L = _lib.lib()

        def e2e_call():
            _lib.check(L.bh_compute_forces_ex(hm.data_ptr(), hx.data_ptr(), hy.data_ptr(), hz.data_ptr(), n,
                                              C.byref(p), hout.data_ptr(), stream.cuda_stream))

        for _ in range(args.warmup):
            e2e_call()
        te = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e2e_call()
            b.record(stream)
            b.synchronize()
            te.append(a.elapsed_time(b))
        e2e_ms = statistics.mean(te)
        if world > 1:
            tt = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_ms = float(tt.item())
        line["e2e"] = {"value": world * n / (e2e_ms * 1e-3), "unit": "forces/s",
                       "ms_per_step": e2e_ms, "h2d_bytes_per_step": 4 * 8 * n,
                       "d2h_bytes_per_step": 3 * 8 * n, "api": "bh_compute_forces_ex (host arrays)"}
        if rank == 0 and world == 1:
            line["cpu_baseline"] = cpu_baseline(n, m, q, args.order, samples=32768)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_baseline(n, m, q, order, samples):
    """CPU restatement of the reference (morton_octree.f90 keys/sort/build/
    quadrupole + barnes_hut walk) on this host's cores: the full tree build
    plus the walk of a seeded sample of targets, scaled to all N targets."""
    import oracle

    x, y, z = (np.ascontiguousarray(q[:, k]) for k in range(3))
    t0 = time.perf_counter()
    tree = oracle.MortonTree(m, x, y, z, L=21, ssa=1.2, use_quadrupole=order >= 4, fma_mode=1)
    t_build = time.perf_counter() - t0
    rng = np.random.default_rng(7)
    tg = rng.choice(n, samples, replace=False)
    t0 = time.perf_counter()
    tree.forces_targets(tg, 1.0, EPS * EPS, THETA * THETA, order >= 4)
    t_walk = time.perf_counter() - t0
    total = t_build + t_walk * n / samples
    del tree
    return {"value": n / total, "unit": "forces/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"full 1M tree build ({t_build:.2f} s) + walk of {samples} seeded targets "
                      f"({t_walk:.2f} s) scaled to N",
            "build_s": t_build, "walk_s_scaled": t_walk * n / samples}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle

    oracle.build()
    n = args.n
    m, q = workload(n, seed=1000)
    samples = 8192
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(n, m, q, args.order, samples)
        if i >= args.warmup:
            vals.append(cb)
    value = statistics.mean(v["value"] for v in vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "forces/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * n / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Hernquist ICs)",
            "config": {"workload": f"hernquist N={n} a=1 r<=100a equal masses seeded", "theta": THETA,
                       "eps": EPS, "order": args.order},
            "cpu_baseline": {"value": value, "unit": "forces/s", "cores": vals[0]["cores"],
                             "kind": "port",
                             "sample": f"per step: full tree build + walk of {samples} seeded targets, scaled to N "
                                       "(the Fortran reference cannot be compiled here: no Fortran compiler)"},
            "e2e": {"value": value, "unit": "forces/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
