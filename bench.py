#!/usr/bin/env python
"""Benchmark of the Barnes-Hut force path on B200.

Headline (default): force evaluations of N = 1,048,576-body Hernquist systems
(a = 1, truncated at 100 a, equal masses, seeded; theta = 0.5, quadrupole,
softening 0.01, FP32 Kahan-compensated group walk: producer/consumer warp
teams, box test plus every member's own MAC), served by the continuous
batching server against the plain single-system call:

  * plain  -- ``bh_system_forces`` per system (keys -> radix sort -> octree ->
    multipoles -> groups -> walk -> status), device-resident inputs, the L2
    flushed before every call;
  * served -- the same systems submitted at once to ``serving.Server``
    (3 lanes, ticks of up to 2 systems, continuous batching), device-resident
    requests prepared ahead (result buffers allocated) and queued together
    with ``submit_many``; p50/p99 latency per request;
  * e2e    -- both again from pinned HOST buffers with the copies included:
    plain through ``bh_compute_forces_ex`` (the api3d drop-in), served with
    host requests;
  * batched -- 512 independent systems (N log-uniform in [1024, 65536], Plummer
    and uniform-density spheres): one batched build + walk (and its CUDA-graph
    replay) with autotuned group/leaf parameters against a loop of plain
    calls;
  * dehnen -- Dehnen's dual-tree method (FP64) on the accuracy system, with its
    error on the same targets;
  * serving_sweep, parareal -- the serving config (Poisson arrivals, rate swept)
    and the batched Parareal config, as ``--serving-sweep`` and ``--parareal``
    print them on their own (single-GPU runs only).

The RMS relative error is measured against the FP64 direct sum on 16,384
seeded targets; served results are checked equal (bit for bit) to the plain
ones.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --serving-sweep     # the serving config: Poisson arrivals, rate swept
  python bench.py --parareal          # the batched Parareal config

One process per GPU (torchrun for N > 1): every rank serves its own systems
(weak scaling, no collective on the data path); times are the max over
ranks.  ``--impl reference`` times the CPU restatement of the reference's
Fortran (the reference cannot be compiled here: no Fortran compiler) on this
host's cores: one full force evaluation of the headline system per step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
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
# Algorithmic flops per interaction, each operation of the reference's formulas
# listed once (a multiply-add counts 2; in the body-body term rsqrt counts 2,
# which gives the usual 20 of the GPU Gems 3 convention).
FLOP_OPS = {
    # morton_octree.f90:676-686 (and the monopole cell term :711-718)
    "body_body": [("d = x_j - x_i", 3), ("r2 = d.d + eps2", 6), ("rsqrt", 2),
                  ("r^-3 = rinv^3", 2), ("m r^-3", 1), ("a += s d", 6)],
    # octree_default.f90:2009-2027 (a10's quadrupole cell term; rsqrt counts 1 here)
    "quad_cell": [("d = c - x_i", 3), ("r2 = d.d + eps2", 6), ("rsqrt", 1),
                  ("powers r^-2 .. r^-7", 6), ("Q d (3 rows of 3 terms)", 15), ("d.Q.d", 5),
                  ("1.5 trQ", 2), ("s = M/r^3 - 1.5 trQ/r^5 + 7.5 dQd/r^7", 7),
                  ("a += s d - 3 Q d / r^5", 15)],
    # octree_default.f90:2033-2082 (a10's octupole cell term, on top of the quadrupole)
    "oct_extra": [("r^-4 and the 7.5, -1.5, -17.5 prefactors", 5), ("pair products of d", 6),
                  ("O_{12..14}.d and its scale", 6), ("three rows of O contracted with d d", 42),
                  ("cubic contraction O:ddd", 17), ("a += r^-3 o", 4)],
}
FLOPS_PP = sum(k for _, k in FLOP_OPS["body_body"])                 # 20
_QUAD = sum(k for _, k in FLOP_OPS["quad_cell"])                    # 60
FLOPS_PC = {1: FLOPS_PP, 4: _QUAD, 8: _QUAD + sum(k for _, k in FLOP_OPS["oct_extra"])}
assert (FLOPS_PP, FLOPS_PC[4], FLOPS_PC[8]) == (20, 60, 140)
METRIC = "forces/s (N=1M, theta=0.5, err<=1e-3 vs FP64): served vs plain; p50/p99 ms"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--bodies", type=int, default=N_DEFAULT, dest="n")
    ap.add_argument("--order", type=int, default=ORDER)
    ap.add_argument("--precision", type=int, default=0,
                    help="0 FP32 group walk, 1 FP64 group walk, 2 per-target FP64, 3 Dehnen")
    ap.add_argument("--group-size", type=int, default=64)
    ap.add_argument("--leaf-cap", type=int, default=8)
    ap.add_argument("--group-span", type=int, default=0)
    ap.add_argument("--mac", type=int, default=1,
                    help="group walk acceptance: 0 the group's box distance, 1 also a node that "
                         "every member's own MAC accepts (default)")
    ap.add_argument("--pipeline", type=int, default=None,
                    help="FP32 walk: 0 one warp per group, 1 producer/consumer warp teams "
                         "(the library default)")
    ap.add_argument("--lanes", type=int, default=3)
    ap.add_argument("--tick-systems", type=int, default=2,
                    help="served: systems of N bodies one lane's tick may hold")
    ap.add_argument("--batch-systems", type=int, default=512)
    ap.add_argument("--split-system", action="store_true",
                    help="strong scaling: every rank takes the same system and walks its share of "
                         "the target groups; one all-reduce combines them (implies --no-extras)")
    ap.add_argument("--serving-sweep", action="store_true",
                    help="instead of the headline line: the serving config (Poisson arrivals, "
                         "rate swept, force and leapfrog requests, N log-uniform in [1024, 2^21] "
                         "over three profiles); prints one JSON line of its own")
    ap.add_argument("--sweep-requests", type=int, default=48)
    ap.add_argument("--parareal", action="store_true",
                    help="instead of the headline line: the batched Parareal config (Plummer "
                         "16384, 64 slices, coarse monopole theta 0.8, fine quadrupole theta 0.3)")
    ap.add_argument("--parareal-bodies", type=int, default=16384)
    ap.add_argument("--parareal-iters", type=int, default=40)
    ap.add_argument("--no-extras", action="store_true",
                    help="plain timed calls only (no serving, error check, e2e, batch or CPU baseline)")
    return ap.parse_args()


def workload(n, seed):
    from hierarquicos_b200.initial_values import generate_initial_values

    m, q, _ = generate_initial_values(n, 100.0, -1.0, True, False, "hernquist", (1.0, 1.0),
                                      seed=seed, velocities=False)
    return m, q


def device_workload(n, seed):
    """Hernquist system drawn on the device: m, x, y, z (n,) CUDA tensors."""
    from hierarquicos_b200.initial_values import generate_initial_values_device

    m, q, _ = generate_initial_values_device(n, 100.0, -1.0, True, False, "hernquist", (1.0, 1.0),
                                             seed=seed, velocities=False)
    return m, q[0].contiguous(), q[1].contiguous(), q[2].contiguous()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.p is not None:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def launches_per_evaluation(n, nsys=1, L=21):
    """Our kernel launches in one build + walk (the pipeline's launch
    sequence: 54 for one system of 2^20 bodies)."""
    scan = 1                                           # one chained-scan launch

    def sort(bits):                                    # digit histograms, their scan, passes
        return 2 + math.ceil(bits / 8)

    keys = 3                                           # reduce, finalize, keys
    particle_sort = sort(3 * L)
    by_system = 0
    if nsys >= 2:
        by_system = 1 + sort(max(1, math.ceil(math.log2(nsys)))) + 1
    first_bits = 1
    while (1 << first_bits) <= n:
        first_bits += 1
    node_sort = sort(first_bits + 5)
    # karras, mark, scan (also writes the node count), compact keys, node sort, bin2cn,
    # records, levels, roots
    tree = 2 + scan + 1 + node_sort + 1 + 1 + 1 + 1
    upward = 22                                        # one launch per level
    groups = 1 + scan + 1                              # flags (and system starts), scan, first
    walk = 1
    return keys + particle_sort + by_system + 1 + tree + upward + groups + walk


def dist_max(x, dev, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


HOST_CPUS = None  # the process's CPUs before bind_to_gpu_node narrowed them


def parse_cpulist(text):
    """'0-3,8,10-11' -> {0, 1, 2, 3, 8, 10, 11}."""
    cpus = set()
    for part in text.strip().split(","):
        if not part:
            continue
        lo, _, hi = part.partition("-")
        cpus.update(range(int(lo), int(hi or lo) + 1))
    return cpus


def bind_to_gpu_node(torch, dev):
    """Binds this process to the CPUs of the GPU's own NUMA node (the PCI
    device's local_cpulist in sysfs), as a deployment pins a GPU's host
    process: pinned host buffers allocated afterwards sit in that node's
    memory, and host<->device copies do not cross the socket link (a copy from
    the other socket's memory runs at a fraction of the bandwidth).  Returns
    what was done, as a sentence for the bench line."""
    global HOST_CPUS
    try:
        pr = torch.cuda.get_device_properties(dev)
        addr = f"{pr.pci_domain_id:04x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        with open(f"/sys/bus/pci/devices/{addr}/local_cpulist") as fh:
            local_cpus = parse_cpulist(fh.read())
        current = os.sched_getaffinity(0)
    except (OSError, AttributeError, ValueError, RuntimeError) as exc:
        return f"unbound (GPU's node not known: {type(exc).__name__})"
    mine = local_cpus & current
    if not mine:
        return "unbound (none of this process's CPUs is on the GPU's node)"
    if mine == current:
        return f"unbound: all {len(current)} CPUs of this process are on the GPU's node"
    HOST_CPUS = current
    os.sched_setaffinity(0, mine)
    return (f"bound to the {len(mine)} CPUs of the GPU's node (sysfs local_cpulist); pinned "
            f"buffers allocated afterwards")


class all_host_cpus:
    """Restores the process's full CPU set for the duration (child processes
    started inside inherit it), then the narrowed one."""

    def __enter__(self):
        self.saved = os.sched_getaffinity(0)
        if HOST_CPUS:
            os.sched_setaffinity(0, HOST_CPUS)
        return self

    def __exit__(self, *a):
        os.sched_setaffinity(0, self.saved)


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
    bound_cpus = bind_to_gpu_node(torch, local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    n = args.n
    K, W = args.steps, args.warmup
    p = _lib.default_params(theta=THETA, eps=EPS, order=args.order, precision=args.precision,
                            group_size=args.group_size, leaf_cap=args.leaf_cap,
                            group_span=args.group_span)
    if args.mac is not None:
        p.mac = args.mac
    if args.pipeline is not None:
        p.pipeline = args.pipeline
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    # K timed + W warm-up systems, drawn on the device (the same systems on
    # every rank when one system is split over the ranks)
    rank_seed = 0 if args.split_system else 97 * rank
    systems = [device_workload(n, seed=1000 + rank_seed + i) for i in range(K + W)]
    out = torch.empty(3 * n, dtype=torch.float64, device=dev)
    if args.split_system:
        args.no_extras = True
        return run_split(args, p, systems, out, flush, dev, local, rank, world)

    # ---- plain: one call per system ----
    sysm = BHSystem(local)
    for i in range(W):
        sysm.forces(*systems[K + i], p, out=out)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t_total, t_build, t_walk = [], [], []
    with ClockSampler(local) as clocks:
        for i in range(K):
            flush.zero_()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ev[0].record(stream)
            sysm.build(*systems[i], p)
            ev[1].record(stream)
            sysm.walk(p, out)
            ev[2].record(stream)
            sysm.sync()          # status, strict-key check (and its rare rebuild)
            ev[3].record(stream)
            ev[3].synchronize()
            t_total.append(ev[0].elapsed_time(ev[3]))
            t_build.append(ev[0].elapsed_time(ev[1]))
            t_walk.append(ev[1].elapsed_time(ev[2]))
        torch.cuda.synchronize()
    plain_ms = dist_max(float(sum(t_total)), dev, world) / K
    plain_value = world * n / (plain_ms * 1e-3)
    f_plain_last = out.clone()

    line = {"metric": METRIC, "value": plain_value, "unit": "forces/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": plain_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 walk (Kahan), f64 keys/moments",
            "data": "synthetic (seeded Hernquist ICs drawn on the device)",
            "config": headline_config(args, n, p.mac, p.pipeline, K, world),
            "plain": {"value": plain_value, "unit": "forces/s", "ms_per_step": plain_ms,
                      "phases_ms": {"build": statistics.mean(t_build),
                                    "walk": statistics.mean(t_walk),
                                    "status": statistics.mean(t_total) - statistics.mean(t_build)
                                    - statistics.mean(t_walk)}},
            "clocks": clocks.summary(),
            "gpu_launches": launches_per_evaluation(n) * K}

    if not args.no_extras:
        from hierarquicos_b200 import serving

        def serve(reqs, warm):
            """Submits ``warm`` and waits, then submits all of ``reqs`` at
            once; returns (device ms from first submission to the last result,
            metrics of ``reqs``)."""
            with serving.Server(p, device=local, lanes=args.lanes,
                                max_tick_bodies=args.tick_systems * n, hbm_budget=150e9) as srv:
                srv.submit_many(warm)
                # the client allocates its requests' result buffers ahead of
                # time (device requests) or pins them (host requests)
                for r in reqs:
                    srv.prepare(r)
                srv.drain(timeout=600)
                torch.cuda.synchronize()
                if world > 1:
                    dist.barrier()
                for ln in srv.lanes:
                    ln.ticks = ln.tick_bodies = 0
                    ln.tick_log.clear()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                t0 = time.perf_counter()
                for r in reqs:
                    r.arrival = t0
                srv.submit_many(reqs)
                srv.drain(timeout=600)
                torch.cuda.synchronize()
                b.record(stream)
                b.synchronize()
                return a.elapsed_time(b), srv.metrics(reqs)

        def dev_reqs(idx):
            return [serving.Request("force", systems[i][0], torch.stack(systems[i][1:4]))
                    for i in idx]

        # ---- served: the same K systems as device-resident requests ----
        reqs = dev_reqs(range(K))
        with ClockSampler(local) as sclocks:
            served_total_ms, met = serve(reqs, dev_reqs(range(K, K + W)))
        served_ms = dist_max(served_total_ms, dev, world) / K
        served_value = world * n / (served_ms * 1e-3)
        # a request served in a two-system tick equals the plain call, bit for bit
        same = bool(torch.equal(reqs[-1].forces.T.reshape(-1), f_plain_last))
        line["value"] = served_value
        line["ms_per_step"] = served_ms
        line["served"] = {"value": served_value, "unit": "forces/s", "ms_per_request": served_ms,
                          "p50_ms": met["p50_ms"], "p99_ms": met["p99_ms"], "ticks": met["ticks"],
                          "mean_tick_bodies": met["mean_tick_bodies"], "lanes": args.lanes,
                          "tick_times": met["tick_times"],
                          "equal_to_plain_bitwise": same}
        line["served_over_plain"] = served_value / plain_value
        line["latency_ms"] = {"p50": met["p50_ms"], "p99": met["p99_ms"],
                              "definition": "all K requests arrive at once; arrival to result ready "
                                            "on the device"}
        line["clocks"] = sclocks.summary()
        line["clocks_plain"] = clocks.summary()
        line["gpu_launches"] = launches_per_evaluation(2 * n, 2) * met["ticks"]

        # ---- accuracy against the FP64 direct sum (plain output of the last system) ----
        mK, xK, yK, zK = systems[K - 1]
        rng = np.random.default_rng(12345 + rank)
        tg = np.sort(rng.choice(n, N_ERR_TARGETS, replace=False))
        ttg = torch.as_tensor(tg, device=dev)
        fd = direct_targets(mK, xK, yK, zK, ttg, 1.0, EPS).T.cpu().numpy()
        f = f_plain_last.view(3, n).T[ttg].cpu().numpy()
        mh = mK.cpu().numpy()
        qh = torch.stack([xK, yK, zK], 1).cpu().numpy()
        err = error_stats(f, fd, mh[tg], qh[tg])
        sysm.build(mK, xK, yK, zK, p)
        sysm.sync()
        fr, cnt = sysm.reference_targets(tg, p, counts=True)
        err_ref = error_stats(fr, fd)
        mean_pp, mean_pc = cnt.mean(axis=0)
        line["accuracy"] = {"targets": N_ERR_TARGETS, "rms_rel": err["rms_rel"],
                            "max_rel": err["max_rel"], "normalised_rms": err.get("normalised_rms"),
                            "reference_walk_rms_rel": err_ref["rms_rel"],
                            "meets_1e-3": err["rms_rel"] <= 1e-3,
                            "served": "identical to plain (bitwise)" if same else "DIFFERS"}

        # ---- Dehnen's dual-tree method on the same system (methods 20/21/22) ----
        pd = _lib.default_params(theta=THETA, eps=EPS, order=args.order,
                                 precision=_lib.BH_PREC_DEHNEN)
        dsys = BHSystem(local)
        dout = torch.empty(3 * n, dtype=torch.float64, device=dev)
        dsys.forces(mK, xK, yK, zK, pd, out=dout)  # sizes its pair lists
        td = []
        for _ in range(3):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            dsys.forces(mK, xK, yK, zK, pd, out=dout)
            b.record(stream)
            b.synchronize()
            td.append(a.elapsed_time(b))
        derr = error_stats(dout.view(3, n).T[ttg].cpu().numpy(), fd, mh[tg], qh[tg])
        line["dehnen"] = {"value": n / (statistics.mean(td) * 1e-3), "unit": "forces/s",
                          "ms_per_call": statistics.mean(td), "theta": THETA, "order": args.order,
                          "rms_rel": derr["rms_rel"], "max_rel": derr["max_rel"],
                          "note": "FP64 build + dual traversal + terms + downward pass, same "
                                  "system and targets as the accuracy check"}
        dsys.close()
        del dout

        # ---- roofline of the walk (dominant kernel) ----
        p.count_stats = 1
        sysm.walk(p, out)
        sysm.sync()
        st = sysm.stats()
        p.count_stats = 0
        peak = np.zeros(3)
        _lib.check(_lib.lib().bh_probe_fma_peak(local, peak.ctypes.data_as(C.c_void_p)))
        fp32_peak = max(peak[0], peak[2])
        alg_flops = n * (mean_pp * FLOPS_PP + mean_pc * FLOPS_PC[args.order])
        exe_flops = float(st[0]) * FLOPS_PP + float(st[1]) * FLOPS_PC[args.order]
        t_w = statistics.mean(t_walk) * 1e-3
        achieved = alg_flops / t_w / 1e12
        traffic = None
        tf = os.path.join(ROOT, "profiles", "walk_dram_traffic.json")
        if os.path.exists(tf):
            with open(tf) as fh:
                traffic = json.load(fh).get("bytes_per_launch_scaled")
        line["roofline"] = {
            "bound": "fp32",
            "kernel": "pipe_walk_kernel" if p.pipeline and args.precision == 0 else "group_walk_kernel",
            "achieved": achieved,
            "peak": fp32_peak / 1e3, "unit": "TFLOP/s", "frac": achieved / (fp32_peak / 1e3),
            "traffic": traffic,
            "peak_source": "FP32 FMA throughput measured by bh_probe_fma_peak in this run, the larger "
                           "of scalar and paired (f32x2) FMA chains "
                           "(MEASURED_PEAKS.json has no FP32 figure; its HBM copy peak is not the bound)",
            "algorithmic_flops_per_launch": alg_flops, "executed_flops_per_launch": exe_flops,
            "executed_over_algorithmic": exe_flops / alg_flops,
            "reference_interactions_per_target": {"body_body": float(mean_pp),
                                                  "body_cell": float(mean_pc)},
            "executed_interactions_per_target": {"body_body": float(st[0]) / n,
                                                 "body_cell": float(st[1]) / n},
            "walk_ms": t_w * 1e3, "fp32_scalar_fma_tflops": peak[0] / 1e3,
            "fp32_paired_fma_tflops": peak[2] / 1e3, "fp64_peak_tflops": peak[1] / 1e3}

        # ---- end to end from pinned host buffers ----
        # each array pinned on its own (empty_like would not keep pin_memory)
        hm, hx, hy, hz = (torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(4))
        hout = torch.empty(3 * n, dtype=torch.float64, pin_memory=True)
        assert all(h.is_pinned() for h in (hm, hx, hy, hz, hout))
        for h, d in zip((hm, hx, hy, hz), systems[0]):
            h.copy_(d.cpu())
        L = _lib.lib()

        def e2e_call():
            _lib.check(L.bh_compute_forces_ex(hm.data_ptr(), hx.data_ptr(), hy.data_ptr(),
                                              hz.data_ptr(), n, C.byref(p), hout.data_ptr(),
                                              stream.cuda_stream))

        for _ in range(W):
            e2e_call()
        te = []
        for _ in range(K):
            flush.zero_()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e2e_call()
            b.record(stream)
            b.synchronize()
            te.append(a.elapsed_time(b))
        plain_e2e_ms = dist_max(statistics.mean(te), dev, world)
        # the host link itself on this box: the call's four input copies
        # (pinned, 32 B/body) and its result copy (24 B/body) alone
        dstage = torch.empty(4 * n, dtype=torch.float64, device=dev)

        def link(fn):
            ts = []
            for i in range(W + K):
                torch.cuda.synchronize()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
                b.synchronize()
                if i >= W:
                    ts.append(a.elapsed_time(b))
            return statistics.median(ts)

        h2d_ms = link(lambda: [dstage[k * n:(k + 1) * n].copy_(h, non_blocking=True)
                               for k, h in enumerate((hm, hx, hy, hz))])
        d2h_ms = link(lambda: hout.copy_(dstage[:3 * n], non_blocking=True))
        del dstage
        # the api3d drop-in from ordinary (pageable) numpy arrays, as the
        # reference's f2py callers pass them: a fresh Fortran-ordered result
        # array per call, as the f2py function returns
        from hierarquicos_b200 import api3d

        pm, px_, py_, pz_ = (h.numpy().copy() for h in (hm, hx, hy, hz))
        for _ in range(W):
            api3d.compute_forces(pm, px_, py_, pz_, THETA, 1.0, EPS, order=args.order, mac=p.mac,
                                 pipeline=p.pipeline)
        tp = []
        for _ in range(K):
            flush.zero_()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            api3d.compute_forces(pm, px_, py_, pz_, THETA, 1.0, EPS, order=args.order, mac=p.mac,
                                 pipeline=p.pipeline)
            b.record(stream)
            b.synchronize()
            tp.append(a.elapsed_time(b))
        pageable_ms = dist_max(statistics.mean(tp), dev, world)
        host_sys = []
        for i in range(K + W):
            mm, xx, yy, zz = systems[i]
            host_sys.append((mm.cpu().numpy(), torch.stack([xx, yy, zz], 1).cpu().numpy()))
        # the client's inputs and result buffers are pinned ahead of time, as the
        # plain call's are
        hreqs = [serving.Server.prepare(serving.Request("force", *host_sys[i])) for i in range(K)]
        hwarm = [serving.Server.prepare(serving.Request("force", *host_sys[K + i]))
                 for i in range(W)]
        served_e2e_total, hmet = serve(hreqs, hwarm)
        served_e2e_ms = dist_max(served_e2e_total, dev, world) / K
        same_host = bool(np.array_equal(hreqs[-1].forces, f_plain_last.view(3, n).T.cpu().numpy()))
        line["e2e"] = {"value": world * n / (served_e2e_ms * 1e-3), "unit": "forces/s",
                       "ms_per_step": served_e2e_ms, "h2d_bytes_per_step": 4 * 8 * n,
                       "d2h_bytes_per_step": 3 * 8 * n,
                       "api": "serving.Server with host requests (pinned in, results copied out)",
                       "host_cpus": bound_cpus,
                       "p50_ms": hmet["p50_ms"], "p99_ms": hmet["p99_ms"],
                       "equal_to_plain_bitwise": same_host,
                       "host_link": {"h2d_ms": h2d_ms, "h2d_GBps": 32 * n / (h2d_ms * 1e6),
                                     "d2h_ms": d2h_ms, "d2h_GBps": 24 * n / (d2h_ms * 1e6),
                                     "note": "the plain call's own copies, timed alone on this "
                                             "box: its floor is the device step plus both"},
                       "plain": {"value": world * n / (plain_e2e_ms * 1e-3), "ms_per_step": plain_e2e_ms,
                                 "ms_min": min(te), "ms_median": statistics.median(te),
                                 "ms_max": max(te),
                                 "api": "bh_compute_forces_ex (pinned host arrays)"},
                       "plain_pageable": {"value": world * n / (pageable_ms * 1e-3),
                                          "ms_per_step": pageable_ms,
                                          "api": "api3d.compute_forces (pageable numpy arrays in, "
                                                 "a new (N,3) Fortran array out)"}}
        del systems, host_sys, hreqs, hwarm, reqs

        # ---- 512 independent systems: batched vs plain loop ----
        line["batched"] = bench_batch(args, p, dev, local, world, rank)

        if rank == 0 and world == 1:
            line["cpu_baseline"] = cpu_baseline(n, args.order)
            # the serving and Parareal configs, each recorded beside the
            # headline; a failure there is reported, not fatal to the line
            for key, fn in (("serving_sweep", lambda: serving_sweep(args, local)),
                            ("parareal", lambda: parareal_summary(args))):
                try:
                    line[key] = fn()
                except Exception as exc:  # noqa: BLE001
                    line[key] = {"error": f"{type(exc).__name__}: {exc}"[:500]}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_split(args, p, systems, out, flush, dev, local, rank, world):
    """One system per step split over the ranks: each rank builds it whole,
    walks its range of target groups and the ranks' outputs are summed (one
    NCCL all-reduce inside the timed step); strong scaling."""
    import torch
    import torch.distributed as dist

    from hierarquicos_b200.shard import sharded_forces
    from hierarquicos_b200.system import BHSystem

    n, K, W = args.n, args.steps, args.warmup
    stream = torch.cuda.current_stream()
    sysm = BHSystem(local)
    for i in range(W):
        sharded_forces(sysm, *systems[K + i], p, out=out, rank=rank, world=world)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    times = []
    with ClockSampler(local) as clocks:
        for i in range(K):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            sharded_forces(sysm, *systems[i], p, out=out, rank=rank, world=world)
            b.record(stream)
            b.synchronize()
            times.append(a.elapsed_time(b))
    ms = dist_max(float(sum(times)), dev, world) / K
    line = {"metric": METRIC, "value": n / (ms * 1e-3), "unit": "forces/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 walk (Kahan), f64 keys/moments",
            "data": "synthetic (seeded Hernquist ICs drawn on the device)",
            "config": {"workload": f"hernquist N={n} a=1 r<=100a equal masses seeded, one system "
                                   f"split over {world} ranks", "theta": THETA, "eps": EPS,
                       "order": args.order, "parallelism": f"target groups split x{world}, "
                                                           "all-reduce of the forces",
                       "l2": "flushed (256 MiB write) before every step"},
            "clocks": clocks.summary(),
            "gpu_launches": launches_per_evaluation(n) * K}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def batch_workload(count, seed):
    """``count`` systems, N log-uniform in [1024, 65536], alternating Plummer
    (b = 1) and uniform-density unit spheres, drawn on the device."""
    import torch

    from hierarquicos_b200.initial_values import generate_initial_values_device

    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(1024), math.log(65536), count)).astype(np.int64)
    ms, xs, ys, zs = [], [], [], []
    for k, nk in enumerate(sizes):
        prof = "plummer" if k % 2 == 0 else "homogeneous"
        m, q, _ = generate_initial_values_device(int(nk), -1.0, -1.0, True, False, prof, (1.0, 1.0),
                                                 seed=seed * 100000 + k, velocities=False)
        ms.append(m)
        xs.append(q[0])
        ys.append(q[1])
        zs.append(q[2])
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    return sizes, off, (torch.cat(ms), torch.cat(xs), torch.cat(ys), torch.cat(zs))


def bench_batch(args, p, dev, local, world, rank):
    import torch

    from hierarquicos_b200 import autotune
    from hierarquicos_b200.system import BHSystem, direct_targets

    stream = torch.cuda.current_stream()
    sizes, off, (m, x, y, z) = batch_workload(args.batch_systems, 77 + rank)
    ntot = int(off[-1])
    pt, rep = autotune.tune(m, x, y, z, off, p, reps=2, use_cache=False)
    out = torch.empty(3 * ntot, dtype=torch.float64, device=dev)
    sysm = BHSystem(local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.mean(ts)

    # plain loop: one call per system, default parameters
    plain = BHSystem(local)
    views = [(m[a:b], x[a:b], y[a:b], z[a:b], out[3 * a:3 * b])
             for a, b in zip(off[:-1].tolist(), off[1:].tolist())]

    def loop():
        for mm, xx, yy, zz, oo in views:
            plain.forces(mm, xx, yy, zz, p, out=oo)

    loop()
    loop_ms = dist_max(timed(loop, 2), dev, world)
    f_loop = out.clone()

    def batched(pp):
        return lambda: sysm.forces_batch(m, x, y, z, off, pp, out=out)

    batched(p)()
    b_default_ms = dist_max(timed(batched(p), max(3, args.steps)), dev, world)
    same = bool(torch.equal(out, f_loop))
    batched(pt)()
    b_ms = dist_max(timed(batched(pt), max(3, args.steps)), dev, world)
    # CUDA graph of the tuned build + walk (status read after each replay)
    sysm.build_batch(m, x, y, z, off, pt)
    sysm.sync()
    sysm.capture(pt, out)

    def replay():
        sysm.replay()
        sysm.sync()

    replay()
    g_ms = dist_max(timed(replay, max(3, args.steps)), dev, world)
    # accuracy of the tuned batch on sampled targets of sampled systems
    rng = np.random.default_rng(5)
    errs = []
    f = out.view(-1)
    for s in rng.choice(len(sizes), 8, replace=False):
        a, b = int(off[s]), int(off[s + 1])
        nb = b - a
        tg = np.sort(rng.choice(nb, min(1024, nb), replace=False))
        tgt = torch.as_tensor(tg, device=dev)
        fd = direct_targets(m[a:b], x[a:b], y[a:b], z[a:b], tgt, p.G, p.eps).T
        fb = torch.stack([f[3 * a + tgt], f[3 * a + nb + tgt], f[3 * a + 2 * nb + tgt]], 1)
        d = torch.linalg.norm(fb - fd, dim=1) / torch.linalg.norm(fd, dim=1)
        errs.append(d.cpu().numpy())
    e = np.concatenate(errs)
    total = world * ntot
    return {"workload": f"{len(sizes)} systems, N log-uniform [1024, 65536] (total {ntot}), "
                        "Plummer b=1 / uniform sphere R=1 alternating, theta 0.5 quadrupole",
            "plain_loop": {"value": total / (loop_ms * 1e-3), "ms": loop_ms},
            "batched_default": {"value": total / (b_default_ms * 1e-3), "ms": b_default_ms,
                                "equal_to_plain_loop_bitwise": same},
            "batched_tuned": {"value": total / (b_ms * 1e-3), "ms": b_ms,
                              "params": {"group_size": pt.group_size, "group_span": pt.group_span,
                                         "leaf_cap": pt.leaf_cap}},
            "graph_replay": {"value": total / (g_ms * 1e-3), "ms": g_ms},
            "speedup_over_plain_loop": loop_ms / min(b_ms, g_ms),
            "rms_rel": float(np.sqrt(np.mean(e * e))), "max_rel": float(e.max()),
            "unit": "forces/s"}


def cpu_baseline_runs(n, order, runs, warmup, seed=1000):
    """The CPU restatement of the reference's Morton path (morton_octree.f90:
    init = keys, merge sort, node build, quadrupole upward pass; forces_par =
    the per-target barnes_hut walk of all N bodies under OpenMP), built with
    the reference's flags (-O3 -march=native -fopenmp) for this host, run in a
    child process on all usable cores with OMP_PROC_BIND=close: ``warmup`` +
    ``runs`` full force evaluations of the seeded Hernquist system.  Returns the
    summary with the per-run times."""
    from oracle.cpu_baseline import child_env, usable_cores

    with all_host_cpus():  # the CPU arm gets every core of the host
        cores = usable_cores()
        r = subprocess.run([sys.executable, "-m", "oracle.cpu_baseline", "--n", str(n), "--runs",
                            str(runs), "--warmup", str(warmup), "--order", str(order), "--seed",
                            str(seed), "--theta", str(THETA), "--eps", str(EPS)],
                           env=child_env(cores), cwd=ROOT, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"CPU baseline failed ({r.returncode}): {r.stderr[-2000:]}")
    for line in r.stdout.splitlines()[::-1]:
        if line.startswith('{"summary"'):
            return json.loads(line)["summary"]
    raise RuntimeError("CPU baseline printed no summary")


def cpu_baseline(n, order, runs=3, warmup=1):
    """``cpu_baseline`` object of the bench line: the median of ``runs`` full
    force evaluations on the host's cores (about 4-5 s each at N = 2^20 on 16
    cores), nothing extrapolated."""
    sm = cpu_baseline_runs(n, order, runs, warmup)
    return {"value": n / sm["median_total_s"], "unit": "forces/s", "cores": sm["threads"],
            "kind": "port",
            "sample": f"{runs} full force evaluations of N={n} (after {warmup} warm-up): tree build "
                      f"(serial, as morton_octree.f90 generate_nodes) + per-target walk of all N "
                      f"targets (OpenMP); median; -O3 -march=native -fopenmp build of the oracle",
            "build_s": sm["median_build_s"], "walk_s": sm["median_walk_s"],
            "per_run_s": sm["per_run_s"]}


def headline_config(args, n, mac, pipeline, K, world):
    """The bench line's ``config``: the same object for both arms."""
    return {"workload": f"hernquist N={n} a=1 r<=100a equal masses seeded, force requests",
            "n_per_request": n, "requests_per_gpu": K, "theta": THETA, "eps": EPS,
            "order": args.order,
            "walk": {0: "fp32-kahan group walk", 1: "fp64 group walk",
                     2: "fp64 per-target", 3: "fp64 dehnen dual tree"}[args.precision],
            "group_size": args.group_size, "leaf_cap": args.leaf_cap,
            "group_span": args.group_span or 2 * args.group_size, "mac": mac,
            "pipeline": pipeline, "keys": "63-bit, strict",
            "l2": "plain: flushed (256 MiB write) before every call; served: every request "
                  "touches > 500 MB of distinct data (inputs larger than L2)",
            "parallelism": f"independent systems per rank x{world}"}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's Fortran path,
    timed on this host's cores (the reference itself is Fortran and no Fortran
    compiler exists on these hosts).  Every step is one full force evaluation
    of the headline system (tree build + walk of all N targets); W warm-up
    steps, then exactly K timed ones.  Under torchrun only rank 0 runs."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.n
    sm = cpu_baseline_runs(n, args.order, args.steps, args.warmup)
    step_s = sm["mean_total_s"]
    value = n / step_s
    from hierarquicos_b200._lib import default_params

    p = default_params()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "forces/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * step_s, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Hernquist ICs)",
            "config": headline_config(args, n, args.mac if args.mac is not None else p.mac,
                                      args.pipeline if args.pipeline is not None else p.pipeline,
                                      args.steps, world),
            "reference_path": "CPU restatement of morton_octree.f90 init + forces_par "
                              "(per-target barnes_hut walk, FP64), -O3 -march=native -fopenmp",
            "cpu_baseline": {"value": value, "unit": "forces/s", "cores": sm["threads"],
                             "kind": "port",
                             "sample": f"per step: one full force evaluation of N={n} (serial tree "
                                       f"build + OpenMP walk of all N targets); the Fortran "
                                       f"reference cannot be compiled here: no Fortran compiler",
                             "build_s": sm["median_build_s"], "walk_s": sm["median_walk_s"],
                             "per_step_s": sm["per_run_s"]},
            "e2e": {"value": value, "unit": "forces/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_serving_sweep(args):
    """The serving config: a seeded request set (force or leapfrog with equal
    odds, 1-100 steps of dt = 1e-3, N log-uniform in [1024, 2^21], Plummer /
    Hernquist / uniform sphere in turn, device-resident, theta 0.5 quadrupole,
    150 GB admission budget).  First the set is submitted at once (capacity:
    requests/s and forces/s); then it arrives as a Poisson stream at fractions
    of that capacity.  Per rate: p50/p99 latency (arrival to result) and
    forces/s over the run."""
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(local)
    print(json.dumps(serving_sweep(args, local)), flush=True)


def serving_sweep(args, local):
    """The serving config's line (see run_serving_sweep) as a dict."""
    import torch

    from hierarquicos_b200 import _lib, serving
    from hierarquicos_b200.initial_values import generate_initial_values_device

    p = _lib.default_params(theta=THETA, eps=EPS, order=args.order, mac=args.mac)
    if args.pipeline is not None:
        p.pipeline = args.pipeline
    rng = np.random.default_rng(2026)
    profiles = ("plummer", "hernquist", "homogeneous")
    specs = []
    for i in range(args.sweep_requests):
        n = int(np.exp(rng.uniform(np.log(1024), np.log(1 << 21))))
        leap = bool(rng.random() < 0.5)
        steps = int(rng.integers(1, 101)) if leap else 0
        m, q, mom = generate_initial_values_device(
            n, 100.0 if profiles[i % 3] == "hernquist" else -1.0, -1.0, True, False,
            profiles[i % 3], (1.0, 1.0), seed=5000 + i, velocities=leap, device=local)
        specs.append((m, q, mom if leap else None, steps))
    torch.cuda.synchronize()

    def requests():
        return [serving.Request("leapfrog", m, q, mom, steps=st, dt=1e-3) if st
                else serving.Request("force", m, q) for m, q, mom, st in specs]

    def run(reqs, rate=None):
        with serving.Server(p, device=local, lanes=args.lanes, hbm_budget=150e9) as srv:
            warm = sorted(requests(), key=lambda r: r.n * r.evals_needed)[:3]
            srv.submit_many(warm)                         # warm-up: the 3 smallest
            for r in reqs:                                # result buffers, ahead of time
                srv.prepare(r)
            srv.drain(timeout=1200)
            if rate is None:                              # all at once
                srv.submit_many(reqs)
            else:                                         # Poisson arrivals
                t_next = time.perf_counter()
                for r, g in zip(reqs, rng.exponential(1.0 / rate, len(reqs))):
                    t_next += g
                    delay = t_next - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                    r.arrival = time.perf_counter()
                    srv.submit(r)
            srv.drain(timeout=1200)
            torch.cuda.synchronize()
            return srv.metrics(reqs)

    cap = run(requests())
    cap_rps = cap["requests"] / cap["wall_s"]
    rates = []
    for load in (0.5, 0.8, 0.95):
        met = run(requests(), rate=load * cap_rps)
        rates.append({"load": load, "rate_rps": load * cap_rps, "p50_ms": met["p50_ms"],
                      "p99_ms": met["p99_ms"], "forces_per_s": met["forces_per_s"],
                      "wall_s": met["wall_s"], "requests": met["requests"],
                      "by_kind": met["by_kind"], "paused_ticks": met["paused_ticks"]})
    sizes = [int(sp[0].numel()) for sp in specs]
    return {
        "metric": "serving: Poisson arrivals, rate swept (p50/p99 latency ms, forces/s)",
        "config": {"workload": "force and leapfrog requests (1-100 steps, dt 1e-3), N log-uniform "
                               "in [1024, 2^21], Plummer / Hernquist / uniform sphere, device "
                               "resident", "requests": args.sweep_requests, "theta": THETA,
                   "eps": EPS, "order": args.order, "mac": p.mac, "pipeline": p.pipeline,
                   "lanes": args.lanes, "hbm_budget": 150e9,
                   "median_n": int(np.median(sizes)), "max_n": int(max(sizes)),
                   "force_evaluations": int(sum(sp[3] + 1 if sp[3] else 1 for sp in specs))},
        "capacity": {"requests_per_s": cap_rps, "forces_per_s": cap["forces_per_s"],
                     "p50_ms": cap["p50_ms"], "p99_ms": cap["p99_ms"], "by_kind": cap["by_kind"]},
        "scheduling": "force requests admitted before integrations; a tick holding force "
                      "requests takes integrations up to 2^22 bodies (at most 8 ticks out in a row)",
        "rates": rates}


def run_parareal(args):
    """The batched Parareal config: Plummer N = 16,384 (equal masses, G = 1,
    b = 1, velocities by von Neumann sampling, seeded), velocity Verlet over
    64 time slices of [0, 1]; coarse propagator symplectic Euler with monopole
    theta = 0.8 forces, 2 steps per slice (dt = 1/128); fine propagator
    velocity Verlet with quadrupole theta = 0.3, 16 steps per slice
    (dt = 1/1024); softening 0.01; stop at the reference's error norm
    <= 1e-20 (parareal/parareal.f90:161,174).  All slices' fine propagators
    run as one batch per step.  Two runs: the FP32 group walk with the FP64
    correction, and the FP64 group walk with the double-double correction.
    For each: the error and the time of every iteration, the time to
    convergence, the sequential fine run over the same slices and the
    distance of the Parareal end state from it."""
    import torch

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    print(json.dumps(parareal_summary(args)), flush=True)


def parareal_summary(args):
    """The batched Parareal config's line (see run_parareal) as a dict."""
    import torch

    from hierarquicos_b200 import parareal as pr
    from hierarquicos_b200.initial_values import generate_initial_values

    n, W, tf, G, eps = args.parareal_bodies, 64, 1.0, 1.0, 0.01
    m, q, p = generate_initial_values(n, -1.0, -1.0, True, False, "plummer", (1.0, 1.0), seed=4,
                                      velocities=True)
    coarse = pr.Propagator("euler", "bh", 2, theta=0.8, order=1)
    runs = []
    for label, prec, corr in (("fp32 group walk, fp64 correction", 0, "fp64"),
                              ("fp64 group walk, double-double correction", 1, "dd")):
        fine = pr.Propagator("verlet", "bh", 16, theta=0.3, order=4, precision=prec)
        # warm-up: builds the handles' workspaces
        pr.integrate_parareal(m, q, p, tf, W, 2, 0.8, G, eps, 1e-20, 16, coarse, fine,
                              correction=corr)
        res = pr.integrate_parareal(m, q, p, tf, W, args.parareal_iters, 0.8, G, eps, 1e-20, 16,
                                    coarse, fine, correction=corr)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        qs, ps = pr.sequential_fine(m, q, p, tf, W, fine, G, eps)
        torch.cuda.synchronize()
        seq_s = time.perf_counter() - t0
        d = np.concatenate([(res.q[-1] - qs[-1]).ravel(), (res.p[-1] - ps[-1]).ravel()])

        def time_to(tol):
            acc = 0.0
            for e, t in zip(res.errors, res.iteration_seconds):
                acc += t
                if e <= tol:
                    return acc
            return None

        runs.append({"run": label, "correction": corr, "fine_precision": prec,
                     "iterations": res.iterations, "converged": res.converged,
                     "errors": res.errors, "iteration_s": res.iteration_seconds,
                     "parareal_s": res.seconds, "sequential_fine_s": seq_s,
                     "speedup_to_convergence": (seq_s / res.seconds) if res.converged else None,
                     "time_to_1e-12_s": time_to(1e-12), "time_to_1e-20_s": time_to(1e-20),
                     "end_state_vs_sequential_fine": float(np.sqrt(np.sum(d * d))) / (6 * n)})
    return {
        "metric": "batched Parareal: error per iteration (reference norm), s per iteration, "
                  "speed-up over the sequential fine run",
        "config": {"workload": f"plummer N={n} b=1 equal masses seeded, velocity Verlet, {W} slices "
                               f"over [0, {tf}]", "coarse": "symplectic Euler, monopole theta 0.8, "
                               "2 steps per slice (dt 1/128)",
                   "fine": "velocity Verlet, quadrupole theta 0.3, 16 steps per slice (dt 1/1024)",
                   "eps": eps, "G": G, "tolerance": 1e-20, "max_iterations": args.parareal_iters},
        "runs": runs}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.serving_sweep:
        run_serving_sweep(args)
    elif args.parareal:
        run_parareal(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
