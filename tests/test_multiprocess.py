"""Multi-process logic of the benchmark on the CPU (gloo, world size 2): the
max-over-ranks timing reduction, and the reference arm under torchrun (rank 0
alone runs and prints one line; the other ranks exit without work)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench

    got = bench.dist_max(10.0 + rank, torch.device("cpu"), world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def _free_port():
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_timings_reduce_to_the_max_over_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 11.0, 1: 11.0}


def test_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--bodies", "4096"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0


@pytest.mark.parametrize("rank", ["1"])
def test_reference_arm_other_ranks_exit_without_work(rank):
    env = dict(os.environ, RANK=rank, WORLD_SIZE="2", LOCAL_RANK=rank)
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--bodies", "4096"], cwd=ROOT,
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_group_ranges_partition_the_groups():
    sys.path.insert(0, ROOT)
    from hierarquicos_b200.shard import group_range

    for n_groups in (0, 1, 5, 16384, 16385):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                g0, g1 = group_range(n_groups, r, world)
                assert 0 <= g0 <= g1 <= n_groups
                assert g1 - g0 in (n_groups // world, n_groups // world + 1)
                seen.extend(range(g0, g1))
            assert seen == list(range(n_groups))


def _shard_worker(rank, world, port, q):
    """Each rank fills only its groups' bodies (zeros elsewhere); the sum over
    the ranks must be every body's value exactly."""
    import numpy as np
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    from hierarquicos_b200.shard import combine, group_range

    rng = np.random.default_rng(7)
    n, n_groups = 1000, 37
    g_first = np.sort(rng.choice(np.arange(1, n), n_groups - 1, replace=False))
    g_first = np.concatenate([[0], g_first, [n]])
    full = rng.standard_normal(3 * n)  # the same "forces" on every rank
    perm = rng.permutation(n)          # sorted position -> original index
    g0, g1 = group_range(n_groups, rank, world)
    out = torch.zeros(3 * n, dtype=torch.float64)
    for i in range(g_first[g0], g_first[g1]):
        o = perm[i]
        for k in range(3):
            out[k * n + o] = full[k * n + o]
    combine(out)
    ok = bool(np.array_equal(out.numpy(), full))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ok))


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_outputs_combine_to_the_full_result(world):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(res.values()), res


def test_rebalance_moves_cut_points_toward_equal_cost():
    import numpy as np

    sys.path.insert(0, ROOT)
    from hierarquicos_b200.shard import rebalance

    rng = np.random.default_rng(3)
    n_groups, world = 16384, 4
    # group cost rises toward the middle (a centrally concentrated system)
    cost = 1.0 + 5.0 * np.exp(-((np.arange(n_groups) - n_groups / 2) / 1500.0) ** 2)
    cost *= rng.uniform(0.8, 1.2, n_groups)
    bounds = [0, 4096, 8192, 12288, 16384]

    def times(b):
        return [cost[b[r]:b[r + 1]].sum() for r in range(world)]

    imb0 = max(times(bounds)) / np.mean(times(bounds))
    for _ in range(6):
        bounds = rebalance(bounds, times(bounds))
        assert bounds[0] == 0 and bounds[-1] == n_groups
        assert all(bounds[i] <= bounds[i + 1] for i in range(world))
    imb = max(times(bounds)) / np.mean(times(bounds))
    assert imb0 > 1.3 and imb < 1.03, (imb0, imb)
    # equal times keep the cut points
    assert rebalance([0, 10, 20, 30], [1.0, 1.0, 1.0]) == [0, 10, 20, 30]
    # empty ranges are allowed and stay ordered
    b = rebalance([0, 0, 50, 100], [0.0, 3.0, 1.0])
    assert b[0] == 0 and b[-1] == 100 and b == sorted(b)


def _balance_worker(rank, world, port, q):
    """Every rank reports its own time; all ranks must agree on the new cut
    points."""
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    from hierarquicos_b200.shard import Balancer

    bal = Balancer(world)
    bal.range(1000, rank)
    got = bal.update(10.0 * (rank + 1))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, (got, bal.bounds)))


def test_balancer_agrees_on_all_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_balance_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1]
    times, bounds = res[0]
    assert times == [10.0, 20.0]
    assert bounds[0] == 0 and bounds[-1] == 1000 and bounds[1] > 500  # rank 1 was slower
