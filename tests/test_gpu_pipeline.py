"""The warp-specialised FP32 walk (pipeline = 1: producer warps walk the tree
and stage batches into a shared-memory ring, consumer warps evaluate them)
gives the same forces, bit for bit, and the same interaction counts as the
one-warp walk (pipeline = 0): the batches, their order and the arithmetic are
the same, only the warps that do the work differ."""
import numpy as np
import pytest

from conftest import hernquist, plummer, xyz

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bh():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from hierarquicos_b200 import system
    from hierarquicos_b200._lib import lib

    lib()
    return system


def clustered(n, seed):
    # a Hernquist sphere with a block of coincident bodies and a tight clump
    m, q = hernquist(n, seed=seed)
    q[10:60] = q[5]
    q[200:1200] = q[200] + 1e-6 * np.random.default_rng(seed).standard_normal((1000, 3))
    return m, q


CASES = [
    ("plummer20k", lambda: plummer(20000, seed=4)),
    ("hernquist50k", lambda: hernquist(50000, seed=5)),
    ("clustered30k", lambda: clustered(30000, seed=6)),
]


def both(s, **kw):
    import torch

    f0 = s.walk(pipeline=0, count_stats=1, **kw)
    s.sync()
    st0 = s.stats().copy()
    f1 = s.walk(pipeline=1, count_stats=1, **kw)
    s.sync()
    st1 = s.stats().copy()
    torch.cuda.synchronize()
    return f0, f1, st0, st1


@pytest.mark.parametrize("name,gen", CASES)
@pytest.mark.parametrize("order", [1, 4, 8])
@pytest.mark.parametrize("group_size", [32, 64])
def test_pipeline_equals_one_warp_walk(bh, name, gen, order, group_size):
    import torch

    m, q = gen()
    s = bh.BHSystem()
    s.build(m, *xyz(q), order=order, group_size=group_size)
    for eps, mac, theta in [(0.0, 0, 0.5), (0.01, 1, 0.6), (0.01, 0, 0.0)]:
        f0, f1, st0, st1 = both(s, order=order, group_size=group_size, eps=eps, mac=mac,
                                theta=theta)
        assert torch.equal(f0, f1), (eps, mac, theta)
        np.testing.assert_array_equal(st0[:2], st1[:2])
        assert torch.isfinite(f1).all()


@pytest.mark.parametrize("out_kind", [0, 1])
def test_pipeline_accelerations_and_batches(bh, out_kind):
    import torch

    sizes = [1, 2, 33, 64, 65, 5000, 17]
    parts = [plummer(k, seed=10 + i) for i, k in enumerate(sizes)]
    m = np.concatenate([p[0] for p in parts])
    q = np.concatenate([p[1] for p in parts])
    off = np.concatenate([[0], np.cumsum(sizes)])
    s = bh.BHSystem()
    kw = dict(order=4, group_size=64, eps=0.02, out_kind=out_kind)
    f0 = s.forces_batch(m, *xyz(q), off, pipeline=0, **kw)
    s.sync()
    f0 = f0.clone()
    f1 = s.forces_batch(m, *xyz(q), off, pipeline=1, **kw)
    s.sync()
    assert torch.equal(f0, f1)


def test_pipeline_group_ranges(bh):
    """A walk over a range of target groups writes the same entries as the
    one-warp walk over that range and leaves the rest untouched."""
    import torch

    m, q = hernquist(40000, seed=8)
    s = bh.BHSystem()
    kw = dict(order=4, group_size=64, eps=0.01)
    s.build(m, *xyz(q), **kw)
    ng = s.info()["n_groups"]
    g0, g1 = ng // 3, (2 * ng) // 3
    outs = []
    for pipe in (0, 1):
        out = torch.full((3 * m.size,), 7.0, dtype=torch.float64, device="cuda")
        s.walk(out=out, groups=(g0, g1), pipeline=pipe, **kw)
        s.sync()
        outs.append(out)
    assert torch.equal(outs[0], outs[1])
    assert (outs[1] == 7.0).any() and (outs[1] != 7.0).any()


def test_pipeline_fp64_ignores_the_switch(bh):
    """pipeline applies to the FP32 walk; the FP64 walk is the same either way."""
    import torch

    m, q = plummer(8000, seed=9)
    s = bh.BHSystem()
    s.build(m, *xyz(q), order=4)
    f0, f1, _, _ = both(s, order=4, precision=1, eps=0.01)
    assert torch.equal(f0, f1)


def test_pipeline_large(bh):
    import torch

    m, q = hernquist(1 << 20, seed=12)
    s = bh.BHSystem()
    s.build(m, *xyz(q), order=4, group_size=64)
    f0, f1, st0, st1 = both(s, order=4, group_size=64, eps=0.01, theta=0.5)
    assert torch.equal(f0, f1)
    np.testing.assert_array_equal(st0[:2], st1[:2])


def test_bounded_wait_gives_up_and_releases_the_block(bh):
    """The walk's mbarrier wait on a barrier that nothing arrives at gives up
    after its limit, raises the block's abort flag, and that flag releases the
    other warp of the block long before its own (about 2 s) limit; afterwards
    the context still runs the force pipeline."""
    import ctypes as C

    import torch
    from hierarquicos_b200._lib import check, lib

    limit = 2_000_000
    out = (C.c_longlong * 5)()
    check(lib().bh_probe_bounded_wait(torch.cuda.current_device(), limit, out))
    gave_up, seen, released, waited, flag = list(out)
    assert seen == 1 and gave_up == 0 and released == 0 and flag == 1
    assert 0 < waited < 100 * limit
    m, q = plummer(3000, seed=2)
    f = bh.BHSystem().forces(m, *xyz(q), eps=0.01)
    torch.cuda.synchronize()
    assert torch.isfinite(f).all()
