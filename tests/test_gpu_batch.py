"""Batches of independent systems: every system of a batch must give exactly
(bit for bit) what a build of that system alone gives -- keys, permutation,
centre of mass, root size and forces -- whatever the other systems are.  The
single-system path is itself checked against the oracle in the parity tests;
here one system of the batch is also checked against the oracle directly."""
import os

import numpy as np
import pytest

from conftest import plummer, xyz

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bh():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from hierarquicos_b200 import system
    from hierarquicos_b200._lib import lib

    lib()
    return system


def uniform_sphere(n, seed):
    from hierarquicos_b200.initial_values import generate_initial_values

    m, q, _ = generate_initial_values(n, -1.0, -1.0, True, False, "homogeneous", (1.0, 1.0),
                                      seed=seed, velocities=False)
    return m, q


def mixed_batch(sizes, seed=0):
    """Plummer and uniform-sphere systems of the given sizes, concatenated,
    with shifted centres so that no two systems share a box."""
    ms, qs = [], []
    for k, n in enumerate(sizes):
        if n <= 2:
            rng = np.random.default_rng(seed + k)
            m, q = np.full(n, 1.0 / n), rng.standard_normal((n, 3))
        elif k % 2 == 0:
            m, q = plummer(n, seed=seed + k)
        else:
            m, q = uniform_sphere(n, seed=seed + k)
        ms.append(m)
        qs.append(q + 10.0 * k)
    return ms, qs


def concat(ms, qs):
    m = np.concatenate(ms)
    q = np.concatenate(qs)
    return m, q


SIZES = [1, 2, 3, 17, 64, 65, 100, 1000, 4096, 5000, 8193, 20000]


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("order", [1, 4, 8])
def test_batch_equals_single_systems(bh, precision, order):
    from hierarquicos_b200.system import offsets_of

    ms, qs = mixed_batch(SIZES, seed=order)
    m, q = concat(ms, qs)
    off = offsets_of(SIZES)
    kw = dict(theta=0.5, eps=0.01, order=order, precision=precision)
    s = bh.BHSystem()
    f = s.forces_batch(m, *xyz(q), off, **kw).cpu().numpy()
    keys, perm = s.keys()
    info = s.batch_info()
    single = bh.BHSystem()
    for k, n in enumerate(SIZES):
        a, b = off[k], off[k + 1]
        fs = single.forces(ms[k], *xyz(qs[k]), **kw).cpu().numpy()
        sk, sp = single.keys()
        assert np.array_equal(keys[a:b], sk), f"keys of system {k}"
        assert np.array_equal(perm[a:b] - a, sp), f"permutation of system {k}"
        assert np.array_equal(f[3 * a:3 * b], fs), f"forces of system {k} (n={n})"
        si = single.info()
        if n >= 2:
            assert info["ssa"][k] == si["ssa"]
            assert np.array_equal(info["com"][k], si["com"])
        else:
            assert info["roots"][k] == -1
            assert np.all(f[3 * a:3 * b] == 0.0)


def test_batch_system_matches_oracle(bh, oracle_mod):
    """One system inside a batch, against the oracle's Morton tree."""
    from hierarquicos_b200.system import offsets_of

    sizes = [300, 4096, 777]
    ms, qs = mixed_batch(sizes, seed=5)
    m, q = concat(ms, qs)
    off = offsets_of(sizes)
    s = bh.BHSystem()
    f = s.forces_batch(m, *xyz(q), off, theta=0.5, eps=0.01, order=4, precision=2,
                       com_mode=0).cpu().numpy()
    keys, perm = s.keys()
    k = 1
    a, b = off[k], off[k + 1]
    ref = oracle_mod.MortonTree(ms[k], *xyz(qs[k]), L=21, use_quadrupole=True, fma_mode=0)
    rkeys, rperm = ref.sorted()
    assert np.array_equal(keys[a:b], rkeys)
    assert np.array_equal(perm[a:b] - a, rperm)
    fr = ref.forces_par(1.0, 1e-4, 0.25, True)
    fb = f[3 * a:3 * b].reshape(3, -1).T
    rel = np.linalg.norm(fb - fr, axis=1) / np.linalg.norm(fr, axis=1)
    assert rel.max() < 1e-9


def test_batch_strict_key_repair(bh, oracle_mod):
    """The body of tests/golden/ambiguous_keys.npz needs the sequential
    centre of mass; inside a batch only its system is re-keyed and rebuilt,
    and every system still equals its lone build."""
    from hierarquicos_b200.system import offsets_of

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ambiguous_keys.npz"))
    amb_m = g["m"]
    amb_q = np.stack([g["x"], g["y"], g["z"]], axis=1)
    ms, qs = mixed_batch([500, 3000], seed=9)
    ms = [ms[0], amb_m, ms[1]]
    qs = [qs[0], amb_q, qs[1]]
    sizes = [len(a) for a in ms]
    m, q = concat(ms, qs)
    off = offsets_of(sizes)
    kw = dict(theta=0.5, eps=0.01, order=4, precision=0, com_mode=0, strict_keys=1)
    s = bh.BHSystem()
    f = s.forces_batch(m, *xyz(q), off, **kw).cpu().numpy()
    keys, perm = s.keys()
    ref = oracle_mod.MortonTree(amb_m, *xyz(amb_q), L=21, use_quadrupole=True, fma_mode=0)
    rkeys, rperm = ref.sorted()
    a, b = off[1], off[2]
    assert np.array_equal(keys[a:b], rkeys) and np.array_equal(perm[a:b] - a, rperm)
    single = bh.BHSystem()
    for k in range(3):
        a, b = off[k], off[k + 1]
        fs = single.forces(ms[k], *xyz(qs[k]), **kw).cpu().numpy()
        assert np.array_equal(f[3 * a:3 * b], fs)


def test_batch_order_independence(bh):
    """A system's result does not depend on its neighbours or its place."""
    from hierarquicos_b200.system import offsets_of

    sizes = [2000, 50, 7000, 333]
    ms, qs = mixed_batch(sizes, seed=21)
    kw = dict(theta=0.6, eps=0.0, order=4)
    s = bh.BHSystem()
    m, q = concat(ms, qs)
    f1 = s.forces_batch(m, *xyz(q), offsets_of(sizes), **kw).cpu().numpy()
    order = [2, 0, 3, 1]
    m2, q2 = concat([ms[i] for i in order], [qs[i] for i in order])
    sizes2 = [sizes[i] for i in order]
    f2 = s.forces_batch(m2, *xyz(q2), offsets_of(sizes2), **kw).cpu().numpy()
    off1, off2 = offsets_of(sizes), offsets_of(sizes2)
    for j, i in enumerate(order):
        assert np.array_equal(f1[3 * off1[i]:3 * off1[i + 1]], f2[3 * off2[j]:3 * off2[j + 1]])


def test_graph_replay_matches_forces(bh):
    import torch

    from hierarquicos_b200._lib import default_params
    from hierarquicos_b200.system import offsets_of

    sizes = [4096, 1500, 9000]
    ms, qs = mixed_batch(sizes, seed=2)
    m, q = concat(ms, qs)
    off = offsets_of(sizes)
    p = default_params(theta=0.5, eps=0.01, order=4)
    s = bh.BHSystem()
    ref = s.forces_batch(m, *xyz(q), off, p).clone()
    dev = torch.device("cuda")
    inputs = [torch.as_tensor(np.ascontiguousarray(a), device=dev) for a in (m, *xyz(q))]
    s.build_batch(*inputs, off, p)
    s.sync()
    out = torch.zeros(3 * m.size, dtype=torch.float64, device=dev)
    s.capture(p, out)
    for _ in range(2):
        out.zero_()
        s.replay()
        s.sync()
        assert torch.equal(out, ref)
    # new positions in the same arrays: the replay picks them up
    m2, q2 = concat(*mixed_batch(sizes, seed=3))
    ref2 = s.forces_batch(m2, *xyz(q2), off, p).clone()
    for t, a in zip(inputs, (m2, *xyz(q2))):
        t.copy_(torch.as_tensor(np.ascontiguousarray(a), device=dev))
    s.build_batch(*inputs, off, p)  # same layout: the graph is kept
    s.sync()
    s.capture(p, out)
    s.replay()
    s.sync()
    assert torch.equal(out, ref2)


def test_batch_rejects_bad_layouts(bh):
    from hierarquicos_b200._lib import BH_ERR_INVALID, BHError

    m, q = plummer(100, seed=1)
    s = bh.BHSystem()
    for off in ([0, 50, 50, 100], [0, 60, 40, 100], [1, 100]):
        with pytest.raises((BHError, ValueError)) as e:
            s.forces_batch(m, *xyz(q), np.array(off), theta=0.5)
        if isinstance(e.value, BHError):
            assert e.value.code == BH_ERR_INVALID
    with pytest.raises(BHError) as e:
        s.forces_batch(m, *xyz(q), np.array([0, 50, 100]), depth=0)
    assert e.value.code == BH_ERR_INVALID
    # a non-finite body fails its batch with BH_ERR_NONFINITE
    q2 = q.copy()
    q2[70, 1] = np.nan
    with pytest.raises(BHError) as e:
        s.forces_batch(m, *xyz(q2), np.array([0, 50, 100]))
    from hierarquicos_b200._lib import BH_ERR_NONFINITE

    assert e.value.code == BH_ERR_NONFINITE
    # and the handle still works afterwards
    f = s.forces_batch(m, *xyz(q), np.array([0, 50, 100]), theta=0.5)
    assert np.isfinite(f.cpu().numpy()).all()


def test_capture_as_the_first_walk_of_a_process():
    """A process whose first walk is recorded into a CUDA graph: the walk's
    one-time launch set-up happens during the capture, and the replay still
    equals a plain evaluation bit for bit (run in a fresh interpreter)."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = f"""
import sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {os.path.join(root, 'tests')!r})
import numpy as np, torch
from conftest import plummer, xyz
from hierarquicos_b200.system import BHSystem
from hierarquicos_b200._lib import default_params
for order in (4, 8):
    m, q = plummer(5000, seed=4)
    p = default_params(theta=0.5, eps=0.01, order=order)
    dev = torch.device('cuda')
    ins = [torch.as_tensor(np.ascontiguousarray(a), device=dev) for a in (m, *xyz(q))]
    s = BHSystem()
    s.build_batch(*ins, np.array([0, 5000]), p)
    s.sync()
    out = torch.zeros(15000, dtype=torch.float64, device=dev)
    s.capture(p, out)
    s.replay()
    s.sync()
    ref = BHSystem().forces(*ins, p)
    torch.cuda.synchronize()
    assert torch.equal(out, ref), order
print('ok')
"""
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
