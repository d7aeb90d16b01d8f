"""Bit-exact parity at the sizes the headline workloads run at: the Hernquist
sphere of 2^20 bodies (a = 1, truncated at 100 a, equal masses) and a 2^21-body
system inside a batch of three (the largest request of the serving mix).

Morton keys, the stable sort permutation and the compact octree topology of
the device must equal the oracle's restatement of morton_octree.f90 (keys
:184-213 and :359-395, argsort :501-560, generate_nodes :420-499) exactly, for
both roundings of the reference's sequential centre of mass (:364-370).

Seed 45 of the 2^20 Hernquist draw puts one body within the rounding margin
of a cell edge (0.08 of the margin), so the strict-key path computes the
reference's sequential centre of mass on the device for that system; the
handle's counters show that it ran, and the keys still equal the oracle's."""
import numpy as np
import pytest

from conftest import hernquist, plummer, xyz
from refcompact import compact_from_reference

pytestmark = pytest.mark.gpu

N20 = 1 << 20
N21 = 1 << 21
AMBIGUOUS_SEED = 45  # a body at 0.08 of the key margin (found by scanning seeds)


@pytest.fixture(scope="module")
def bh():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from hierarquicos_b200 import system
    from hierarquicos_b200._lib import lib

    lib()
    return system


@pytest.fixture(scope="module")
def c2():
    return hernquist(N20, seed=0)


def oracle_sorted(oracle_mod, m, q, com_mode):
    keys, _, _, _ = oracle_mod.morton_keys(m, *xyz(q), L=21, ssa=1.2, fma_mode=com_mode)
    perm = oracle_mod.argsort(keys)
    return keys[perm], perm


def check_topology(d, rmeta, rch, rnch):
    assert d["meta"].shape[0] == rmeta.shape[0]
    np.testing.assert_array_equal(d["meta"], rmeta)
    used = np.arange(8)[None, :] < rnch[:, None]
    np.testing.assert_array_equal(np.where(used, d["child"], 0), rch)


@pytest.mark.parametrize("com_mode", [0, 1])
def test_keys_and_permutation_at_2_20(bh, oracle_mod, c2, com_mode):
    m, q = c2
    s = bh.BHSystem()
    s.build(m, *xyz(q), com_mode=com_mode)
    s.sync()
    keys, perm = s.keys()
    rkeys, rperm = oracle_sorted(oracle_mod, m, q, com_mode)
    assert np.array_equal(keys, rkeys)
    assert np.array_equal(perm, rperm)
    s.close()


def test_topology_at_2_20(bh, oracle_mod, c2):
    m, q = c2
    s = bh.BHSystem()
    s.build(m, *xyz(q), com_mode=1)
    s.sync()
    ref = oracle_mod.MortonTree(m, *xyz(q), L=21, use_quadrupole=False, fma_mode=1)
    _, rmeta, rch, rnch = compact_from_reference(ref.nodes())
    del ref
    d = s.nodes()
    check_topology(d, rmeta, rch, rnch)
    # the reference's level order: level_begin brackets each level
    lb, lev = d["level_begin"], d["meta"][:, 2]
    for v in range(len(lb) - 1):
        assert np.all(lev[lb[v]:lb[v + 1]] == v)
    s.close()


@pytest.mark.parametrize("com_mode", [0, 1])
def test_strict_key_check_on_a_real_ambiguous_system(bh, oracle_mod, com_mode):
    m, q = hernquist(N20, seed=AMBIGUOUS_SEED)
    s = bh.BHSystem()
    s.build(m, *xyz(q), com_mode=com_mode, strict_keys=1)
    s.sync()
    checks, rebuilds = s.key_checks()
    assert checks == 1, "the margin check should have fired for this system"
    assert rebuilds in (0, 1)
    keys, perm = s.keys()
    rkeys, rperm = oracle_sorted(oracle_mod, m, q, com_mode)
    assert np.array_equal(keys, rkeys)
    assert np.array_equal(perm, rperm)
    # a system without ambiguous bodies never takes the slow path
    m4, q4 = plummer(4096, seed=0)
    s.build(m4, *xyz(q4), strict_keys=1)
    s.sync()
    assert s.key_checks()[0] == 1
    s.close()


def test_2_21_system_inside_a_batch(bh, oracle_mod):
    """The 2^21-body Hernquist system between a Plummer and a uniform sphere:
    its keys, permutation and compact octree equal the oracle's for the system
    alone (its nodes are picked out of the batch's and renumbered)."""
    from hierarquicos_b200.system import offsets_of

    m1, q1 = hernquist(N21, seed=11)
    m0, q0 = plummer(70000, seed=12)
    m2, q2 = plummer(30000, seed=13, b=0.3)
    ms, qs = [m0, m1, m2], [q0 - 50.0, q1, q2 + 50.0]
    sizes = [a.size for a in ms]
    off = offsets_of(sizes)
    m, q = np.concatenate(ms), np.concatenate(qs)
    s = bh.BHSystem()
    s.build_batch(m, *xyz(q), off, com_mode=1)
    s.sync()
    keys, perm = s.keys()
    a, b = off[1], off[2]
    rkeys, rperm = oracle_sorted(oracle_mod, m1, q1, 1)
    assert np.array_equal(keys[a:b], rkeys)
    assert np.array_equal(perm[a:b] - a, rperm)
    d = s.nodes()
    meta, child = d["meta"], d["child"]
    sel = np.nonzero((meta[:, 0] >= a) & (meta[:, 0] < b))[0]
    local = np.full(meta.shape[0], -1, np.int64)
    local[sel] = np.arange(sel.size)
    lm = meta[sel].astype(np.int64)
    lm[:, 0] -= a
    used = np.arange(8)[None, :] < lm[:, 3:4]
    lc = np.where(used, child[sel].astype(np.int64), 0)  # entries past nchild are unset
    lc = np.where(lc >= 0, local[np.maximum(lc, 0)], ~(~lc - a))
    lc = np.where(used, lc, 0)
    ref = oracle_mod.MortonTree(m1, *xyz(q1), L=21, use_quadrupole=False, fma_mode=1)
    _, rmeta, rch, rnch = compact_from_reference(ref.nodes())
    del ref
    assert lm.shape[0] == rmeta.shape[0]
    np.testing.assert_array_equal(lm, rmeta)
    np.testing.assert_array_equal(lc, rch)
    s.close()
