"""Parity of the CUDA pipeline with the CPU oracle, layer by layer, through
the C ABI: keys and permutation (bit-exact), octree topology (exact), moments
(FP64 rounding), forces (reference walk: FP64 rounding; group walk: the
tolerances stated below) and the FP64 direct sum."""
import numpy as np
import pytest

from conftest import hernquist, plummer, xyz
from refcompact import compact_from_reference, exact_octupole

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bh():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from hierarquicos_b200 import system
    from hierarquicos_b200._lib import lib

    lib()
    return system


def build(bh, m, q, **kw):
    s = bh.BHSystem()
    x, y, z = xyz(q)
    s.build(m, x, y, z, **kw)
    s.sync()
    return s


CASES = [
    ("plummer4096", lambda: plummer(4096, seed=0)),
    ("hernquist20k", lambda: hernquist(20000, seed=3)),
    ("plummer65k", lambda: plummer(65536, seed=7)),
]


@pytest.mark.parametrize("name,gen", CASES)
@pytest.mark.parametrize("com_mode", [0, 1])
def test_keys_and_permutation_bit_exact(bh, oracle_mod, name, gen, com_mode):
    m, q = gen()
    s = build(bh, m, q, com_mode=com_mode)
    keys, perm = s.keys()
    ref = oracle_mod.MortonTree(m, *xyz(q), L=21, ssa=1.2, use_quadrupole=False, fma_mode=com_mode)
    rkeys, rperm = ref.sorted()
    assert np.array_equal(keys, rkeys)
    assert np.array_equal(perm, rperm)
    info = s.info()
    np.testing.assert_array_equal(info["depth"], 21)
    assert info["ssa"] == ref.ssa


def test_keys_with_duplicates_and_ties(bh, oracle_mod):
    # coincident bodies and bodies sharing a cell: ties must keep the
    # original order (stable sort, morton_octree.f90:537-538)
    m, q = plummer(3000, seed=11)
    q[100:140] = q[7]
    q[500:520] = q[501] + 1e-12
    s = build(bh, m, q)
    keys, perm = s.keys()
    rkeys, rperm = oracle_mod.MortonTree(m, *xyz(q), L=21, use_quadrupole=False, fma_mode=1).sorted()
    assert np.array_equal(keys, rkeys)
    assert np.array_equal(perm, rperm)


@pytest.mark.parametrize("L", [4, 9, 15])
def test_keys_shallow_depth(bh, oracle_mod, L):
    m, q = plummer(5000, seed=2)
    s = build(bh, m, q, depth=L)
    keys, perm = s.keys()
    rkeys, rperm = oracle_mod.MortonTree(m, *xyz(q), L=L, use_quadrupole=False, fma_mode=1).sorted()
    assert np.array_equal(keys, rkeys)
    assert np.array_equal(perm, rperm)


def test_auto_depth_matches_choose_depth(bh, oracle_mod):
    # L = 0: smallest depth with unique keys (choose_depth, morton_octree.f90:217-244)
    m, q = plummer(300, seed=5)
    s = build(bh, m, q, depth=0)
    ref = oracle_mod.MortonTree(m, *xyz(q), L=0, use_quadrupole=False, fma_mode=1)
    assert s.info()["depth"] == ref.L
    keys, perm = s.keys()
    rkeys, rperm = ref.sorted()
    assert np.array_equal(keys, rkeys) and np.array_equal(perm, rperm)


@pytest.mark.parametrize("name,gen", CASES[:2])
def test_topology_matches_reference(bh, oracle_mod, name, gen):
    m, q = gen()
    s = build(bh, m, q)
    ref = oracle_mod.MortonTree(m, *xyz(q), L=21, use_quadrupole=True, fma_mode=1)
    _, rmeta, rch, rnch = compact_from_reference(ref.nodes())
    d = s.nodes()
    assert d["meta"].shape[0] == rmeta.shape[0]
    np.testing.assert_array_equal(d["meta"], rmeta)
    used = np.arange(8)[None, :] < rnch[:, None]
    np.testing.assert_array_equal(np.where(used, d["child"], 0), rch)
    # parents are consistent with children
    for j in range(1, d["meta"].shape[0]):
        p = d["parent"][j]
        assert j in d["child"][p, : d["meta"][p, 3]]
    # level_begin matches the reference's level ordering
    lb = d["level_begin"]
    lev = d["meta"][:, 2]
    for v in range(len(lb) - 1):
        assert np.all(lev[lb[v]:lb[v + 1]] == v)


def test_moments_match_reference(bh, oracle_mod):
    m, q = hernquist(20000, seed=4)
    s = build(bh, m, q, order=8)
    ref = oracle_mod.MortonTree(m, *xyz(q), L=21, use_quadrupole=True, fma_mode=1)
    nodes = ref.nodes()
    ids, rmeta, _, _ = compact_from_reference(nodes)
    d = s.nodes()
    com = d["com"]
    np.testing.assert_allclose(com[:, 3], nodes["mass"][ids], rtol=1e-12, atol=0)
    np.testing.assert_allclose(com[:, :3], nodes["qcm"][ids], rtol=0, atol=1e-12 * np.abs(q).max())
    # quadrupole: scale by m * size^2 of the node
    size2 = nodes["size2"][ids]
    scale = (nodes["mass"][ids] * size2)[:, None]
    assert np.max(np.abs(d["quad"] - nodes["quad"][ids]) / scale) < 1e-10
    # octupole against the exact third moments of the node's particles
    keys, perm = s.keys()
    sm, sx = m[perm], q[perm]
    oct_ref = exact_octupole(sm, sx, d["meta"], com)
    scale3 = (nodes["mass"][ids] * size2 ** 1.5)[:, None]
    assert np.max(np.abs(d["oct"] - oct_ref) / scale3) < 1e-9


@pytest.mark.parametrize("order", [1, 4, 8])
def test_reference_walk_matches_oracle(bh, oracle_mod, order):
    # per-target FP64 walk with the reference's semantics vs the restated
    # barnes_hut (morton_octree.f90:627-766) on the same Morton tree; order 8
    # adds the octupole terms of octree_default.f90:1012-1063 on both sides
    # (the oracle sums each node's third moments directly, the device
    # translates them upward), so all three orders agree to FP64 rounding
    m, q = plummer(4096, seed=0)
    theta, eps = 0.5, 0.01
    s = build(bh, m, q, order=order)
    f = s.walk(order=order, precision=2, theta=theta, eps=eps)
    s.sync()
    f = f.view(3, -1).T.cpu().numpy()
    ref = oracle_mod.MortonTree(m, *xyz(q), L=21, use_quadrupole=order >= 4, fma_mode=1)
    fr = ref.forces_par(1.0, eps * eps, theta * theta, 8 if order == 8 else order == 4)
    rel = np.linalg.norm(f - fr, axis=1) / np.linalg.norm(fr, axis=1)
    assert rel.max() < 1e-9, rel.max()


@pytest.mark.parametrize("order", [1, 4, 8])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("group_size", [32, 64])
@pytest.mark.parametrize("mac,theta", [(0, 0.5), (1, 0.5), (1, 0.3), (1, 0.7)])
def test_group_walk_accuracy(bh, oracle_mod, order, precision, group_size, mac, theta):
    """Group walk vs the FP64 direct sum and vs the reference walk.

    mac 0 accepts a node by the group's box distance; mac 1 also accepts one
    that passes every member's own MAC and holds no member.  Tolerances: the
    group walk's RMS relative error against the direct sum is at most 1.05x the
    reference walk's + 2e-6 (FP32 rounding), and its RMS relative difference
    from the reference walk's forces is below 2x the reference walk's own
    error."""
    m, q = plummer(4096, seed=1)
    eps = 0.01
    s = build(bh, m, q, order=order, group_size=group_size)
    f = s.walk(order=order, precision=precision, theta=theta, eps=eps, group_size=group_size,
               mac=mac)
    s.sync()
    f = f.view(3, -1).T.cpu().numpy()
    fd = oracle_mod.direct_forces(m, *xyz(q), 1.0, eps * eps)
    fr = oracle_mod.MortonTree(m, *xyz(q), L=21, use_quadrupole=order >= 4, fma_mode=1).forces_par(
        1.0, eps * eps, theta * theta, 8 if order == 8 else order == 4)

    def rms(a, b):
        r = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
        return np.sqrt(np.mean(r ** 2))

    e_gpu, e_ref = rms(f, fd), rms(fr, fd)
    assert e_gpu <= 1.05 * e_ref + 2e-6, (e_gpu, e_ref)
    assert rms(f, fr) <= 2.0 * e_ref + 2e-6


def test_direct_matches_oracle(bh, oracle_mod):
    import torch

    m, q = hernquist(3000, seed=9)
    fd = oracle_mod.direct_forces(m, *xyz(q), 1.0, 1e-4)
    g = bh.direct_targets(torch.as_tensor(m, device="cuda"), *[torch.as_tensor(a, device="cuda")
                                                               for a in xyz(q)], None, 1.0, 1e-2)
    g = g.T.cpu().numpy()
    np.testing.assert_allclose(g, fd, rtol=1e-11, atol=1e-14 * np.abs(fd).max())


def test_api3d_compute_forces(bh, oracle_mod):
    from hierarquicos_b200 import api3d

    m, q = plummer(2048, seed=3)
    x, y, z = xyz(q)
    f = api3d.compute_forces(m, x, y, z, 0.5, 1.0, 0.01, True)
    assert f.shape == (2048, 3) and f.flags.f_contiguous
    fd = api3d.compute_forces_direct(m, x, y, z, 1.0, 0.01)
    rel = np.linalg.norm(f - fd, axis=1) / np.linalg.norm(fd, axis=1)
    assert np.sqrt(np.mean(rel ** 2)) < 2e-3
    fo = oracle_mod.direct_forces(m, x, y, z, 1.0, 1e-4)
    np.testing.assert_allclose(fd, fo, rtol=1e-11, atol=1e-14 * np.abs(fo).max())
    # accelerations
    a = api3d.compute_forces(m, x, y, z, 0.5, 1.0, 0.01, True, accelerations=True)
    np.testing.assert_allclose(a * m[:, None], f, rtol=1e-12, atol=1e-15 * np.abs(f).max())


@pytest.mark.parametrize("strict", [1, 2])
def test_strict_keys_repair_ambiguous_body(bh, oracle_mod, strict):
    """tests/golden/ambiguous_keys.npz holds an input where the device's
    parallel centre of mass and the reference's sequential one put one body in
    different cells (made by tests/golden/make_ambiguous.py).  With strict keys
    the device detects the body inside the rounding margin, computes the
    sequential sum and rebuilds: keys, permutation and forces then match the
    reference's.  Without the check the key would differ."""
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ambiguous_keys.npz"))
    m, x, y, z = g["m"], g["x"], g["y"], g["z"]
    ref = oracle_mod.MortonTree(m, x, y, z, L=21, use_quadrupole=True, fma_mode=0)
    rkeys, rperm = ref.sorted()
    s = bh.BHSystem()
    f = s.forces(m, x, y, z, com_mode=0, strict_keys=strict, precision=2, theta=0.5, eps=0.01)
    keys, perm = s.keys()
    assert np.array_equal(keys, rkeys) and np.array_equal(perm, rperm)
    fr = ref.forces_par(1.0, 1e-4, 0.25, True)
    f = f.view(3, -1).T.cpu().numpy()
    rel = np.linalg.norm(f - fr, axis=1) / np.linalg.norm(fr, axis=1)
    assert rel.max() < 1e-9
    s2 = bh.BHSystem()
    s2.build(m, x, y, z, com_mode=0, strict_keys=0)
    s2.sync()
    k2, _ = s2.keys()
    assert not np.array_equal(k2, rkeys), "the fast path alone should miss this body"
