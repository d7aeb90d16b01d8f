"""Dehnen's dual-tree method on the device (precision BH_PREC_DEHNEN, the
reference's methods 20/21/22) against the oracle's restatement of
octree_default.f90:1095-1712.

The oracle runs the method over its Morton tree, whose topology the device
build reproduces, and over the reference's insertion tree, which shares the
root cube; the device forces must agree with both to FP64 rounding of the
expansion coefficients (the terms are summed in another order, moments are
translated instead of summed directly).  Tolerance, written in each test:
RMS relative difference per body <= 1e-10, largest <= 1e-7.  Every system of a
batch gets, bit for bit, what it gets alone."""
import numpy as np
import pytest

from conftest import hernquist, plummer, xyz

pytestmark = pytest.mark.gpu

RMS_TOL, MAX_TOL = 1e-10, 1e-7


@pytest.fixture(scope="module")
def bh():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from hierarquicos_b200 import system
    from hierarquicos_b200._lib import lib

    lib()
    return system


def dehnen_gpu(bh, m, q, theta, eps, order, **kw):
    s = bh.BHSystem()
    f = s.forces(m, *xyz(q), theta=theta, eps=eps, order=order, precision=3, **kw)
    return f.view(3, -1).T.cpu().numpy()


def rel_diff(a, b):
    r = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
    return float(np.sqrt(np.mean(r ** 2))), float(r.max())


CASES = [("plummer4096", lambda: plummer(4096, seed=0)),
         ("hernquist20k", lambda: hernquist(20000, seed=3))]


@pytest.mark.parametrize("name,gen", CASES)
@pytest.mark.parametrize("order", [1, 4, 8])
@pytest.mark.parametrize("theta", [0.3, 0.6, 1.0])
def test_dehnen_matches_oracle(bh, oracle_mod, name, gen, order, theta):
    m, q = gen()
    eps = 0.01
    f = dehnen_gpu(bh, m, q, theta, eps, order)
    fo = oracle_mod.MortonTree(m, *xyz(q), L=21).dehnen(1.0, eps * eps, theta * theta, order)
    rms, mx = rel_diff(f, fo)
    assert rms <= RMS_TOL and mx <= MAX_TOL, (rms, mx)


@pytest.mark.parametrize("method", [20, 21, 22])
def test_octree_mirror_matches_reference_tree(bh, oracle_mod, method):
    """OctreeType with methods 20-22 (pre_init + init + dehnen_eval) against the
    oracle's insertion tree, the reference's own."""
    m, q = plummer(3000, seed=4)
    x, y, z = xyz(q)
    t = bh.Octree().pre_init(m, method).init(x, y, z)
    f = t.dehnen_eval(0.5 ** 2, 1e-4, 1.0).T
    fo = oracle_mod.Octree(m, method).init(x, y, z).forces(0.5 ** 2, 1.0, 1e-4)
    rms, mx = rel_diff(f, fo)
    assert rms <= RMS_TOL and mx <= MAX_TOL, (rms, mx)


def test_dehnen_error_against_direct_sum(bh, oracle_mod):
    """Error of the device result against the FP64 direct sum equals the
    oracle's (the same approximation), and falls with theta."""
    m, q = hernquist(8000, seed=6)
    x, y, z = xyz(q)
    fd = oracle_mod.direct_forces(m, x, y, z, 1.0, 1e-4)
    t = oracle_mod.MortonTree(m, x, y, z, L=21)
    prev = None
    for th in (0.9, 0.6, 0.3):
        f = dehnen_gpu(bh, m, q, th, 0.01, 4)
        e = np.linalg.norm(f - fd) / np.linalg.norm(fd)
        fo = t.dehnen(1.0, 1e-4, th * th, 4)
        eo = np.linalg.norm(fo - fd) / np.linalg.norm(fd)
        assert abs(e / eo - 1.0) < 1e-6, (th, e, eo)
        if prev is not None:
            assert e < prev
        prev = e


def test_dehnen_batch_equals_single_systems(bh):
    from hierarquicos_b200.system import offsets_of

    sizes = [1, 2, 3, 64, 1000, 4096, 777]
    ms, qs = [], []
    for k, n in enumerate(sizes):
        if n <= 2:
            rng = np.random.default_rng(k)
            m, q = np.full(n, 1.0 / n), rng.standard_normal((n, 3))
        else:
            m, q = plummer(n, seed=30 + k)
        ms.append(m)
        qs.append(q + 10.0 * k)
    m, q = np.concatenate(ms), np.concatenate(qs)
    off = offsets_of(sizes)
    kw = dict(theta=0.6, eps=0.01, order=4, precision=3)
    s = bh.BHSystem()
    f = s.forces_batch(m, *xyz(q), off, **kw).cpu().numpy()
    single = bh.BHSystem()
    for k, n in enumerate(sizes):
        a, b = off[k], off[k + 1]
        fs = single.forces(ms[k], *xyz(qs[k]), **kw).cpu().numpy()
        assert np.array_equal(f[3 * a:3 * b], fs), f"system {k} (n={n})"
    assert np.all(f[0:3] == 0.0)  # a lone body feels nothing
    # the traversal's lists have one order whatever the schedule: run to run
    # the bits do not change
    f2 = s.forces_batch(m, *xyz(q), off, **kw).cpu().numpy()
    assert np.array_equal(f, f2)


def test_dehnen_two_bodies_is_exact(bh):
    m = np.array([0.3, 0.7])
    q = np.array([[0.0, 0.0, 0.0], [1.0, 2.0, -0.5]])
    f = dehnen_gpu(bh, m, q, 0.5, 0.0, 4)
    d = q[1] - q[0]
    fe = 0.3 * 0.7 * d / np.linalg.norm(d) ** 3
    np.testing.assert_allclose(f[0], fe, rtol=1e-14)
    np.testing.assert_allclose(f[1], -fe, rtol=1e-14)


def test_dehnen_coincident_bodies(bh, oracle_mod):
    m, q = plummer(2000, seed=8)
    q = q.copy()
    q[100:110] = q[100]     # coincident bodies (softened): one node of identical keys
    f = dehnen_gpu(bh, m, q, 0.5, 0.01, 4)
    assert np.all(np.isfinite(f))
    fo = oracle_mod.MortonTree(m, *xyz(q), L=21).dehnen(1.0, 1e-4, 0.25, 4)
    rms, mx = rel_diff(f, fo)
    assert rms <= RMS_TOL and mx <= MAX_TOL, (rms, mx)


def test_dehnen_massless_bodies(bh, oracle_mod):
    """Massless bodies feel nothing (force = m a) and exert nothing; nodes of
    massless bodies only are skipped.  (The reference's arithmetic gives such
    nodes a 0/0 centre of mass; the device build gives them a finite one.)
    The massive bodies' forces carry Dehnen's own error against the direct
    sum, the level the oracle reaches on the same bodies without the massless
    ones."""
    m, q = plummer(3000, seed=6)
    m = m.copy()
    m[::7] = 0.0
    f = dehnen_gpu(bh, m, q, 0.5, 0.01, 4)
    assert np.all(np.isfinite(f))
    assert np.all(f[::7] == 0.0)
    sel = m > 0
    fd = oracle_mod.direct_forces(m, *xyz(q), 1.0, 1e-4)
    e = np.linalg.norm(f[sel] - fd[sel]) / np.linalg.norm(fd[sel])
    qs = q[sel]
    fo = oracle_mod.MortonTree(m[sel], *xyz(qs), L=21).dehnen(1.0, 1e-4, 0.25, 4)
    eo = np.linalg.norm(fo - fd[sel]) / np.linalg.norm(fd[sel])
    assert e <= 2.0 * eo, (e, eo)


def test_dehnen_refused_where_lists_cannot_be_sized(bh):
    import ctypes as C

    import torch

    from hierarquicos_b200 import _lib

    m, q = plummer(512, seed=2)
    s = bh.BHSystem()
    x, y, z = xyz(q)
    s.build(m, x, y, z, order=4)
    s.sync()
    out = torch.empty(3 * 512, dtype=torch.float64, device="cuda")
    p = _lib.default_params(order=4, precision=3)
    rc = _lib.lib().bh_system_capture(s._h, C.byref(p), out.data_ptr())
    assert rc == _lib.BH_ERR_INVALID
    dm, dx, dy, dz = (torch.as_tensor(a, device="cuda") for a in (m, x, y, z))
    rc = _lib.lib().bh_compute_forces_noalloc(dm.data_ptr(), dx.data_ptr(), dy.data_ptr(),
                                              dz.data_ptr(), 512, C.byref(p), out.data_ptr(), None)
    assert rc == _lib.BH_ERR_INVALID
