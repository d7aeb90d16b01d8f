"""Edge cases through the C ABI: tiny systems, coincident and massless bodies,
degenerate geometry, invalid input and errors reported as status codes."""
import numpy as np
import pytest

from conftest import plummer, xyz

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    import torch

    assert torch.cuda.is_available()
    from hierarquicos_b200 import api3d

    return api3d


def test_single_body_has_no_force(api):
    f = api.compute_forces([1.0], [0.3], [0.1], [-2.0], 0.5, 1.0, 0.0, True)
    assert f.shape == (1, 3) and np.all(f == 0.0)


def test_two_bodies_exact(api):
    m = np.array([2.0, 3.0])
    x, y, z = np.array([0.0, 1.0]), np.array([0.0, 2.0]), np.array([0.0, -2.0])
    for order in (1, 4, 8):
        f = api.compute_forces(m, x, y, z, 0.5, 1.0, 0.0, order=order)
        d = np.array([1.0, 2.0, -2.0])
        exact = 1.0 * 2.0 * 3.0 * d / 27.0
        np.testing.assert_allclose(f[0], exact, rtol=2e-6)
        np.testing.assert_allclose(f[1], -exact, rtol=2e-6)


def test_ten_point_fixture_3d(api, oracle_mod):
    # the 2-D fixture of fortran/morton/test_morton.f90:30-39 (z = 0), unit
    # masses, theta 0.1, eps 0.01, automatic depth
    pts = np.array([[0.45931272, 0.22315240], [0.40157369, 0.21211072], [0.70372114, 0.64428738],
                    [0.20444018, 0.68014233], [0.73388286, 0.59264995], [0.68856885, 0.48249009],
                    [0.48843330, 0.28037004], [0.15927911, 0.69084037], [0.30486200, 0.50604824],
                    [0.59676033, 0.80020091]])
    m = np.ones(10)
    x, y, z = pts[:, 0].copy(), pts[:, 1].copy(), np.zeros(10)
    from hierarquicos_b200.system import BHSystem

    s = BHSystem()
    s.build(m, x, y, z, depth=0)
    s.sync()
    ref = oracle_mod.MortonTree(m, x, y, z, L=0, use_quadrupole=True, fma_mode=1)
    assert s.info()["depth"] == ref.L
    k, p = s.keys()
    rk, rp = ref.sorted()
    assert np.array_equal(k, rk) and np.array_equal(p, rp)
    f = s.walk(depth=0, precision=2, theta=0.1, eps=0.01)
    s.sync()
    f = f.view(3, -1).T.cpu().numpy()
    fr = ref.forces_par(1.0, 1e-4, 0.01, True)
    np.testing.assert_allclose(f, fr, rtol=1e-12, atol=1e-13)


def test_coincident_bodies(api, oracle_mod):
    m, q = plummer(2000, seed=4)
    q[10:30] = q[10]
    x, y, z = xyz(q)
    f = api.compute_forces(m, x, y, z, 0.5, 1.0, 0.01, True)
    fd = api.compute_forces_direct(m, x, y, z, 1.0, 0.01)
    assert np.all(np.isfinite(f))
    rel = np.linalg.norm(f - fd, axis=1) / np.linalg.norm(fd, axis=1)
    assert np.sqrt(np.mean(rel ** 2)) < 2e-3


def test_massless_bodies(api):
    m, q = plummer(3000, seed=6)
    m = m.copy()
    m[::7] = 0.0
    x, y, z = xyz(q)
    f = api.compute_forces(m, x, y, z, 0.5, 1.0, 0.01, True)
    fd = api.compute_forces_direct(m, x, y, z, 1.0, 0.01)
    assert np.all(np.isfinite(f))
    assert np.all(f[::7] == 0.0)
    sel = m > 0
    rel = np.linalg.norm(f[sel] - fd[sel], axis=1) / np.linalg.norm(fd[sel], axis=1)
    assert np.sqrt(np.mean(rel ** 2)) < 2e-3


def test_planar_and_linear_systems(api, oracle_mod):
    # flat and linear systems: net forces nearly cancel in the middle, so the
    # relative error is large for the reference too; ours must not be worse
    rng = np.random.default_rng(0)
    n = 3000
    m = np.full(n, 1.0 / n)
    for zero_axes in ((2,), (1, 2)):
        q = rng.standard_normal((n, 3))
        for a in zero_axes:
            q[:, a] = 0.0
        x, y, z = xyz(q)
        f = api.compute_forces(m, x, y, z, 0.5, 1.0, 0.05, True)
        fd = api.compute_forces_direct(m, x, y, z, 1.0, 0.05)
        fr = oracle_mod.MortonTree(m, x, y, z, 21, 1.2, True, fma_mode=1).forces_par(
            1.0, 0.05 ** 2, 0.25, True)

        def rms(a):
            rel = np.linalg.norm(a - fd, axis=1) / np.linalg.norm(fd, axis=1)
            return np.sqrt(np.mean(rel ** 2))

        assert np.all(np.isfinite(f))
        assert rms(f) <= 1.05 * rms(fr) + 1e-6, (rms(f), rms(fr))


def test_nonfinite_input_is_an_error(api):
    m, q = plummer(500, seed=1)
    q[3, 1] = np.nan
    with pytest.raises(api.BHError) as e:
        api.compute_forces(m, *xyz(q), 0.5, 1.0, 0.0, True)
    assert e.value.code == 4


def test_invalid_arguments(api):
    m, q = plummer(100, seed=1)
    with pytest.raises(api.BHError) as e:
        api.compute_forces(m, *xyz(q), 0.5, 1.0, 0.0, order=3)
    assert e.value.code == 1
    with pytest.raises(api.BHError):
        api.compute_forces(m, *xyz(q), -1.0, 1.0, 0.0, True)
    with pytest.raises(api.BHError):
        api.compute_forces(m[:50], *xyz(q), 0.5, 1.0, 0.0, True)
    from hierarquicos_b200.system import BHSystem

    for bad in (dict(pipeline=2), dict(pipeline=-1), dict(mac=2)):
        with pytest.raises(api.BHError) as e:
            BHSystem().forces(m, *xyz(q), **bad)
        assert e.value.code == 1, bad


def test_theta_zero_is_direct(api):
    m, q = plummer(1500, seed=8)
    x, y, z = xyz(q)
    f = api.compute_forces(m, x, y, z, 0.0, 1.0, 0.01, True, precision=1)
    fd = api.compute_forces_direct(m, x, y, z, 1.0, 0.01)
    np.testing.assert_allclose(f, fd, rtol=1e-10, atol=1e-13 * np.abs(fd).max())


def test_results_independent_of_call_history(api):
    # the same system alone and after other systems: identical bits
    m, q = plummer(4000, seed=12)
    x, y, z = xyz(q)
    f1 = api.compute_forces(m, x, y, z, 0.5, 1.0, 0.01, True)
    m2, q2 = plummer(30000, seed=13)
    api.compute_forces(m2, *xyz(q2), 0.7, 1.0, 0.0, order=8)
    f2 = api.compute_forces(m, x, y, z, 0.5, 1.0, 0.01, True)
    assert np.array_equal(f1, f2)


@pytest.mark.parametrize("parts", [2, 3, 8])
def test_walk_over_group_ranges_equals_full_walk(parts):
    """Sharding one system's targets: walking the target groups in disjoint
    ranges, each into a zeroed output, and summing the outputs gives the full
    walk bit for bit (the combine step of a multi-GPU run)."""
    import torch

    from hierarquicos_b200.shard import group_range
    from hierarquicos_b200.system import BHSystem

    m, q = plummer(20000, seed=21)
    x, y, z = xyz(q)
    s = BHSystem()
    kw = dict(theta=0.5, eps=0.01, order=4)
    full = s.forces(m, x, y, z, **kw).clone()
    ng = s.info()["n_groups"]
    total = torch.zeros_like(full)
    for r in range(parts):
        out = torch.zeros_like(full)
        s.walk(out=out, groups=group_range(ng, r, parts), **kw)
        s.sync()
        total += out
    assert torch.equal(total, full)
