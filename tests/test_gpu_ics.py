"""Initial conditions drawn on the device: the same distributions as the host
generator (which follows initial_values/*.f90), checked statistically, plus
the exact post-conditions (centre of mass and total momentum at zero,
masses, determinism)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def iv():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from hierarquicos_b200 import initial_values

    return initial_values


CASES = [("plummer", -1.0, (1.0, 1.0)), ("hernquist", 100.0, (1.0, 1.0)),
         ("homogeneous", -1.0, (1.0, 1.0)), ("uniform_sphere", 1.0, (1.0, 1.0)),
         ("uniform", 1.0, (1.0, 1.0))]


@pytest.mark.parametrize("pr,size,pp", CASES)
def test_positions_follow_the_host_distribution(iv, pr, size, pp):
    from scipy.stats import ks_2samp

    n = 40000
    m, q, _ = iv.generate_initial_values_device(n, size, 1.0, True, False, pr, pp, seed=3,
                                                velocities=False)
    mh, qh, _ = iv.generate_initial_values(n, size, 1.0, True, False, pr, pp, seed=3,
                                           velocities=False)
    r = np.linalg.norm(q.cpu().numpy(), axis=0)
    rh = np.linalg.norm(qh, axis=1)
    assert ks_2samp(r, rh).pvalue > 1e-3
    for k in range(3):  # isotropy: each axis alike (up to the centre-of-mass shift,
        # which far-out bodies of an untruncated profile dominate)
        a, b = q[k].cpu().numpy(), qh[:, k]
        assert ks_2samp(a - np.median(a), b - np.median(b)).pvalue > 1e-3
    np.testing.assert_array_equal(m.cpu().numpy(), mh)


@pytest.mark.parametrize("pr,n", [("plummer", 40000), ("hernquist", 12000)])
def test_speeds_follow_the_host_distribution(iv, pr, n):
    from scipy.stats import ks_2samp

    size = 100.0 if pr == "hernquist" else -1.0
    m, _, p = iv.generate_initial_values_device(n, size, -1.0, True, False, pr, (1.0, 1.0), seed=5)
    mh, _, ph = iv.generate_initial_values(n, size, -1.0, True, False, pr, (1.0, 1.0), seed=5)
    v = np.linalg.norm(p.cpu().numpy(), axis=0) / m.cpu().numpy()
    vh = np.linalg.norm(ph, axis=1) / mh
    assert ks_2samp(v, vh).pvalue > 1e-3


def test_centre_of_mass_momentum_masses_and_determinism(iv):
    n = 30000
    m, q, p = iv.generate_initial_values_device(n, -1.0, -1.0, False, False, "plummer",
                                                (1.0, 1.0), seed=11)
    m, q, p = m.cpu().numpy(), q.cpu().numpy(), p.cpu().numpy()
    assert abs(m.sum() - 1.0) < 1e-12 and m.min() > 0
    assert np.abs((m * q).sum(axis=1)).max() < 1e-12
    assert np.abs(p.sum(axis=1)).max() < 1e-15
    m2, q2, p2 = iv.generate_initial_values_device(n, -1.0, -1.0, False, False, "plummer",
                                                   (1.0, 1.0), seed=11)
    assert np.array_equal(q, q2.cpu().numpy()) and np.array_equal(p, p2.cpu().numpy())
    _, q3, _ = iv.generate_initial_values_device(n, -1.0, -1.0, False, False, "plummer",
                                                 (1.0, 1.0), seed=12)
    assert not np.array_equal(q, q3.cpu().numpy())
    _, q4, p4 = iv.generate_initial_values_device(1000, -1.0, -1.0, True, True, "plummer",
                                                  (1.0, 1.0), seed=1)
    assert np.all(q4[2].cpu().numpy() == 0) and np.all(p4[2].cpu().numpy() == 0)


def test_plummer_is_in_virial_equilibrium(iv):
    from hierarquicos_b200 import integrate as ig

    n = 16384
    m, q, p = iv.generate_initial_values_device(n, -1.0, -1.0, True, False, "plummer",
                                                (1.0, 1.0), seed=2)
    st = ig.BatchState.single(m, q, p)
    d = ig.diagnostics(st, 1.0, 0.0)[0]
    kin, pot = d[1], d[2]
    assert abs(2 * kin / abs(pot) - 1.0) < 0.05
