"""Accuracy of the production walk on the large Hernquist system over the
opening-angle x multipole grid: N = 2^20 (a = 1, truncated at 100 a, equal
masses, seeded), theta in {0.3, 0.5, 0.7} x order in {1, 4, 8}, RMS relative
error on 16,384 seeded targets against the FP64 direct sum over all N sources.

Bound: the FP32 group walk (pipelined, both acceptance tests) is at most 1.05x
the error of the reference's own per-target FP64 walk on the same targets +
2e-6 (FP32 rounding) -- the per-target walk with the reference's MAC
(morton_octree.f90:627-766 for orders 1/4, octree_default.f90:895-1078 for
order 8) -- and theta 0.5 quadrupole meets the 1e-3 bound of the headline
metric.  The FP32 compensated walk against the all-FP64 walk (same groups,
same acceptance): their RMS relative difference is below 1e-6, far under the
truncation error."""
import numpy as np
import pytest

from conftest import hernquist, xyz

pytestmark = pytest.mark.gpu

N = 1 << 20
N_TARGETS = 16384


@pytest.fixture(scope="module")
def system_and_direct():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from hierarquicos_b200 import system

    m, q = hernquist(N, seed=2024)
    dev = "cuda"
    M, X, Y, Z = (torch.as_tensor(a, device=dev) for a in (m, *xyz(q)))
    tg = np.sort(np.random.default_rng(7).choice(N, N_TARGETS, replace=False))
    fd = system.direct_targets(M, X, Y, Z, tg, 1.0, 0.01).cpu().numpy().T
    s = system.BHSystem()
    s.build(M, X, Y, Z, order=8)
    s.sync()
    return system, s, (M, X, Y, Z), tg, fd


def rms(f, fd):
    e = np.linalg.norm(f - fd, axis=1) / np.linalg.norm(fd, axis=1)
    return float(np.sqrt(np.mean(e * e)))


@pytest.mark.parametrize("order", [1, 4, 8])
@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_walk_error_grid(system_and_direct, order, theta):
    import torch

    _, s, _, tg, fd = system_and_direct
    fr = s.reference_targets(tg, theta=theta, eps=0.01, order=order)
    e_ref = rms(fr, fd)
    t = torch.as_tensor(tg, device="cuda")
    for mac in (0, 1):
        f = s.walk(theta=theta, eps=0.01, order=order, mac=mac)
        s.sync()
        e = rms(f.view(3, -1)[:, t].T.cpu().numpy(), fd)
        print(f"order {order} theta {theta} mac {mac}: rms {e:.3e} (reference walk {e_ref:.3e})")
        assert e <= 1.05 * e_ref + 2e-6, (order, theta, mac, e, e_ref)
        if order == 4 and theta == 0.5:
            assert e <= 1e-3
        f64 = s.walk(theta=theta, eps=0.01, order=order, mac=mac, precision=1)
        s.sync()
        d = rms(f.view(3, -1).T.cpu().numpy(), f64.view(3, -1).T.cpu().numpy())
        print(f"    FP32 vs FP64 walk: rms rel difference {d:.2e}")
        assert d < 1e-6, (order, theta, mac, d)
