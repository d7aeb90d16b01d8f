"""The serving loop: continuous batching, HBM admission, and results that do
not depend on the mix (each request gets, bit for bit, what it gets alone
through the plain single-system path)."""
import numpy as np
import pytest

from conftest import plummer, xyz

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sv():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from hierarquicos_b200 import serving

    return serving


def ic(n, seed, velocities=False, profile="plummer"):
    from hierarquicos_b200.initial_values import generate_initial_values

    par = (1.0, 1.0)
    size = 100.0 if profile == "hernquist" else -1.0
    return generate_initial_values(n, size, -1.0, True, False, profile, par, seed=seed,
                                   velocities=velocities)


PARAMS = dict(theta=0.5, eps=0.01, order=4)


def plain_forces(m, q):
    from hierarquicos_b200.system import BHSystem

    f = BHSystem().forces(m, *xyz(q), **PARAMS)
    return f.view(3, -1).T.cpu().numpy()


def plain_leapfrog(m, q, p, steps, dt):
    from hierarquicos_b200 import integrate as ig

    st = ig.BatchState.single(m, q.T, p.T)
    ig.verlet(st, ig.ForceField("bh", **PARAMS), steps, dt)
    return st.q.T.cpu().numpy(), st.p.T.cpu().numpy()


def mixed_requests(sv, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(count):
        n = int(np.exp(rng.uniform(np.log(100), np.log(20000))))
        prof = ["plummer", "hernquist", "homogeneous"][k % 3]
        if rng.random() < 0.5:
            m, q, _ = ic(n, seed * 100 + k, profile=prof)
            reqs.append(sv.Request("force", m, q))
        else:
            m, q, p = ic(n, seed * 100 + k, velocities=True, profile="plummer")
            reqs.append(sv.Request("leapfrog", m, q, p, steps=int(rng.integers(1, 8)), dt=1e-3))
    return reqs


def check_against_plain(r):
    if r.kind == "force":
        assert np.array_equal(r.forces, plain_forces(r.m, r.q)), f"request {r.id}"
    else:
        qe, pe = plain_leapfrog(r.m, r.q, r.p, r.steps, r.dt)
        assert np.array_equal(r.q_out, qe) and np.array_equal(r.p_out, pe), f"request {r.id}"


def test_mixed_stream_matches_plain_path(sv):
    reqs = mixed_requests(sv, 16, seed=1)
    with sv.Server(hbm_budget=40e9, max_tick_bodies=1 << 20, **PARAMS) as srv:
        for r in reqs:
            srv.submit(r)
        srv.drain(timeout=300)
        met = srv.metrics()
    assert met["requests"] == len(reqs)
    assert met["p99_ms"] >= met["p50_ms"] > 0
    for r in reqs:
        assert r.error is None
        check_against_plain(r)


def test_same_alone_and_in_the_mix(sv):
    """The same request served alone and arriving in the middle of a busy
    stream gives identical results."""
    import time

    m, q, p = ic(5000, 77, velocities=True)
    alone = sv.Request("leapfrog", m, q, p, steps=6)
    with sv.Server(max_tick_bodies=1 << 20, hbm_budget=40e9, **PARAMS) as srv:
        srv.submit(alone)
        srv.drain(timeout=120)
    others = mixed_requests(sv, 12, seed=2)
    mixed = sv.Request("leapfrog", m, q, p, steps=6)
    with sv.Server(max_tick_bodies=1 << 20, hbm_budget=40e9, **PARAMS) as srv:
        for k, r in enumerate(others):
            srv.submit(r)
            if k == 5:
                srv.submit(mixed)
            time.sleep(0.002)
        srv.drain(timeout=300)
        lanes = {r.lane for r in others + [mixed]}
    assert np.array_equal(alone.q_out, mixed.q_out)
    assert np.array_equal(alone.p_out, mixed.p_out)
    assert len(lanes) >= 1


def test_admission_respects_the_hbm_budget(sv):
    reqs = [sv.Request("force", *ic(20000, 300 + k)[:2]) for k in range(8)]
    per = sv.Server.footprint(20000)
    ws = 2 * sv.WORKSPACE_BYTES_PER_BODY * (1 << 16)
    budget = ws + 2.5 * per  # room for two resident requests at a time
    with sv.Server(hbm_budget=budget, max_tick_bodies=1 << 16, **PARAMS) as srv:
        for r in reqs:
            srv.submit(r)
        srv.drain(timeout=300)
        assert srv.max_resident <= budget - ws
        assert srv.max_resident >= per
    for r in reqs:
        assert r.t_admit >= r.arrival
        check_against_plain(r)


def test_refuses_requests_that_cannot_fit(sv):
    m, q, _ = ic(3000, 5)
    srv = sv.Server(max_tick_bodies=1024, hbm_budget=1e9, **PARAMS)
    with pytest.raises(ValueError):
        srv.submit(sv.Request("force", m, q))
    with pytest.raises(ValueError):
        sv.Request("leapfrog", m, q, None, steps=3)


@pytest.mark.parametrize("lanes", [1, 2])
def test_device_requests_match_plain_path(sv, lanes):
    """Device-resident requests (CUDA tensors in, CUDA tensors out), mixed with
    host requests and leapfrog runs of different lengths that join and leave
    while others run: every result equals the plain path's bit for bit."""
    import torch

    dev = torch.device("cuda", 0)
    host = mixed_requests(sv, 6, seed=5)
    dev_reqs, ref = [], []
    for k in range(6):
        n = [700, 3000, 12000, 5000, 900, 20000][k]
        if k % 2 == 0:
            m, q, _ = ic(n, 500 + k, profile="hernquist")
            dev_reqs.append(sv.Request("force", torch.as_tensor(m, device=dev),
                                       torch.as_tensor(q.T.copy(), device=dev)))
            ref.append(("force", m, q))
        else:
            m, q, p = ic(n, 500 + k, velocities=True)
            steps = 2 + k
            dev_reqs.append(sv.Request("leapfrog", torch.as_tensor(m, device=dev),
                                       torch.as_tensor(q, device=dev),
                                       torch.as_tensor(p, device=dev), steps=steps, dt=1e-3))
            ref.append(("leapfrog", m, q, p, steps))
    with sv.Server(lanes=lanes, max_tick_bodies=1 << 16, hbm_budget=40e9, **PARAMS) as srv:
        for a, b in zip(host, dev_reqs):
            srv.submit(a)
            srv.submit(b)
        srv.drain(timeout=300)
    for r in host:
        assert r.error is None
        check_against_plain(r)
    for r, e in zip(dev_reqs, ref):
        assert r.error is None
        if e[0] == "force":
            assert r.forces.is_cuda and r.forces.shape == (r.n, 3)
            assert np.array_equal(r.forces.cpu().numpy(), plain_forces(e[1], e[2]))
        else:
            qe, pe = plain_leapfrog(e[1], e[2], e[3], e[4], 1e-3)
            assert np.array_equal(r.q_out.cpu().numpy(), qe)
            assert np.array_equal(r.p_out.cpu().numpy(), pe)


def test_submit_many_queues_a_group_at_once(sv):
    """Requests submitted together (submit_many) get the plain path's results
    bit for bit; a group holding a request that cannot fit is refused before
    any of it is queued."""
    reqs = mixed_requests(sv, 8, seed=11)
    with sv.Server(lanes=2, max_tick_bodies=1 << 16, hbm_budget=40e9, **PARAMS) as srv:
        out = srv.submit_many(reqs)
        assert out == reqs and all(r.arrival is not None for r in reqs)
        srv.drain(timeout=300)
    for r in reqs:
        assert r.error is None
        check_against_plain(r)
    m, q, _ = ic(3000, 6)
    small = sv.Request("force", *ic(500, 7)[:2])
    srv = sv.Server(max_tick_bodies=1024, hbm_budget=1e9, **PARAMS)
    with pytest.raises(ValueError):
        srv.submit_many([small, sv.Request("force", m, q)])
    assert len(srv._pending) == 0


def test_paused_integrations_match_plain_path(sv):
    """With a small force_tick_bodies the lanes make integrations sit ticks
    out while force requests run (and force requests are admitted first); the
    results are still exactly the plain path's, and some ticks did pause."""
    reqs = mixed_requests(sv, 16, seed=5)
    with sv.Server(hbm_budget=40e9, max_tick_bodies=1 << 20, force_tick_bodies=3000,
                   max_pause_ticks=2, **PARAMS) as srv:
        srv.submit_many(reqs)
        srv.drain(timeout=300)
        met = srv.metrics()
    assert met["requests"] == len(reqs)
    assert met["paused_ticks"] > 0
    assert set(met["by_kind"]) <= {"force", "leapfrog"}
    for r in reqs:
        assert r.error is None
        check_against_plain(r)
