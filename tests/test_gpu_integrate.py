"""Time integration and Parareal on the device against the CPU restatement
of the reference's integrators (oracle/integrate.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ig():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from hierarquicos_b200 import integrate

    return integrate


def plummer_state(n, seed):
    from hierarquicos_b200.initial_values import generate_initial_values

    return generate_initial_values(n, -1.0, -1.0, True, False, "plummer", (1.0, 1.0), seed=seed)


def test_kick_drift_bit_exact(ig):
    """One fused kick-kick-drift launch equals the reference's update order,
    evaluated in numpy (no contraction), bit for bit, on a batch of 3 systems."""
    import torch

    rng = np.random.default_rng(0)
    sizes = [5, 300, 1000]
    off = ig.offsets_of(sizes)
    n = off[-1]
    m = rng.random(n) + 0.1
    q = rng.standard_normal((n, 3))
    p = rng.standard_normal((n, 3))
    f = rng.standard_normal(3 * n)
    st = ig.BatchState(m, q.T, p.T, off)
    for k1, k2, dt in [(0.0, 5e-4, 1e-3), (5e-4, 5e-4, 1e-3), (5e-4, 0.0, 0.0), (1e-2, 0.0, 1e-2)]:
        ig.kick_drift(st, torch.as_tensor(f, device="cuda"), k1, k2, dt)
        for s in range(3):
            a, b = off[s], off[s + 1]
            fs = f[3 * a:3 * b].reshape(3, -1).T
            if k1:
                p[a:b] = p[a:b] + k1 * fs
            if k2:
                p[a:b] = p[a:b] + k2 * fs
            if dt:
                q[a:b] = q[a:b] + (dt * p[a:b]) / m[a:b, None]
        assert np.array_equal(st.p.T.cpu().numpy(), p)
        assert np.array_equal(st.q.T.cpu().numpy(), q)


def test_verlet_direct_matches_oracle(ig, oracle_mod):
    from oracle import integrate as oi

    m, q, p = plummer_state(256, seed=4)
    G, eps, dt, steps = 1.0, 0.05, 1e-3, 20
    st = ig.BatchState.single(m, q.T, p.T)
    field = ig.ForceField("direct", G=G, eps=eps)
    ig.verlet(st, field, steps, dt)

    def forces(mm, qq):
        return oracle_mod.direct_forces(mm, qq[:, 0], qq[:, 1], qq[:, 2], G, eps * eps)

    qr, pr = oi.verlet(m, q, p, dt, steps, forces)
    np.testing.assert_allclose(st.q.T.cpu().numpy(), qr, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(st.p.T.cpu().numpy(), pr, rtol=1e-10, atol=1e-16)


def test_symplectic_euler_bh_reference_walk_matches_oracle(ig, oracle_mod):
    """Coarse propagator with the reference-semantics FP64 walk against the
    oracle's Morton-tree forces (same tree, same MAC)."""
    from oracle import integrate as oi

    m, q, p = plummer_state(2048, seed=5)
    G, eps, theta, dt, steps = 1.0, 0.01, 0.8, 1e-2, 3
    st = ig.BatchState.single(m, q.T, p.T)
    field = ig.ForceField("bh", theta=theta, eps=eps, order=1, precision=2, com_mode=0)
    ig.symplectic_euler(st, field, steps, dt)

    def forces(mm, qq):
        t = oracle_mod.MortonTree(mm, qq[:, 0], qq[:, 1], qq[:, 2], L=21, use_quadrupole=False,
                                  fma_mode=0)
        return t.forces_par(G, eps * eps, theta * theta, False)

    qr, pr = oi.symplectic_euler(m, q, p, dt, steps, forces)
    np.testing.assert_allclose(st.q.T.cpu().numpy(), qr, rtol=1e-10, atol=1e-13)
    np.testing.assert_allclose(st.p.T.cpu().numpy(), pr, rtol=1e-7, atol=1e-14)


def test_diagnostics_match_oracle(ig):
    from oracle import integrate as oi

    m, q, p = plummer_state(700, seed=6)
    m2, q2, p2 = plummer_state(300, seed=7)
    st = ig.BatchState(np.concatenate([m, m2]), np.concatenate([q, q2]).T,
                       np.concatenate([p, p2]).T, ig.offsets_of([700, 300]))
    d = ig.diagnostics(st, 1.0, 0.02)
    for s, (mm, qq, pp) in enumerate([(m, q, p), (m2, q2, p2)]):
        r = oi.diagnostics(mm, qq, pp, 1.0, 0.02)
        np.testing.assert_allclose(d[s, :3], r[:3], rtol=1e-12)
        np.testing.assert_allclose(d[s, 3:], r[3:], rtol=1e-9, atol=1e-15)


def test_verlet_bh_conserves_energy(ig):
    m, q, p = plummer_state(4096, seed=8)
    st = ig.BatchState.single(m, q.T, p.T)
    e0 = ig.diagnostics(st, 1.0, 0.01)[0]
    field = ig.ForceField("bh", theta=0.5, eps=0.01, order=4)
    ig.verlet(st, field, 100, 1e-3)
    e1 = ig.diagnostics(st, 1.0, 0.01)[0]
    assert abs(e1[0] - e0[0]) / abs(e0[0]) < 2e-4
    assert np.abs(e1[3:6] - e0[3:6]).max() < 1e-5


def test_batch_integration_equals_single(ig):
    """Each system of an integrated batch follows the trajectory it has alone,
    bit for bit."""
    parts = [plummer_state(n, seed=20 + n) for n in (100, 2000, 777)]
    off = ig.offsets_of([len(a[0]) for a in parts])
    st = ig.BatchState(np.concatenate([a[0] for a in parts]),
                       np.concatenate([a[1] for a in parts]).T,
                       np.concatenate([a[2] for a in parts]).T, off)
    field = ig.ForceField("bh", theta=0.6, eps=0.01, order=4)
    ig.verlet(st, field, 5, 1e-3)
    for s, (m, q, p) in enumerate(parts):
        one = ig.BatchState.single(m, q.T, p.T)
        ig.verlet(one, ig.ForceField("bh", theta=0.6, eps=0.01, order=4), 5, 1e-3)
        _, qb, pb = st.system(s)
        assert np.array_equal(qb, one.q.T.cpu().numpy())
        assert np.array_equal(pb, one.p.T.cpu().numpy())


def test_graph_replayed_field_follows_the_plain_trajectory(ig):
    """A field that replays its recorded build + walk gives the plain field's
    trajectory bit for bit: velocity Verlet on a batch, and symplectic Euler on
    one scratch state refilled between windows (the Parareal coarse sweep)."""
    parts = [plummer_state(n, seed=40 + n) for n in (3000, 1200)]
    off = ig.offsets_of([len(a[0]) for a in parts])
    args = (np.concatenate([a[0] for a in parts]), np.concatenate([a[1] for a in parts]).T,
            np.concatenate([a[2] for a in parts]).T, off)
    runs = []
    for graph in (False, True):
        st = ig.BatchState(*args)
        field = ig.ForceField("bh", theta=0.6, eps=0.01, order=4, graph=graph)
        ig.verlet(st, field, 6, 1e-3)
        runs.append((st.q.cpu().numpy(), st.p.cpu().numpy()))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])

    m, q, p = plummer_state(2500, seed=47)
    ends = []
    for graph in (False, True):
        one = ig.BatchState.single(m, q.T, p.T)
        field = ig.ForceField("bh", theta=0.8, eps=0.01, order=1, graph=graph)
        seen = []
        for w in range(3):
            if w:  # the next window starts from a perturbed copy, in the same tensors
                one.q.copy_(one.q * (1.0 + 1e-3 * w))
            ig.symplectic_euler(one, field, 2, 1e-2)
            seen.append((one.q.cpu().numpy(), one.p.cpu().numpy()))
        ends.append(seen)
    for (qa, pa), (qb, pb) in zip(*ends):
        assert np.array_equal(qa, qb) and np.array_equal(pa, pb)

    # parameters changed between calls are recorded anew, not replayed stale
    import torch

    one = ig.BatchState.single(m, q.T, p.T)
    field = ig.ForceField("bh", theta=0.8, eps=0.01, order=1, graph=True)
    f = torch.empty(3 * one.n, dtype=torch.float64, device=one.device)
    field(one, f)
    field(one, f)  # replayed
    field.params.theta = 0.4
    field(one, f)
    ref = ig.ForceField("bh", theta=0.4, eps=0.01, order=1)(one, torch.empty_like(f))
    assert torch.equal(f, ref)


def test_parareal_matches_oracle_direct(ig, oracle_mod):
    """The reference's Parareal with direct-force propagators, device against
    the CPU restatement: same iterates (to FP64 rounding of the force sums)
    and the same error curve."""
    from hierarquicos_b200 import parareal as pr
    from oracle import integrate as oi

    m, q, p = plummer_state(64, seed=9)
    G, eps, tf, W, itmax = 1.0, 0.05, 0.4, 6, 5
    coarse = pr.Propagator("euler", "direct", 1)
    fine = pr.Propagator("verlet", "direct", 8)
    res = pr.integrate_parareal(m, q, p, tf, W, itmax, 0.5, G, eps, 0.0, 8, coarse, fine)

    def forces(mm, qq):
        return oracle_mod.direct_forces(mm, qq[:, 0], qq[:, 1], qq[:, 2], G, eps * eps)

    window = tf / W
    U, errs, its = oi.parareal(
        m, q, p, tf, W, itmax, 0.0,
        lambda mm, qq, pp: oi.symplectic_euler(mm, qq, pp, window, 1, forces),
        lambda mm, qq, pp: oi.verlet(mm, qq, pp, window / 8, 8, forces))
    assert res.iterations == its
    for i in range(W):
        np.testing.assert_allclose(res.q[i], U[i][0], rtol=1e-11, atol=1e-13)
        np.testing.assert_allclose(res.p[i], U[i][1], rtol=1e-9, atol=1e-14)
    big = [k for k, e in enumerate(errs) if e > 1e-13]
    np.testing.assert_allclose(np.array(res.errors)[big], np.array(errs)[big], rtol=1e-5)


def test_parareal_becomes_stationary_at_the_fine_solution(ig):
    """With deterministic propagators the iteration stops changing (error 0)
    after at most num_windows iterations, at the sequential fine solution."""
    from hierarquicos_b200 import parareal as pr

    m, q, p = plummer_state(512, seed=10)
    G, eps, tf, W = 1.0, 0.02, 0.25, 5
    coarse = pr.Propagator("euler", "bh", 1, theta=0.8, order=1)
    fine = pr.Propagator("verlet", "bh", 10, theta=0.3, order=4)
    res = pr.integrate_parareal(m, q, p, tf, W, W + 2, 0.8, G, eps, 1e-20, 10, coarse, fine)
    assert res.converged and res.errors[-1] <= 1e-20
    qs, ps = pr.sequential_fine(m, q, p, tf, W, fine, G, eps)
    np.testing.assert_allclose(res.q, qs, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(res.p, ps, rtol=1e-9, atol=1e-15)


def test_parareal_double_double_correction(ig, oracle_mod):
    """The double-double correction: hi + lo is the exact value of
    (G_new + F) - G_old, so hi is the FP64 correction rounded once (it may
    differ from the twice-rounded FP64 form by an ulp) and |lo| is at most half
    an ulp of hi; the error curve is that of the FP64 correction."""
    from hierarquicos_b200 import parareal as pr

    m, q, p = plummer_state(64, seed=9)
    G, eps, tf, W, itmax = 1.0, 0.05, 0.4, 6, 5
    coarse = pr.Propagator("euler", "direct", 1)
    fine = pr.Propagator("verlet", "direct", 8)
    a = pr.integrate_parareal(m, q, p, tf, W, itmax, 0.5, G, eps, 0.0, 8, coarse, fine)
    b = pr.integrate_parareal(m, q, p, tf, W, itmax, 0.5, G, eps, 0.0, 8, coarse, fine,
                              correction="dd")
    assert b.q_lo is not None and b.iterations == a.iterations
    np.testing.assert_allclose(b.q, a.q, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(b.p, a.p, rtol=1e-10, atol=1e-15)
    assert np.all(np.abs(b.q_lo) <= 0.5 * np.spacing(np.abs(b.q)))
    assert np.all(np.abs(b.p_lo) <= 0.5 * np.spacing(np.abs(b.p)))
    big = [k for k, e in enumerate(a.errors) if e > 1e-13]
    np.testing.assert_allclose(np.array(b.errors)[big], np.array(a.errors)[big], rtol=1e-5)
    # once a window's coarse value stops changing, G_new = G_old and the exact
    # correction is F itself (lo = 0); after one iteration the later windows
    # still move, and their corrections carry low parts
    c = pr.integrate_parareal(m, q, p, tf, W, 2, 0.5, G, eps, 0.0, 8, coarse, fine,
                              correction="dd")
    assert np.any(c.q_lo[2:] != 0.0) or np.any(c.p_lo[2:] != 0.0)
    assert np.all(np.abs(c.q_lo) <= 0.5 * np.spacing(np.abs(c.q)))


def test_parareal_reference_example_config(ig, oracle_mod):
    """The configuration of parareal/main.f90 (N = 1000 in the cube [-10, 10]^3,
    m = 1/N, p = 0, G = 1, eps = 0.5, tf = 10, 30 windows, 16 fine Verlet steps
    per window, direct forces in both propagators -- its "PARAREAL (direct)"
    run) on seeded positions: the device's error curve equals the restated
    integrate_parareal's and falls geometrically until the FP64 floor."""
    from hierarquicos_b200 import parareal as pr
    from oracle import integrate as oi

    N, G, eps, tf, W, qntt, itmax = 1000, 1.0, 0.5, 10.0, 30, 16, 5
    rng = np.random.Generator(np.random.PCG64(0))
    m = np.full(N, 1.0 / N)
    q = 10.0 * (2.0 * rng.random((N, 3)) - 1.0)
    p = np.zeros((N, 3))
    coarse = pr.Propagator("euler", "direct", 1)
    fine = pr.Propagator("verlet", "direct", qntt)
    res = pr.integrate_parareal(m, q, p, tf, W, itmax, -1.0, G, eps, 1e-20, qntt, coarse, fine)

    def forces(mm, qq):
        return oracle_mod.direct_forces(mm, qq[:, 0], qq[:, 1], qq[:, 2], G, eps * eps)

    window = tf / W
    _, errs, its = oi.parareal(
        m, q, p, tf, W, itmax, 1e-20,
        lambda mm, qq, pp: oi.symplectic_euler(mm, qq, pp, window, 1, forces),
        lambda mm, qq, pp: oi.verlet(mm, qq, pp, window / qntt, qntt, forces))
    assert res.iterations == its
    big = [k for k, e in enumerate(errs) if e > 1e-12]
    assert len(big) >= 3
    np.testing.assert_allclose(np.array(res.errors)[big], np.array(errs)[big], rtol=1e-5)
    e = np.array(res.errors)
    assert np.all(e[1:len(big)] < 1e-2 * e[:len(big) - 1])  # each iteration gains > 2 decades
