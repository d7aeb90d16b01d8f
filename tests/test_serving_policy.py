"""Scheduling policy of the serving loop, on the host (no device work):
admission order (force requests before integrations, FIFO within a kind, a
request that does not fit passed over a bounded number of times) and the
per-tick choice of which integrations run beside force requests."""
import collections
import threading
import types

import numpy as np


def req(kind, n, steps=0):
    from hierarquicos_b200.serving import Request

    p = np.zeros((n, 3)) if kind == "leapfrog" else None
    return Request(kind, np.full(n, 1.0 / n), np.zeros((n, 3)), p, steps=steps)


def fake_server(pending, budget_bodies, tick_bodies, max_passed=3, force_tick_bodies=None):
    from hierarquicos_b200.serving import Server

    s = object.__new__(Server)
    s._cv = threading.Condition()
    s._pending = collections.deque(pending)
    s._resident = 0
    s.max_resident = 0
    s.workspace_bytes = 0
    s.hbm_budget = float(Server.footprint(budget_bodies))
    s.max_tick_bodies = tick_bodies
    s.max_tick_systems = 4096
    s.max_passed = max_passed
    s.force_tick_bodies = force_tick_bodies
    s.max_pause_ticks = 2
    return s


def lane(server, active=()):
    return types.SimpleNamespace(server=server, active=list(active), index=0)


def test_admission_takes_force_requests_first_then_fifo():
    from hierarquicos_b200.serving import Server

    a, b, c, d = req("leapfrog", 100, 5), req("force", 100), req("leapfrog", 100, 3), req("force", 50)
    s = fake_server([a, b, c, d], budget_bodies=10_000, tick_bodies=10_000)
    got = Server._admit(s, lane(s))
    assert got == [b, d, a, c]
    assert not s._pending


def test_admission_passes_over_a_request_that_does_not_fit_a_bounded_number_of_times():
    from hierarquicos_b200.serving import Server

    big, small = req("force", 900), req("force", 100)
    s = fake_server([big, small], budget_bodies=10_000, tick_bodies=1000, max_passed=2)
    ln = lane(s, active=[req("leapfrog", 500, 10)])
    assert Server._admit(s, ln) == [small]           # big does not fit the tick: passed over
    s._pending.append(req("force", 10))
    assert len(Server._admit(s, ln)) == 1            # passed over a second time
    later = req("force", 10)
    s._pending.append(later)
    assert Server._admit(s, ln) == []                # big has waited long enough: it blocks
    assert list(s._pending) == [big, later]
    ln.active = []
    assert Server._admit(s, ln) == [big, later]


def test_tick_runs_integrations_beside_force_requests_within_the_budget():
    from hierarquicos_b200.serving import _Lane

    s = fake_server([], 1, 1, force_tick_bodies=1000)
    ln = lane(s)
    f = req("force", 400)
    l1, l2, l3 = req("leapfrog", 300, 9), req("leapfrog", 700, 9), req("leapfrog", 200, 9)
    l1._last_tick, l2._last_tick, l3._last_tick = 5, 3, 4
    run, paused = _Lane._schedule(ln, [l1, f, l2, l3])
    # least recently run first: l2 (700) does not fit the 600 left, l3 (200) and l1 (300) do
    assert run == [f, l3, l1] and paused == [l2]
    # an integration that has sat out max_pause_ticks ticks runs regardless
    l2._paused = 2
    run, paused = _Lane._schedule(ln, [l1, f, l2, l3])
    assert run == [f, l2] and paused == [l3, l1]
    # without force requests every system runs
    run, paused = _Lane._schedule(ln, [l1, l2, l3])
    assert run == [l1, l2, l3] and paused == []
    # scheduling switched off
    s.force_tick_bodies = None
    assert _Lane._schedule(ln, [f, l1, l2, l3]) == ([f, l1, l2, l3], [])
