"""Serving: a request loop with continuous batching and HBM admission.

Requests are force evaluations or leapfrog integrations (velocity Verlet in
momentum form, the reference's integrator, benchmarks/integration_verlet/
integration.f90:110-172) of independent systems of any size.  The server
keeps every admitted request's particles on the device until it finishes, and
advances ALL of a lane's active requests together: one tick is one batched
force evaluation (one build and one walk over all of the lane's systems) and
one kick-drift launch with per-system coefficients, so a request admitted
while others are running joins the very next tick.

Design for one GPU:
  * ``lanes`` independent lanes (default 2), each a host thread with its own
    engine workspace and CUDA streams.  While one lane waits for its tick's
    status on the host, the other lane's tick runs on the GPU, so the device
    stays busy and the lanes' work overlaps.
  * admission by HBM footprint: a request is admitted (FIFO) when its resident
    bytes fit in ``hbm_budget`` next to the lanes' fixed workspaces and the
    requests already resident; otherwise it waits until finished requests
    release memory.  A request larger than a lane's tick capacity is refused.
  * inputs arrive in pinned host memory and are copied on a copy stream;
    results go back on another copy stream, overlapping the next tick.
  * results do not depend on the mix: every system in a batch gets exactly
    (bit for bit) the result it gets alone.

Latency of a request = completion of its result copy to the host minus its
arrival time; ``Server.metrics()`` reports p50/p99 and throughput.
"""
from __future__ import annotations

import collections
import dataclasses
import itertools
import threading
import time

import numpy as np
import torch

from ._lib import BHParams, check, default_params, lib
from .integrate import as_device
from .system import BHSystem, _dptr

STATE_BYTES_PER_BODY = 8 + 24 + 24          # m, q, p (FP64)
RESIDENT_BYTES_PER_BODY = 2 * STATE_BYTES_PER_BODY + 24 + 24  # + tick copy, forces, coefficients
# engine workspace (keys, sort, tree, moments, groups: 520) + the lane's two
# state buffers and forces (136)
WORKSPACE_BYTES_PER_BODY = 656

_ids = itertools.count()


@dataclasses.dataclass(eq=False)
class Request:
    """A force evaluation (``kind='force'``) or ``steps`` leapfrog steps of
    length ``dt`` (``kind='leapfrog'``) of one system.  m (n,), q (n,3),
    p (n,3) momenta (leapfrog only)."""

    kind: str
    m: np.ndarray
    q: np.ndarray
    p: np.ndarray | None = None
    steps: int = 0
    dt: float = 1e-3
    arrival: float | None = None
    id: int = dataclasses.field(default_factory=lambda: next(_ids))
    # filled by the server
    forces: np.ndarray | None = None     # (n, 3) for force requests
    q_out: np.ndarray | None = None      # (n, 3) final positions (leapfrog)
    p_out: np.ndarray | None = None
    t_admit: float | None = None
    t_done: float | None = None
    lane: int = -1
    error: str | None = None

    def __post_init__(self):
        if self.kind not in ("force", "leapfrog"):
            raise ValueError("kind must be 'force' or 'leapfrog'")
        # device-resident request: CUDA tensors in (m (n,), q and p (3, n)),
        # results stay on the device
        self.on_device = isinstance(self.m, torch.Tensor) and self.m.is_cuda
        self.n = int(self.m.numel() if self.on_device else np.asarray(self.m).size)
        if self.kind == "leapfrog" and (self.steps < 1 or self.p is None):
            raise ValueError("a leapfrog request needs momenta and steps >= 1")
        self._done = threading.Event()
        self._evals = 0  # force evaluations done
        self._last_tick = -1  # last tick of its lane that evaluated it
        self._paused = 0      # ticks sat out in a row
        self._passed = 0      # admission rounds in which a later request went first

    @property
    def evals_needed(self) -> int:
        return 1 if self.kind == "force" else self.steps + 1

    @property
    def latency(self) -> float | None:
        return None if self.t_done is None else self.t_done - self.arrival

    def wait(self, timeout=None) -> bool:
        return self._done.wait(timeout)


_ROWS = ("m", "x", "y", "z", "px", "py", "pz")


class _Lane:
    """One host thread and its device buffers, all allocated once: the engine
    workspace, two (7, max_tick_bodies) state buffers used in turn (m, x, y,
    z, px, py, pz of every active system, back to back), the forces of a tick
    and the per-system offsets and kick coefficients.  A tick gathers the
    systems still running and the newly admitted ones into the other state
    buffer, so the tick itself allocates no device memory."""

    def __init__(self, server: "Server", index: int):
        self.server = server
        self.index = index
        dev = server.device
        cap, cap_s = server.max_tick_bodies, server.max_tick_systems
        with torch.cuda.device(dev):
            self.stream = torch.cuda.Stream(dev)
            # host copies go through the server's two copy streams, shared by
            # the lanes: in the order the lanes enqueue them, at the full
            # bandwidth of each direction
            self.h2d = server.h2d
            self.d2h = server.d2h
            self.sys = BHSystem(dev.index).reserve(cap, cap_s)
            self.buf = [torch.empty(7, cap, dtype=torch.float64, device=dev) for _ in range(2)]
            self.out = torch.empty(3 * cap, dtype=torch.float64, device=dev)
            self.d_off = torch.empty(cap_s + 1, dtype=torch.int64, device=dev)
            self.d_coef = torch.empty(3 * cap_s, dtype=torch.float64, device=dev)
        self.h_off = torch.empty(cap_s + 1, dtype=torch.int64, pin_memory=True)
        self.h_coef = torch.empty(3 * cap_s, dtype=torch.float64, pin_memory=True)
        self.cur = 0                       # buffer holding the running systems
        self.pos: dict[int, int] = {}      # request id -> its first body in buf[cur]
        self.d2h_done: torch.cuda.Event | None = None
        self.active: list[Request] = []
        self.fresh: list[Request] = []     # admitted, not yet in a state buffer
        self.done_q: collections.deque = collections.deque()
        self.done_cv = threading.Condition()
        self.ticks = 0
        self.tick_bodies = 0
        self.paused_ticks = 0              # integrations that sat a tick out
        # per tick: host seconds spent enqueuing it and CUDA events around its
        # device work (read by Server.metrics)
        self.tick_log: collections.deque = collections.deque(maxlen=4096)
        self.thread = threading.Thread(target=self._run, name=f"bh-lane-{index}", daemon=True)
        self.finisher = threading.Thread(target=self._finish_loop, name=f"bh-done-{index}",
                                         daemon=True)

    def close(self):
        """Frees the lane's device memory (after its threads have ended)."""
        self.sys.close()
        self.buf = []
        self.out = self.d_off = self.d_coef = None

    def _schedule(self, act: list[Request]) -> tuple[list[Request], list[Request]]:
        """Which of the lane's systems this tick evaluates.  Without force
        requests in the lane every system runs.  With some, the force requests
        run and integrations join them only while the tick stays within the
        server's ``force_tick_bodies`` (least recently run first); the others
        sit this tick out, their state carried over unchanged.  An integration
        that has sat out ``max_pause_ticks`` ticks in a row runs regardless,
        so a stream of force requests cannot stall it."""
        srv = self.server
        forces = [r for r in act if r.kind == "force"]
        if not forces or srv.force_tick_bodies is None:
            return act, []
        budget = srv.force_tick_bodies - sum(r.n for r in forces)
        run, paused = list(forces), []
        for r in sorted((r for r in act if r.kind == "leapfrog"), key=lambda r: r._last_tick):
            if r.n <= budget or r._paused >= srv.max_pause_ticks:
                run.append(r)
                budget -= r.n
            else:
                paused.append(r)
        return run, paused

    # -- one tick: forces of every running system, then the per-system kicks --
    def _tick(self):
        srv = self.server
        run, paused = self._schedule(self.active + self.fresh)
        act = run + paused  # running systems first: the tick evaluates [0, n)
        nrun = len(run)
        sizes = [r.n for r in act]
        off = np.zeros(len(act) + 1, np.int64)
        off[1:] = np.cumsum(sizes)
        n = int(off[nrun])
        src, dst = self.buf[self.cur], self.buf[1 - self.cur]
        t_host = time.perf_counter()
        ev_begin = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(self.stream):
            ev_begin.record(self.stream)
            if self.d2h_done is not None:  # the previous results have left `out` and `dst`
                self.stream.wait_event(self.d2h_done)
            # host inputs of new requests: copied on the copy stream straight
            # into their place in the new state buffer
            host_new = [(i, r) for i, r in enumerate(act) if r in self.fresh and not r.on_device]
            if host_new:
                self.h2d.wait_event(ev_begin)
                with torch.cuda.stream(self.h2d):
                    for i, r in host_new:
                        a, b = int(off[i]), int(off[i + 1])
                        for k, name in enumerate(_ROWS):
                            if name in r._pinned:
                                dst[k, a:b].copy_(r._pinned[name], non_blocking=True)
                    ev_in = torch.cuda.Event()
                    ev_in.record(self.h2d)
            for i, r in enumerate(act):
                a, b = int(off[i]), int(off[i + 1])
                if r.id in self.pos:                      # running: its current state
                    p0 = self.pos[r.id]
                    dst[:, a:b].copy_(src[:, p0:p0 + r.n], non_blocking=True)
                elif r.on_device:                         # new, device inputs
                    for k, name in enumerate(_ROWS):
                        if name in r._pinned:
                            dst[k, a:b].copy_(r._pinned[name], non_blocking=True)
                if r.kind == "force" and r.id not in self.pos:
                    dst[4:7, a:b].zero_()                 # no momenta: the kick is a no-op
            if host_new:
                self.stream.wait_event(ev_in)
            out = self.out[:3 * n]
            self.sys.forces_batch(dst[0, :n], dst[1, :n], dst[2, :n], dst[3, :n], off[:nrun + 1],
                                  srv.params, out=out)
            if any(r.kind == "leapfrog" for r in run):
                coef = self.h_coef.numpy()
                for i, r in enumerate(run):
                    c = (0.0, 0.0, 0.0)
                    if r.kind == "leapfrog":
                        h = 0.5 * r.dt
                        k = r._evals
                        c = (0.0, h, r.dt) if k == 0 else ((h, h, r.dt) if k < r.steps
                                                           else (h, 0.0, 0.0))
                    coef[3 * i:3 * i + 3] = c
                self.h_off.numpy()[:nrun + 1] = off[:nrun + 1]
                self.d_coef[:3 * nrun].copy_(self.h_coef[:3 * nrun], non_blocking=True)
                self.d_off[:nrun + 1].copy_(self.h_off[:nrun + 1], non_blocking=True)
                check(lib().bh_kick_drift_systems(
                    _dptr(dst[0]), _dptr(out), _dptr(dst[1]), _dptr(dst[2]), _dptr(dst[3]),
                    _dptr(dst[4]), _dptr(dst[5]), _dptr(dst[6]), _dptr(self.d_off), nrun, n,
                    _dptr(self.d_coef), self.stream.cuda_stream))
            for r in run:
                r._evals += 1
                r._last_tick = self.ticks
                r._paused = 0
            for r in paused:
                r._paused += 1
            # device results: copied into the request's own buffers
            finished, keep = [], []
            for i, r in enumerate(act):
                a, b = int(off[i]), int(off[i + 1])
                if i < nrun and r._evals >= r.evals_needed:
                    finished.append((r, a, b))
                    if r.on_device:
                        if r.kind == "force":
                            r._dev_result["f"].copy_(out[3 * a:3 * b].view(3, b - a),
                                                     non_blocking=True)
                        else:
                            for k, name in enumerate(_ROWS[1:], start=1):
                                r._dev_result[name].copy_(dst[k, a:b], non_blocking=True)
                else:
                    keep.append((r, a))
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(self.stream)
        self.tick_log.append((time.perf_counter() - t_host, ev_begin, ev))
        # host results on the copy stream
        host_done = [(r, a, b) for r, a, b in finished if not r.on_device]
        if host_done:
            self.d2h.wait_event(ev)
            with torch.cuda.stream(self.d2h):
                for r, a, b in host_done:
                    if r.kind == "force":
                        r._host_out["f"].copy_(out[3 * a:3 * b], non_blocking=True)
                    else:
                        for k, name in enumerate(_ROWS[1:], start=1):
                            r._host_out[name].copy_(dst[k, a:b], non_blocking=True)
                self.d2h_done = torch.cuda.Event()
                self.d2h_done.record(self.d2h)
        with self.done_cv:
            for r, a, b in finished:
                done = torch.cuda.Event()
                done.record(self.d2h if not r.on_device else self.stream)
                self.done_q.append((r, done))
            self.done_cv.notify()
        self.cur = 1 - self.cur
        self.pos = {r.id: a for r, a in keep}
        self.active = [r for r, _ in keep]
        self.fresh = []
        self.ticks += 1
        self.tick_bodies += n
        self.paused_ticks += len(paused)

    def _run(self):
        srv = self.server
        torch.cuda.set_device(srv.device)
        try:
            while True:
                self.fresh = srv._admit(self)
                if not self.active and not self.fresh:
                    if srv._stopping and srv._idle():
                        break
                    with srv._cv:
                        srv._cv.wait(0.01)
                    continue
                self._tick()
        except Exception as e:  # a failed tick fails its requests, not the server
            for r in self.active + self.fresh:
                r.error = str(e)
                r.t_done = time.perf_counter()
                srv._release(r)
                r._done.set()
            self.active = []
            self.fresh = []
            srv._lane_error = e
        finally:
            with self.done_cv:
                self.done_q.append(None)
                self.done_cv.notify()

    def _finish_loop(self):
        torch.cuda.set_device(self.server.device)
        while True:
            with self.done_cv:
                while not self.done_q:
                    self.done_cv.wait()
                item = self.done_q.popleft()
            if item is None:
                return
            r, ev = item
            ev.synchronize()
            r.t_done = time.perf_counter()
            if r.on_device:
                do = r._dev_result
                if r.kind == "force":
                    r.forces = do["f"].T
                else:
                    r.q_out = torch.stack([do["x"], do["y"], do["z"]], dim=1)
                    r.p_out = torch.stack([do["px"], do["py"], do["pz"]], dim=1)
                self.server._release(r)
                r._done.set()
                continue
            ho = r._host_out
            if r.kind == "force":
                r.forces = ho["f"].numpy().reshape(3, r.n).T
            else:
                r.q_out = np.stack([ho["x"].numpy(), ho["y"].numpy(), ho["z"].numpy()], axis=1)
                r.p_out = np.stack([ho["px"].numpy(), ho["py"].numpy(), ho["pz"].numpy()], axis=1)
            self.server._release(r)
            r._done.set()


class Server:
    """Continuous-batching force server on one GPU.

    ``params``: engine parameters (theta, eps, order, ...; default theta 0.5,
    quadrupole).  ``hbm_budget``: bytes the server may hold on the device.
    ``max_tick_bodies``: bodies of one lane's tick (bounds the lanes'
    workspaces and a tick's latency).  ``force_tick_bodies``: while a lane
    holds force requests its ticks take integrations only up to this many
    bodies in all (the rest sit the tick out, at most ``max_pause_ticks`` in a
    row).  Admission takes force requests before integrations, FIFO within
    each kind, and lets a later request that fits go ahead of one that does
    not, until the one passed over has waited ``max_passed`` rounds."""

    def __init__(self, params: BHParams | None = None, device=None, hbm_budget: float = 150e9,
                 max_tick_bodies: int = 1 << 23, lanes: int = 2, max_tick_systems: int = 4096,
                 force_tick_bodies: int | None = 1 << 22, max_pause_ticks: int = 8,
                 max_passed: int = 64, **kw):
        self.device = as_device(device)
        # scheduling: force requests are admitted ahead of integrations, and a
        # tick that holds force requests takes integrations only up to
        # force_tick_bodies bodies (None: every active system runs every tick)
        self.force_tick_bodies = None if force_tick_bodies is None else int(force_tick_bodies)
        self.max_pause_ticks = int(max_pause_ticks)
        self.max_passed = int(max_passed)
        self.params = params if params is not None else default_params(**kw)
        self.hbm_budget = float(hbm_budget)
        self.max_tick_bodies = int(max_tick_bodies)
        self.max_tick_systems = int(min(max_tick_systems, max_tick_bodies))
        self.workspace_bytes = lanes * WORKSPACE_BYTES_PER_BODY * self.max_tick_bodies
        if self.workspace_bytes >= self.hbm_budget:
            raise ValueError("hbm_budget does not cover the lanes' workspaces")
        self._cv = threading.Condition()
        self._pending: collections.deque[Request] = collections.deque()
        self._resident = 0
        self.max_resident = 0
        self._stopping = False
        self._inflight = 0
        self._lane_error = None
        self.completed: list[Request] = []
        with torch.cuda.device(self.device):
            self.h2d = torch.cuda.Stream(self.device)
            self.d2h = torch.cuda.Stream(self.device)
        self.lanes = [_Lane(self, i) for i in range(lanes)]
        self._lane_bodies = [0] * lanes
        self._started = False

    @staticmethod
    def footprint(n: int) -> int:
        """Device bytes a request of n bodies holds while it is resident."""
        return RESIDENT_BYTES_PER_BODY * n

    # -- client side --
    def _check_fits(self, r: Request) -> None:
        if r.n > self.max_tick_bodies:
            raise ValueError(f"request of {r.n} bodies exceeds a lane's tick ({self.max_tick_bodies})")
        if self.footprint(r.n) > self.hbm_budget - self.workspace_bytes:
            raise ValueError("request larger than the HBM budget")

    def submit(self, r: Request) -> Request:
        self._check_fits(r)
        self.prepare(r)
        if r.arrival is None:
            r.arrival = time.perf_counter()
        with self._cv:
            self._pending.append(r)
            self._inflight += 1
            self._cv.notify_all()
        return r

    def submit_many(self, requests) -> list[Request]:
        """Submits requests that arrive together: all are checked and prepared
        first, then queued at once, so the lanes see the whole group when they
        wake.  (Submitting them one by one lets the lanes start ticks on the
        first arrivals while the client, competing with them for the
        interpreter lock, is still submitting the rest: fewer systems per tick
        and idle gaps on the device.)  Arrival times not set are set to the
        moment of queueing."""
        rs = list(requests)
        for r in rs:
            self._check_fits(r)
        for r in rs:
            self.prepare(r)
        now = time.perf_counter()
        for r in rs:
            if r.arrival is None:
                r.arrival = now
        with self._cv:
            self._pending.extend(rs)
            self._inflight += len(rs)
            self._cv.notify_all()
        return rs

    @staticmethod
    def prepare(r: Request) -> Request:
        """Puts a request's inputs where the server reads them (pinned host
        buffers for host arrays) and allocates its pinned result buffers.  A
        client that prepares its requests ahead of time keeps these copies
        out of the requests' latency; ``submit`` prepares the others."""
        if getattr(r, "_pinned", None) is not None:
            return r
        Server._pin(r)
        return r

    @staticmethod
    def _pin(r: Request):
        if r.on_device:
            # the inputs are read in place; the result buffers are allocated
            # here, on the client's thread, so a lane's tick allocates nothing
            q = r.q if r.q.shape[0] == 3 else r.q.T
            d = {"m": r.m, "x": q[0], "y": q[1], "z": q[2]}
            dev, f64 = r.m.device, torch.float64
            if r.kind == "leapfrog":
                p = r.p if r.p.shape[0] == 3 else r.p.T
                d.update(px=p[0], py=p[1], pz=p[2])
                r._dev_result = {k: torch.empty(r.n, dtype=f64, device=dev) for k in _ROWS[1:]}
            else:
                r._dev_result = {"f": torch.empty(3, r.n, dtype=f64, device=dev)}
            r._pinned = d
            return

        def pin(a):
            t = torch.empty(len(a), dtype=torch.float64, pin_memory=True)
            t.numpy()[:] = a
            return t

        m = np.asarray(r.m, np.float64)
        q = np.asarray(r.q, np.float64)
        host = {"m": pin(m), "x": pin(q[:, 0]), "y": pin(q[:, 1]), "z": pin(q[:, 2])}
        if r.kind == "leapfrog":
            p = np.asarray(r.p, np.float64)
            host.update(px=pin(p[:, 0]), py=pin(p[:, 1]), pz=pin(p[:, 2]))
            r._host_out = {k: torch.empty(r.n, dtype=torch.float64, pin_memory=True)
                           for k in ("x", "y", "z", "px", "py", "pz")}
        else:
            r._host_out = {"f": torch.empty(3 * r.n, dtype=torch.float64, pin_memory=True)}
        r._pinned = host

    def start(self) -> "Server":
        if not self._started:
            self._started = True
            for ln in self.lanes:
                ln.thread.start()
                ln.finisher.start()
        return self

    def drain(self, timeout: float | None = None) -> None:
        """Waits until every submitted request has finished."""
        t_end = None if timeout is None else time.perf_counter() + timeout
        with self._cv:
            while self._inflight > 0:
                if self._lane_error is not None:
                    raise RuntimeError(f"lane failed: {self._lane_error}")
                left = None if t_end is None else t_end - time.perf_counter()
                if left is not None and left <= 0:
                    raise TimeoutError("requests still running")
                self._cv.wait(0.05 if left is None else min(0.05, left))

    def stop(self) -> None:
        with self._cv:
            self._stopping = True
            self._cv.notify_all()
        for ln in self.lanes:
            if ln.thread.is_alive():
                ln.thread.join()
            if ln.finisher.is_alive():
                ln.finisher.join()
        # free the lanes' device memory now, at a known point, rather than
        # whenever the garbage collector reaches the server
        torch.cuda.synchronize(self.device)
        for ln in self.lanes:
            ln.close()

    def __enter__(self):
        return self.start()

    def __exit__(self, *a):
        self.stop()

    # -- lane side --
    def _idle(self) -> bool:
        return not self._pending

    def _admit(self, lane: _Lane) -> list[Request]:
        """Admission of pending requests into this lane while they fit the HBM
        budget and the lane's tick capacity: force requests first, then
        integrations, FIFO within each kind.  A request that does not fit is
        passed over for later ones that do; once it has been passed over
        ``max_passed`` times nothing behind it is admitted until it fits."""
        out = []
        with self._cv:
            room = self.hbm_budget - self.workspace_bytes
            bodies = sum(r.n for r in lane.active)
            systems = len(lane.active)
            order = sorted(range(len(self._pending)),
                           key=lambda i: (self._pending[i].kind != "force", i))
            taken = set()
            for i in order:
                r = self._pending[i]
                fp = self.footprint(r.n)
                if (self._resident + fp > room or bodies + r.n > self.max_tick_bodies
                        or systems + 1 > self.max_tick_systems):
                    r._passed += 1
                    if r._passed > self.max_passed:
                        break
                    continue
                systems += 1
                taken.add(i)
                self._resident += fp
                self.max_resident = max(self.max_resident, self._resident)
                bodies += r.n
                r.t_admit = time.perf_counter()
                r.lane = lane.index
                out.append(r)
            if taken:
                self._pending = collections.deque(
                    r for i, r in enumerate(self._pending) if i not in taken)
        return out

    def _release(self, r: Request):
        with self._cv:
            self._resident -= self.footprint(r.n)
            self._inflight -= 1
            self.completed.append(r)
            self._cv.notify_all()

    # -- reporting --
    def metrics(self, requests=None) -> dict:
        rs = [r for r in (requests if requests is not None else self.completed)
              if r.t_done is not None and r.error is None]
        if not rs:
            return {}
        lat = np.array([r.latency for r in rs]) * 1e3
        t0 = min(r.arrival for r in rs)
        t1 = max(r.t_done for r in rs)
        forces = sum(r.n * r.evals_needed for r in rs)
        host_ms, dev_ms, gap_ms = [], [], []
        for ln in self.lanes:
            prev = None
            for h, b, e in ln.tick_log:
                if not e.query():
                    continue
                host_ms.append(h * 1e3)
                dev_ms.append(b.elapsed_time(e))
                if prev is not None:
                    gap_ms.append(prev.elapsed_time(b))  # device idle of the lane between ticks
                prev = e
        ticks = {"host_ms_mean": float(np.mean(host_ms)) if host_ms else None,
                 "device_ms_mean": float(np.mean(dev_ms)) if dev_ms else None,
                 "device_ms_max": float(np.max(dev_ms)) if dev_ms else None,
                 "lane_gap_ms_mean": float(np.mean(gap_ms)) if gap_ms else None,
                 "lane_gap_ms_max": float(np.max(gap_ms)) if gap_ms else None}
        by_kind = {}
        for kind in ("force", "leapfrog"):
            lk = np.array([r.latency for r in rs if r.kind == kind]) * 1e3
            if lk.size:
                by_kind[kind] = {"requests": int(lk.size), "p50_ms": float(np.percentile(lk, 50)),
                                 "p99_ms": float(np.percentile(lk, 99))}
        return {"requests": len(rs), "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                "by_kind": by_kind,
                "paused_ticks": sum(ln.paused_ticks for ln in self.lanes),
                "wall_s": t1 - t0, "forces": int(forces), "forces_per_s": forces / (t1 - t0),
                "ticks": sum(ln.ticks for ln in self.lanes),
                "mean_tick_bodies": sum(ln.tick_bodies for ln in self.lanes)
                / max(1, sum(ln.ticks for ln in self.lanes)),
                "max_resident_bytes": self.max_resident, "tick_times": ticks}
