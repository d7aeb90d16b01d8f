"""Parareal on the device, with every window's fine propagator in one batch.

Mirrors ``integrate_parareal`` (parareal/parareal.f90:97-186): windows of
length tf / num_windows; an initial coarse sweep U_0; then per iteration the
fine propagator F of every window started from the previous iterate, and the
sequential correction

    U_{k+1,i+1} = (G(U_{k+1,i}) + F(U_{k,i})) - G(U_{k,i}),

with the error NORM2(U_{k+1,last} - U_{k,last}) / (6 N) and the stop at
error <= maxerror.  The reference's propagators are ``G_til`` (symplectic
Euler, Barnes-Hut quadrupole, one step of the window length) and ``F_til``
(velocity Verlet, FP64 direct forces, qntt steps); both are ``Propagator``
choices here, and so is a Barnes-Hut fine propagator.

B200 design: the windows are independent systems, so the fine propagators of
all windows run as ONE batch -- each fine step is one build and one walk over
num_windows - 1 systems -- and the coarse values G(U_{k,i}) of the previous
sweep are kept, so each iteration runs one sequential coarse sweep.  State
and correction are FP64 on the device (the reference uses REAL(16); FP64
limits how far below ~1e-16 relative the iterates can settle, but the
iteration becomes exactly stationary once a window's input stops changing,
because every propagator here is deterministic bit for bit).  The correction
can also be carried in double-double (``correction="dd"``).
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np
import torch

from ._lib import default_params
from .integrate import BatchState, ForceField, as_device, symplectic_euler, verlet


@dataclasses.dataclass
class Propagator:
    """One window of integration: ``scheme`` 'verlet' or 'euler', ``steps``
    steps of window / steps each, forces ``kind`` 'bh' (theta, order) or
    'direct'."""

    scheme: str = "verlet"
    kind: str = "direct"
    steps: int = 16
    theta: float = 0.5
    order: int = 4
    precision: int = 0

    def field(self, G: float, eps: float, device=None, graph: bool = False) -> ForceField:
        p = default_params(theta=self.theta, G=G, eps=eps, order=self.order,
                           precision=self.precision)
        return ForceField(self.kind, p, device, graph=graph)

    def run(self, st: BatchState, field: ForceField, window: float) -> None:
        dt = window / self.steps
        if self.scheme == "verlet":
            verlet(st, field, self.steps, dt)
        elif self.scheme == "euler":
            symplectic_euler(st, field, self.steps, dt)
        else:
            raise ValueError(f"unknown scheme {self.scheme!r}")


def reference_coarse(theta: float) -> Propagator:
    """G_til of the reference: one symplectic Euler step per window, BH quadrupole."""
    return Propagator("euler", "bh", 1, theta, 4)


def reference_fine(qntt: int) -> Propagator:
    """F_til of the reference: qntt velocity-Verlet steps, FP64 direct forces."""
    return Propagator("verlet", "direct", qntt)


@dataclasses.dataclass
class PararealResult:
    q: np.ndarray            # (num_windows, N, 3): state at the start of each window
    p: np.ndarray
    errors: list
    iterations: int
    seconds: float
    converged: bool
    iteration_seconds: list = dataclasses.field(default_factory=list)
    q_lo: np.ndarray | None = None  # correction "dd": low parts of the state (q + q_lo)
    p_lo: np.ndarray | None = None


def _two_sum(a: torch.Tensor, b: torch.Tensor):
    """s + e = a + b exactly, s = fl(a + b) (Knuth's TwoSum; every torch
    elementwise operation here is one separately rounded FP64 operation)."""
    s = a + b
    bb = s - a
    e = (a - (s - bb)) + (b - bb)
    return s, e


def _dd_correction(g: torch.Tensor, f: torch.Tensor, g_old: torch.Tensor):
    """(G(U_{k+1}) + F(U_k)) - G(U_k) of parareal.f90:153-156 in double-double:
    the three FP64 terms are added with TwoSum and the result is returned as
    a normalised pair (hi, lo) with hi + lo within 2^-104 relative of the exact
    sum (hi is the exact sum rounded to FP64 up to one ulp)."""
    s, e1 = _two_sum(g, f)
    t, e2 = _two_sum(s, -g_old)
    lo = e1 + e2
    hi = t + lo
    lo = lo - (hi - t)
    return hi, lo


def _window(st: BatchState, i: int, n: int):
    return slice(i * n, (i + 1) * n)


def integrate_parareal(m, q0, p0, tf: float, num_windows: int, n_itermax: int, theta: float,
                       G: float, eps: float, maxerror: float, qntt: int,
                       coarse: Propagator | None = None, fine: Propagator | None = None,
                       verbose: bool = False, device=None,
                       correction: str = "fp64") -> PararealResult:
    """Parareal with the reference's arguments (parareal/parareal.f90:97);
    ``coarse``/``fine`` default to the reference's G_til / F_til.

    ``correction`` "fp64" evaluates the update (G_new + F) - G_old in FP64 as
    the source text reads; "dd" evaluates it exactly (double-double, see
    _dd_correction) and keeps each window's state as an FP64 pair hi + lo: the
    propagators start from hi, the error norm is taken on hi + lo, and the
    low parts are returned in q_lo / p_lo.  The reference works in REAL(16)
    (113-bit significand); the pair carries 106 bits of the state between
    iterations while the propagators themselves stay FP64."""
    if correction not in ("fp64", "dd"):
        raise ValueError("correction must be 'fp64' or 'dd'")
    dd = correction == "dd"
    coarse = coarse or reference_coarse(theta)
    fine = fine or reference_fine(qntt)
    dev = as_device(device)
    m = np.ascontiguousarray(m, np.float64)
    n = m.size
    W = num_windows
    window = tf / W
    # the coarse propagator steps one scratch state window after window:
    # its evaluations replay one recorded graph
    cfield = coarse.field(G, eps, dev, graph=True)
    ffield = fine.field(G, eps, dev)

    # U[k]: all windows' starting states, one batch of W systems
    offs = np.arange(W + 1, dtype=np.int64) * n
    mW = np.tile(m, W)
    U = BatchState(mW, np.zeros((3, W * n)), np.zeros((3, W * n)), offs, dev)
    tq0 = torch.as_tensor(np.asarray(q0, np.float64).T.copy(), device=dev)
    tp0 = torch.as_tensor(np.asarray(p0, np.float64).T.copy(), device=dev)
    U.q[:, :n] = tq0
    U.p[:, :n] = tp0
    one = BatchState.single(m, tq0, tp0, dev)  # scratch for the coarse sweep

    def coarse_of(q, p):
        one.q.copy_(q)
        one.p.copy_(p)
        coarse.run(one, cfield, window)
        return one.q.clone(), one.p.clone()

    # initial coarse sweep; G(U_{0,i}) = U_{0,i+1}
    for i in range(W - 1):
        gq, gp = coarse_of(U.q[:, _window(U, i, n)], U.p[:, _window(U, i, n)])
        U.q[:, _window(U, i + 1, n)] = gq
        U.p[:, _window(U, i + 1, n)] = gp
    Gq_old = U.q[:, n:].clone()
    Gp_old = U.p[:, n:].clone()

    fin_offs = np.arange(W, dtype=np.int64) * n
    mW1 = U.m[:(W - 1) * n]
    q_lo = torch.zeros_like(U.q)  # low parts of the state (correction "dd")
    p_lo = torch.zeros_like(U.p)
    errors = []
    it_seconds = []
    iterations = 1
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    converged = False
    for _ in range(n_itermax - 1):
        iterations += 1
        t_it = time.perf_counter()
        # fine propagators of windows 0..W-2, one batch
        Fst = BatchState(mW1, U.q[:, :(W - 1) * n].contiguous(),
                         U.p[:, :(W - 1) * n].contiguous(), fin_offs, dev)
        fine.run(Fst, ffield, window)
        # sequential correction
        Uq = U.q.clone()
        Up = U.p.clone()
        Uq_lo = q_lo.clone()
        Up_lo = p_lo.clone()
        Gq_new = torch.empty_like(Gq_old)
        Gp_new = torch.empty_like(Gp_old)
        for i in range(W - 1):
            w = _window(U, i, n)
            gq, gp = coarse_of(Uq[:, w], Up[:, w])
            Gq_new[:, w] = gq
            Gp_new[:, w] = gp
            w1 = _window(U, i + 1, n)
            if dd:
                Uq[:, w1], Uq_lo[:, w1] = _dd_correction(gq, Fst.q[:, w], Gq_old[:, w])
                Up[:, w1], Up_lo[:, w1] = _dd_correction(gp, Fst.p[:, w], Gp_old[:, w])
            else:
                Uq[:, w1] = (gq + Fst.q[:, w]) - Gq_old[:, w]
                Up[:, w1] = (gp + Fst.p[:, w]) - Gp_old[:, w]
        last = _window(U, W - 1, n)
        if dd:
            # (hi + lo) - (hi' + lo'): the hi difference is exact for close
            # values (Sterbenz), the lo difference is far below it
            dq = (Uq[:, last] - U.q[:, last]) + (Uq_lo[:, last] - q_lo[:, last])
            dp = (Up[:, last] - U.p[:, last]) + (Up_lo[:, last] - p_lo[:, last])
        else:
            dq = Uq[:, last] - U.q[:, last]
            dp = Up[:, last] - U.p[:, last]
        d = torch.cat([dq.reshape(-1), dp.reshape(-1)])
        err = float(torch.sqrt(torch.sum(d * d))) / (6 * n)
        errors.append(err)
        U.q.copy_(Uq)
        U.p.copy_(Up)
        q_lo, p_lo = Uq_lo, Up_lo
        Gq_old, Gp_old = Gq_new, Gp_new
        it_seconds.append(time.perf_counter() - t_it)  # float() above synchronised
        if verbose:
            print(f"Iter.: {iterations:4d} / Error: {err:12.4e}", flush=True)
        if err <= maxerror:
            converged = True
            break
    torch.cuda.synchronize(dev)
    seconds = time.perf_counter() - t0
    q = U.q.T.reshape(W, n, 3).cpu().numpy()
    p = U.p.T.reshape(W, n, 3).cpu().numpy()
    res = PararealResult(q, p, errors, iterations, seconds, converged, it_seconds)
    if dd:
        res.q_lo = q_lo.T.reshape(W, n, 3).cpu().numpy()
        res.p_lo = p_lo.T.reshape(W, n, 3).cpu().numpy()
    return res


def sequential_fine(m, q0, p0, tf: float, num_windows: int, fine: Propagator, G: float,
                    eps: float, device=None):
    """The fine propagator run window after window (the exact solution that
    Parareal converges to): states at the start of every window."""
    dev = as_device(device)
    m = np.ascontiguousarray(m, np.float64)
    st = BatchState.single(m, np.asarray(q0, np.float64).T, np.asarray(p0, np.float64).T, dev)
    field = fine.field(G, eps, dev, graph=True)  # one state stepped throughout: replayed
    qs, ps = [st.q.T.cpu().numpy()], [st.p.T.cpu().numpy()]
    for _ in range(num_windows - 1):
        fine.run(st, field, tf / num_windows)
        qs.append(st.q.T.cpu().numpy())
        ps.append(st.p.T.cpu().numpy())
    return np.stack(qs), np.stack(ps)
