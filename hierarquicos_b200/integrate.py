"""Device-resident time integration of batches of systems.

Replaces the reference's integrators that call the force path:
velocity Verlet in momentum form (benchmarks/integration_verlet/integration.f90:
110-172, and the fine propagator ``F_til`` of parareal/parareal.f90:43-68) and
the symplectic Euler coarse propagator ``G_til`` (parareal/parareal.f90:8-41).
The state (positions, momenta, masses) stays on the device in FP64; forces
come from the Barnes-Hut engine (one build + walk per step for the whole
batch) or from the FP64 direct sum.  The kick and drift updates run in one
kernel with the reference's operation order (see ``bh_kick_drift``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import BH_ERR_NOT_BUILT, BHError, BHParams, check, default_params, lib
from .system import BHSystem, _dptr, _stream, offsets_of


class BatchState:
    """Positions, momenta and masses of a batch of systems, on the device.

    ``q``/``p`` are (3, N) float64 tensors (rows x, y, z; N = all bodies of all
    systems, concatenated by system), ``m`` is (N,), ``offsets`` the nsys + 1
    host offsets."""

    def __init__(self, m, q, p, offsets, device=None):
        dev = as_device(device)
        self.device = dev
        self.m = torch.as_tensor(np.ascontiguousarray(m, np.float64), device=dev) \
            if not isinstance(m, torch.Tensor) else m.to(dev, torch.float64).contiguous()
        self.q = _rows(q, dev)
        self.p = _rows(p, dev)
        n = self.m.numel()
        self.offsets = np.ascontiguousarray(offsets, np.int64)
        if self.offsets[0] != 0 or self.offsets[-1] != n:
            raise ValueError("offsets must be [0, ..., N]")
        self.d_offsets = torch.as_tensor(self.offsets, device=dev)
        self.n = n
        self.nsys = self.offsets.size - 1

    @classmethod
    def single(cls, m, q, p, device=None):
        return cls(m, q, p, [0, len(m)], device)

    def system(self, s):
        """(m, q (n_s,3), p (n_s,3)) of system s, as numpy arrays."""
        a, b = self.offsets[s], self.offsets[s + 1]
        return (self.m[a:b].cpu().numpy(), self.q[:, a:b].T.cpu().numpy(),
                self.p[:, a:b].T.cpu().numpy())

    def clone(self) -> "BatchState":
        c = object.__new__(BatchState)
        c.__dict__.update(self.__dict__)
        c.q = self.q.clone()
        c.p = self.p.clone()
        return c


def as_device(device=None) -> torch.device:
    """A CUDA device from None (the current one), an index or a torch.device."""
    if isinstance(device, torch.device):
        return device if device.index is not None else torch.device(
            "cuda", torch.cuda.current_device())
    return torch.device("cuda", torch.cuda.current_device() if device is None else int(device))


def _rows(a, dev) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        t = a.to(dev, torch.float64).clone()  # the state is the integrator's own
    else:
        t = torch.as_tensor(np.asarray(a, np.float64), device=dev)
    if t.shape[0] != 3:
        t = t.T
    return t.contiguous()


class ForceField:
    """Forces of a batch: Barnes-Hut (``kind='bh'``) or FP64 direct sum
    (``kind='direct'``), written in the walk's per-system block layout.

    With ``graph=True`` a Barnes-Hut field records its build + walk into a CUDA
    graph after the first evaluation of a state and replays it while it is
    called with the same state tensors, layout and output (an integrator
    stepping one state): one launch instead of one per kernel, for the small
    systems whose evaluation is launch-bound.  Every replay is followed by the
    same status check (strict keys, stack growth) as a plain call, and gives
    the same bits.  The graph writes into a buffer of the field's own, which
    is copied into the caller's output."""

    def __init__(self, kind: str = "bh", params: BHParams | None = None, device=None,
                 graph: bool = False, **kw):
        if kind not in ("bh", "direct"):
            raise ValueError("kind must be 'bh' or 'direct'")
        self.kind = kind
        self.params = params if params is not None else default_params(**kw)
        self.sys = BHSystem(as_device(device).index) if kind == "bh" else None
        self.graph = graph and kind == "bh"
        self._graph_key = None
        self._graph_out = None

    def __call__(self, st: BatchState, out: torch.Tensor) -> torch.Tensor:
        x, y, z = st.q[0], st.q[1], st.q[2]
        if self.kind == "bh":
            if not self.graph:
                return self.sys.forces_batch(st.m, x, y, z, st.offsets, self.params, out=out)
            # the graph writes into the field's own buffer (callers often hand
            # a fresh output per call), copied out afterwards
            key = (st.m.data_ptr(), x.data_ptr(), y.data_ptr(), z.data_ptr(), st.n,
                   st.offsets.tobytes(), bytes(self.params))  # changed parameters record anew
            if key == self._graph_key:
                try:
                    self.sys.replay()
                except BHError as e:
                    # a workspace that grew since (stack, layout) dropped the
                    # graph: evaluate normally and record it again
                    if e.code != BH_ERR_NOT_BUILT:
                        raise
                else:
                    self.sys.sync()
                    out.copy_(self._graph_out)
                    return out
            if self._graph_out is None or self._graph_out.numel() != 3 * st.n:
                self._graph_out = torch.empty(3 * st.n, dtype=torch.float64, device=out.device)
            self.sys.forces_batch(st.m, x, y, z, st.offsets, self.params, out=self._graph_out)
            self.sys.capture(self.params, self._graph_out)  # the next call replays it
            self._graph_key = key
            out.copy_(self._graph_out)
            return out
        p = self.params
        for s in range(st.nsys):
            a, b = int(st.offsets[s]), int(st.offsets[s + 1])
            check(lib().bh_direct_targets_device(
                _dptr(st.m[a:b]), _dptr(x[a:b]), _dptr(y[a:b]), _dptr(z[a:b]), b - a, None, b - a,
                p.G, p.eps, 0, _dptr(out[3 * a:3 * b]), _stream()))
        return out


def kick_drift(st: BatchState, f: torch.Tensor | None, kick1: float, kick2: float,
               drift: float) -> None:
    """p += kick1 f; p += kick2 f; q += (drift p) / m (each skipped when its
    coefficient is 0), for every body of the batch."""
    check(lib().bh_kick_drift(
        _dptr(st.m), _dptr(f) if f is not None else None, _dptr(st.q[0]), _dptr(st.q[1]),
        _dptr(st.q[2]), _dptr(st.p[0]), _dptr(st.p[1]), _dptr(st.p[2]), _dptr(st.d_offsets),
        st.nsys, st.n, kick1, kick2, drift, _stream()))


def verlet(st: BatchState, field: ForceField, nsteps: int, dt: float,
           f: torch.Tensor | None = None) -> torch.Tensor:
    """nsteps velocity-Verlet steps (parareal/parareal.f90:55-63).  ``f``, if
    given, holds the forces at the current positions (otherwise they are
    computed first).  Returns the forces at the final positions."""
    if f is None:
        f = torch.empty(3 * st.n, dtype=torch.float64, device=st.device)
        field(st, f)
    if nsteps <= 0:
        return f
    h = 0.5 * dt
    kick_drift(st, f, 0.0, h, dt)
    field(st, f)
    for _ in range(nsteps - 1):
        kick_drift(st, f, h, h, dt)
        field(st, f)
    kick_drift(st, f, h, 0.0, 0.0)
    return f


def symplectic_euler(st: BatchState, field: ForceField, nsteps: int, dt: float) -> None:
    """nsteps of the reference's coarse propagator (parareal/parareal.f90:20-35):
    forces, p += dt f, q += dt p / m."""
    f = torch.empty(3 * st.n, dtype=torch.float64, device=st.device)
    for _ in range(nsteps):
        field(st, f)
        kick_drift(st, f, dt, 0.0, dt)


def diagnostics(st: BatchState, G: float = 1.0, eps: float = 0.0) -> np.ndarray:
    """(nsys, 9): total energy, kinetic, potential, linear momentum (3),
    angular momentum (3) per system (parareal/api3d.f90:108-153)."""
    scratch = torch.empty(8 * st.n, dtype=torch.float64, device=st.device)
    out = torch.empty(9 * st.nsys, dtype=torch.float64, device=st.device)
    check(lib().bh_diagnostics(
        _dptr(st.m), _dptr(st.q[0]), _dptr(st.q[1]), _dptr(st.q[2]), _dptr(st.p[0]),
        _dptr(st.p[1]), _dptr(st.p[2]), _dptr(st.d_offsets), st.nsys, st.n, G, eps,
        _dptr(scratch), _dptr(out), _stream()))
    return out.view(st.nsys, 9).cpu().numpy()


__all__ = ["BatchState", "ForceField", "kick_drift", "verlet", "symplectic_euler", "diagnostics",
           "offsets_of"]
