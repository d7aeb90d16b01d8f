"""Device-resident Barnes-Hut systems over the C ABI.

``BHSystem`` owns one device workspace (``bh_system``) and runs the pipeline
on CUDA tensors: build (keys, radix sort, octree, multipoles, groups) and walk.
It replaces the reference's tree objects, ``OctreeType`` (pre_init + init +
forces_groups, fortran/octree_default.f90:178-387, 1811-1831) and
``morton_tree_type`` (init + forces_par, fortran/morton/morton_octree.f90:73-180);
thin mirrors of those two interfaces are ``MortonTree`` and ``Octree`` below.

PyTorch is used for device memory and the current stream only.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import BHParams, check, default_params, lib

ORDER_OF_METHOD = {10: 1, 11: 4, 12: 8, 20: 1, 21: 4, 22: 8, 30: 1, 31: 4, 32: 8}


def _dptr(t: torch.Tensor) -> int:
    assert t.is_cuda and t.is_contiguous()
    return t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _f64(a, device) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=device)


class BHSystem:
    """One device workspace; grows on demand, reused across calls."""

    def __init__(self, device: int | None = None):
        if device is None:
            device = torch.cuda.current_device()
        self.device = device
        h = C.c_void_p()
        check(lib().bh_system_create(C.byref(h), device))
        self._h = h
        self.n = 0
        self._inputs = None

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().bh_system_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- pipeline --
    def build(self, m, x, y, z, params: BHParams | None = None, **kw) -> "BHSystem":
        dev = torch.device("cuda", self.device)
        m, x, y, z = (_f64(a, dev) for a in (m, x, y, z))
        p = params if params is not None else default_params(**kw)
        self._inputs = (m, x, y, z)  # keep alive for the asynchronous build
        self.n = m.numel()
        check(lib().bh_system_build(self._h, _dptr(m), _dptr(x), _dptr(y), _dptr(z), self.n,
                                    C.byref(p), _stream()))
        return self

    def walk(self, params: BHParams | None = None, out: torch.Tensor | None = None,
             groups: tuple[int, int] | None = None, **kw):
        """Group walk into ``out``; ``groups=(g0, g1)`` walks only target groups
        [g0, g1) and leaves the other bodies' entries of ``out`` as they are."""
        p = params if params is not None else default_params(**kw)
        if out is None:
            out = torch.empty(3 * self.n, dtype=torch.float64, device=f"cuda:{self.device}")
        if groups is None:
            check(lib().bh_system_walk(self._h, C.byref(p), _dptr(out), _stream()))
        else:
            check(lib().bh_system_walk_groups(self._h, C.byref(p), int(groups[0]), int(groups[1]),
                                              _dptr(out), _stream()))
        return out

    def sync(self):
        check(lib().bh_system_sync(self._h, _stream()))

    def forces(self, m, x, y, z, params: BHParams | None = None, out=None, **kw) -> torch.Tensor:
        """Build + walk + sync; returns the SoA (3N,) float64 device tensor."""
        dev = torch.device("cuda", self.device)
        m, x, y, z = (_f64(a, dev) for a in (m, x, y, z))
        p = params if params is not None else default_params(**kw)
        n = m.numel()
        if out is None:
            out = torch.empty(3 * n, dtype=torch.float64, device=dev)
        self._inputs = (m, x, y, z)
        self.n = n
        check(lib().bh_system_forces(self._h, _dptr(m), _dptr(x), _dptr(y), _dptr(z), n,
                                     C.byref(p), _dptr(out), _stream()))
        return out

    def reserve(self, n: int, nsys: int = 1) -> "BHSystem":
        """Allocates the workspace for batches of up to n bodies in up to nsys
        systems, so that builds within those bounds allocate nothing."""
        check(lib().bh_system_reserve(self._h, int(n), int(nsys)))
        return self

    # -- batches of independent systems --
    def build_batch(self, m, x, y, z, offsets, params: BHParams | None = None,
                    **kw) -> "BHSystem":
        """Builds every system of a batch at once.  System s owns entries
        [offsets[s], offsets[s+1]) of the concatenated m, x, y, z."""
        dev = torch.device("cuda", self.device)
        m, x, y, z = (_f64(a, dev) for a in (m, x, y, z))
        off = _offsets(offsets, m.numel())
        p = params if params is not None else default_params(**kw)
        self._inputs = (m, x, y, z)
        self._offsets = off
        self.n = m.numel()
        check(lib().bh_system_build_batch(self._h, _dptr(m), _dptr(x), _dptr(y), _dptr(z),
                                          off.ctypes.data_as(C.c_void_p), off.size - 1,
                                          C.byref(p), _stream()))
        return self

    def forces_batch(self, m, x, y, z, offsets, params: BHParams | None = None, out=None,
                     **kw) -> torch.Tensor:
        """Build + walk + sync of a batch; returns the (3N,) float64 device
        tensor whose entries [3 off_s, 3 off_{s+1}) are system s's SoA forces."""
        dev = torch.device("cuda", self.device)
        m, x, y, z = (_f64(a, dev) for a in (m, x, y, z))
        off = _offsets(offsets, m.numel())
        p = params if params is not None else default_params(**kw)
        n = m.numel()
        if out is None:
            out = torch.empty(3 * n, dtype=torch.float64, device=dev)
        self._inputs = (m, x, y, z)
        self._offsets = off
        self.n = n
        check(lib().bh_system_forces_batch(self._h, _dptr(m), _dptr(x), _dptr(y), _dptr(z),
                                           off.ctypes.data_as(C.c_void_p), off.size - 1,
                                           C.byref(p), _dptr(out), _stream()))
        return out

    def batch_info(self) -> dict:
        nsys = self._offsets.size - 1
        roots = np.empty(nsys, np.int32)
        com4 = np.empty((nsys, 4))
        ssa = np.empty(nsys)
        check(lib().bh_system_batch_info(self._h, roots.ctypes.data_as(C.c_void_p),
                                         com4.ctypes.data_as(C.c_void_p),
                                         ssa.ctypes.data_as(C.c_void_p)))
        return dict(roots=roots, com=com4[:, :3], mass=com4[:, 3], ssa=ssa)

    def capture(self, params: BHParams, out: torch.Tensor) -> None:
        """Records build + walk of the current batch (same input tensors,
        layout and parameters) into a CUDA graph held by the handle."""
        self._graph_out = out
        check(lib().bh_system_capture(self._h, C.byref(params), _dptr(out)))

    def replay(self) -> None:
        check(lib().bh_system_replay(self._h, _stream()))

    # -- introspection --
    def info(self) -> dict:
        n, L, nn, ng = C.c_int64(), C.c_int(), C.c_int64(), C.c_int64()
        com4 = np.zeros(4)
        ssa = C.c_double()
        check(lib().bh_system_info(self._h, C.byref(n), C.byref(L), C.byref(nn), C.byref(ng),
                                   com4.ctypes.data_as(C.c_void_p), C.byref(ssa)))
        return dict(n=n.value, depth=L.value, n_nodes=nn.value, n_groups=ng.value, com=com4[:3],
                    mass=com4[3], ssa=ssa.value)

    def keys(self):
        keys = np.empty(self.n, np.uint64)
        perm = np.empty(self.n, np.int32)
        check(lib().bh_system_get_keys(self._h, keys.ctypes.data_as(C.c_void_p),
                                       perm.ctypes.data_as(C.c_void_p)))
        return keys, perm

    def nodes(self) -> dict:
        info = self.info()
        M = info["n_nodes"]
        d = dict(meta=np.empty((M, 4), np.int32), child=np.empty((M, 8), np.int32),
                 parent=np.empty(M, np.int32), com=np.empty((M, 4)), quad=np.zeros((M, 6)),
                 oct=np.zeros((M, 14)), level_begin=np.zeros(info["depth"] + 2, np.int32))
        check(lib().bh_system_get_nodes(self._h, *[d[k].ctypes.data_as(C.c_void_p) for k in
                                                   ("meta", "child", "parent", "com", "quad",
                                                    "oct", "level_begin")]))
        return d

    def groups(self) -> np.ndarray:
        ng = self.info()["n_groups"]
        g = np.empty(ng + 1, np.int32)
        check(lib().bh_system_get_groups(self._h, g.ctypes.data_as(C.c_void_p)))
        return g

    def key_checks(self) -> tuple[int, int]:
        """(sequential centre-of-mass checks, rebuilds) of the strict-key path
        since this handle was created."""
        c = np.zeros(2, np.int64)
        check(lib().bh_system_get_key_checks(self._h, c.ctypes.data_as(C.c_void_p)))
        return int(c[0]), int(c[1])

    def stats(self) -> np.ndarray:
        s = np.zeros(4, np.uint64)
        check(lib().bh_system_get_stats(self._h, s.ctypes.data_as(C.c_void_p)))
        return s

    def reference_targets(self, targets, params: BHParams | None = None, counts: bool = False,
                          **kw):
        """Per-target FP64 walk with the reference's MAC (original indices).

        Returns (forces (k,3) float64 numpy[, counts (k,2) body-body, cell])."""
        dev = torch.device("cuda", self.device)
        t = torch.as_tensor(np.ascontiguousarray(targets, dtype=np.int64), device=dev)
        k = t.numel()
        p = params if params is not None else default_params(**kw)
        out = torch.empty(3 * k, dtype=torch.float64, device=dev)
        cnt = torch.empty(2 * k, dtype=torch.int64, device=dev) if counts else None
        check(lib().bh_system_reference_targets(self._h, C.byref(p), _dptr(t), k, _dptr(out),
                                                _dptr(cnt) if counts else None, _stream()))
        f = out.view(3, k).T.cpu().numpy()
        if counts:
            return f, cnt.view(k, 2).cpu().numpy()
        return f


def _offsets(offsets, n: int) -> np.ndarray:
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    if off.ndim != 1 or off.size < 2 or off[0] != 0 or off[-1] != n:
        raise ValueError("offsets must be [0, ..., N] with N the total number of bodies")
    return off


def offsets_of(sizes) -> np.ndarray:
    """Batch offsets from the system sizes."""
    return np.concatenate([[0], np.cumsum(np.asarray(sizes, np.int64))]).astype(np.int64)


def direct_targets(m, x, y, z, targets=None, G: float = 1.0, eps: float = 0.0,
                   out_kind: int = 0) -> torch.Tensor:
    """FP64 direct sum on the device for the given ORIGINAL target indices (all
    if None); returns a (3, k) float64 device tensor."""
    dev = m.device if isinstance(m, torch.Tensor) and m.is_cuda else torch.device("cuda")
    m, x, y, z = (_f64(a, dev) for a in (m, x, y, z))
    n = m.numel()
    if targets is None:
        t = None
        k = n
    else:
        t = torch.as_tensor(np.ascontiguousarray(targets, dtype=np.int64), device=dev) \
            if not isinstance(targets, torch.Tensor) else targets.to(dev, torch.int64).contiguous()
        k = t.numel()
    out = torch.empty(3 * k, dtype=torch.float64, device=dev)
    check(lib().bh_direct_targets_device(_dptr(m), _dptr(x), _dptr(y), _dptr(z), n,
                                         _dptr(t) if t is not None else None, k, G, eps, out_kind,
                                         _dptr(out), _stream()))
    return out.view(3, k)


class MortonTree:
    """Mirror of morton_tree_type (morton_octree.f90:46-180).

    ``MortonTree(N, ms, qs, L, ssa, use_quadrupole)`` builds the tree (qs is
    (3,N) like the Fortran or (N,3)); ``forces_par(G, eps2, theta2, mult_par)``
    returns forces (3,N) in the original order, as the Fortran function does."""

    def __init__(self, N, ms, qs, L: int = 21, ssa: float = 1.2, use_quadrupole: bool = True,
                 **kw):
        qs = np.asarray(qs, np.float64)
        if qs.shape == (3, N):
            qs = qs.T
        self.N = N
        self.use_quadrupole = use_quadrupole
        self.sys = BHSystem()
        self._kw = kw
        self.params = default_params(depth=L, amp=ssa, order=4 if use_quadrupole else 1, **kw)
        self.sys.build(ms, qs[:, 0], qs[:, 1], qs[:, 2], self.params)
        self.sys.sync()
        self.depth = self.sys.info()["depth"]

    def forces_par(self, G: float, eps2: float, theta2: float, mult_par: bool | None = None,
                   num_threads: int | None = None) -> np.ndarray:
        mult = self.use_quadrupole if mult_par is None else mult_par
        p = default_params(**self._kw)
        p.depth, p.amp = self.params.depth, self.params.amp
        p.theta, p.G, p.eps = float(np.sqrt(theta2)), G, float(np.sqrt(eps2))
        p.order = 4 if mult else 1
        out = self.sys.walk(p)
        self.sys.sync()
        return out.view(3, self.N).cpu().numpy()

    forces_seq = forces_par


class Octree:
    """Mirror of OctreeType's force methods (octree_default.f90:90-170).

    ``pre_init(m, method, group_size=64)`` with method 10/11/12 (classic BH,
    monopole/quadrupole/octupole), 20/21/22 (Dehnen's dual-tree method) or
    30/31/32 (grouped BH); ``init(x, y, z)``; ``forces_groups(theta2, G, eps2)``
    (and ``dehnen_eval(theta2, eps2, G)`` for 20-22) returns forces (3,N).
    Methods 10-12 run the per-target reference walk, 20-22 the device dual
    traversal, 30-32 the warp-cooperative group walk."""

    def __init__(self):
        self.sys = None

    def pre_init(self, m, method: int = 31, collide: bool = False, radii=None,
                 group_size: int = 64):
        if method not in ORDER_OF_METHOD:
            raise ValueError(f"method {method} not identified (10-12, 20-22, 30-32)")
        self.m = np.ascontiguousarray(m, np.float64)
        self.N = self.m.size
        self.method = method
        self.multipole = ORDER_OF_METHOD[method]
        self.group_size = 64 if group_size > 32 else 32
        self.sys = BHSystem()
        return self

    def init(self, x, y, z):
        if self.sys is None:
            raise RuntimeError("Not allocated! Run pre_init first!")
        p = default_params(order=self.multipole, group_size=self.group_size)
        self.sys.build(self.m, x, y, z, p)
        self.sys.sync()
        return self

    def dehnen_eval(self, theta2: float, potsoft2: float, G: float, forces=None, nt_par=None):
        """octree_default.f90:1676-1712 (dehnen_eval): argument order as there."""
        if self.method not in (20, 21, 22):
            raise ValueError("dehnen_eval needs method 20, 21 or 22")
        return self.forces_groups(theta2, G, potsoft2, forces)

    def forces_groups(self, theta2: float, G: float, eps2: float, forces=None, nt=None):
        prec = {1: _lib.BH_PREC_REFERENCE, 2: _lib.BH_PREC_DEHNEN, 3: _lib.BH_PREC_FP32}[
            self.method // 10]
        p = default_params(order=self.multipole, group_size=self.group_size, precision=prec,
                           theta=float(np.sqrt(theta2)), G=G, eps=float(np.sqrt(eps2)))
        out = self.sys.walk(p)
        self.sys.sync()
        f = out.view(3, self.N).cpu().numpy()
        if forces is not None:
            forces[...] = f
        return f
