"""CPU oracle for the Barnes-Hut force path -- TEST INFRASTRUCTURE ONLY.

A ctypes wrapper around ``bh_oracle.c``, the C restatement of the reference's
Fortran (fortran/morton/morton_octree.f90, fortran/octree_default.f90,
fortran/direct_forces.f90).  Only the tests, the smoke check and the benchmark's
CPU-baseline leg import this package, and only as the checker; the product
library never does.

Parity pinning: the reference itself cannot be compiled here (no Fortran
compiler) and its own tests store no expected keys, topologies or forces, so
this oracle is pinned statistically against the force-error statistics the
reference recorded (benchmarks/forces_time_and_error/out/), not bit-for-bit.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libbh_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(
        os.path.join(_HERE, "bh_oracle.c")
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def _host_tag() -> str:
    """The CPU model and flags of this host, hashed: a -march=native build is
    only valid on a host with the same tag."""
    import hashlib
    import platform

    info = platform.machine()
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith(("model name", "flags")):
                    info += line
                if line.startswith("flags"):
                    break
    except OSError:
        pass
    return hashlib.sha1(info.encode()).hexdigest()[:12]


def use_native_build() -> str:
    """Switches this process to the timed CPU-baseline build of the same
    source (the reference's flags: -O3 -march=native -fopenmp, contraction
    allowed), compiled for this host on first use.  Call before anything
    else in the process uses the oracle; the parity checks use the default
    build."""
    global _SO
    if _lib is not None:
        raise RuntimeError("use_native_build() must come before the oracle is first loaded")
    rel = os.path.join("_build", f"native-{_host_tag()}")
    so = os.path.join(_HERE, rel, "libbh_oracle.so")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(
            os.path.join(_HERE, "bh_oracle.c")):
        subprocess.run(["make", "-s", "-C", _HERE, "fast", f"FASTDIR={rel}"], check=True)
    _SO = so
    return so


def lib():
    global _lib
    if _lib is None:
        if _SO.endswith(os.path.join("_build", "libbh_oracle.so")):
            build()
        L = C.CDLL(_SO)
        L.orc_last_error.restype = C.c_char_p
        L.orc_argsort.argtypes = [C.c_int64, _u64p, _i32p]
        L.orc_morton_keys.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, C.c_int, C.c_double, C.c_int,
                                      _u64p, C.POINTER(C.c_int), _dp, C.POINTER(C.c_double)]
        L.orc_morton_build.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, C.c_int, C.c_double, C.c_int,
                                       C.c_int, C.POINTER(C.c_void_p)]
        L.orc_morton_free.argtypes = [C.c_void_p]
        L.orc_morton_info.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int),
                                      C.POINTER(C.c_double), _dp]
        L.orc_morton_get_sorted.argtypes = [C.c_void_p, _u64p, _i32p]
        L.orc_morton_get_levels.argtypes = [C.c_void_p, _i64p, _i64p]
        L.orc_morton_get_nodes.argtypes = [C.c_void_p] + [C.c_void_p] * 12
        L.orc_morton_forces.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int,
                                        _dp, C.c_int]
        L.orc_morton_octupoles.argtypes = [C.c_void_p]
        L.orc_morton_forces_targets.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                                C.c_int, C.c_int64, _i64p, _dp, C.c_void_p, C.c_int]
        L.orc_morton_dehnen.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int,
                                        _dp, C.POINTER(C.c_int64)]
        L.orc_octree_create.argtypes = [C.c_int64, _dp, C.c_int, C.c_int, C.c_int64,
                                        C.POINTER(C.c_void_p)]
        L.orc_octree_init.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_octree_free.argtypes = [C.c_void_p]
        L.orc_octree_info.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int64)]
        L.orc_octree_get_nodes.argtypes = [C.c_void_p] + [C.c_void_p] * 11
        L.orc_octree_forces.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _dp, C.c_int]
        L.orc_octree_forces_targets.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                                C.c_int64, _i64p, _dp, C.c_void_p, C.c_int]
        L.orc_direct_forces.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, C.c_double, C.c_double, _dp]
        L.orc_direct_forces_targets.argtypes = [C.c_int64, _dp, _dp, _dp, _dp, C.c_double,
                                                C.c_double, C.c_int64, _i64p, _dp, C.c_int]
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _check(rc: int) -> None:
    if rc != 0:
        raise OracleError(f"oracle error {rc}: {lib().orc_last_error().decode()}")


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def num_threads() -> int:
    return int(lib().orc_num_threads())


def argsort(keys) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    perm = np.empty(keys.size, np.int32)
    _check(lib().orc_argsort(keys.size, keys, perm))
    return perm


def morton_keys(m, x, y, z, L: int = 21, ssa: float = 1.2, fma_mode: int = 0):
    """Keys in original order (morton_octree.f90:359-395).

    Returns (keys, L, com4, ssa_scaled)."""
    m, x, y, z = map(_f64, (m, x, y, z))
    n = m.size
    keys = np.empty(n, np.uint64)
    Lout = C.c_int(0)
    com4 = np.zeros(4)
    ssa_out = C.c_double(0.0)
    _check(lib().orc_morton_keys(n, m, x, y, z, L, ssa, fma_mode, keys, C.byref(Lout), com4,
                                 C.byref(ssa_out)))
    return keys, Lout.value, com4, ssa_out.value


class MortonTree:
    """morton_tree_type (morton_octree.f90:46-111): init + forces_par."""

    def __init__(self, m, x, y, z, L: int = 21, ssa: float = 1.2, use_quadrupole: bool = True,
                 fma_mode: int = 0):
        m, x, y, z = map(_f64, (m, x, y, z))
        self.n = m.size
        h = C.c_void_p()
        _check(lib().orc_morton_build(self.n, m, x, y, z, L, ssa, fma_mode, int(use_quadrupole),
                                      C.byref(h)))
        self._h = h
        nn = C.c_int64(0)
        Lc = C.c_int(0)
        s = C.c_double(0)
        com4 = np.zeros(4)
        lib().orc_morton_info(h, C.byref(nn), C.byref(Lc), C.byref(s), com4)
        self.nnodes, self.L, self.ssa, self.com4 = nn.value, Lc.value, s.value, com4

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.orc_morton_free(h)
            self._h = None

    def sorted(self):
        keys = np.empty(self.n, np.uint64)
        perm = np.empty(self.n, np.int32)
        lib().orc_morton_get_sorted(self._h, keys, perm)
        return keys, perm

    def levels(self):
        b = np.empty(self.L + 1, np.int64)
        e = np.empty(self.L + 1, np.int64)
        lib().orc_morton_get_levels(self._h, b, e)
        return b, e

    def nodes(self) -> dict:
        nn = self.nnodes
        d = dict(
            prefix=np.empty(nn, np.int64), level=np.empty(nn, np.int32), size2=np.empty(nn),
            first=np.empty(nn, np.int32), last=np.empty(nn, np.int32), parent=np.empty(nn, np.int32),
            nchild=np.empty(nn, np.int32), child=np.empty((nn, 8), np.int32),
            next=np.empty(nn, np.int32), mass=np.empty(nn), qcm=np.empty((nn, 3)),
            quad=np.empty((nn, 6)),
        )
        order = ["prefix", "level", "size2", "first", "last", "parent", "nchild", "child", "next",
                 "mass", "qcm", "quad"]
        lib().orc_morton_get_nodes(self._h, *[_ptr(d[k]) for k in order])
        return d

    def _mult(self, mult) -> int:
        """True/False (the reference's quadrupole switch) or 8: the octupole
        terms of octree_default.f90:1012-1063 over this tree."""
        if mult is None or mult is True:
            return 1
        if mult == 8:
            _check(lib().orc_morton_octupoles(self._h))
            return 8
        return int(bool(mult))

    def forces_par(self, G: float, eps2: float, theta2: float, mult: bool | int | None = None,
                   nthreads: int = 0) -> np.ndarray:
        """Forces (N,3) in original order; memory layout SoA like api3d."""
        out = np.empty(3 * self.n)
        _check(lib().orc_morton_forces(self._h, G, eps2, theta2, self._mult(mult), out, nthreads))
        return out.reshape(3, self.n).T

    def dehnen(self, G: float, eps2: float, theta2: float, mult: int = 4, pairs: bool = False):
        """Dehnen's dual-tree method (octree_default.f90:1095-1712) over this
        Morton tree: forces (N,3) in original order; with pairs=True also the
        number of mutual interactions."""
        out = np.empty(3 * self.n)
        npairs = C.c_int64(0)
        _check(lib().orc_morton_dehnen(self._h, G, eps2, theta2, int(mult), out, C.byref(npairs)))
        f = out.reshape(3, self.n).T
        return (f, npairs.value) if pairs else f

    def forces_targets(self, targets, G, eps2, theta2, mult=True, nthreads: int = 0):
        """(forces (k,3), counts (k,2) = body-body, cell) for ORIGINAL indices."""
        t = np.ascontiguousarray(targets, dtype=np.int64)
        out = np.empty(3 * t.size)
        cnt = np.empty(2 * t.size, np.int64)
        _check(lib().orc_morton_forces_targets(self._h, G, eps2, theta2, self._mult(mult), t.size,
                                               t, out, _ptr(cnt), nthreads))
        return out.reshape(3, t.size).T, cnt.reshape(t.size, 2)


class Octree:
    """OctreeType (octree_default.f90:90-170): pre_init + init + forces.
    method 10-12 classic BH, 20-22 Dehnen's dual-tree method (forces() runs
    dehnen_eval), 30-32 grouped BH; the last digit picks monopole, quadrupole
    or octupole."""

    def __init__(self, m, method: int = 11, group_size: int = 64, max_nodes: int = 0):
        m = _f64(m)
        self.n = m.size
        self.method = method
        h = C.c_void_p()
        _check(lib().orc_octree_create(self.n, m, method, group_size, max_nodes, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.orc_octree_free(h)
            self._h = None

    def init(self, x, y, z):
        _check(lib().orc_octree_init(self._h, _f64(x), _f64(y), _f64(z)))
        nn = C.c_int64(0)
        md = C.c_int(0)
        ng = C.c_int64(0)
        lib().orc_octree_info(self._h, C.byref(nn), C.byref(md), C.byref(ng))
        self.nnodes, self.most_depth, self.ngroups = nn.value, md.value, ng.value
        return self

    def nodes(self) -> dict:
        nn = self.nnodes
        d = dict(center=np.empty((nn, 3)), halfside=np.empty(nn), L2=np.empty(nn), mass=np.empty(nn),
                 qcm=np.empty((nn, 3)), particle=np.empty(nn, np.int32), type=np.empty(nn, np.int32),
                 child=np.empty((nn, 8), np.int32), depth=np.empty(nn, np.int32),
                 quad=np.empty((nn, 6)), oct=np.empty((nn, 14)))
        order = ["center", "halfside", "L2", "mass", "qcm", "particle", "type", "child", "depth",
                 "quad", "oct"]
        lib().orc_octree_get_nodes(self._h, *[_ptr(d[k]) for k in order])
        return d

    def forces(self, theta2: float, G: float, eps2: float, nthreads: int = 0) -> np.ndarray:
        out = np.empty(3 * self.n)
        _check(lib().orc_octree_forces(self._h, theta2, G, eps2, out, nthreads))
        return out.reshape(3, self.n).T

    def forces_targets(self, targets, theta2, G, eps2, nthreads: int = 0):
        t = np.ascontiguousarray(targets, dtype=np.int64)
        out = np.empty(3 * t.size)
        cnt = np.empty(2 * t.size, np.int64)
        _check(lib().orc_octree_forces_targets(self._h, theta2, G, eps2, t.size, t, out, _ptr(cnt),
                                               nthreads))
        return out.reshape(3, t.size).T, cnt.reshape(t.size, 2)


def direct_forces(m, x, y, z, G: float = 1.0, eps2: float = 0.0) -> np.ndarray:
    """direct_forces.f90:18-38 (sequential, Newton's 3rd law); (N,3)."""
    m, x, y, z = map(_f64, (m, x, y, z))
    out = np.empty(3 * m.size)
    _check(lib().orc_direct_forces(m.size, m, x, y, z, G, eps2, out))
    return out.reshape(3, m.size).T


def direct_forces_targets(m, x, y, z, targets, G: float = 1.0, eps2: float = 0.0,
                          nthreads: int = 0) -> np.ndarray:
    m, x, y, z = map(_f64, (m, x, y, z))
    t = np.ascontiguousarray(targets, dtype=np.int64)
    out = np.empty(3 * t.size)
    _check(lib().orc_direct_forces_targets(m.size, m, x, y, z, G, eps2, t.size, t, out, nthreads))
    return out.reshape(3, t.size).T
