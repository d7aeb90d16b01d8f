"""Drop-in for the reference's f2py module ``api_mod`` (fortran/api3d.f90).

Same names, argument order and meaning as the Fortran module:

* ``compute_forces(m, x, y, z, theta, G, eps, quad)`` -> forces (N,3)
  (fortran/api3d.f90:20-41, REAL(16) twin parareal/api3d.f90:20-44);
* ``compute_forces_direct(m, x, y, z, G, eps)`` -> forces (N,3)
  (fortran/api3d.f90:43-72);
* ``generate_tree(m, x, y, z, quad)`` (fortran/api3d.f90:9-18).

theta and eps are passed unsquared and squared inside, as parareal/api3d.f90:30
does.  ``quad`` selects the quadrupole (True) or the monopole (False/None), as
the Fortran optional argument does; ``order=8`` asks for the octupole.  The
result is a Fortran-ordered (N,3) float64 array, i.e. the same memory layout as
the f2py return value.  Where the Fortran stops the process (STOP) these raise
``BHError``.  Every call builds a fresh tree, as the Fortran does, but reuses a
device workspace.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import BHError, check, default_params, lib  # noqa: F401  (BHError re-exported)

__all__ = ["compute_forces", "compute_forces_direct", "generate_tree", "BHError"]


def _vec(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64).reshape(-1)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def compute_forces(m, x, y, z, theta, G, eps, quad=None, order: int | None = None,
                   accelerations: bool = False, **params) -> np.ndarray:
    m, x, y, z = map(_vec, (m, x, y, z))
    n = m.size
    if not (x.size == y.size == z.size == n):
        raise BHError(1, "m, x, y, z must have the same length")
    if order is None:
        order = 4 if quad else 1
    p = default_params(theta=float(theta), G=float(G), eps=float(eps), order=int(order),
                       out_kind=1 if accelerations else 0, **params)
    out = np.empty((n, 3), dtype=np.float64, order="F")
    check(lib().bh_compute_forces_ex(_ptr(m), _ptr(x), _ptr(y), _ptr(z), n, C.byref(p),
                                     out.ctypes.data_as(C.c_void_p), None))
    return out


def compute_forces_direct(m, x, y, z, G, eps, accelerations: bool = False) -> np.ndarray:
    m, x, y, z = map(_vec, (m, x, y, z))
    n = m.size
    out = np.empty((n, 3), dtype=np.float64, order="F")
    check(lib().bh_compute_forces_direct(_ptr(m), _ptr(x), _ptr(y), _ptr(z), n, float(G),
                                         float(eps), 1 if accelerations else 0,
                                         out.ctypes.data_as(C.c_void_p), None))
    return out


def generate_tree(m, x, y, z, quad=None):
    """Builds the octree (and the quadrupoles when quad is true) and discards
    it, like the Fortran subroutine; returns the tree's summary."""
    from .system import BHSystem

    s = BHSystem()
    s.build(m, x, y, z, default_params(order=4 if quad else 1))
    s.sync()
    info = s.info()
    s.close()
    return info
