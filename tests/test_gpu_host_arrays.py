"""The host-array entry points (bh_compute_forces_ex, bh_compute_forces_direct,
api3d) with pinned and with ordinary pageable host memory.

Pinned arrays are copied straight by the copy engines; pageable ones are
staged through pinned chunks by the library's host threads.  Both must give
the device-array path's result bit for bit, for sizes that end inside a
chunk, span many chunks or hold a single body, and a device pointer passed as
a host array is refused.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import hernquist, plummer

pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch

    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)))
    assert t.is_pinned()
    return t


@pytest.mark.parametrize("n,seed", [(1, 1), (1000, 2), (65536 + 3, 3), (300_001, 4),
                                    (1 << 20, 5)])
def test_pageable_and_pinned_arrays_give_the_device_result(n, seed):
    import torch

    from hierarquicos_b200 import _lib, api3d
    from hierarquicos_b200.system import BHSystem

    m, q = (hernquist if n > 1000 else plummer)(n, seed=seed)
    x, y, z = (np.ascontiguousarray(q[:, k]) for k in range(3))
    p = _lib.default_params(theta=0.5, eps=0.01, order=4)
    dev = [torch.as_tensor(a, device="cuda") for a in (m, x, y, z)]
    ref = BHSystem().forces(*dev, params=p).view(3, n).T.cpu().numpy()

    # pageable numpy arrays in, a fresh Fortran-ordered (n, 3) array out
    got = api3d.compute_forces(m, x, y, z, 0.5, 1.0, 0.01, order=4)
    assert got.flags.f_contiguous and got.shape == (n, 3)
    assert np.array_equal(got, ref)

    # pinned arrays in and out
    hm, hx, hy, hz = (_pinned(a) for a in (m, x, y, z))
    hout = torch.empty(3 * n, dtype=torch.float64, pin_memory=True)
    lib = _lib.lib()
    rc = lib.bh_compute_forces_ex(hm.data_ptr(), hx.data_ptr(), hy.data_ptr(), hz.data_ptr(), n,
                                  C.byref(p), hout.data_ptr(), None)
    assert rc == 0, _lib.last_error()
    assert np.array_equal(hout.numpy().reshape(3, n).T, ref)

    # mixed: pinned inputs, pageable result
    out = np.empty(3 * n, dtype=np.float64)
    rc = lib.bh_compute_forces_ex(hm.data_ptr(), hx.data_ptr(), hy.data_ptr(), hz.data_ptr(), n,
                                  C.byref(p), out.ctypes.data_as(C.c_void_p), None)
    assert rc == 0, _lib.last_error()
    assert np.array_equal(out.reshape(3, n).T, ref)


def test_direct_sum_from_pageable_arrays():
    import torch

    from hierarquicos_b200 import api3d
    from hierarquicos_b200.system import direct_targets

    n = 70_001
    m, q = plummer(n, seed=6)
    x, y, z = (np.ascontiguousarray(q[:, k]) for k in range(3))
    got = api3d.compute_forces_direct(m, x, y, z, 1.0, 0.01)
    dev = [torch.as_tensor(a, device="cuda") for a in (m, x, y, z)]
    ref = direct_targets(*dev, G=1.0, eps=0.01).T.cpu().numpy()
    assert np.array_equal(got, ref)


def test_device_pointer_in_place_of_a_host_array_is_refused():
    import torch

    from hierarquicos_b200 import _lib

    n = 512
    m, q = plummer(n, seed=7)
    x, y, z = (np.ascontiguousarray(q[:, k]) for k in range(3))
    p = _lib.default_params()
    lib = _lib.lib()
    dm = torch.as_tensor(m, device="cuda")
    out = np.empty(3 * n, dtype=np.float64)
    rc = lib.bh_compute_forces_ex(dm.data_ptr(), x.ctypes.data, y.ctypes.data, z.ctypes.data, n,
                                  C.byref(p), out.ctypes.data_as(C.c_void_p), None)
    assert rc == _lib.BH_ERR_INVALID
    assert "device pointer" in _lib.last_error()
    dout = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    rc = lib.bh_compute_forces_ex(m.ctypes.data, x.ctypes.data, y.ctypes.data, z.ctypes.data, n,
                                  C.byref(p), dout.data_ptr(), None)
    assert rc == _lib.BH_ERR_INVALID
    # the library is still usable afterwards
    rc = lib.bh_compute_forces_ex(m.ctypes.data, x.ctypes.data, y.ctypes.data, z.ctypes.data, n,
                                  C.byref(p), out.ctypes.data_as(C.c_void_p), None)
    assert rc == 0, _lib.last_error()
