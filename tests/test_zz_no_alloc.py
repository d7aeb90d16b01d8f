"""The allocation-free entry point, bh_compute_forces_noalloc.

It serves callers that must not allocate device memory themselves or through
this library -- for instance a program whose device memory is owned by another
allocator, or a time-step loop that cannot afford the device-wide stall a
cudaMalloc may cause.  All its scratch space is one fixed array inside the
library, which limits it to BH_NOALLOC_MAX_N bodies.  These tests call it
through the C ABI and compare it with bh_system_forces, the allocating entry
point, on the same inputs; this file is collected last so that a failure here
stops a -x run only after every other test has run."""
import ctypes as C

import numpy as np
import pytest

from conftest import hernquist, plummer, xyz

pytestmark = pytest.mark.gpu


def _device_arrays(m, q):
    import torch

    return [torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")
            for a in (m, *xyz(q))]


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    import torch

    from hierarquicos_b200 import _lib
    from hierarquicos_b200.system import BHSystem

    assert torch.cuda.is_available()
    lib = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [("plummer", plummer(6000, seed=21), dict(theta=0.5, eps=0.01, order=4)),
             ("hernquist", hernquist(_lib.BH_NOALLOC_MAX_N, seed=22), dict(theta=0.7, eps=0.0, order=8))]
    for name, (m, q), kw in cases:       # two calls in a row, different systems and parameters
        n = m.size
        dm, dx, dy, dz = _device_arrays(m, q)
        p = _lib.default_params(**kw)
        out = torch.full((3 * n,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.bh_compute_forces_noalloc(dm.data_ptr(), dx.data_ptr(), dy.data_ptr(),
                                           dz.data_ptr(), n, C.byref(p), out.data_ptr(), stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        ref = BHSystem().forces(dm, dx, dy, dz, params=p)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.all(np.isfinite(a)), name
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-14 * np.abs(b).max(), err_msg=name)


def test_noalloc_rejects_systems_above_its_limit():
    import torch

    from hierarquicos_b200 import _lib

    lib = _lib.lib()
    n = _lib.BH_NOALLOC_MAX_N + 1
    m, q = plummer(n, seed=23)
    dm, dx, dy, dz = _device_arrays(m, q)
    out = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    p = _lib.default_params()
    rc = lib.bh_compute_forces_noalloc(dm.data_ptr(), dx.data_ptr(), dy.data_ptr(), dz.data_ptr(),
                                       n, C.byref(p), out.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.BH_ERR_INVALID
    assert str(_lib.BH_NOALLOC_MAX_N) in _lib.last_error()
