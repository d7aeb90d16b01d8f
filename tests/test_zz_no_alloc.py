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
        # the same kernels in the same order: equal bit for bit
        assert np.array_equal(a, b), name


def test_noalloc_allocates_no_device_memory():
    """After a first call has looked the fixed array up, calls of other sizes
    and parameters leave the device's free memory and torch's allocator as
    they were (the output and inputs are the caller's, made beforehand)."""
    import torch

    from hierarquicos_b200 import _lib

    lib = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    inputs = []
    for n, seed in ((300, 31), (5000, 32), (_lib.BH_NOALLOC_MAX_N, 33)):
        m, q = hernquist(n, seed=seed)
        dm, dx, dy, dz = _device_arrays(m, q)
        inputs.append((n, dm, dx, dy, dz, torch.empty(3 * n, dtype=torch.float64, device="cuda")))

    def call(n, dm, dx, dy, dz, out, **kw):
        p = _lib.default_params(**kw)
        rc = lib.bh_compute_forces_noalloc(dm.data_ptr(), dx.data_ptr(), dy.data_ptr(),
                                           dz.data_ptr(), n, C.byref(p), out.data_ptr(), stream)
        assert rc == 0, _lib.last_error()

    call(*inputs[0])  # warm: the first call on the device looks the array up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for args in inputs:
        for kw in (dict(order=4, theta=0.5, eps=0.01), dict(order=8, theta=0.3),
                   dict(order=1, precision=1), dict(order=4, precision=2, theta=0.6)):
            call(*args, **kw)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_small_theta_fits_its_fixed_stacks():
    """theta = 0.05 on the largest clustered system: the fixed walk stacks hold
    every node of the tree, so the walk completes (no BH_ERR_CAPACITY) and
    equals the allocating entry point's result."""
    import torch

    from hierarquicos_b200 import _lib
    from hierarquicos_b200.system import BHSystem

    lib = _lib.lib()
    n = _lib.BH_NOALLOC_MAX_N
    m, q = hernquist(n, seed=34)
    dm, dx, dy, dz = _device_arrays(m, q)
    for kw in (dict(theta=0.05, eps=0.0, order=4), dict(theta=0.05, order=1, group_size=32)):
        p = _lib.default_params(**kw)
        out = torch.empty(3 * n, dtype=torch.float64, device="cuda")
        rc = lib.bh_compute_forces_noalloc(dm.data_ptr(), dx.data_ptr(), dy.data_ptr(),
                                           dz.data_ptr(), n, C.byref(p), out.data_ptr(),
                                           torch.cuda.current_stream().cuda_stream)
        assert rc == 0, _lib.last_error()
        ref = BHSystem().forces(dm, dx, dy, dz, params=p)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), ref.cpu().numpy())


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


def test_noalloc_refuses_a_capturing_stream():
    """The call synchronises its stream, so on a stream that is being captured
    it returns BH_ERR_INVALID and queues nothing: the replayed graph holds only
    the caller's own work."""
    import torch

    from hierarquicos_b200 import _lib

    lib = _lib.lib()
    n = 256
    m, q = plummer(n, seed=24)
    dm, dx, dy, dz = _device_arrays(m, q)
    out = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    p = _lib.default_params()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        out.add_(1.0)
        rc = lib.bh_compute_forces_noalloc(dm.data_ptr(), dx.data_ptr(), dy.data_ptr(),
                                           dz.data_ptr(), n, C.byref(p), out.data_ptr(),
                                           s.cuda_stream)
    assert rc == _lib.BH_ERR_INVALID
    assert "captur" in _lib.last_error()
    g.replay()
    torch.cuda.synchronize()
    assert torch.all(out == 1.0)
