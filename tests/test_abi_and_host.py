"""CPU-only checks of the C ABI library and the host-side code: the library
loads and exports every function the header declares (no GPU call is made),
the ctypes struct matches the C layout, and the host helpers behave."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hierarquicos_bh.h")


def header_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(bh_\w+)\s*\(", src, re.M)))


@pytest.fixture(scope="module")
def built_lib():
    from hierarquicos_b200 import build

    return build.build()


def test_library_exports_every_header_function(built_lib):
    from hierarquicos_b200 import _lib

    declared = header_functions()
    assert declared == sorted(_lib.EXPORTED)
    out = subprocess.run(["nm", "-D", "--defined-only", built_lib], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (bh_\w+)", out))
    missing = set(declared) - exported
    assert not missing, missing


def test_library_loads_without_gpu(built_lib):
    from hierarquicos_b200 import _lib

    L = _lib.lib()
    assert L.bh_version().decode().startswith("hierarquicos-b200")
    p = _lib.default_params()
    assert (p.theta, p.order, p.depth, p.amp, p.group_size) == (0.5, 4, 21, 1.2, 64)


def test_params_struct_layout_matches_c(built_lib):
    # compile a tiny C program against the header and compare offsets
    from hierarquicos_b200._lib import BHParams

    code = r'''
#include <stddef.h>
#include <stdio.h>
#include "hierarquicos_bh.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(bh_params), offsetof(bh_params, amp),
         offsetof(bh_params, group_size), offsetof(bh_params, strict_keys),
         offsetof(bh_params, pipeline), offsetof(bh_params, precision), offsetof(bh_params, order));
  return 0;
}
'''
    import tempfile

    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(src, "w").write(code)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        vals = list(map(int, subprocess.run([exe], capture_output=True, text=True).stdout.split()))
    mine = [C.sizeof(BHParams), BHParams.amp.offset, BHParams.group_size.offset,
            BHParams.strict_keys.offset, BHParams.pipeline.offset, BHParams.precision.offset,
            BHParams.order.offset]
    assert vals == mine


def test_unknown_parameter_is_rejected(built_lib):
    from hierarquicos_b200._lib import default_params

    with pytest.raises(TypeError):
        default_params(thetta=0.3)


def test_initial_values_profiles():
    from hierarquicos_b200.initial_values import generate_initial_values

    m, q, p = generate_initial_values(20000, -1.0, -1.0, True, False, "plummer", (1.0, 1.0), seed=1)
    r = np.linalg.norm(q, axis=1)
    assert abs(np.median(r) - 1.3048) < 0.05          # Plummer half-mass radius 1.305 b
    assert np.allclose((m[:, None] * q).sum(0), 0.0, atol=1e-12)
    assert np.allclose(p.sum(0), 0.0, atol=1e-14)
    ke = 0.5 * np.sum(np.sum(p * p, axis=1) / m)
    assert abs(ke - 3 * np.pi / 64) < 0.02              # Plummer kinetic energy, G = M = b = 1
    m, q, _ = generate_initial_values(20000, 100.0, -1.0, True, False, "hernquist", (1.0, 1.0),
                                      seed=2, velocities=False)
    r = np.linalg.norm(q, axis=1)
    assert r.max() <= 100.0 + 1e-9 + np.abs((m[:, None] * q).sum(0)).max() * 2
    # truncated at 100 a: half of the kept mass inside r with r^2/(1+r)^2 = 0.5 * (100/101)^2
    target = 0.5 * (100 / 101) ** 2
    rh = np.sqrt(target) / (1 - np.sqrt(target))
    assert abs(np.median(r) - rh) < 0.1
    m, q, _ = generate_initial_values(20000, -1.0, -1.0, True, False, "homogeneous", (1.0, 1.0),
                                      seed=3, velocities=False)
    assert np.linalg.norm(q, axis=1).max() < 1.0 + 0.05


def test_error_stats():
    from hierarquicos_b200.metrics import error_stats

    rng = np.random.default_rng(0)
    fd = rng.standard_normal((100, 3))
    f = fd * (1 + 1e-3)
    s = error_stats(f, fd)
    assert abs(s["rms_rel"] - 1e-3) < 1e-9 and abs(s["max_rel"] - 1e-3) < 1e-9


def test_bench_cpu_binding_helpers():
    """The bench's NUMA binding: sysfs cpulist parsing, no change without a
    GPU, and the full CPU set restored around the CPU arm's child process."""
    import os
    import sys

    import torch

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    assert bench.parse_cpulist("0-3,8,10-11\n") == {0, 1, 2, 3, 8, 10, 11}
    assert bench.parse_cpulist("5") == {5}
    before = os.sched_getaffinity(0)
    if not torch.cuda.is_available():
        assert bench.bind_to_gpu_node(torch, 0).startswith("unbound")
        assert os.sched_getaffinity(0) == before
    saved = bench.HOST_CPUS
    try:
        one = {min(before)}
        bench.HOST_CPUS = before
        os.sched_setaffinity(0, one)
        with bench.all_host_cpus():
            assert os.sched_getaffinity(0) == before
        assert os.sched_getaffinity(0) == one
    finally:
        bench.HOST_CPUS = saved
        os.sched_setaffinity(0, before)
