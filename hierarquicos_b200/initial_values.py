"""Seeded initial conditions with the reference's density profiles.

Mirrors ``initial_values_mod.generate_initial_values``
(initial_values/initial_values.f90:51-173) and the profile modules
(initial_values/plummer.f90, hernquist.f90, homogeneous.f90): radii by inverting
the cumulative mass profile (rejected above ``size_qs`` when it is >= 0),
isotropic directions (initial_values.f90:355-381), von Neumann sampling of the
speeds from the ergodic distribution function, equal masses 1/N (or random
masses normalised to 1), momenta instead of velocities, and the centre of mass
and the total momentum moved to zero.

The random stream is NumPy's PCG64 seeded with ``seed``; gfortran's
RANDOM_NUMBER stream cannot be reproduced, so draws are statistically, not
bitwise, equivalent to the reference's.
"""
from __future__ import annotations

import math

import numpy as np

PI = 4.0 * math.atan(1.0)
M0 = 1.0


def plummer_inverse_P(x, b):
    """plummer.f90:53-62."""
    return x ** (1.0 / 3.0) * b / np.sqrt(1.0 - x ** (2.0 / 3.0))


def plummer_potential(r, G, b):
    """plummer.f90:64-77."""
    return -G * M0 / np.sqrt(r ** 2 + b ** 2)


def plummer_edf_norm(x):
    """plummer.f90:92-98."""
    return (1.0 - x ** 2) ** 3.5


PLUMMER_MAXIMUM_PDF = 0.0922108113291  # plummer.f90:100-104


def hernquist_inverse_P(x, a):
    """hernquist.f90:158-171."""
    return a * np.sqrt(x) / (1.0 - np.sqrt(x))


def hernquist_potential(r, G, a):
    """hernquist.f90:173-186."""
    return -G * M0 / (a + r)


def hernquist_edf_norm(r, x, G, a):
    """hernquist.f90:200-212."""
    E = np.sqrt(-hernquist_potential(r, G, a) * (1.0 - x ** 2))
    edf = 1.0 / (8.0 * math.sqrt(2.0) * a * PI ** 3)
    edf = edf / np.sqrt(1.0 - E) ** 5.0
    edf = edf * 3.0 * np.arcsin(np.sqrt(E))
    return edf + edf * np.sqrt(E * (1.0 - E)) * (1.0 - 2.0 * E) * (8.0 * E ** 2 - 8.0 * E - 3.0)


def hernquist_maximum_pdf(r, G, a):
    """hernquist.f90:214-247: first sign change of d/dq [q^2 f(E)] by centred
    finite differences with h = 1e-3, vectorised over r."""
    r = np.asarray(r, np.float64)
    h = 0.001

    def der(x):
        return ((x + h) ** 2 * hernquist_edf_norm(r, x + h, G, a)
                - (x - h) ** 2 * hernquist_edf_norm(r, x - h, G, a)) / (2.0 * h)

    x = h
    before = der(x)
    maximum = np.ones_like(r)
    done = np.zeros(r.shape, bool)
    while x + h < 1.0 and not done.all():
        x = x + h
        nxt = der(x)
        hit = (~done) & (before * nxt <= 0)
        if hit.any():
            maximum[hit] = (x * x * hernquist_edf_norm(r, x, G, a))[hit]
            done |= hit
        before = nxt
    return maximum


def homogeneous_sphere_inverse_P(x, R):
    """homogeneous.f90:48-61."""
    return R * (x * M0) ** (1.0 / 3.0)


def _truncated_radii(rng, n, inv, size_qs):
    out = np.empty(n)
    k = 0
    while k < n:
        x = rng.random(max(1024, int((n - k) * 1.1)))
        r = inv(x)
        if size_qs >= 0:
            r = r[r <= size_qs]
        take = min(n - k, r.size)
        out[k:k + take] = r[:take]
        k += take
    return out


def _von_neumann(rng, n, maximum, pdf):
    """Speed fraction q with density proportional to pdf(q, idx); accepted when
    maximum * u < pdf (initial_values.f90:245-254, 336-349)."""
    q = np.empty(n)
    todo = np.arange(n)
    for _ in range(10000):
        if todo.size == 0:
            break
        y = rng.random(todo.size)
        qv = rng.random(todo.size)
        mx = maximum if np.isscalar(maximum) else maximum[todo]
        ok = mx * y < pdf(qv, todo)
        q[todo[ok]] = qv[ok]
        todo = todo[~ok]
    if todo.size:
        raise RuntimeError("Too many attempts to sample with von Neumann, try again")
    return q


def cartesian_from_radius(rng, r, two_d=False):
    """initial_values.f90:355-381: isotropic directions for radii r; (N,3)."""
    n = r.size
    phi = 2.0 * PI * rng.random(n)
    if two_d:
        cos_t = np.zeros(n)
        sin_t = np.ones(n)
    else:
        cos_t = 2.0 * rng.random(n) - 1.0
        sin_t = np.sqrt(1.0 - cos_t * cos_t)
    return np.stack([r * sin_t * np.cos(phi), r * sin_t * np.sin(phi), r * cos_t], axis=1)


def generate_initial_values(N: int, size_qs: float = -1.0, size_ps: float = -1.0,
                            nm: bool = True, td: bool = False, pr: str = "plummer",
                            pp=(1.0, 1.0), seed: int = 0, velocities: bool = True):
    """Returns (m (N,), qs (N,3), ps (N,3)) like initial_values.f90:51-173.

    pr: 'uniform', 'uniform_sphere', 'plummer', 'homogeneous', 'hernquist';
    pp = (G, b) / (G, R) / (G, a).  velocities=False skips the (costly)
    speed sampling and returns zero momenta; positions are unaffected because
    they are drawn first from their own stream."""
    rng = np.random.Generator(np.random.PCG64(seed))
    vrng = np.random.Generator(np.random.PCG64([seed, 1]))
    if nm:
        m = np.full(N, 1.0 / N)
    else:
        m = rng.random(N)
        while m.min() == 0.0:
            m = rng.random(N)
        m = m / m.sum()
    G, par = float(pp[0]), float(pp[1])
    vr = None
    if pr == "uniform":
        qs = size_qs * (2.0 * rng.random((N, 3)) - 1.0)
        ps = size_ps * (2.0 * vrng.random((N, 3)) - 1.0) if velocities else np.zeros((N, 3))
    elif pr == "uniform_sphere":
        r = size_qs * (2.0 * rng.random(N) - 1.0)
        qs = cartesian_from_radius(rng, r, td)
        if velocities:
            vr = size_ps * (2.0 * vrng.random(N) - 1.0)
    elif pr == "plummer":
        r = _truncated_radii(rng, N, lambda x: plummer_inverse_P(x, par), size_qs)
        qs = cartesian_from_radius(rng, r, td)
        if velocities:
            v_esc = np.sqrt(-2.0 * plummer_potential(r, G, par))
            q = _von_neumann(vrng, N, PLUMMER_MAXIMUM_PDF, lambda qv, idx: qv * qv * plummer_edf_norm(qv))
            vr = q * v_esc
    elif pr == "homogeneous":
        r = _truncated_radii(rng, N, lambda x: homogeneous_sphere_inverse_P(x, par), size_qs)
        qs = cartesian_from_radius(rng, r, td)
        if velocities:
            vr = size_ps * (2.0 * vrng.random(N) - 1.0)
    elif pr == "hernquist":
        r = _truncated_radii(rng, N, lambda x: hernquist_inverse_P(x, par), size_qs)
        qs = cartesian_from_radius(rng, r, td)
        if velocities:
            v_esc = np.sqrt(-2.0 * hernquist_potential(r, G, par))
            mx = hernquist_maximum_pdf(r, G, par)
            q = _von_neumann(vrng, N, mx,
                             lambda qv, idx: qv * qv * hernquist_edf_norm(r[idx], qv, G, par))
            vr = v_esc * q
    else:
        raise ValueError(f'Unknow density profile: "{pr}"')
    if pr in ("uniform_sphere", "plummer", "homogeneous", "hernquist"):
        ps = cartesian_from_radius(vrng, vr, td) if vr is not None else np.zeros((N, 3))
    if velocities and size_ps >= 0:
        big = np.abs(ps).max()
        if big > size_ps:
            ps = ps * size_ps / big
    if td:
        ps[:, 2] = 0.0
        qs[:, 2] = 0.0
    ps = ps * m[:, None]
    ps = ps - ps.sum(axis=0) / N
    com = (m[:, None] * qs).sum(axis=0) / m.sum()
    qs = qs - com
    return m, np.ascontiguousarray(qs), np.ascontiguousarray(ps)


PROFILES = {"uniform": 0, "uniform_sphere": 1, "plummer": 2, "homogeneous": 3, "hernquist": 4}


def generate_initial_values_device(N: int, size_qs: float = -1.0, size_ps: float = -1.0,
                                   nm: bool = True, td: bool = False, pr: str = "plummer",
                                   pp=(1.0, 1.0), seed: int = 0, velocities: bool = True,
                                   device=None):
    """The same distributions as ``generate_initial_values``, drawn on the GPU
    by ``bh_generate_ics`` (counter-based streams, so not the host's draws).
    Returns CUDA tensors m (N,), q (3, N), p (3, N) (rows x, y, z)."""
    import ctypes as C

    import torch

    from ._lib import check, lib

    if pr not in PROFILES:
        raise ValueError(f'Unknow density profile: "{pr}"')
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    m = torch.empty(N, dtype=torch.float64, device=dev)
    q = torch.empty(3, N, dtype=torch.float64, device=dev)
    p = torch.empty(3, N, dtype=torch.float64, device=dev)
    scratch = torch.empty(2400, dtype=torch.float64, device=dev)
    check(lib().bh_generate_ics(PROFILES[pr], N, float(size_qs), float(size_ps), int(td), int(nm),
                                float(pp[0]), float(pp[1]), C.c_uint64(seed & (2**64 - 1)),
                                int(velocities), m.data_ptr(), q.data_ptr(), p.data_ptr(),
                                scratch.data_ptr(), torch.cuda.current_stream(dev).cuda_stream))
    return m, q, p
