"""CPU restatement of the reference's integrators and Parareal driver --
TEST INFRASTRUCTURE ONLY (imported by the tests as the checker).

Follows, in FP64 numpy with the same operation order:
  * velocity Verlet in momentum form, ``F_til`` (parareal/parareal.f90:43-68)
    and ``test_integration_verlet_bh`` (benchmarks/integration_verlet/
    integration.f90:110-172);
  * symplectic Euler, ``G_til`` (parareal/parareal.f90:8-41);
  * the Parareal iteration ``integrate_parareal`` (parareal/parareal.f90:97-186):
    coarse initial sweep, fine propagators of all windows from the previous
    iterate, sequential correction U_{k+1,i+1} = G(U_{k+1,i}) + F(U_{k,i}) -
    G(U_{k,i}), error NORM2(U_{k+1,last} - U_{k,last}) / (6 N) and the stop at
    error <= maxerror;
  * the diagnostics total_energy / total_linear_momentum /
    total_angular_momentum (parareal/api3d.f90:108-153).
The reference runs these in REAL(16); this restatement (like the device code)
uses FP64.  Forces come from a callable ``forces(m, q) -> (N, 3)``.
"""
from __future__ import annotations

import numpy as np


def verlet(m, q, p, dt, nsteps, forces):
    """F_til: forces at the start, then per step p_half = p + (0.5 dt) f;
    q = q + (dt p_half) / m; f = F(q); p = p_half + (0.5 dt) f."""
    q = np.array(q, np.float64)
    p = np.array(p, np.float64)
    mm = np.asarray(m, np.float64)[:, None]
    f = forces(m, q)
    h = 0.5 * dt
    for _ in range(nsteps):
        p_half = p + h * f
        q = q + (dt * p_half) / mm
        f = forces(m, q)
        p = p_half + h * f
    return q, p


def symplectic_euler(m, q, p, dt, nsteps, forces):
    """G_til: per step f = F(q); p = p + dt f; q = q + (dt p) / m."""
    q = np.array(q, np.float64)
    p = np.array(p, np.float64)
    mm = np.asarray(m, np.float64)[:, None]
    for _ in range(nsteps):
        f = forces(m, q)
        p = p + dt * f
        q = q + (dt * p) / mm
    return q, p


def parareal(m, q0, p0, tf, num_windows, n_itermax, maxerror, coarse, fine):
    """integrate_parareal with propagators ``coarse(m, q, p)`` and
    ``fine(m, q, p)`` over one window each.  Returns (U, errors, iterations)
    where U[i] = (q, p) at the start of window i + 1 (U[0] = initial state)."""
    U = [(np.array(q0, np.float64), np.array(p0, np.float64))]
    for i in range(num_windows - 1):
        U.append(coarse(m, *U[i]))
    errors = []
    iterations = 1
    for _ in range(n_itermax - 1):
        iterations += 1
        Ft = [None] + [fine(m, *U[i]) for i in range(num_windows - 1)]
        Un = [U[0]]
        for i in range(num_windows - 1):
            gn = coarse(m, *Un[i])
            go = coarse(m, *U[i])
            qn = (gn[0] + Ft[i + 1][0]) - go[0]
            pn = (gn[1] + Ft[i + 1][1]) - go[1]
            Un.append((qn, pn))
        n = len(m)
        d = np.concatenate([(Un[-1][0] - U[-1][0]).ravel(), (Un[-1][1] - U[-1][1]).ravel()])
        err = float(np.sqrt(np.sum(d * d))) / (6 * n)
        errors.append(err)
        U = Un
        if err <= maxerror:
            break
    return U, errors, iterations


def diagnostics(m, q, p, G=1.0, eps=0.0):
    """(E, kinetic, potential, P(3), J(3)) as in parareal/api3d.f90:108-153."""
    m = np.asarray(m, np.float64)
    q = np.asarray(q, np.float64)
    p = np.asarray(p, np.float64)
    kin = float(np.sum(0.5 * np.sum(p * p, axis=1) / m))
    pot = 0.0
    for a in range(1, len(m)):
        d = q[:a] - q[a]
        r = np.sqrt(np.sum(d * d, axis=1) + eps * eps)
        pot += float(np.sum(-G * m[a] * m[:a] / r))
    P = p.sum(axis=0)
    J = np.cross(q, p).sum(axis=0)
    return np.concatenate([[kin + pot, kin, pot], P, J])
