"""Force-error metrics of the reference harness -- TEST INFRASTRUCTURE ONLY.

Restates benchmarks/test_forces.f90:66-127 (evaluate_error_on_accelerations)
and the relative L2 error of benchmarks/dehnen/forces_dehnen.f90.
"""
from __future__ import annotations

import numpy as np


def reference_errors(ms, qs, forces, forces_dir) -> np.ndarray:
    """errors(1..7) of test_forces.f90:66-127.

    ms (N,), qs (N,3), forces / forces_dir (N,3).  errors[0] is the normalised
    RMS acceleration error sqrt((||a - a_dir|| / sum m/|q|^2)^2 / N) (:126),
    errors[1:4] the force sum (:86-88), errors[4:7] the torque sum q x F
    (:100-103)."""
    ms = np.asarray(ms, np.float64)
    qs = np.asarray(qs, np.float64)
    f = np.asarray(forces, np.float64)
    fd = np.asarray(forces_dir, np.float64)
    n = ms.size
    err = np.zeros(7)
    err[1:4] = f.sum(axis=0)
    acc = f / ms[:, None]
    acc_dir = fd / ms[:, None]
    a_scale = np.sum(ms / np.einsum("ij,ij->i", qs, qs))
    err[4:7] = np.cross(qs, f).sum(axis=0)
    err[0] = np.sqrt((np.linalg.norm(acc - acc_dir) / a_scale) ** 2 / n)
    return err


def normalised_rms(ms, qs, forces, forces_dir) -> float:
    """forces_time_and_error.f90:287-308 (the metric of the recorded tables)."""
    return float(reference_errors(ms, qs, forces, forces_dir)[0])


def relative_l2(forces, forces_dir) -> float:
    """||a - a_dir|| / ||a_dir|| (forces_dehnen.f90, error2)."""
    f = np.asarray(forces, np.float64)
    fd = np.asarray(forces_dir, np.float64)
    return float(np.linalg.norm(f - fd) / np.linalg.norm(fd))


def per_target_relative(forces, forces_dir) -> np.ndarray:
    """|F_i - F_dir,i| / |F_dir,i| for every target."""
    f = np.asarray(forces, np.float64)
    fd = np.asarray(forces_dir, np.float64)
    return np.linalg.norm(f - fd, axis=1) / np.linalg.norm(fd, axis=1)
