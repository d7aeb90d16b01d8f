"""Force-error statistics reported with every result.

The reference reports the normalised RMS acceleration error of
benchmarks/test_forces.f90:126 and the relative L2 error of
benchmarks/dehnen/forces_dehnen.f90; results here are also summarised by the
per-target relative error |F - F_dir| / |F_dir| (RMS and max).
"""
from __future__ import annotations

import numpy as np


def error_stats(forces, forces_dir, masses=None, positions=None) -> dict:
    """forces / forces_dir: (k,3) for the same k targets."""
    f = np.asarray(forces, np.float64)
    fd = np.asarray(forces_dir, np.float64)
    diff = np.linalg.norm(f - fd, axis=1)
    ref = np.linalg.norm(fd, axis=1)
    rel = diff / np.where(ref > 0, ref, np.inf)
    out = dict(rms_rel=float(np.sqrt(np.mean(rel ** 2))), max_rel=float(rel.max()),
               median_rel=float(np.median(rel)),
               l2_rel=float(np.linalg.norm(f - fd) / np.linalg.norm(fd)))
    if masses is not None and positions is not None:
        m = np.asarray(masses, np.float64)
        q = np.asarray(positions, np.float64)
        acc = (f - fd) / m[:, None]
        a_scale = np.sum(m / np.einsum("ij,ij->i", q, q))
        out["normalised_rms"] = float(np.sqrt((np.linalg.norm(acc) / a_scale) ** 2 / m.size))
    return out
