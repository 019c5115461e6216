"""Seeded synthetic beams with the benchmark configurations' distributions.

The reference benchmarks no public dataset; these generators stand in for its
workloads (numpy ``default_rng(seed)``; the reference's Julia RNG streams are
not reproducible outside Julia).  All return (pos, mom) as N x 3 float64.
"""
from __future__ import annotations

import numpy as np


def uniform(N: int, seed: int = 0):
    """Positions i.i.d. Uniform[0,1]^3, momenta all zero."""
    rng = np.random.default_rng(seed)
    pos = rng.random((N, 3))
    return pos, np.zeros((N, 3))


def gaussian_bunch(N: int, seed: int = 0, sigma=(1.0, 1.0, 0.1), uz=(200.0, 0.2), uxy=0.01):
    """Relativistic Gaussian bunch: x ~ N(0, sigma), u_z ~ N(uz), u_x,u_y ~ N(0, uxy)."""
    rng = np.random.default_rng(seed)
    pos = rng.normal(0.0, 1.0, (N, 3)) * np.asarray(sigma)
    mom = np.empty((N, 3))
    mom[:, 0] = rng.normal(0.0, uxy, N)
    mom[:, 1] = rng.normal(0.0, uxy, N)
    mom[:, 2] = rng.normal(uz[0], uz[1], N)
    return pos, mom


def beamlets(N: int, seed: int = 0, nbeam: int = 8, sigma=(0.3, 0.3, 0.03), uz=(100.0, 0.1), uxy=0.005):
    """Mixture of equal-weight Gaussian beamlets with centres Uniform[-5,5]^3."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-5.0, 5.0, (nbeam, 3))
    which = np.repeat(np.arange(nbeam), -(-N // nbeam))[:N]
    pos = centres[which] + rng.normal(0.0, 1.0, (N, 3)) * np.asarray(sigma)
    mom = np.empty((N, 3))
    mom[:, 0] = rng.normal(0.0, uxy, N)
    mom[:, 1] = rng.normal(0.0, uxy, N)
    mom[:, 2] = rng.normal(uz[0], uz[1], N)
    return pos, mom


def rel_l2(a, b) -> float:
    """||a - b||_2 / ||b||_2 over all particles and components (inf if b == 0 and a != b)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = float(np.linalg.norm(b))
    d = float(np.linalg.norm(a - b))
    if nb == 0.0:
        return 0.0 if d == 0.0 else float("inf")
    return d / nb
