"""Shared test helpers: seeded synthetic inputs and rotation distances."""
from __future__ import annotations

import os

import numpy as np
from scipy.spatial.transform import Rotation as R

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def euler_dist_deg(a1, b1, g1, a2, b2, g2):
    """Geodesic distance (degrees) between rotations given as Euler triples (same convention)."""
    r1 = R.from_euler("ZYZ", np.stack([a1, b1, g1], -1).reshape(-1, 3))
    r2 = R.from_euler("ZYZ", np.stack([a2, b2, g2], -1).reshape(-1, 3))
    return np.rad2deg((r1.inv() * r2).magnitude()).reshape(np.shape(a1))


def synthetic_sigma(rng, B, Lmax, noise=0.3):
    """sigma_b = sum_l w_l conj(D^l(R_b)) + noise; f(R) = Re sum D(R) sigma peaks at R_b."""
    from oracle import wigner as W

    n = W.dsize(Lmax)
    a = rng.uniform(0, 2 * np.pi, B)
    b = np.arccos(rng.uniform(-1, 1, B))
    g = rng.uniform(0, 2 * np.pi, B)
    D = W.wigner_D(a, b, g, Lmax)
    ls, _, _ = W.lmm(Lmax)
    w = np.exp(-(ls / (0.6 * Lmax)) ** 2) * (2 * ls + 1)
    sig = np.conj(D) * w + noise * (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n))) * w / (2 * ls + 1)
    return sig.astype(np.complex64), np.stack([a, b, g], -1)
