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


# ------------------------------------------------------------------ synthetic volumes
def blob_template(rng, N, n_blobs, centre_radius, sigma_range, amp_range=(0.5, 1.0), mask_radius=None,
                  lobes=None):
    """Sum of isotropic Gaussians, float32; centres uniform in a ball (or two lobes)."""
    g = np.arange(N) - N // 2
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    vol = np.zeros((N, N, N), dtype=np.float64)
    for i in range(n_blobs):
        if lobes:
            (r_l, off) = lobes[i % len(lobes)]
            d = rng.standard_normal(3)
            c = np.array(off) + d / np.linalg.norm(d) * r_l * rng.uniform() ** (1 / 3)
        else:
            d = rng.standard_normal(3)
            c = d / np.linalg.norm(d) * centre_radius * rng.uniform() ** (1 / 3)
        s = rng.uniform(*sigma_range)
        a = rng.uniform(*amp_range)
        vol += a * np.exp(-((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) / (2 * s * s))
    if mask_radius is not None:
        r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
        vol *= np.clip((mask_radius + 2 - r) / 4, 0, 1)
    return vol.astype(np.float32)


def haar_quaternions(rng, n):
    """(w, x, y, z) unit quaternions, Haar-distributed."""
    q = rng.standard_normal((n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def rotate_volumes_reference(vols, quats):
    """src/matcha/utils/volume_rotation.py:49-125 (permute_before_sample=False), torch CPU.

    ZYZ angles of each quaternion -> scipy rotation matrix -> trilinear grid_sample of the
    (odd-padded) volume at R @ (x, y, z) with align_corners=True.
    """
    import torch
    import torch.nn.functional as TF

    v = torch.from_numpy(np.asarray(vols, dtype=np.float32)).unsqueeze(1)
    b, _, d, h, w = v.shape
    pad = (0, 1 if w % 2 == 0 else 0, 0, 1 if h % 2 == 0 else 0, 0, 1 if d % 2 == 0 else 0)
    v = TF.pad(v, pad)
    dp, hp, wp = v.shape[2:]
    mats = R.from_quat(np.roll(quats, -1, axis=1)).as_matrix()
    rot = torch.tensor(mats, dtype=torch.float32)
    dr = torch.linspace(-1, 1, dp)
    hr = torch.linspace(-1, 1, hp)
    wr = torch.linspace(-1, 1, wp)
    wg, hg, dg = torch.meshgrid(dr, hr, wr, indexing="ij")
    coords = torch.stack([dg.flatten(), hg.flatten(), wg.flatten()], 0)
    rc = (rot @ coords).permute(0, 2, 1).reshape(b, dp, hp, wp, 3)
    out = TF.grid_sample(v, rc, mode="bilinear", align_corners=True)
    return out[:, 0, :d, :h, :w].numpy()


def alignment_error_deg(alpha, beta, gamma, quats_true):
    """Angle of the tracker after update_rotation_estimate (src/matcha/utils/rotation_ops.py:23-34)
    starting from the true rotation, as src/matcha/example.py:208-220 measures it."""
    est = R.from_euler("ZYZ", np.stack([alpha, beta, gamma], -1))
    q = est.as_quat()  # (x, y, z, w)
    q_wxyz = np.roll(q, 1, axis=1)
    q_wxyz[:, [1, 3]] = q_wxyz[:, [3, 1]]
    sw = R.from_quat(np.roll(q_wxyz, -1, axis=1))
    tr = R.from_quat(np.roll(quats_true, -1, axis=1))
    return np.rad2deg((tr * sw.inv()).magnitude())


def make_subtomograms(template, rng, B, max_shift, snr_db=0.0, mask_radius=None):
    """Synthetic subtomograms as the benchmark draws them, on the host: the template rotated
    by Haar rotations (rotate_volumes_reference), shifted by uniform offsets in
    [-max_shift, max_shift]^3 (Fourier phase ramp, (z, y, x) order), plus white Gaussian
    noise at ``snr_db`` measured by the signal power inside the spherical mask
    (src/matcha/example.py:93-124).  Returns (float32 volumes, quaternions, shifts)."""
    N = template.shape[0]
    q = haar_quaternions(rng, B)
    shifts = rng.uniform(-max_shift, max_shift, (B, 3))
    vols = rotate_volumes_reference(np.repeat(template[None], B, 0), q).astype(np.float64)
    k = np.fft.fftfreq(N)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    g = np.arange(N) - N // 2
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    mask = np.sqrt(x ** 2 + y ** 2 + z ** 2) < (0.45 * N if mask_radius is None else mask_radius)
    for i in range(B):
        ph = np.exp(-2j * np.pi * (kz * shifts[i, 0] + ky * shifts[i, 1] + kx * shifts[i, 2]))
        v = np.fft.ifftn(np.fft.fftn(vols[i]) * ph).real
        power = np.mean(v[mask] ** 2)
        vols[i] = v + rng.standard_normal(v.shape) * np.sqrt(power * 10.0 ** (-snr_db / 10.0))
    return vols.astype(np.float32), q, shifts


def quat_dist_deg(q1, q2):
    """Rotation angle between (w, x, y, z) quaternions, degrees."""
    r1 = R.from_quat(np.roll(np.asarray(q1, dtype=np.float64), -1, axis=-1))
    r2 = R.from_quat(np.roll(np.asarray(q2, dtype=np.float64), -1, axis=-1))
    return np.rad2deg((r1.inv() * r2).magnitude())
