"""Oracle (test infrastructure only): the subtomogram preparation of every alternation,
restated in numpy.

Follows BatchProcessor._extract_rotated_batch (src/matcha/align_subtomograms.py:240-252):
  * shifted patch      extract_subtomogram_patch_batch (src/matcha/utils/io_utils.py:113-178,
                       normalize=True, set_coords_to_zero=False): grid_sample of the volume at
                       voxel + shift through the normalised grid 2 g / (N - 1) - 1
  * normalisation      normalise / mean / std (src/matcha/utils/volume_ops.py:17-35) in the
                       hard spherical mask distance < radius about N // 2 (volume_ops.py:6-14
                       with sigma 0, setup_utils.py:274-281), then times the mask
  * rotation           rotate_volumes (src/matcha/utils/volume_rotation.py:8-125): Euler ZYZ
                       angles of the tracker (quaternionic's to_euler_angles), scipy's
                       from_euler('ZYZ', degrees=True) matrix, grid_sample of the odd-padded
                       volume at R (x, y, z) on linspace(-1, 1) grids, cropped back
Every grid_sample is trilinear with align_corners=True and zero padding (oracle.shift.trilinear).
Only tests, the smoke check and the CPU baseline may import this module.
"""
from __future__ import annotations

import numpy as np
from scipy.spatial.transform import Rotation as R

from .shift import trilinear


def spherical_mask(N, radius):
    c = N // 2
    z, y, x = np.ogrid[:N, :N, :N]
    return (np.sqrt((z - c) ** 2 + (y - c) ** 2 + (x - c) ** 2) < radius).astype(np.float64)


def euler_zyz_deg(q_wxyz):
    """np.rad2deg(quaternionic.array(q).to_euler_angles) for the tracker q (w, x, y, z)."""
    q = np.asarray(q_wxyz, dtype=np.float64)
    n = (q ** 2).sum(-1)
    a = np.arctan2(q[..., 3], q[..., 0]) + np.arctan2(-q[..., 1], q[..., 2])
    b = 2 * np.arccos(np.sqrt((q[..., 0] ** 2 + q[..., 3] ** 2) / n))
    g = np.arctan2(q[..., 3], q[..., 0]) - np.arctan2(-q[..., 1], q[..., 2])
    return np.rad2deg(np.stack([a, b, g], -1))


def extract_patch(vol, shift_xyz):
    """The patch of one (N, N, N) volume at voxel + shift (x, y, z order)."""
    N = vol.shape[0]
    size = N - 1
    z, y, x = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")

    def unnorm(g):
        n = 2 * g / size - 1
        return ((n + 1) / 2) * size

    return trilinear(vol, unnorm(z + shift_xyz[2]), unnorm(y + shift_xyz[1]), unnorm(x + shift_xyz[0]))


def normalise_masked(patch, mask):
    m = (patch * mask).sum() / mask.sum()
    sd = np.sqrt((patch ** 2 * mask).sum() / mask.sum() - m ** 2)
    return (patch - m) / sd * mask


def rotate_volume(vol, q_wxyz):
    """rotate_volumes_in_batches for one volume and tracker quaternion."""
    N = vol.shape[0]
    pad = 1 if N % 2 == 0 else 0
    P = N + pad
    v = np.zeros((P, P, P), dtype=vol.dtype)
    v[:N, :N, :N] = vol
    rot = R.from_euler("ZYZ", euler_zyz_deg(q_wxyz), degrees=True).as_matrix()
    r = np.linspace(-1, 1, P)
    zg, yg, xg = np.meshgrid(r, r, r, indexing="ij")
    coords = np.stack([xg.ravel(), yg.ravel(), zg.ravel()], 0)  # (x, y, z) of each output voxel
    rx, ry, rz = (rot @ coords).reshape(3, P, P, P)
    half = (P - 1) / 2
    out = trilinear(v, (rz + 1) * half, (ry + 1) * half, (rx + 1) * half)
    return out[:N, :N, :N]


def prepare(volumes, shift_xyz, tracker, radius):
    """(B, N, N, N) volumes -> the expansion's input of the alternation."""
    volumes = np.asarray(volumes, dtype=np.float64)
    mask = spherical_mask(volumes.shape[1], radius)
    out = np.empty_like(volumes)
    for b in range(volumes.shape[0]):
        p = normalise_masked(extract_patch(volumes[b], np.asarray(shift_xyz[b], dtype=np.float64)), mask)
        out[b] = rotate_volume(p, tracker[b])
    return out
