"""Oracle (test infrastructure only): the RELION-style FFT shift match, restated in numpy.

Follows src/matcha/core/ShiftMatcher.py:
  * reference preparation      load_reference_full :456-472 (apply_soft_mask :377-408,
                               gridding_correct :411-439, get_mask_full :442-453)
  * masks                      src/matcha/utils/setup_utils.py:239-270
  * rotate the reference       rotate_complex_volume :491-537 (trilinear, align_corners=True,
                               zero padding, torch.grid_sample semantics)
  * shifted patch              extract_shifted_patch_batch :558-616 (set_coords_to_zero=True,
                               normalize=False)
  * background fill            apply_cosine_mask :540-555
  * local upsampled DFT        compute_shift :94-282 (mode "local", space "complex",
                               normalization None, score_normalization True) and
                               _upsampled_dft :46-91
  * one micro-batch            estimate_shift_like_relion :619-674
Returned shifts are in the reference's (x, y, z) order (flip of the (dim1, dim2, dim3)
result) with its sub-pixel grid of 1/upsample_factor.  Only tests, the smoke check and
the CPU baseline may import this module.
"""
from __future__ import annotations

import numpy as np
from scipy.spatial.transform import Rotation as R


# ---------------------------------------------------------------- reference preparation
def apply_soft_mask(vol, ori_size, pixel_size, ini_high, width_fmask_edge=6.0):
    if ini_high <= 0:
        return vol
    radius = ori_size * pixel_size / ini_high - width_fmask_edge / 2.0
    radius_p = radius + width_fmask_edge
    ft = np.fft.fftshift(np.fft.fftn(vol, norm="forward"))
    zd, yd, xd = vol.shape
    zz, yy, xx = np.indices(vol.shape)
    r = np.sqrt((xx - xd // 2) ** 2 + (yy - yd // 2) ** 2 + (zz - zd // 2) ** 2)
    mask = np.ones_like(r)
    mask[r > radius_p] = 0
    tz = (r >= radius) & (r <= radius_p)
    mask[tz] = 0.5 - 0.5 * np.cos(np.pi * (radius_p - r[tz]) / width_fmask_edge)
    ft *= mask
    return np.fft.ifftn(np.fft.ifftshift(ft), norm="forward").real.astype(np.float64)


def gridding_correct(vol, ori_size, padding_factor=1.0):
    z, y, x = vol.shape
    kk, ii, jj = np.meshgrid(np.arange(-z // 2, z // 2), np.arange(-y // 2, y // 2), np.arange(-x // 2, x // 2),
                             indexing="ij")
    rval = np.sqrt(kk ** 2 + ii ** 2 + jj ** 2) / (ori_size * padding_factor)
    sinc = np.ones_like(rval)
    nz = rval > 0
    sinc[nz] = np.sin(np.pi * rval[nz]) / (np.pi * rval[nz])
    corr = sinc ** 2
    corr[corr == 0] = 1.0
    return vol / corr


def get_mask_full(shape):
    nz, ny, nx = shape
    cz, cy = nz // 2, ny // 2
    Z, Y, X = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    kp = np.where(Z < cz, Z, Z - nz)
    ip = np.where(Y < cy, Y, Y - ny)
    jp = np.where(X < cy, X, X - nx)
    return (kp ** 2 + ip ** 2 + jp ** 2) <= nz // 2 * nz // 2


def load_reference_full(ref, volume_size, voxel_size):
    ref = np.asarray(ref, dtype=np.float64)
    iref = apply_soft_mask(ref, volume_size, voxel_size, 4.0, 2.0)
    g = gridding_correct(iref, volume_size, 1.0)
    h = int(volume_size // 2)
    faux = np.fft.fftn(np.roll(g, (-h, -h, -h), axis=(0, 1, 2)), norm="forward")
    mask = np.fft.fftshift(get_mask_full(faux.shape), axes=(0, 1, 2))
    return np.fft.fftshift(faux, axes=(0, 1, 2)) * mask


def compute_masks(shape, radius, cosine_width=5.0):
    z, y, x = shape
    if radius < 0:
        radius = x / 2.0
    radius_p = radius + cosine_width
    zz, yy, xx = np.meshgrid(np.arange(-z // 2, z // 2), np.arange(-y // 2, y // 2), np.arange(-x // 2, x // 2),
                             indexing="ij")
    r = np.sqrt(xx ** 2 + yy ** 2 + zz ** 2)
    inner = r < radius
    outer = r > radius_p
    cos_m = (~inner) & (~outer)
    raised = 0.5 + 0.5 * np.cos(np.pi * (radius_p - r[cos_m]) / cosine_width)
    return outer, cos_m, raised


# ---------------------------------------------------------------- trilinear sampling
def trilinear(vol, iz, iy, ix):
    """torch.grid_sample(mode='bilinear', align_corners=True, padding_mode='zeros') at
    unnormalised indices; vol (D, H, W) real or complex."""
    D, H, W = vol.shape
    z0, y0, x0 = np.floor(iz), np.floor(iy), np.floor(ix)
    out = np.zeros(np.shape(iz), dtype=vol.dtype)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                zc, yc, xc = z0 + dz, y0 + dy, x0 + dx
                w = (1 - np.abs(iz - zc)) * (1 - np.abs(iy - yc)) * (1 - np.abs(ix - xc))
                ok = (zc >= 0) & (zc < D) & (yc >= 0) & (yc < H) & (xc >= 0) & (xc < W)
                zi = np.clip(zc, 0, D - 1).astype(int)
                yi = np.clip(yc, 0, H - 1).astype(int)
                xi = np.clip(xc, 0, W - 1).astype(int)
                out += np.where(ok, w * vol[zi, yi, xi], 0)
    return out


def euler_zyz_deg_from_quat_conj(q_wxyz):
    """np.rad2deg(quaternionic.array(q.conj()).to_euler_angles) (ShiftMatcher.py:913)."""
    q = np.asarray(q_wxyz, dtype=np.float64) * np.array([1, -1, -1, -1])
    n = (q ** 2).sum(-1)
    a = np.arctan2(q[..., 3], q[..., 0]) + np.arctan2(-q[..., 1], q[..., 2])
    b = 2 * np.arccos(np.sqrt((q[..., 0] ** 2 + q[..., 3] ** 2) / n))
    g = np.arctan2(q[..., 3], q[..., 0]) - np.arctan2(-q[..., 1], q[..., 2])
    return np.rad2deg(np.stack([a, b, g], -1))


def rotate_reference_half(ref_shifted, angles_deg):
    """rotate_complex_volume(..., pad_for_rfft_slicing=True)[..., N//2:] for each angle triple."""
    N = ref_shifted.shape[0]
    de = N + ((N + 1) % 2)
    c = (de - 1) / 2
    w = N + 1
    z, y, x = np.meshgrid(np.arange(N), np.arange(N), np.arange(w), indexing="ij")
    base = np.stack([x - c, y - c, z - c], 0).reshape(3, -1)
    out = []
    for ang in np.atleast_2d(angles_deg):
        rb = R.from_euler("ZYZ", ang, degrees=True).as_matrix()
        rot = rb @ base + c
        v = trilinear(ref_shifted, rot[2], rot[1], rot[0]).reshape(N, N, w)
        out.append(v[:, :, N // 2:])
    return np.array(out)


def extract_shifted_patch(vol, shift_zyx):
    """extract_shifted_patch_batch with set_coords_to_zero=True, normalize=False, one shift."""
    N = vol.shape[0]
    f = np.asarray(shift_zyx, dtype=np.float64)[::-1]  # torch.flip(shift_zyx)
    i, j, k = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    patch = trilinear(vol, i + f[0], j + f[1], k + f[2])
    for dim in range(3):
        a = abs(f[dim])
        if a - np.floor(a) > 0:
            idx = [slice(None)] * 3
            idx[dim] = int(np.floor(a)) if f[dim] < 0 else -int(np.ceil(a))
            patch[tuple(idx)] = 0
    return patch


def apply_cosine_mask(vol, outer, cos_m, raised):
    bg = vol[outer].sum() + (raised * vol[cos_m]).sum()
    wsum = outer.sum() + raised.sum()
    avg = bg / wsum if wsum > 0 else 0.0
    v = vol.copy()
    v[outer] = avg
    v[cos_m] = (1 - raised) * vol[cos_m] + raised * avg
    return v


def fftfreq(n, d):
    return np.fft.fftfreq(n, d=d)


def local_upsampled_peak(src, tgt, uf, radius):
    """compute_shift(mode='local', space='complex', normalization=None, score_normalization=True)."""
    prod = np.conj(src) * tgt
    window = 2 * radius + 1
    U = int(np.ceil(uf * window))
    dft = np.floor(U / 2.0)
    data = np.conj(prod)
    for dim in (2, 1, 0):
        n = data.shape[dim]
        rows = np.arange(U) - dft
        kern = np.exp(-2j * np.pi * rows[:, None] * fftfreq(n, uf)[None, :])
        data = np.moveaxis(np.tensordot(data, kern, axes=([dim], [1])), -1, dim)
    val = np.conj(data).real / (np.linalg.norm(tgt) * np.linalg.norm(src))
    flat = int(np.argmax(val))
    peak = np.array(np.unravel_index(flat, val.shape), dtype=np.float64)
    shift = (peak - dft) / uf
    return shift, float(val.max()), val


def estimate_shift_like_relion(ref_fourier, subtomo, shift_zyx, angles_deg, uf, radius, box_size=None,
                               voxel_size=1.0, return_parts=False):
    """One subtomogram: (shift in (x, y, z) order, normalised score)."""
    N = subtomo.shape[0]
    rot = rotate_reference_half(ref_fourier, angles_deg)[0]
    rot = np.fft.ifftshift(rot, axes=(0, 1)) * get_mask_full((N, N, N // 2 + 1))
    patch = extract_shifted_patch(np.asarray(subtomo, np.float64), shift_zyx)
    box = float(N if box_size is None else box_size)
    outer, cos_m, raised = compute_masks((N, N, N), box / (2.0 * voxel_size), 5.0)
    patch = apply_cosine_mask(patch, outer, cos_m, raised)
    h = N // 2
    sub = np.fft.rfftn(np.roll(patch, (-h, -h, -h), axis=(0, 1, 2)), norm="forward")
    shift, score, val = local_upsampled_peak(rot, sub, uf, radius)
    out = (shift[::-1], score)
    if return_parts:
        return out, dict(rot=rot, patch=patch, sub=sub, grid=val)
    return out


def shift_score_and_grad(ref_fourier, subtomo, shift_zyx, angles_deg, s_xyz, box_size=None, voxel_size=1.0):
    """The correlation the upsampled DFT of local_upsampled_peak samples, as a function of a
    continuous shift s (x, y, z): c(s) = Re sum_m prod[m] exp(2 pi i s . f(m)) / (|tgt| |src|)
    with prod = conj(src) tgt and f = (fftfreq(N), fftfreq(N), fftfreq(N/2+1)) on the (z, y, x)
    data axes; returns (c, dc/ds in (x, y, z))."""
    _, parts = estimate_shift_like_relion(ref_fourier, subtomo, shift_zyx, angles_deg, 1, 0, box_size=box_size,
                                          voxel_size=voxel_size, return_parts=True)
    src, tgt = parts["rot"], parts["sub"]
    prod = np.conj(src) * tgt
    n0, n1, n2 = prod.shape
    f0, f1, f2 = np.meshgrid(np.fft.fftfreq(n0), np.fft.fftfreq(n1), np.fft.fftfreq(n2), indexing="ij")
    s = np.asarray(s_xyz, dtype=np.float64)
    e = prod * np.exp(2j * np.pi * (s[2] * f0 + s[1] * f1 + s[0] * f2))
    den = np.linalg.norm(tgt) * np.linalg.norm(src)
    c = e.real.sum() / den
    g = np.array([(2j * np.pi * f2 * e).real.sum(), (2j * np.pi * f1 * e).real.sum(),
                  (2j * np.pi * f0 * e).real.sum()]) / den
    return c, g
