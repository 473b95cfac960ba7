"""Gradient of the alignment score with respect to each subtomogram's rotation.

The score the orientation search maximises is f(alpha, beta, gamma) = Re sum_l D^l sigma_l
(src/matcha/core/Matcha.py:369-403), a function on SO(3) through the intrinsic z-y-z angles the
search returns.  ``RotationScore`` evaluates it at R(omega) = Rz(a) Ry(b) Rz(g) exp([omega]x)
for so(3) coordinates omega (B, 3) in the body frame of the base rotation, and its backward
gives df/domega: the Euler gradient from the CUDA derivative sweep (``mtb_score_derivatives``,
the same sweep the Newton step uses), mapped through the z-y-z Euler kinematics
(body rate = T(b, g) d(a, b, g)/dt) and the right Jacobian of exp.  Near beta = 0 or pi the
Euler angles are singular and the mapping loses precision; the gradient itself is defined
there, but this route to it is not used there.

Not covered: gradients with respect to the shift and to the template's Fourier-Laguerre
coefficients.
"""
from __future__ import annotations

import torch


def _hat(w):
    z = torch.zeros_like(w[..., 0])
    return torch.stack([torch.stack([z, -w[..., 2], w[..., 1]], -1),
                        torch.stack([w[..., 2], z, -w[..., 0]], -1),
                        torch.stack([-w[..., 1], w[..., 0], z], -1)], -2)


def so3_exp(w):
    """Rotation matrices exp([w]x) (Rodrigues), float64."""
    th = torch.linalg.norm(w, dim=-1)[..., None, None]
    K = _hat(w)
    small = th < 1e-8
    ths = torch.where(small, torch.ones_like(th), th)
    a = torch.where(small, 1.0 - th ** 2 / 6.0, torch.sin(ths) / ths)
    b = torch.where(small, 0.5 - th ** 2 / 24.0, (1.0 - torch.cos(ths)) / ths ** 2)
    eye = torch.eye(3, dtype=w.dtype, device=w.device).expand(K.shape)
    return eye + a * K + b * (K @ K)


def right_jacobian(w):
    """Jr(w): exp([w + dw]x) = exp([w]x) exp([Jr(w) dw]x) to first order."""
    th = torch.linalg.norm(w, dim=-1)[..., None, None]
    K = _hat(w)
    small = th < 1e-6
    ths = torch.where(small, torch.ones_like(th), th)
    c1 = torch.where(small, 0.5 - th ** 2 / 24.0, (1.0 - torch.cos(ths)) / ths ** 2)
    c2 = torch.where(small, 1.0 / 6.0 - th ** 2 / 120.0, (ths - torch.sin(ths)) / ths ** 3)
    eye = torch.eye(3, dtype=w.dtype, device=w.device).expand(K.shape)
    return eye - c1 * K + c2 * (K @ K)


def zyz_matrix(a, b, g):
    """Rz(a) Ry(b) Rz(g), float64."""
    ca, sa, cb, sb, cg, sg = torch.cos(a), torch.sin(a), torch.cos(b), torch.sin(b), torch.cos(g), torch.sin(g)
    return torch.stack([torch.stack([ca * cb * cg - sa * sg, -ca * cb * sg - sa * cg, ca * sb], -1),
                        torch.stack([sa * cb * cg + ca * sg, -sa * cb * sg + ca * cg, sa * sb], -1),
                        torch.stack([-sb * cg, sb * sg, cb], -1)], -2)


def zyz_angles(R):
    """(a, b, g) with Rz(a) Ry(b) Rz(g) = R, b in [0, pi]."""
    b = torch.arccos(torch.clamp(R[..., 2, 2], -1.0, 1.0))
    a = torch.atan2(R[..., 1, 2], R[..., 0, 2])
    g = torch.atan2(R[..., 2, 1], -R[..., 2, 0])
    return a, b, g


def euler_to_body(b, g):
    """T with body angular velocity = T d(a, b, g)/dt for Rz(a) Ry(b) Rz(g)."""
    sb, cb, sg, cg = torch.sin(b), torch.cos(b), torch.sin(g), torch.cos(g)
    z = torch.zeros_like(b)
    return torch.stack([torch.stack([-sb * cg, sg, z], -1),
                        torch.stack([sb * sg, cg, z], -1),
                        torch.stack([cb, z, torch.ones_like(b)], -1)], -2)


class RotationScore(torch.autograd.Function):
    """f_b(omega_b) for omega (B, 3) float64 around base angles (B, 3); sigma (B, Dsize)
    complex64 on the device; matcher a ``Matcha`` whose L_max >= L."""

    @staticmethod
    def forward(ctx, omega, base_angles, sigma, matcher, L):
        w = omega.detach().to(torch.float64)
        base = base_angles.to(device=w.device, dtype=torch.float64)
        R = zyz_matrix(base[:, 0], base[:, 1], base[:, 2]) @ so3_exp(w)
        a, b, g = zyz_angles(R)
        f, grad_e, _ = matcher.score_derivatives(sigma, a, b, g, L)
        ctx.save_for_backward(w, b, g, grad_e.to(torch.float64))
        return f.to(omega.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        w, b, g, grad_e = ctx.saved_tensors
        # df/domega = Jr^T T^{-T} df/d(a, b, g)
        gb = torch.linalg.solve(euler_to_body(b, g).transpose(-1, -2), grad_e[..., None])
        gw = (right_jacobian(w).transpose(-1, -2) @ gb)[..., 0]
        return grad_out.to(torch.float64)[:, None] * gw, None, None, None, None


def rotation_score(omega, base_angles, sigma, matcher, L=None):
    """Differentiable score of each subtomogram at the rotation R_zyz(base) exp([omega]x)."""
    return RotationScore.apply(omega, base_angles, sigma, matcher, matcher.Lmax if L is None else L)
