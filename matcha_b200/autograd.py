"""Gradients of the alignment scores: rotation (so(3)), correlation coefficients, template
coefficients and shift, as ``torch.autograd.Function``s over the CUDA kernels.

The reference differentiates only inside its Newton step (Euler gradient and Hessian,
src/matcha/core/WignerDGradients.py:155-302) and has no backward pass.  Here:

* ``rotation_score(omega, base_angles, sigma, matcher, L)``: f_b = Re sum_l D^l(R_b) sigma_b
  (src/matcha/core/Matcha.py:184, :288) at R_b = Rz(a) Ry(b) Rz(g) exp([omega_b]x), omega in
  the body frame of the base rotation.  Forward: ``mtb_score_derivatives``.  Backward
  (``mtb_score_backward``): the kernel regenerates D(R_b) from the angles (nothing is stored
  by the forward) and returns, in one sweep, df/dsigma = conj(D) and the body-frame gradient
  from the generators of the representation applied to sigma; the chain rule through exp
  is the right Jacobian Jr(omega)^T.  No Euler-angle kinematics, so beta = 0 or pi is not
  special.
* ``template_sigma(a_template, correlator, L)``: sigma of the correlator's last expanded batch
  against template coefficients (CrossCorrelationMatcher.py:183-212), differentiable in the
  template (``mtb_sigma_backward_template``, the adjoint of the contraction).
* ``shift_score(shift_xyz, shifter, subtomos, shift_zyx, rot)``: the shift match's correlation
  at a continuous shift (the function its upsampled DFT samples, ShiftMatcher.py:46-91) and
  its gradient (``mtb_shift_score_grad``).
* ``summed_aligned_correlation``: the sum over a batch of the rotation scores (through the
  template) and the shift scores, differentiable in every subtomogram's so(3) coordinates and
  shift and in the template's coefficients.

Complex gradients follow PyTorch's convention (d/dRe + i d/dIm of the real loss).
"""
from __future__ import annotations

import torch

from . import _native as nat


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
    """(a, b, g) with Rz(a) Ry(b) Rz(g) = R, b in [0, pi].  At b = 0 or pi only a + g (or
    a - g) is defined; the split chosen gives the same rotation."""
    sb = torch.sqrt(R[..., 0, 2] ** 2 + R[..., 1, 2] ** 2)
    b = torch.atan2(sb, R[..., 2, 2])
    gimbal = sb < 1e-12
    # beta = 0: R = Rz(a + g); beta = pi: R[0, 0] = -cos(a - g), R[1, 0] = -sin(a - g); g = 0 there
    up = R[..., 2, 2] > 0
    a_g = torch.where(up, torch.atan2(R[..., 1, 0], R[..., 0, 0]), torch.atan2(-R[..., 1, 0], -R[..., 0, 0]))
    a = torch.where(gimbal, a_g, torch.atan2(R[..., 1, 2], R[..., 0, 2]))
    g = torch.where(gimbal, torch.zeros_like(a), torch.atan2(R[..., 2, 1], -R[..., 2, 0]))
    b = torch.where(gimbal, torch.where(up, torch.zeros_like(b), torch.full_like(b, torch.pi)), b)
    return a, b, g


def euler_to_body(b, g):
    """T with body angular velocity = T d(a, b, g)/dt for Rz(a) Ry(b) Rz(g); the Euler gradient
    of a function is T^T times its body-frame gradient."""
    sb, cb, sg, cg = torch.sin(b), torch.cos(b), torch.sin(g), torch.cos(g)
    z = torch.zeros_like(b)
    return torch.stack([torch.stack([-sb * cg, sg, z], -1),
                        torch.stack([sb * sg, cg, z], -1),
                        torch.stack([cb, z, torch.ones_like(b)], -1)], -2)


def _f32(t):
    return t.to(torch.float32).contiguous()


class RotationScore(torch.autograd.Function):
    """f_b(omega_b) for omega (B, 3) float64 around base angles (B, 3); sigma (B, >= Dsize(L))
    complex64 on the device (differentiable); matcher a ``Matcha`` whose L_max >= L."""

    @staticmethod
    def forward(ctx, omega, sigma, base_angles, matcher, L):
        w = omega.detach().to(torch.float64)
        base = base_angles.to(device=w.device, dtype=torch.float64)
        R = zyz_matrix(base[:, 0], base[:, 1], base[:, 2]) @ so3_exp(w)
        a, b, g = (_f32(x) for x in zyz_angles(R))
        sig = sigma.detach().contiguous()
        f, _, _ = matcher.score_derivatives(sig, a, b, g, L)
        ctx.save_for_backward(w, sig, a, b, g)
        ctx.L = int(L)
        return f.to(torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        w, sig, a, b, g = ctx.saved_tensors
        B, L = sig.shape[0], ctx.L
        weight = _f32(grad_out)
        need_sigma = ctx.needs_input_grad[1]
        grad_sigma = torch.zeros_like(sig) if need_sigma else None
        grad_body = torch.empty((B, 3), device=sig.device, dtype=torch.float64)
        lib = nat.load()
        with torch.cuda.device(sig.device):
            nat.check(lib.mtb_score_backward(nat.ptr(sig), sig.stride(0), B, L, nat.ptr(a), nat.ptr(b), nat.ptr(g),
                                             nat.ptr(weight), nat.ptr(grad_sigma),
                                             grad_sigma.stride(0) if need_sigma else 0, nat.ptr(grad_body),
                                             nat.stream_ptr(sig.device)), "mtb_score_backward")
        grad_omega = (right_jacobian(w).transpose(-1, -2) @ grad_body[..., None])[..., 0]
        return grad_omega, grad_sigma, None, None, None


def rotation_score(omega, base_angles, sigma, matcher, L=None):
    """Differentiable score of each subtomogram at the rotation R_zyz(base) exp([omega]x)."""
    return RotationScore.apply(omega, sigma, base_angles, matcher, matcher.Lmax if L is None else L)


class TemplateSigma(torch.autograd.Function):
    """sigma (B, Dsize(L)) of the correlator's last expanded batch against template
    coefficients a_template (ne + 1,) complex64 (the padded vector set_template keeps)."""

    @staticmethod
    def forward(ctx, a_template, correlator, L):
        sig = correlator.sigma_from_template(a_template.detach().contiguous(), L)
        ctx.correlator, ctx.L, ctx.B = correlator, int(L), sig.shape[0]
        return sig

    @staticmethod
    def backward(ctx, grad_sigma):
        cc = ctx.correlator
        g = grad_sigma.contiguous()
        out = torch.empty((cc.fle.ne + 1,), device=g.device, dtype=torch.complex64)
        with torch.cuda.device(g.device):
            nat.check(cc.fle._lib.mtb_sigma_backward_template(cc.fle._h, nat.ptr(cc._coeffs), cc._coeffs.stride(0),
                                                             nat.ptr(g), g.stride(0), ctx.B, ctx.L, nat.ptr(out),
                                                             nat.stream_ptr(g.device)),
                      "mtb_sigma_backward_template")
        return out, None, None


def template_sigma(a_template, correlator, L):
    return TemplateSigma.apply(a_template, correlator, L)


class ShiftScore(torch.autograd.Function):
    """The shift match's correlation of each subtomogram at continuous shifts (B, 3) (x, y, z)."""

    @staticmethod
    def forward(ctx, shift_xyz, shifter, subtomos, shift_zyx, rot):
        s = _f32(shift_xyz.detach())
        score, grad = shifter.score_and_gradient(subtomos, shift_zyx, rot, s)
        ctx.save_for_backward(grad)
        return score.to(shift_xyz.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad_out[:, None].to(grad.dtype) * grad, None, None, None, None


def shift_score(shift_xyz, shifter, subtomos, shift_zyx, rot):
    return ShiftScore.apply(shift_xyz, shifter, subtomos, shift_zyx, rot)


def summed_aligned_correlation(step, volumes, omega, base_angles, a_template, shift_xyz, shift_zyx, rot):
    """The summed aligned correlation of a batch: sum_b f_b(R_b exp(omega_b); sigma_b(aT)) +
    sum_b c_b(s_b), for an ``AlignmentStep`` (its correlator, matcher and shifter):
    volumes (B, N, N, N) are expanded (the template-independent half of sigma), sigma comes
    from ``a_template`` (ne + 1,) complex64 through ``template_sigma``, the rotation scores at
    the base angles (B, 3) moved by omega (B, 3), the shift scores at shift_xyz (B, 3) for
    subtomograms ``volumes`` at the prior shift_zyx with rotation matrices rot (B, 9).
    Differentiable in omega, a_template and shift_xyz."""
    step.correlator.expand(volumes)
    sig = template_sigma(a_template, step.correlator, step.cfg.L)
    f = rotation_score(omega, base_angles, sig, step.matcher, step.cfg.L)
    c = shift_score(shift_xyz, step.shifter, volumes, shift_zyx, rot)
    return f.sum() + c.to(f.dtype).sum()
