"""Denoiser-in-the-loop training on the native projector.

The reference trains a 3-D U-Net inside its reconstruction loop
(FL/example/demo.py:396-475): every step the denoised estimate C_d =
net(C) is projected with ``forward_emission_batch_autograd``
(FL/cuda_lib/autograd.py:37-77; attenuation held fixed), the loss
1e3 * MSE(Pf, I) + Poisson(Pf, I) + 0.1 * TV(C_d) (FL/ml_lib/ml_loss.py:6-16)
is back-propagated into the network and Adam takes a step; every few steps
the attenuation is rebuilt and C refreshed by 20 MLEM iterations.  Its
unrolled model (UnrolledBatchMLEM_vanilla, FL/ml_lib/ml_model.py:285-365)
alternates MLEM steps and the denoiser but calls the non-differentiable
``mlem_cuda_batch`` and leaves the denoiser call unfinished.

Here:
* ``ratio_backprojection`` is P^T(I / max(P C, 1e-6)) as an autograd Function
  whose backward is its exact vector-Jacobian product, P^T D P g with
  D = -I / (P C)^2 where P C > 1e-6 (one forward and one backward projection
  on the native kernels);
* ``mlem_step`` is one MLEM update (atten_cuda.cpp:321-342) differentiable in
  C: C * back / (sens + beta * huber(C)), clamped at 0;
* ``UnrolledMLEM`` alternates ``mlem_step`` and a denoiser after a warm-up,
  gradients flowing through both;
* ``DenoiserInLoop`` is the demo's training step, projecting through the
  fixed attenuation (the reference's choice) or through a given projector --
  ``xrf.XRFProjector``, so that the loss also sees the self-absorption of C_d.
The network itself is the caller's (the reference's U-Net weights are not
distributed with it).
"""
import torch

from .cuda_lib.atten_cuda import backward_emission_batch, forward_emission_batch
from .cuda_lib.autograd import forward_emission_batch_autograd
from .grad_recon import gradient_loss

__all__ = ["poisson_loss_image", "huber_term", "ratio_backprojection", "mlem_step",
           "sensitivity", "UnrolledMLEM", "DenoiserInLoop"]


def poisson_loss_image(pred, target, eps=1e-6):
    """mean(pred - target * log(pred)), pred clamped below at eps
    (FL/ml_lib/ml_loss.py:6-8)."""
    pred = pred.clamp_min(eps)
    return (pred - target * torch.log(pred)).mean()


def huber_term(C, delta):
    """sum over the four in-plane neighbours of clip(C - C_nbr, -delta, delta)
    (huber_grad_batch, atten_cuda_kernel.cu:495-616), differentiable in C."""
    g = torch.zeros_like(C)
    d = C[..., 1:, :] - C[..., :-1, :]
    d = d.clamp(-delta, delta)
    g = g + torch.nn.functional.pad(d, (0, 0, 1, 0)) - torch.nn.functional.pad(d, (0, 0, 0, 1))
    d = (C[..., :, 1:] - C[..., :, :-1]).clamp(-delta, delta)
    g = g + torch.nn.functional.pad(d, (1, 0)) - torch.nn.functional.pad(d, (0, 1))
    return g


class _RatioBackprojection(torch.autograd.Function):
    @staticmethod
    def forward(ctx, C, atten, em, theta, I):
        Pf = forward_emission_batch(atten, C.contiguous(), em, theta)
        keep = Pf > 1e-6
        Pf = Pf.clamp_min(1e-6)
        back = backward_emission_batch(atten, (I / Pf).contiguous(), em, theta)
        ctx.save_for_backward(atten, em, theta, I, Pf, keep)
        return back

    @staticmethod
    def backward(ctx, g):
        atten, em, theta, I, Pf, keep = ctx.saved_tensors
        Pg = forward_emission_batch(atten, g.contiguous(), em, theta)
        w = torch.where(keep, -I / (Pf * Pf), torch.zeros_like(Pf)) * Pg
        return backward_emission_batch(atten, w.contiguous(), em, theta), None, None, None, None


def ratio_backprojection(C, atten, em, theta, I):
    """P^T (I / max(P C, 1e-6)) for C (R, B, H, W), differentiable in C."""
    return _RatioBackprojection.apply(C, atten, em, theta, I)


def sensitivity(atten, em, theta):
    """max(P^T 1, 1e-6) (atten_cuda.cpp:308-314)."""
    A, B, H, W = atten.shape
    ones = torch.ones((A, B, W), dtype=atten.dtype, device=atten.device)
    return backward_emission_batch(atten, ones, em, theta).clamp_min(1e-6)


def mlem_step(C, atten, em, theta, I, sens, beta=1e-3, delta=0.01):
    """One MLEM update of mlem_cuda_batch (atten_cuda.cpp:321-342),
    differentiable in C: max(C * back / (sens + beta * huber(C)), 0)."""
    back = ratio_backprojection(C, atten, em, theta, I)
    den = sens + beta * huber_term(C, delta) if beta > 0 else sens
    return torch.relu(C * back / den)


class UnrolledMLEM(torch.nn.Module):
    """n_iter MLEM steps with the denoiser applied after each step from
    warmup_iters on (FL/ml_lib/ml_model.py:285-365).  The denoiser maps
    (R, B, H, W) to the same shape.  fine_tune=False detaches between steps."""

    def __init__(self, denoiser, n_iter=10, beta=0.1, delta=0.01, warmup_iters=3):
        super().__init__()
        self.denoiser = denoiser
        self.n_iter = n_iter
        self.beta = beta
        self.delta = delta
        self.warmup_iters = warmup_iters

    def forward(self, C_init, atten, em, theta, I, fine_tune=True):
        sens = sensitivity(atten, em, theta)
        C = C_init.clone()
        for k in range(self.n_iter):
            C = mlem_step(C, atten, em, theta, I, sens, self.beta, self.delta)
            if k >= self.warmup_iters:
                C = self.denoiser(C)
            if not fine_tune:
                C = C.detach()
        return C


class DenoiserInLoop:
    """The training step of FL/example/demo.py:396-475 for one element.

    denoiser    module mapping C (R, B, H, W) to C_d of the same shape.
    atten, em, theta, I   the projector's inputs (A, B, H, W), (A, R), (A,), (A, B, W).
    projector   None: the fixed-attenuation projector (the reference's
                forward_emission_batch_autograd); or a callable C_d -> Pf
                (A, B, W) that is differentiable in C_d, e.g. a lambda over
                xrf.XRFProjector for the gradient through mu.
    weights     (mse, poisson, tv) of the loss; the demo's (1e3, 1, 0.1).
    """

    def __init__(self, denoiser, atten, em, theta, I, projector=None, lr=1e-5,
                 weights=(1e3, 1.0, 0.1), params=None):
        self.denoiser = denoiser
        self.atten, self.em, self.theta, self.I = atten, em, theta, I
        self.projector = projector
        self.weights = weights
        ps = [p for p in (params if params is not None else denoiser.parameters()) if p.requires_grad]
        self.opt = torch.optim.Adam(ps, lr=lr)
        self.history = []

    def loss(self, C):
        C_d = self.denoiser(C)
        if self.projector is None:
            Pf = forward_emission_batch_autograd(self.atten, C_d, self.em, self.theta)
        else:
            Pf = self.projector(C_d)
        Pf = Pf.clamp_min(0)
        mse = torch.nn.functional.mse_loss(Pf, self.I)
        poi = poisson_loss_image(Pf, self.I)
        tv = gradient_loss(C_d)
        wm, wp, wt = self.weights
        return wm * mse + wp * poi + wt * tv, C_d, (float(mse), float(poi), float(tv))

    def step(self, C):
        """One Adam step on the denoiser; returns (total loss, C_d detached)."""
        self.opt.zero_grad(set_to_none=True)
        total, C_d, parts = self.loss(C.detach())
        total.backward()
        self.opt.step()
        self.history.append((float(total),) + parts)
        return float(total), C_d.detach()
