"""Gradient-based reconstruction through the self-absorption model.

The reference's gradient loop (FL/example/demo.py:413-475) differentiates
the projector only (`forward_emission_batch_autograd`, attenuation held
fixed) and recomputes the attenuation outside the graph.  Here the loss is
differentiated through the attenuation too: `XRFProjector` rebuilds the
attenuation of each angle chunk from the current concentrations inside the
forward and again inside the hand-written adjoint, so nothing of size
angles x volume is stored between them.

Loss (per step):  mean((P(C) - I)^2) / mean(I^2) + tv_weight * TV(C), with
TV the reference's `gradient_loss` (FL/ml_lib/ml_loss.py:13-16): the mean
absolute in-plane differences along rows and along columns.  The misfit is
relative (1 for C = 0) so that its gradient does not sink under Adam's
epsilon when the projections are small numbers.  Optimiser: Adam on C,
FP32, with C clamped at zero after each step.
"""
import numpy as np
import torch

from .xrf import XRFProjector

__all__ = ["gradient_loss", "GradientRecon"]


def gradient_loss(x):
    """Mean |x[..., 1:, :] - x[..., :-1, :]| + mean |x[..., :, 1:] - x[..., :, :-1]|
    (FL/ml_lib/ml_loss.py:13-16)."""
    dx = x[..., 1:, :] - x[..., :-1, :]
    dy = x[..., :, 1:] - x[..., :, :-1]
    return dx.abs().mean() + dy.abs().mean()


class GradientRecon:
    """Adam reconstruction of C (L, S, H, W) from projections I (L, A, S, W).

    param, angles_deg, mask, shape, fixed_frac, incident, chunk: as
    `XRFProjector`.  tv_weight: weight of `gradient_loss`.  lr: Adam step.
    """

    def __init__(self, param, angles_deg, mask, shape, fixed_frac=None, incident="own",
                 tv_weight=1e-3, lr=1e-2, device="cuda", chunk=0):
        self.proj = XRFProjector(param, angles_deg, mask, shape, fixed_frac=fixed_frac,
                                 incident=incident, device=device, chunk=chunk)
        self.tv_weight = float(tv_weight)
        self.lr = float(lr)
        self.device = self.proj.device

    def loss(self, C, I):
        """(total, misfit, tv) for C with requires_grad as needed."""
        misfit = torch.mean((self.proj(C) - I) ** 2) / torch.mean(I.detach() ** 2)
        tv = gradient_loss(C)
        return misfit + self.tv_weight * tv, misfit, tv

    def gradient(self, C, I):
        """d loss / d C (a new tensor) and the loss value."""
        Cv = C.detach().clone().requires_grad_(True)
        total, _, _ = self.loss(Cv, I)
        total.backward()
        return Cv.grad, float(total.detach())

    def run(self, I, C0=None, n_steps=200, history=None):
        """n_steps of Adam from C0 (default ones); returns C.  `history`, if a
        list, receives the loss after every step."""
        L = self.proj.L
        S, H, W = self.proj.shape
        if C0 is None:
            C = torch.ones((L, S, H, W), dtype=torch.float32, device=self.device)
        else:
            C = torch.as_tensor(C0, dtype=torch.float32, device=self.device).clone()
        C.requires_grad_(True)
        opt = torch.optim.Adam([C], lr=self.lr)
        I = I.contiguous()
        for _ in range(int(n_steps)):
            opt.zero_grad(set_to_none=True)
            total, _, _ = self.loss(C, I)
            total.backward()
            opt.step()
            with torch.no_grad():
                C.clamp_(min=0.0)
            if history is not None:
                history.append(float(total.detach()))
        return C.detach()


def misfit_np(Pf, I):
    """Host helper: mean squared misfit in FP64."""
    return float(np.mean((np.asarray(Pf, np.float64) - np.asarray(I, np.float64)) ** 2))
