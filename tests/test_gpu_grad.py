"""Gradient reconstruction through the self-absorption model: the hand-written
adjoint against torch autograd of an operator-level composition in FP64 on
the GPU, the full loss gradient against FP64 central differences of the
oracle, and Adam steps that lower the loss."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from fl_correction_b200.detector_mask import generate_detector_mask
from fl_correction_b200.grad_recon import GradientRecon, gradient_loss
from tests import torch_model as TM
from tests.helpers import T, rel_err
from tests.test_gpu_xrf import _case

pytestmark = pytest.mark.gpu


def test_adjoint_matches_torch_autograd_fp64_on_gpu():
    p, angles, mask, frac, rng = _case(31, n_ch=3, L=2, S=4, N=16, A=6)
    S, N = frac.shape[1], frac.shape[-1]
    rec = GradientRecon(p, angles, mask, (S, N, N), fixed_frac=frac[2:])
    proj = rec.proj
    th, cx, cf, em = (proj.theta.cpu().numpy(), proj.coef_x.cpu().numpy(),
                      proj.coef_f.cpu().numpy(), proj.em.cpu().numpy())
    C64 = torch.tensor(frac[:2], dtype=torch.float64, device="cuda", requires_grad=True)
    fr = torch.cat([C64, torch.tensor(frac[2:], dtype=torch.float64, device="cuda")])
    Pf64 = TM.xrf_project(fr, th, cx, cf, mask, em)
    g = rng.standard_normal(tuple(Pf64.shape)).astype(np.float32)
    (Pf64 * torch.tensor(g, dtype=torch.float64, device="cuda")).sum().backward()
    dC = proj.adjoint(T(frac[:2]), T(g)).cpu().numpy()
    assert rel_err(dC, C64.grad.cpu().numpy()) < 2e-5


def _oracle_loss(recon, frac, mask, C, I, tv_weight):
    proj = recon.proj
    f = frac.copy()
    f[:C.shape[0]] = C
    Pf = O.xrf_project(f, proj.theta.cpu().numpy(), proj.coef_x.cpu().numpy(),
                       proj.coef_f.cpu().numpy(), mask, proj.em.cpu().numpy())
    tv = float(gradient_loss(torch.tensor(C, dtype=torch.float64)))
    return float(np.mean((Pf - I) ** 2) / np.mean(I ** 2)) + tv_weight * tv


def test_loss_gradient_matches_fp64_central_differences():
    # the cfg2 check (FD, eps = 1e-4, random voxels, FP64) at a small size
    p, angles, mask, frac, rng = _case(32, n_ch=3, L=2, S=3, N=16, A=5)
    S, N = frac.shape[1], frac.shape[-1]
    rec = GradientRecon(p, angles, mask, (S, N, N), fixed_frac=frac[2:], tv_weight=1e-3)
    C = frac[:2].astype(np.float64)
    I = rec.proj.project(T(C * 0.8 + 0.1)).cpu().numpy().astype(np.float64)
    g, _ = rec.gradient(T(C), T(I))
    g = g.cpu().numpy()
    eps = 1e-4
    for _ in range(16):
        idx = tuple(int(rng.integers(0, n)) for n in C.shape)
        Cp, Cm = C.copy(), C.copy()
        Cp[idx] += eps
        Cm[idx] -= eps
        f64 = frac.astype(np.float64)
        fd = (_oracle_loss(rec, f64, mask, Cp, I, 1e-3)
              - _oracle_loss(rec, f64, mask, Cm, I, 1e-3)) / (2 * eps)
        assert abs(g[idx] - fd) <= 2e-3 * np.abs(g).max(), (idx, g[idx], fd)


def test_adam_steps_lower_the_loss():
    p, angles, mask, frac, rng = _case(33, n_ch=2, L=2, S=4, N=24, A=12)
    S, N = frac.shape[1], frac.shape[-1]
    rec = GradientRecon(p, angles, mask, (S, N, N), tv_weight=1e-3, lr=1e-2)
    I = rec.proj.project(T(frac))
    hist = []
    C = rec.run(I, n_steps=40, history=hist)
    assert hist[-1] < 0.25 * hist[0]
    assert float(C.min()) >= 0.0
