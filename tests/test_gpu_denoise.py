"""Denoiser-in-the-loop training (fl_correction_b200/denoise.py): the
differentiable MLEM step against the native MLEM iteration and against FP64
torch autograd of the projector model (tests/torch_model.py), and the
training step of FL/example/demo.py:396-475 on a small problem."""
import numpy as np
import pytest
import torch

from fl_correction_b200 import denoise
from fl_correction_b200.cuda_lib import atten_cuda as AC
from tests import torch_model as TM
from tests.helpers import T, projector_case, rel_err

pytestmark = pytest.mark.gpu


def _case(seed=0, A=10, B=2, H=20, W=20):
    rng = np.random.default_rng(seed)
    atten, C, em, th = projector_case(rng, A, B, 1, H, W)
    C = C + 0.2
    I = np.stack([TM.project(torch.tensor(atten[a], dtype=torch.float64),
                             torch.tensor(C[0], dtype=torch.float64), float(em[a, 0]),
                             th[a]).numpy() for a in range(A)]) * rng.uniform(0.9, 1.1, (A, B, W))
    return atten, C, em, th, I


def _p64(atten, C, em, th):
    """P C in FP64 torch: (A, B, W)."""
    return torch.stack([TM.project(atten[a], C[0], float(em[a, 0]), th[a]) for a in range(len(th))])


def test_mlem_step_equals_native_iteration():
    atten, C, em, th, I = _case(1)
    a, c, e, t, i = T(atten), T(C), T(em), T(th), T(I)
    for beta in (0.0, 1e-3):
        sens = denoise.sensitivity(a, e, t)
        got = denoise.mlem_step(c, a, e, t, i, sens, beta, 0.01)
        ref = AC.mlem_cuda_batch(c, a, e, t, i, 1, beta, 0.01)
        assert rel_err(got.detach().cpu().numpy(), ref.cpu().numpy()) < 1e-5


def test_ratio_backprojection_vjp_matches_fp64_autograd():
    atten, C, em, th, I = _case(2)
    a, e, t, i = T(atten), T(em), T(th), T(I)
    rng = np.random.default_rng(3)
    g = rng.standard_normal(C.shape).astype(np.float32)
    c = T(C).requires_grad_(True)
    back = denoise.ratio_backprojection(c, a, e, t, i)
    (got,) = torch.autograd.grad(back, c, T(g))
    # FP64: back(C) = P^T (I / P C) = d/dC' <I / P C, P C'>; its vjp by double autograd
    a64 = torch.tensor(atten, dtype=torch.float64)
    I64 = torch.tensor(I, dtype=torch.float64)
    C64 = torch.tensor(C, dtype=torch.float64, requires_grad=True)
    r = I64 / _p64(a64, C64, em, th)
    Cp = torch.zeros_like(C64, requires_grad=True)
    (b64,) = torch.autograd.grad((r * _p64(a64, Cp, em, th)).sum(), Cp, create_graph=True)
    assert rel_err(back.detach().cpu().numpy(), b64.detach().numpy()) < 1e-5
    (ref,) = torch.autograd.grad(b64, C64, torch.tensor(g, dtype=torch.float64))
    assert rel_err(got.cpu().numpy(), ref.numpy()) < 1e-4


def test_unrolled_mlem_gradient_reaches_the_denoiser():
    atten, C, em, th, I = _case(4)
    a, e, t, i = T(atten), T(em), T(th), T(I)
    net = torch.nn.Conv2d(1, 1, 3, padding=1, bias=False).cuda()
    with torch.no_grad():
        net.weight.zero_()
        net.weight[0, 0, 1, 1] = 1.0
    den = lambda x: net(x.reshape(-1, 1, *x.shape[-2:])).reshape(x.shape)  # noqa: E731
    model = denoise.UnrolledMLEM(den, n_iter=4, beta=0.0, warmup_iters=2)
    out = model(torch.ones_like(T(C)), a, e, t, i)
    out.sum().backward()
    assert net.weight.grad is not None and torch.isfinite(net.weight.grad).all()
    assert float(net.weight.grad.abs().sum()) > 0
    # identity denoiser: the unrolled model is 4 plain MLEM iterations
    ref = AC.mlem_cuda_batch(torch.ones_like(T(C)), a, e, t, i, 4, 0.0, 0.01)
    assert rel_err(out.detach().cpu().numpy(), ref.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("through_mu", [False, True])
def test_training_step_lowers_the_loss(through_mu):
    from fl_correction_b200 import phantoms
    from fl_correction_b200.detector_mask import generate_detector_mask
    from fl_correction_b200.recon import CorrectedMLEM
    from fl_correction_b200.xrf import XRFProjector
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(6)
    N, A = 24, 18
    conc = phantoms.ellipsoid_grains(N, rng)[None]
    angles = np.linspace(0, 180, A, endpoint=False)
    param = phantoms.xrf_params(["Fe"], A, 12.0, 4e-4)
    mask = generate_detector_mask(13.309, 13.309, N)
    s = CorrectedMLEM(param, angles, mask, (N, N, N), device=dev)
    truth = torch.from_numpy(conc).to(dev)
    s.recompute_attenuation(truth)
    I = s.project(truth)[0].contiguous()                     # (A, S, W)
    C = s.run(I[None], n_iter=5, recompute_every=5)          # (1, S, H, W)
    net = torch.nn.Conv3d(1, 1, 3, padding=1).to(dev)
    with torch.no_grad():
        net.weight.zero_()
        net.weight[0, 0, 1, 1, 1] = 0.7
        net.bias.zero_()
    den = lambda x: net(x[None])[0]  # noqa: E731
    proj = None
    if through_mu:
        xp = XRFProjector(param, angles, mask, (N, N, N), device=dev)
        proj = lambda Cd: xp(Cd)[0]  # noqa: E731
    loop = denoise.DenoiserInLoop(den, s.atten[0], s.em[0], s.theta, I, projector=proj, lr=1e-2,
                                  params=net.parameters())
    first, _ = loop.step(C)
    for _ in range(15):
        last, _ = loop.step(C)
    assert np.isfinite(last) and last < first
