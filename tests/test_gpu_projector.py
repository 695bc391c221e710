"""Projector parity: forward_emission[_batch] / backward_emission[_batch]
through the C ABI against the FP64 oracle (atten_cuda_kernel.cu:91-446)."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from fl_correction_b200.cuda_lib import atten_cuda as AC
from fl_correction_b200.cuda_lib import autograd as AG
from tests.helpers import TOL_MAP, T, projector_case, rel_err

pytestmark = pytest.mark.gpu

SPECIAL = [0.0, math.pi / 2, math.pi, -math.pi / 2, math.pi / 4, 3 * math.pi / 4, 1e-7, 2.9]

CASES = [(8, 2, 1, 24, 24), (8, 3, 2, 20, 28), (8, 1, 3, 33, 17), (1, 1, 1, 2, 2),
         (5, 4, 1, 64, 64), (12, 2, 1, 96, 96), (6, 2, 1, 200, 200),
         # an odd slice count (the two-slice forward's last CTA has one slice),
         # non-square slices, a width without a compile-time instance
         (7, 5, 1, 48, 40), (6, 3, 1, 50, 70)]


@pytest.mark.parametrize("A,B,R,H,W", CASES)
def test_forward_batch(A, B, R, H, W):
    rng = np.random.default_rng(A * 1000 + H)
    atten, C, em, th = projector_case(rng, A, B, R, H, W, SPECIAL[:A] if A <= 8 else None)
    out = AC.forward_emission_batch(T(atten), T(C), T(em), T(th)).cpu().numpy()
    assert out.shape == (A, B, W)
    assert rel_err(out, O.fwd_emission(atten, C, em, th)) < TOL_MAP


@pytest.mark.parametrize("A,B,R,H,W", CASES)
def test_backward_batch(A, B, R, H, W):
    rng = np.random.default_rng(A * 1000 + H + 1)
    atten, C, em, th = projector_case(rng, A, B, R, H, W, SPECIAL[:A] if A <= 8 else None)
    ratio = rng.random((A, B, W)).astype(np.float32)
    out = AC.backward_emission_batch(T(atten), T(ratio), T(em), T(th)).cpu().numpy()
    assert out.shape == (R, B, H, W)
    assert rel_err(out, O.bwd_emission(atten, ratio, em, th)) < TOL_MAP


def test_single_slice_forms():
    rng = np.random.default_rng(11)
    atten, C, em, th = projector_case(rng, 9, 1, 2, 30, 30)
    a1, c1 = atten[:, 0], C[:, 0]
    out = AC.forward_emission(T(a1), T(c1), T(em), T(th)).cpu().numpy()
    assert out.shape == (9, 30)
    assert rel_err(out, O.fwd_emission(a1, c1, em, th)) < TOL_MAP
    ratio = rng.random((9, 30)).astype(np.float32)
    back = AC.backward_emission(T(a1), T(ratio), T(em), T(th)).cpu().numpy()
    assert back.shape == (2, 30, 30)
    assert rel_err(back, O.bwd_emission(a1, ratio, em, th)) < TOL_MAP


def test_adjoint_dot_product_full_size():
    # 128^3 slab of the benchmark geometry, 120 angles, FP32 on the GPU
    A, B, H = 120, 8, 128
    g = torch.Generator(device="cuda").manual_seed(0)
    atten = torch.rand((A, B, H, H), device="cuda", generator=g)
    C = torch.rand((1, B, H, H), device="cuda", generator=g)
    y = torch.rand((A, B, H), device="cuda", generator=g)
    em = torch.full((A, 1), 0.02, device="cuda")
    th = torch.linspace(0, math.pi, A + 1, device="cuda")[:-1].contiguous()
    lhs = (AC.forward_emission_batch(atten, C, em, th).double() * y.double()).sum()
    rhs = (C.double() * AC.backward_emission_batch(atten, y, em, th).double()).sum()
    assert abs(float(lhs - rhs)) <= 1e-5 * abs(float(lhs))


def test_linearity_full_size():
    A, B, H = 120, 16, 128
    g = torch.Generator(device="cuda").manual_seed(1)
    atten = torch.rand((A, B, H, H), device="cuda", generator=g)
    X = torch.rand((1, B, H, H), device="cuda", generator=g)
    Y = torch.rand((1, B, H, H), device="cuda", generator=g)
    em = torch.full((A, 1), 0.5, device="cuda")
    th = torch.linspace(0, math.pi, A + 1, device="cuda")[:-1].contiguous()
    P = lambda c: AC.forward_emission_batch(atten, c, em, th).double()
    lhs = P(2 * X + 3 * Y)
    rhs = 2 * P(X) + 3 * P(Y)
    assert float((lhs - rhs).abs().max() / rhs.abs().max()) < TOL_MAP


def test_deterministic_forward():
    rng = np.random.default_rng(5)
    atten, C, em, th = projector_case(rng, 16, 4, 1, 64, 64)
    a, c, e, t = T(atten), T(C), T(em), T(th)
    r1 = AC.forward_emission_batch(a, c, e, t)
    r2 = AC.forward_emission_batch(a, c, e, t)
    assert torch.equal(r1, r2)


def test_autograd_matches_backward():
    rng = np.random.default_rng(6)
    atten, C, em, th = projector_case(rng, 7, 2, 1, 20, 20)
    Ct = T(C).requires_grad_(True)
    Pf = AG.forward_emission_batch_autograd(T(atten), Ct, T(em), T(th))
    w = T(rng.random(Pf.shape))
    (Pf * w).sum().backward()
    ref = O.bwd_emission(atten, w.cpu().numpy(), em, th)
    assert rel_err(Ct.grad.cpu().numpy(), ref) < TOL_MAP
    C1 = T(C[:, 0]).requires_grad_(True)
    P1 = AG.forward_emission_autograd(T(atten[:, 0]), C1, T(em), T(th))
    P1.sum().backward()
    ref1 = O.bwd_emission(atten[:, 0], np.ones((7, 20)), em, th)
    assert rel_err(C1.grad.cpu().numpy(), ref1) < TOL_MAP


def test_shape_errors_raise():
    a = torch.zeros((3, 2, 8, 8), device="cuda")
    with pytest.raises(RuntimeError, match="n_ref"):
        AC.forward_emission_batch(a, torch.zeros((2, 2, 8, 8), device="cuda"),
                                  torch.ones((3, 1), device="cuda"), torch.zeros(3, device="cuda"))
    with pytest.raises(RuntimeError):
        AC.forward_emission_batch(a, torch.zeros((1, 3, 8, 8), device="cuda"),
                                  torch.ones((3, 1), device="cuda"), torch.zeros(3, device="cuda"))
    with pytest.raises(RuntimeError, match="float32"):
        AC.forward_emission_batch(a.double(), a.double()[:1], torch.ones((3, 1), device="cuda"),
                                  torch.zeros(3, device="cuda"))


def test_non_contiguous_inputs():
    rng = np.random.default_rng(7)
    atten, C, em, th = projector_case(rng, 6, 2, 1, 16, 16)
    at = T(atten).transpose(2, 3).contiguous().transpose(2, 3)   # same values, strided
    assert not at.is_contiguous()
    out = AC.forward_emission_batch(at, T(C), T(em), T(th)).cpu().numpy()
    assert rel_err(out, O.fwd_emission(atten, C, em, th)) < TOL_MAP


@pytest.mark.parametrize("mode", [1, 2, 3, 4])
@pytest.mark.parametrize("A,B,R,H,W", [(8, 3, 2, 20, 28), (5, 2, 1, 64, 64), (1, 1, 1, 2, 2),
                                       (4, 2, 1, 112, 112)])
def test_backward_splat_variants(mode, A, B, R, H, W):
    # shared-atomic splat, nine-phase splat, gather and column segments (of 2
    # samples at 64^2, 5 at 112^2) give the same transpose
    from fl_correction_b200 import tune
    rng = np.random.default_rng(A * 1000 + H + 7)
    atten, C, em, th = projector_case(rng, A, B, R, H, W, SPECIAL[:A] if A <= 8 else None)
    ratio = rng.random((A, B, W)).astype(np.float32)
    old = tune.get_knob("proj.bwd")
    tune.set_knob("proj.bwd", mode)
    try:
        out = AC.backward_emission_batch(T(atten), T(ratio), T(em), T(th)).cpu().numpy()
        C0 = np.ones_like(C)
        I = O.fwd_emission(atten, C, em, th)
        mout = AC.mlem_cuda_batch(T(C0), T(atten), T(em), T(th), T(I), 3, 0.0, 0.01).cpu().numpy()
    finally:
        tune.set_knob("proj.bwd", old)
    assert rel_err(out, O.bwd_emission(atten, ratio, em, th)) < TOL_MAP
    assert rel_err(mout, O.mlem(C0, atten, em, th, I, 3, 0.0, 0.01)) < 1e-4

