"""Algebraic properties of the oracle: exact transposes (dot-product tests in
FP64) and MLEM invariants."""
import numpy as np

from oracle import oracle as O
from fl_correction_b200.detector_mask import generate_detector_mask
from tests.helpers import projector_case, rel_err


def _dot(a, b):
    return float(np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64)))


def test_projector_adjoint_fp64():
    rng = np.random.default_rng(1)
    for (A, B, R, H, W) in [(7, 2, 2, 24, 24), (5, 1, 1, 17, 23)]:
        atten, C, em, th = projector_case(rng, A, B, R, H, W)
        y = rng.random((A, B, W))
        lhs = _dot(O.fwd_emission(atten, C, em, th), y)
        rhs = _dot(C, O.bwd_emission(atten, y, em, th))
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_projector_datten_is_derivative():
    rng = np.random.default_rng(2)
    atten, C, em, th = projector_case(rng, 6, 2, 1, 12, 12)
    g = rng.random((6, 2, 12))
    d = O.fwd_emission_datten(g, C, em, th)
    dA = rng.random(atten.shape)
    eps = 1e-3
    lhs = (_dot(O.fwd_emission(atten + eps * dA, C, em, th), g) -
           _dot(O.fwd_emission(atten - eps * dA, C, em, th), g)) / (2 * eps)
    assert abs(lhs - _dot(d, dA)) <= 1e-9 * abs(lhs)


def test_rotation_adjoint_fp64():
    rng = np.random.default_rng(3)
    x = rng.random((2, 19, 19))
    y = rng.random((2, 19, 19))
    for th in (0.0, 0.4, 2.2):
        assert abs(_dot(O.rotate(x, th), y) - _dot(x, O.rotate_adjoint(y, th))) < 1e-10


def test_cone_adjoint_fp64():
    rng = np.random.default_rng(4)
    mask = generate_detector_mask(13.309, 13.309, 16)
    x = rng.random((1, 7, 16, 16))
    y = rng.random((1, 7, 16, 16))
    assert abs(_dot(O.cone_beam(x, mask), y) - _dot(x, O.cone_beam_adjoint(y, mask))) < 1e-9


def test_cone_slab_matches_full():
    rng = np.random.default_rng(5)
    mask = generate_detector_mask(13.309, 13.309, 12)
    x = rng.random((2, 9, 12, 12))
    full = O.cone_beam(x, mask)
    slab = O.cone_beam_slab(x, mask, 3, 6)
    assert np.allclose(slab[:, 3:6], full[:, 3:6], rtol=0, atol=1e-14)
    assert np.all(slab[:, :3] == 0)


def test_mlem_keeps_consistent_solution():
    # noise-free data generated from C_true: C_true is a fixed point (beta=0)
    rng = np.random.default_rng(6)
    atten, C, em, th = projector_case(rng, 9, 2, 1, 16, 16)
    C = C + 0.5
    I = O.fwd_emission(atten, C, em, th)
    out = O.mlem(C, atten, em, th, I, 5, beta=0.0)
    # pixels no ray reaches (sens clamped to 1e-6, back = 0) drop to zero
    seen = O.bwd_emission(atten, np.ones((9, 2, 16)), em, th) > 1e-3
    assert np.abs(out - C)[seen].max() < 1e-10
    assert np.all(out[~seen] == 0)


def test_mlem_nonnegative_and_huber():
    rng = np.random.default_rng(7)
    atten, C, em, th = projector_case(rng, 9, 2, 2, 16, 16)
    I = O.fwd_emission(atten, C, em, th) * rng.uniform(0.5, 1.5, (9, 2, 16))
    out = O.mlem(np.ones_like(C), atten, em, th, I, 10, beta=1e-3, delta=0.01)
    assert np.all(out >= 0)
    g = O.huber_grad(C, 0.05)
    assert np.abs(g).max() <= 4 * 0.05 + 1e-15


def test_xrf_adjoint_matches_finite_differences():
    # the full-mu adjoint (projector + attenuation) against central differences
    rng = np.random.default_rng(5)
    n_ch, S, N, A, L = 3, 3, 8, 3, 2
    frac = rng.random((n_ch, S, N, N)) * 0.8
    th = np.array([0.3, 1.7, -2.4], np.float32)
    cx = rng.uniform(0.02, 0.1, (A, n_ch))
    cf = rng.uniform(0.02, 0.1, (A, L, n_ch))
    mask = rng.random((3, 4, 5))
    em = rng.uniform(0.5, 2, (L, A))
    for inc in ["own", "all", "none"]:
        Pf = O.xrf_project(frac, th, cx, cf, mask, em, inc)
        g = rng.standard_normal(Pf.shape)
        dC = O.xrf_project_adjoint(frac, th, cx, cf, mask, em, g, inc)
        for _ in range(2):
            d = np.zeros_like(frac)
            d[:L] = rng.standard_normal((L, S, N, N))
            eps = 1e-6
            jp = _dot(g, O.xrf_project(frac + eps * d, th, cx, cf, mask, em, inc))
            jm = _dot(g, O.xrf_project(frac - eps * d, th, cx, cf, mask, em, inc))
            fd = (jp - jm) / (2 * eps)
            an = _dot(dC, d[:L])
            assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (inc, fd, an)


def test_xrf_project_equals_atten_then_projector():
    # forward = per-angle attenuation maps followed by the projector
    rng = np.random.default_rng(6)
    n_ch, S, N, A, L = 2, 2, 10, 2, 2
    frac = rng.random((n_ch, S, N, N)) * 0.8
    th = np.array([0.9, -1.1], np.float32)
    cx = rng.uniform(0.02, 0.1, (A, n_ch))
    cf = rng.uniform(0.02, 0.1, (A, L, n_ch))
    mask = rng.random((3, 3, 3))
    em = rng.uniform(0.5, 2, (L, A))
    Pf = O.xrf_project(frac, th, cx, cf, mask, em, "own")
    for a in range(A):
        fr = O.rotate(frac, th[a])
        E = np.exp(-O.cone_beam(np.einsum("ij,jshw->ishw", cf[a], fr), mask))
        for l in range(L):
            att = O.incident_scan(fr[l:l + 1] * cx[a, l])[0] * E[l]
            ref = O.fwd_emission(att[None], frac[l:l + 1], em[l, a].reshape(1, 1), th[a:a + 1])[0]
            assert rel_err(Pf[l, a], ref) < 1e-12


def test_xrf_adjoint_matches_torch_autograd_fp64():
    # a third, independent composition: torch operators (grid_sample, cumprod,
    # conv3d, gathers) differentiated by autograd in FP64
    import torch
    from tests import torch_model as TM
    rng = np.random.default_rng(8)
    n_ch, S, N, A, L = 3, 3, 10, 3, 2
    frac = rng.random((n_ch, S, N, N)) * 0.8
    th = np.array([0.3, 1.7, -2.4], np.float32)
    cx = rng.uniform(0.02, 0.1, (A, n_ch))
    cf = rng.uniform(0.02, 0.1, (A, L, n_ch))
    mask = generate_detector_mask(13.309, 13.309, N)
    em = rng.uniform(0.5, 2, (L, A))
    for inc in ["own", "all", "none"]:
        ref = O.xrf_project(frac, th, cx, cf, mask, em, inc)
        C = torch.tensor(frac[:L], dtype=torch.float64, requires_grad=True)
        Pf = TM.xrf_project(torch.cat([C, torch.tensor(frac[L:])]), th, cx, cf, mask, em, inc)
        assert rel_err(Pf.detach().numpy(), ref) < 1e-6
        g = rng.standard_normal(ref.shape)
        (Pf * torch.tensor(g)).sum().backward()
        assert rel_err(C.grad.numpy(), O.xrf_project_adjoint(frac, th, cx, cf, mask, em, g, inc)) < 1e-6
