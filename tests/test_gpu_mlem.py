"""MLEM parity: mlem_cuda[_batch] (FL/cuda_lib/atten_cuda.cpp:244-345) and
the numpy drivers of FL/torch_recon.py against the FP64 oracle after 20
iterations (bar 1e-4)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from fl_correction_b200 import _lib, torch_recon
from fl_correction_b200.cuda_lib import atten_cuda as AC
from tests.helpers import TOL_MLEM, T, projector_case, rel_err

pytestmark = pytest.mark.gpu


def _problem(rng, A, B, R, H, W):
    atten, C, em, th = projector_case(rng, A, B, R, H, W)
    I = O.fwd_emission(atten, C, em, th) * rng.uniform(0.8, 1.2, (A, B, W))
    return atten, C, em, th, I


@pytest.mark.parametrize("A,B,R,H,W", [(12, 4, 1, 64, 64), (9, 3, 2, 20, 28), (30, 2, 1, 48, 48)])
@pytest.mark.parametrize("beta", [1e-3, 0.0])
def test_mlem_batch_20_iterations(A, B, R, H, W, beta):
    rng = np.random.default_rng(A + H)
    atten, C, em, th, I = _problem(rng, A, B, R, H, W)
    C0 = np.ones_like(C)
    out = AC.mlem_cuda_batch(T(C0), T(atten), T(em), T(th), T(I), 20, beta, 0.01).cpu().numpy()
    assert rel_err(out, O.mlem(C0, atten, em, th, I, 20, beta, 0.01)) < TOL_MLEM


def test_mlem_unfused_path_large_slice():
    # 200x200 slices do not fit the fused kernel's shared memory.  (With very
    # few angles the pixels that only the corner of a footprint reaches have a
    # sensitivity made of FP32 fractions whose absolute error ~ulp(200) is
    # comparable to the value itself, so 30 angles keep the problem well posed.)
    rng = np.random.default_rng(2)
    atten, C, em, th, I = _problem(rng, 30, 1, 1, 200, 200)
    C0 = np.ones_like(C)
    out = AC.mlem_cuda_batch(T(C0), T(atten), T(em), T(th), T(I), 20, 1e-3, 0.01).cpu().numpy()
    assert rel_err(out, O.mlem(C0, atten, em, th, I, 20, 1e-3, 0.01)) < TOL_MLEM


def test_mlem_single_slice():
    rng = np.random.default_rng(3)
    atten, C, em, th, I = _problem(rng, 10, 1, 1, 32, 32)
    out = AC.mlem_cuda(T(C[:, 0] * 0 + 1), T(atten[:, 0]), T(em), T(th), T(I[:, 0]), 20).cpu().numpy()
    ref = O.mlem(np.ones_like(C[:, 0]), atten[:, 0], em, th, I[:, 0], 20, 1e-3, 0.01)
    assert rel_err(out, ref) < TOL_MLEM


def test_graph_and_eager_agree_and_input_untouched():
    rng = np.random.default_rng(4)
    atten, C, em, th, I = _problem(rng, 12, 4, 1, 32, 32)
    C0 = T(np.ones_like(C))
    keep = C0.clone()
    out_graph = AC.mlem_cuda_batch(C0, T(atten), T(em), T(th), T(I), 7)
    assert torch.equal(C0, keep)
    C1 = C0.clone()
    ws_b = _lib.query("flc_mlem_workspace_bytes", 12, 4, 1, 32, 32)
    ws = _lib.workspace(ws_b, "cuda")
    a, e, t, i = T(atten), T(em), T(th), T(I)
    _lib.call("flc_mlem", _lib.ptr(C1), _lib.ptr(a), _lib.ptr(e), _lib.ptr(t), _lib.ptr(i), 7,
              1e-3, 0.01, 12, 4, 1, 32, 32, _lib.ptr(ws), ws_b, 0, _lib.stream())
    # same iterations; the backward's shared-memory atomics sum in run-dependent order
    assert rel_err(C1.cpu().numpy(), out_graph.cpu().numpy()) < 1e-5


def test_numpy_drivers():
    rng = np.random.default_rng(5)
    A, S, H = 15, 3, 24
    atten, C, em, th, I = _problem(rng, A, S, 1, H, H)
    angles = th.astype(np.float64) * 180 / np.pi
    em1 = em[:, 0].astype(np.float64)
    out = torch_recon.torch_mlem_recon_batch(np.ones_like(C), I, angles, atten=atten, em_cs=em1,
                                             rho=2.0, pix=0.5, n_iter=20)
    th32 = (angles / 180 * np.pi).astype(np.float32)
    ref = O.mlem(np.ones_like(C), atten, (em1 * 2.0 * 0.5)[:, None], th32, I, 20, 1e-3, 0.01)
    assert rel_err(out, ref) < TOL_MLEM
    out1 = torch_recon.torch_mlem_recon(np.ones((1, H, H)), I[:, 0], angles, atten=atten[:, 0],
                                        em_cs=em1, rho=2.0, pix=0.5, n_iter=20)
    ref1 = O.mlem(np.ones((1, H, H)), atten[:, 0], (em1 * 2.0 * 0.5)[:, None], th32, I[:, 0], 20,
                  1e-3, 0.01)
    assert rel_err(out1, ref1) < TOL_MLEM


def test_huber_api():
    rng = np.random.default_rng(6)
    C = rng.random((2, 3, 17, 19)).astype(np.float32)
    g = torch.empty((2, 3, 17, 19), device="cuda")
    AC.huber_grad_batch(T(C), g, 0.05)
    assert rel_err(g.cpu().numpy(), O.huber_grad(C, 0.05)) < 1e-6


@pytest.mark.parametrize("shapes,beta", [([(12, 4, 32), (30, 3, 32), (7, 5, 32)], 1e-3),
                                         ([(24, 16, 64), (24, 16, 64), (24, 16, 64)], 0.0),
                                         ([(9, 2, 20)], 1e-3),
                                         # uneven slice sizes in one launch
                                         # (angle counts that keep each problem well posed)
                                         ([(24, 3, 40), (16, 2, 24), (36, 4, 64), (48, 2, 96)], 1e-3)])
def test_mlem_multi_matches_per_problem(shapes, beta):
    """flc_mlem_multi (one persistent launch per iteration for all problems)
    against flc_mlem per problem and the oracle."""
    rng = np.random.default_rng(len(shapes) + int(beta * 1e3))
    Cs, ats, ems, ths, Is, refs = [], [], [], [], [], []
    for (A, B, N) in shapes:
        atten, C, em, th, I = _problem(rng, A, B, 1, N, N)
        Cs.append(T(np.ones_like(C)))
        ats.append(T(atten)); ems.append(T(em)); ths.append(T(th)); Is.append(T(I))
        refs.append(O.mlem(np.ones_like(C), atten, em, th, I, 7, beta, 0.01))
    singles = [AC.mlem_cuda_batch(c.clone(), a, e, t, i, 7, beta, 0.01)
               for c, a, e, t, i in zip(Cs, ats, ems, ths, Is)]
    _lib.mlem_multi(Cs, ats, ems, ths, Is, 7, beta, 0.01)
    for c, s1, ref in zip(Cs, singles, refs):
        assert rel_err(c.cpu().numpy(), s1.cpu().numpy()) < 1e-5
        assert rel_err(c.cpu().numpy(), ref) < TOL_MLEM


def test_corrected_mlem_multi_equals_per_element():
    from fl_correction_b200 import phantoms
    from fl_correction_b200.detector_mask import generate_detector_mask
    from fl_correction_b200.recon import CorrectedMLEM
    rng = np.random.default_rng(8)
    N, A = 32, 24
    conc = phantoms.voronoi_grains(N, rng, 2, n_seeds=12)
    conc = (conc * 0.4).astype(np.float32)
    angles = np.linspace(0, 180, A, endpoint=False)
    param = phantoms.xrf_params(["Fe", "Ni"], A, 14.0, 4e-4)
    mask = generate_detector_mask(13.309, 13.309, N)
    outs = []
    for multi in (False, True):
        s = CorrectedMLEM(param, angles, mask, (N, N, N), multi=multi)
        truth = torch.from_numpy(conc).cuda()
        s.recompute_attenuation(truth)
        I = s.project(truth).contiguous()
        outs.append(s.run(I, n_iter=6, recompute_every=3).cpu().numpy())
    assert rel_err(outs[1], outs[0]) < 1e-5
