"""Parity against the reference's own CUDA kernels: fixtures recorded from
the reference extension (tests/golden/ref_gpu.npz, made by
tests/golden/make_golden_refgpu.py) and, when the prebuilt extension is
present in oracle/_ref, a live side-by-side on fresh inputs."""
import os

import numpy as np
import pytest
import torch

from fl_correction_b200.cuda_lib import atten_cuda as AC
from tests.helpers import GOLDEN, TOL_MAP, TOL_MLEM, T, projector_case, rel_err

pytestmark = pytest.mark.gpu
REF_SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                      "ref_atten_cuda.so")


@pytest.fixture(scope="module")
def g():
    p = os.path.join(GOLDEN, "ref_gpu.npz")
    if not os.path.exists(p):
        pytest.skip("reference GPU fixtures not recorded")
    return np.load(p)


def test_cone_fixtures(g):
    assert rel_err(AC.cal_atten_cuda(T(g["cone_mu"]), T(g["cone_mask"])).cpu().numpy(),
                   g["cone_out"]) < TOL_MAP
    assert rel_err(AC.cal_atten_cuda(T(g["cone_mu"]), T(g["cone_gmask"])).cpu().numpy(),
                   g["cone_gout"]) < TOL_MAP


def test_projector_fixtures(g):
    a, c, e, t, r = (T(g[k]) for k in ("p_atten", "p_C", "p_em", "p_theta", "p_ratio"))
    assert rel_err(AC.forward_emission_batch(a, c, e, t).cpu().numpy(), g["p_fwd_batch"]) < TOL_MAP
    assert rel_err(AC.backward_emission_batch(a, r, e, t).cpu().numpy(), g["p_bwd_batch"]) < TOL_MAP
    assert rel_err(AC.forward_emission(a[:, 0].contiguous(), c[:, 0].contiguous(), e, t).cpu().numpy(),
                   g["p_fwd"]) < TOL_MAP
    assert rel_err(AC.backward_emission(a[:, 0].contiguous(), r[:, 0].contiguous(), e, t).cpu().numpy(),
                   g["p_bwd"]) < TOL_MAP


def test_mlem_fixtures(g):
    a, e, t, I = (T(g[k]) for k in ("p_atten", "p_em", "p_theta", "m_I"))
    C0 = torch.ones_like(T(g["p_C"]))
    assert rel_err(AC.mlem_cuda_batch(C0, a, e, t, I, 20, 1e-3, 0.01).cpu().numpy(), g["m_beta"]) < TOL_MLEM
    assert rel_err(AC.mlem_cuda_batch(C0, a, e, t, I, 20, 0.0, 0.01).cpu().numpy(), g["m_nobeta"]) < TOL_MLEM
    out = AC.mlem_cuda(C0[:, 0].contiguous(), a[:, 0].contiguous(), e, t, I[:, 0].contiguous(), 20)
    assert rel_err(out.cpu().numpy(), g["m_single"]) < TOL_MLEM


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_SO):
        pytest.skip("reference extension not built (python oracle/build_ref.py)")
    from oracle.build_ref import load_built
    return load_built()


def test_live_side_by_side(ref):
    rng = np.random.default_rng(9)
    atten, C, em, th = projector_case(rng, 30, 8, 1, 64, 64)
    a, c, e, t = T(atten), T(C), T(em), T(th)
    assert rel_err(AC.forward_emission_batch(a, c, e, t).cpu().numpy(),
                   ref.forward_emission_batch(a, c, e, t).cpu().numpy()) < TOL_MAP
    r = T(rng.random((30, 8, 64)))
    assert rel_err(AC.backward_emission_batch(a, r, e, t).cpu().numpy(),
                   ref.backward_emission_batch(a, r, e, t).cpu().numpy()) < TOL_MAP
    import fl_correction_b200.detector_mask as dm
    mask = T(dm.generate_detector_mask(13.309, 13.309, 32))
    mu = T(rng.random((2, 16, 32, 32)) * 0.05)
    assert rel_err(AC.cal_atten_cuda(mu, mask).cpu().numpy(), ref.cal_atten_cuda(mu, mask).cpu().numpy()) < TOL_MAP
    I = ref.forward_emission_batch(a, c, e, t) * 1.1
    C0 = torch.ones_like(c)
    assert rel_err(AC.mlem_cuda_batch(C0, a, e, t, I, 20).cpu().numpy(),
                   ref.mlem_cuda_batch(C0, a, e, t, I, 20).cpu().numpy()) < TOL_MLEM
