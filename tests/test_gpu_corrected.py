"""Parity of the corrected MLEM itself (recon.CorrectedMLEM, the benchmarked
loop) on the 64^3 x 60-angle workload exactly as the benchmark configuration
states it: ellipsoid phantom, Fe K-alpha, Poisson noise at 1e4 counts, 20
iterations with the attenuation rebuilt every 5.  Compared with two
compositions that share none of this repository's kernels: the FP64 oracle
(tests/compose.py) and the reference's own kernels (cal_atten_cuda and
mlem_cuda_batch of FL/cuda_lib, built from its sources into oracle/_ref)
driven by the reference's torch steps.  Bar: 1e-4 (max|a-b|/max|b|), the
bar of 20 MLEM iterations."""
import os

import numpy as np
import pytest
import torch

from fl_correction_b200 import phantoms
from fl_correction_b200.detector_mask import generate_detector_mask
from fl_correction_b200.recon import CorrectedMLEM
from tests import compose
from tests.helpers import TOL_MLEM, rel_err

pytestmark = pytest.mark.gpu
REF_SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                      "ref_atten_cuda.so")


@pytest.fixture(scope="module")
def cfg0():
    wl = phantoms.make_workload(0)
    N = wl.N
    dev = torch.device("cuda", 0)
    mask = generate_detector_mask(wl.mask_angle, wl.mask_angle, N)
    solver = CorrectedMLEM(wl.param, wl.angles, mask, (N, N, N), device=dev)
    truth = torch.from_numpy(wl.conc).to(dev)
    solver.recompute_attenuation(truth)
    I = solver.project(truth)
    g = torch.Generator(device=dev).manual_seed(wl.seed)
    scale = wl.noise_max_counts / float(I.max())
    I = (torch.poisson(I * scale, generator=g) / scale).contiguous()
    C = solver.run(I, n_iter=wl.n_iter, recompute_every=wl.recompute_every)
    torch.cuda.synchronize()
    return wl, mask, I, C


def test_cfg0_corrected_mlem_vs_fp64_oracle(cfg0):
    wl, mask, I, C = cfg0
    N = wl.N
    ref = compose.oracle_corrected_mlem(wl.param, wl.angles, mask, I.cpu().numpy(),
                                        np.ones((1, N, N, N)), wl.n_iter, wl.recompute_every)
    e = compose.relative_errors(C.cpu().numpy(), ref)
    print("cfg0 vs oracle", e)
    assert rel_err(C.cpu().numpy(), ref) < TOL_MLEM


def test_cfg0_corrected_mlem_vs_reference_kernels(cfg0):
    if not os.path.exists(REF_SO):
        pytest.skip("reference extension not built (python oracle/build_ref.py)")
    from oracle.build_ref import load_built
    refext = load_built()
    wl, mask, I, C = cfg0
    N = wl.N
    fixed = torch.ones((1, N, N, N), device=I.device)
    Cr = compose.reference_corrected_mlem(refext, wl.param, wl.angles, mask, I, fixed,
                                          wl.n_iter, wl.recompute_every)
    e = compose.relative_errors(C.cpu().numpy(), Cr.cpu().numpy())
    print("cfg0 vs reference", e)
    assert rel_err(C.cpu().numpy(), Cr.cpu().numpy()) < TOL_MLEM


def test_cal_frac_feedback_vs_reference_kernels():
    """The corrected loop with the reference's own feedback step (cal_frac,
    FL/example/demo.py:249-265) on a smaller workload of the same kind."""
    if not os.path.exists(REF_SO):
        pytest.skip("reference extension not built (python oracle/build_ref.py)")
    from oracle.build_ref import load_built
    refext = load_built()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(3)
    N, A = 40, 36
    conc = phantoms.ellipsoid_grains(N, rng)[None]
    angles = np.linspace(0, 180, A, endpoint=False)
    param = phantoms.xrf_params(["Fe"], A, 12.0, 1.6e-4)
    mask = generate_detector_mask(13.309, 13.309, N)
    solver = CorrectedMLEM(param, angles, mask, (N, N, N), device=dev, feedback="cal_frac")
    truth = torch.from_numpy(conc).to(dev)
    solver.recompute_attenuation(truth)
    I = solver.project(truth).contiguous()
    C = solver.run(I, n_iter=10, recompute_every=5)
    Cr = compose.reference_corrected_mlem(refext, param, angles, mask, I,
                                          torch.ones((1, N, N, N), device=dev), 10, 5,
                                          feedback="cal_frac")
    assert rel_err(C.cpu().numpy(), Cr.cpu().numpy()) < TOL_MLEM


def test_concurrent_elements_match_the_sequential_loop():
    # the elements' MLEM chains on one stream each (the default) against one
    # after another on the caller's stream: 3 elements at 96^3 x 90 angles,
    # 10 iterations with a rebuild every 5, from the same projections
    wl = phantoms.make_workload(2)
    N = wl.N
    dev = torch.device("cuda", 0)
    mask = generate_detector_mask(wl.mask_angle, wl.mask_angle, N)
    frac = wl.frac()
    L = len(wl.elements)
    out = {}
    for conc in (False, True):
        s = CorrectedMLEM(wl.param, wl.angles, mask, (N, N, N), fixed_frac=frac[L:], device=dev,
                          concurrent=conc)
        truth = torch.from_numpy(wl.conc).to(dev)
        s.recompute_attenuation(truth)
        I = s.project(truth).contiguous()
        ev = []
        out[conc] = s.run(I, n_iter=10, recompute_every=5, mlem_events=ev).cpu().numpy()
        assert sum(v for _, _, v in ev) == 10 * L
    assert rel_err(out[True], out[False]) < 1e-6
