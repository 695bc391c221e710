"""The row-band backward projection (no global atomics) against the FP64
oracle: forced at small sizes through the "proj.band" knob, and where it runs
by itself, on slices whose image does not fit in shared memory (256^2); the
lean kernels at 192^2 beside it.  Backward projection, sensitivity (ratio 1,
clamped) and 20 MLEM iterations."""
import contextlib

import numpy as np
import pytest

from oracle import oracle as O
from fl_correction_b200 import _lib
from fl_correction_b200.cuda_lib import atten_cuda as AC
from tests.helpers import TOL_MAP, TOL_MLEM, T, projector_case, rel_err

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def band_forced(on=True):
    lib = _lib.load()
    assert lib.flc_tune_set(b"proj.band", 1 if on else 0) == 0
    try:
        yield
    finally:
        lib.flc_tune_set(b"proj.band", 0)


def _bwd(rng, A, B, R, H, W, angles=None):
    atten, _, em, th = projector_case(rng, A, B, R, H, W, angles)
    ratio = rng.uniform(0.5, 1.5, (A, B, W)).astype(np.float32)
    out = AC.backward_emission_batch(T(atten), T(ratio), T(em), T(th)).cpu().numpy()
    return out, O.bwd_emission(atten, ratio, em, th)


@pytest.mark.parametrize("A,B,R,H,W", [(12, 3, 1, 40, 40), (9, 2, 2, 30, 36), (16, 1, 1, 64, 64),
                                       (7, 2, 1, 37, 23)])
def test_band_backward_forced(A, B, R, H, W):
    rng = np.random.default_rng(A * H + W)
    with band_forced():
        out, ref = _bwd(rng, A, B, R, H, W)
    assert rel_err(out, ref) < TOL_MAP


def test_band_backward_axis_angles():
    """0, 45, 90, ... degrees: the line orientation switches at |cos| = |sin|,
    and samples land exactly on band edges."""
    rng = np.random.default_rng(11)
    angles = np.deg2rad(np.arange(0, 360, 22.5)).astype(np.float32)
    with band_forced():
        out, ref = _bwd(rng, len(angles), 2, 1, 48, 48, angles)
    assert rel_err(out, ref) < TOL_MAP


def test_band_sensitivity_forced():
    rng = np.random.default_rng(5)
    A, B, H, W = 10, 2, 44, 44
    atten, _, em, th = projector_case(rng, A, B, 1, H, W)
    # P^T 1, the sensitivity of the MLEM driver before its clamp
    ones = np.ones((A, B, W), np.float32)
    with band_forced():
        out = AC.backward_emission_batch(T(atten), T(ones), T(em), T(th)).cpu().numpy()
    assert rel_err(out, O.bwd_emission(atten, ones, em, th)) < TOL_MAP


@pytest.mark.parametrize("beta", [1e-3, 0.0])
def test_band_mlem_forced(beta):
    rng = np.random.default_rng(17)
    A, B, R, H, W = 12, 2, 1, 48, 48
    atten, C, em, th = projector_case(rng, A, B, R, H, W)
    I = O.fwd_emission(atten, C, em, th) * rng.uniform(0.8, 1.2, (A, B, W))
    C0 = np.ones_like(C)
    with band_forced():
        out = AC.mlem_cuda_batch(T(C0), T(atten), T(em), T(th), T(I), 20, beta, 0.01).cpu().numpy()
    assert rel_err(out, O.mlem(C0, atten, em, th, I, 20, beta, 0.01)) < TOL_MLEM


@pytest.mark.parametrize("N", [192, 256])
def test_large_slice_backward(N):
    """256^2 does not fit the lean kernel (the band kernel runs by itself);
    192^2 does."""
    rng = np.random.default_rng(N)
    out, ref = _bwd(rng, 12, 2, 1, N, N)
    assert rel_err(out, ref) < TOL_MAP


@pytest.mark.parametrize("N", [192, 256])
def test_large_slice_mlem(N):
    rng = np.random.default_rng(N + 1)
    A, B = 30, 2
    atten, C, em, th = projector_case(rng, A, B, 1, N, N)
    I = O.fwd_emission(atten, C, em, th) * rng.uniform(0.8, 1.2, (A, B, N))
    C0 = np.ones_like(C)
    out = AC.mlem_cuda_batch(T(C0), T(atten), T(em), T(th), T(I), 20, 1e-3, 0.01).cpu().numpy()
    assert rel_err(out, O.mlem(C0, atten, em, th, I, 20, 1e-3, 0.01)) < TOL_MLEM


def test_band_matches_lean_bitwise_order_free():
    """The band and lean backward add the same products in different orders:
    equal to FP32 rounding."""
    rng = np.random.default_rng(23)
    atten, _, em, th = projector_case(rng, 20, 3, 1, 64, 64)
    ratio = rng.uniform(0.5, 1.5, (20, 3, 64)).astype(np.float32)
    lean = AC.backward_emission_batch(T(atten), T(ratio), T(em), T(th)).cpu().numpy()
    with band_forced():
        band = AC.backward_emission_batch(T(atten), T(ratio), T(em), T(th)).cpu().numpy()
    assert rel_err(band, lean) < 2e-6
