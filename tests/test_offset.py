"""detector_offset_angle != 0 (FL/torch_functions.py:134-166): the path sum
toward a detector at 90 - offset degrees to the beam.  The semantics here
(torch_functions.torch_xrf_atten_3D): rotate mu_f by the offset onto a
padded canvas at the same pixel size, cone path sum toward the right, rotate
back, crop; checked against the same composition in FP64 by the oracle, and
against the plain path when the offset vanishes."""
import math

import numpy as np
import pytest

from fl_correction_b200.torch_functions import offset_canvas
from tests.helpers import rel_err


def _rotated_hw(H, W, theta):
    # the canvas size rule of FL/torch_image_util.py:5-10
    c, s = abs(math.cos(theta)), abs(math.sin(theta))
    return int(H * c + W * s + 0.5), int(W * c + H * s + 0.5)


@pytest.mark.parametrize("H,deg", [(20, 15.0), (21, -30.0), (64, 8.0), (33, 90.0)])
def test_canvas_holds_the_rotated_slice_with_whole_padding(H, deg):
    phi = deg / 180 * math.pi
    n = offset_canvas(H, H, phi)
    assert n >= max(_rotated_hw(H, H, phi)) and n >= H
    assert (n - H) % 2 == 0 and 2 <= n - max(max(_rotated_hw(H, H, phi)), H) <= 3


def _oracle_offset(frac, cf, mask, phi):
    from oracle import oracle as O
    mu = np.einsum("ij,jshw->ishw", np.asarray(cf, np.float64), np.asarray(frac, np.float64))
    H, W = mu.shape[-2:]
    n = offset_canvas(H, W, phi)
    pr, pc = (n - H) // 2, (n - W) // 2
    mc = np.zeros(mu.shape[:2] + (n, n))
    mc[..., pr:pr + H, pc:pc + W] = mu
    res = O.rotate(O.cone_beam(O.rotate(mc, np.float32(phi)), mask), np.float32(-phi))
    return np.exp(-res[..., pr:pr + H, pc:pc + W])


@pytest.mark.gpu
@pytest.mark.parametrize("deg", [15.0, -25.0])
def test_offset_path_sum_matches_fp64_composition(deg):
    import torch
    from fl_correction_b200.detector_mask import generate_detector_mask
    from fl_correction_b200.torch_functions import coef_xrf, torch_xrf_atten_3D
    from tests.helpers import atten_param
    rng = np.random.default_rng(11)
    p = atten_param()
    n_ch, S, N = 3, 5, 20
    frac = (rng.random((n_ch, S, N, N)) * 0.8).astype(np.float32)
    frac[:, :, 5:12, 4:15] += 0.3
    mask = generate_detector_mask(13.309, 13.309, N)
    got = torch_xrf_atten_3D(torch.tensor(frac, device="cuda"), p, mask, detector_offset_angle=deg)
    phi = float(np.float32(deg / 180 * np.pi))
    ref = _oracle_offset(frac, coef_xrf(p), mask.astype(np.float32), phi)
    assert rel_err(got, ref) < 1e-5


def test_small_offset_converges_to_the_plain_path():
    """As the offset shrinks, the rotate / path sum / rotate-back composition
    (FP64) approaches the plain path sum.  The bilinear rotations smear mu by
    a fraction of a pixel near the slice edges, where the plain result is 1
    on the detector side: there the difference shrinks only in proportion to
    the offset (0.25 at 0.6 degrees on a 24-pixel slice), so the bound is on
    the mean and on the interior."""
    from fl_correction_b200.detector_mask import generate_detector_mask
    from fl_correction_b200.torch_functions import coef_xrf
    from oracle import oracle as O
    from tests.helpers import atten_param
    rng = np.random.default_rng(12)
    cf = coef_xrf(atten_param())
    frac = (rng.random((3, 4, 24, 24)) * 0.5).astype(np.float32)
    mask = generate_detector_mask(13.309, 13.309, 24).astype(np.float32)
    mu = np.einsum("ij,jshw->ishw", np.asarray(cf, np.float64), frac.astype(np.float64))
    plain = np.exp(-O.cone_beam(mu, mask))
    means = []
    for deg in (5.0, 0.6, 0.2):
        d = np.abs(_oracle_offset(frac, cf, mask, float(np.float32(deg / 180 * np.pi))) - plain)
        means.append(d.mean())
        if deg <= 0.6:
            assert d[..., 3:-3, 3:-3].max() < 0.05
    assert means[0] > means[1] > means[2] and means[2] < 0.003


@pytest.mark.gpu
def test_small_offset_takes_the_rotated_branch():
    """0.6 degrees (just above the 1e-2 rad threshold of the plain branch)
    against the FP64 composition."""
    import torch
    from fl_correction_b200.detector_mask import generate_detector_mask
    from fl_correction_b200.torch_functions import coef_xrf, torch_xrf_atten_3D
    from tests.helpers import atten_param
    rng = np.random.default_rng(12)
    p = atten_param()
    frac = (rng.random((3, 4, 24, 24)) * 0.5).astype(np.float32)
    mask = generate_detector_mask(13.309, 13.309, 24)
    near = torch_xrf_atten_3D(torch.tensor(frac, device="cuda"), p, mask, detector_offset_angle=0.6)
    ref = _oracle_offset(frac, coef_xrf(p), mask.astype(np.float32), float(np.float32(0.6 / 180 * np.pi)))
    assert rel_err(near, ref) < 1e-5
