"""cal_frac (FL/core.py:159-205) on the device (flc_cal_frac), against
goldens recorded from the reference's own cal_frac (threshold mask at its
fallback value 1: scikit-image is absent where the goldens were made), and
the oracle's numpy restatement pinned against the same goldens."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import golden_cpu, golden_meta, rel_err

CASES = [("calfrac_default", dict(scale_range=[0.02, 0.98], enable_scale=True, scale_limit=0.95)),
         ("calfrac_plain", dict(scale_range=[], enable_scale=False)),
         ("calfrac_other", dict(scale_range=[0.1, 0.7], enable_scale=True, scale_limit=0.5))]


@pytest.mark.parametrize("key,kw", CASES)
def test_oracle_restatement_matches_reference(key, kw):
    g = golden_cpu()
    got = O.cal_frac(g["calfrac_img"], **kw)
    assert np.array_equal(got.astype(np.float64), g[key])


@pytest.mark.gpu
@pytest.mark.parametrize("key,kw", CASES)
def test_device_cal_frac_matches_reference(key, kw):
    import torch
    from fl_correction_b200.core import cal_frac
    g = golden_cpu()
    r = cal_frac(torch.tensor(g["calfrac_img"], device="cuda"), **kw)
    got = r["frac"].cpu().numpy()
    # FP32 throughout, as numpy on FP32 volumes; only the division may round
    # differently from numpy's
    assert rel_err(got, g[key]) < 1e-6
    if key == "calfrac_default":
        assert rel_err(r["img_sum"].cpu().numpy(), g["calfrac_default_sum"]) < 1e-7


@pytest.mark.gpu
def test_device_cal_frac_order_statistics_at_size():
    # exact ranks on a volume with many ties and a wide range
    import torch
    from fl_correction_b200.core import cal_frac
    rng = np.random.default_rng(5)
    img = rng.choice(np.array([0.0, 0.25, 0.5, 1.0, 3.0, 1e-30], np.float32), size=(2, 40, 64, 64))
    img = (img * rng.uniform(0.5, 1.5, img.shape)).astype(np.float32)
    for kw in CASES:
        got = cal_frac(torch.tensor(img, device="cuda"), **kw[1])["frac"].cpu().numpy()
        ref = O.cal_frac(img, **kw[1])
        assert rel_err(got, ref) < 1e-6
