"""torch_2D_xray_atten_with_ref and its vectorised form
(FL/torch_functions.py:181-215, :247-330): the FP64 oracle against the
reference's own outputs, and the native kernel (flc_xray_atten_ref2d)
against both."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import golden_cpu, golden_meta

KEYS = ("C", "C_other", "theta", "cs_ref", "rho")


def _case():
    g = golden_cpu()
    return [g["xray2d_" + k] for k in KEYS] + [golden_meta()["xray2d_pix"]]


@pytest.mark.parametrize("variant,key", [(0, "xray2d_out"), (1, "xray2d_vec_out")])
def test_oracle_matches_reference(variant, key):
    ref = golden_cpu()[key]
    out = O.xray_atten_ref2d(*_case(), variant=variant)
    assert out.shape == ref.shape
    assert np.abs(out - ref).max() <= 1e-5 * np.abs(ref).max()


def test_the_two_forms_differ_where_the_reference_does():
    """The vectorised form's product includes row h: its values are the
    plain form's times f[h] (up to its own eps, floor and rotation)."""
    g = golden_cpu()
    a, b = g["xray2d_out"], g["xray2d_vec_out"]
    assert np.all(a[:, -1] == 1) and np.all(b[:, -1] == 1)
    assert np.abs(a - b).max() > 1e-2


def test_rejects_bad_arguments():
    from fl_correction_b200 import _lib
    lib = _lib.load()
    assert lib.flc_xray_atten_ref2d_workspace_bytes() >= 4
    args = [None] * 5 + [0.05, None, 1, 1, 8, 8, 0, None, 0, None]
    assert lib.flc_xray_atten_ref2d(*args) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("variant,key", [(0, "xray2d_out"), (1, "xray2d_vec_out")])
def test_kernel_matches_reference_and_oracle(variant, key):
    import torch
    from fl_correction_b200 import torch_functions as tf
    C, Co, th, cs, rho, pix = _case()
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (C, Co, th, cs, rho)]
    fn = tf.torch_2D_xray_atten_with_ref if variant == 0 else \
        tf.torch_2D_xray_atten_with_ref_vectorize
    out = fn(*t, pix).cpu().numpy()
    ref = golden_cpu()[key]
    assert np.abs(out - ref).max() <= 1e-5 * np.abs(ref).max()
    orc = O.xray_atten_ref2d(C, Co, th, cs, rho, pix, variant=variant)
    assert np.abs(out - orc).max() <= 1e-5 * np.abs(orc).max()


@pytest.mark.gpu
def test_kernel_square_slice_many_angles():
    """A 64^2 slice at 90 angles (scalar rho) against the oracle."""
    import torch
    from fl_correction_b200 import torch_functions as tf
    rng = np.random.default_rng(5)
    N, A, R = 64, 90, 2
    C = rng.random((R, N, N)).astype(np.float32)
    Co = np.zeros((N, N), np.float32)
    th = np.linspace(0, np.pi, A, endpoint=False).astype(np.float32)
    cs = (rng.random((A, R)) * 0.4).astype(np.float32)
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(a).to(dev) for a in (C, Co, th, cs)]
    for v, fn in ((0, tf.torch_2D_xray_atten_with_ref),
                  (1, tf.torch_2D_xray_atten_with_ref_vectorize)):
        out = fn(*t, 3.0, 0.1).cpu().numpy()
        orc = O.xray_atten_ref2d(C, Co, th, cs, np.full((N, N), 3.0), 0.1, variant=v)
        assert np.abs(out - orc).max() <= 2e-5 * np.abs(orc).max()
