"""generate_detector_mask against the reference's masks, and the rank-one
factorisation the separable cone kernel relies on."""
import numpy as np
import pytest

from fl_correction_b200.detector_mask import factor_mask, generate_detector_mask
from tests.helpers import golden_cpu, golden_meta


@pytest.mark.parametrize("idx", range(6))
def test_mask_matches_reference(idx):
    a, b, L = golden_meta()["mask_cases"][idx]
    ref = golden_cpu()[f"mask{idx}"]
    m = generate_detector_mask(a, b, L)
    assert m.shape == ref.shape
    # float64 masks; the kernels consume them as float32 (7 significant digits)
    assert np.abs(m - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("L", [16, 64, 128, 256])
def test_config_mask_shapes_and_planes(L):
    m = generate_detector_mask(13.309, 13.309, L)
    expect = {16: (3, 16, 3), 64: (15, 64, 15), 128: (29, 128, 29), 256: (59, 256, 59)}[L]
    assert m.shape == expect
    assert np.all(m[:, 0, :] == 0)           # the voxel itself is excluded
    assert np.all(m >= 0)


def test_factorisation_is_exact():
    m = generate_detector_mask(13.309, 13.309, 64)
    u, v = factor_mask(m)
    rec = np.einsum("dz,dy->zdy", u.astype(np.float64), v.astype(np.float64))
    assert np.abs(rec - m).max() <= 1e-6 * m.max()


def test_factorisation_rejects_general_mask():
    rng = np.random.default_rng(0)
    assert factor_mask(rng.random((5, 7, 3))) is None


@pytest.mark.parametrize("idx", range(6))
def test_device_mask_shape_query(idx):
    import ctypes
    from fl_correction_b200 import _lib
    a, b, L = golden_meta()["mask_cases"][idx]
    Mz, Mx, My, nb = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_size_t()
    _lib.call("flc_detector_mask_shape", float(a), float(b), int(L), ctypes.byref(Mz),
              ctypes.byref(Mx), ctypes.byref(My), ctypes.byref(nb))
    assert (Mz.value, Mx.value, My.value) == golden_cpu()[f"mask{idx}"].shape
    assert nb.value > 0


def test_device_mask_rejects_bad_arguments():
    from fl_correction_b200 import _lib
    lib = _lib.load()
    assert lib.flc_detector_mask_shape(0.0, 10.0, 16, None, None, None, None) == 1
    assert lib.flc_detector_mask_shape(10.0, 10.0, 0, None, None, None, None) == 1
    assert lib.flc_detector_mask(10.0, 10.0, 16, None, None, None, None, 0, None) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("idx", range(6))
def test_device_mask_matches_reference(idx):
    from fl_correction_b200.detector_mask import detector_mask_device
    a, b, L = golden_meta()["mask_cases"][idx]
    ref = golden_cpu()[f"mask{idx}"]
    u, v, shape, dense = detector_mask_device(a, b, L, dense=True)
    assert shape == ref.shape
    # the reference's numba mask rounds its FP32 trigonometry differently in
    # the last places (the host restatement meets it to the same bound)
    assert np.abs(dense.cpu().numpy() - ref).max() <= 1e-6 * np.abs(ref).max()
    host = generate_detector_mask(a, b, L)
    assert np.abs(dense.cpu().numpy() - host).max() <= 1e-12 * np.abs(host).max()
    rec = np.einsum("dz,dy->zdy", u.cpu().numpy().astype(np.float64), v.cpu().numpy().astype(np.float64))
    assert np.abs(rec - ref).max() <= 1e-6 * np.abs(ref).max()
