"""CPU checks of the test-side compositions in tests/compose.py: the restated
reference steps equal the reference's own torch functions (goldens recorded
from FL/torch_functions.py by tests/golden/make_golden.py), and the FP64
oracle composition of the corrected loop is self-consistent on a slab."""
import numpy as np
import torch

from oracle import oracle as O
from tests import compose
from tests.helpers import atten_param, golden_cpu, rel_err


class _CpuRef:
    """Stands in for the reference extension on the CPU: cal_atten_cuda by
    the oracle's restatement of atten_kernel (atten_cuda_kernel.cu:10-57)."""

    @staticmethod
    def cal_atten_cuda(mu, mask):
        return torch.tensor(O.cone_ref(mu.numpy(), mask.numpy()), dtype=torch.float32)


def test_reference_steps_match_reference_torch_functions():
    g = golden_cpu()
    p = atten_param()
    comps, elems = p["elem_compound"], p["elem_type"]
    cs, rho, pix = p["cs"], p["rho"], p["pix"]
    cx = np.array([[float(cs[f"{c}-x"]) * rho[c] * pix for c in comps]], np.float32)
    cf = np.array([[[float(cs[f"{c}-{e}"]) * rho[c] * pix for c in comps] for e in elems]],
                  np.float32)
    frac = torch.tensor(g["atten_frac"])
    th = float(g["pipe_theta"])
    att = compose.reference_atten(_CpuRef, frac, [th], cx, cf, g["xrf_mask"])
    ref = g["pipe_atten_x"][:len(elems)] * g["pipe_atten_xrf"][:len(elems)]
    assert rel_err(att[:, 0].numpy(), ref) < 2e-6


def test_rot90_matches_reference():
    g = golden_cpu()
    x = torch.tensor(g["r90_x"])
    assert np.array_equal(compose._rot90(x, "clock").numpy(), g["r90_clock"])
    assert np.array_equal(compose._rot90(x, "c-clock").numpy(), g["r90_cclock"])


def test_bounded_fractions():
    C = np.array([[[0.5, 1.4, -0.2]], [[0.7, 0.1, 0.3]]])
    f = compose.bounded_fractions(C)
    assert np.allclose(f[:, 0, 0], [0.5 / 1.2, 0.7 / 1.2])
    assert np.allclose(f[:, 0, 1], [1.0 / 1.1, 0.1 / 1.1])
    assert np.allclose(f[:, 0, 2], [0.0, 0.3])


def test_oracle_slab_equals_full_volume():
    """The slab form of the oracle composition gives the full-volume result
    on its valid slices (the cone couples hz = Mz // 2 planes per rebuild)."""
    from fl_correction_b200 import phantoms
    from fl_correction_b200.detector_mask import generate_detector_mask
    rng = np.random.default_rng(3)
    N, A, S = 12, 6, 16
    angles = np.linspace(0, 180, A, endpoint=False)
    param = phantoms.xrf_params(["Fe"], A, 12.0, 2e-3)
    mask = generate_detector_mask(25.0, 25.0, N)
    hz = mask.shape[0] // 2
    fixed = np.ones((1, S, N, N))
    I = rng.uniform(0.5, 1.5, (1, A, S, N))
    full = compose.oracle_corrected_mlem(param, angles, mask, I, fixed, 4, 2)
    k = 2                                   # rebuilds
    z0, z1 = 5, 7
    lo, hi = max(0, z0 - k * hz), min(S, z1 + k * hz)
    slab = compose.oracle_corrected_mlem(param, angles, mask, I[:, :, lo:hi], fixed[:, lo:hi], 4, 2,
                                         z_range=(z0 - lo, z1 - lo))
    assert hz >= 1 and lo > 0
    assert np.allclose(slab[:, z0 - lo:z1 - lo], full[:, z0:z1], rtol=1e-12, atol=0)


def test_relative_errors():
    e = compose.relative_errors(np.array([1.0, 2.0, 0.0011]), np.array([1.0, 2.2, 0.001]), 1e-2)
    assert abs(e["max_abs_over_max"] - 0.2 / 2.2) < 1e-12
    assert abs(e["pointwise_max_rel"] - 0.2 / 2.2) < 1e-12   # 0.001 is below the floor
