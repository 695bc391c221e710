"""The CPU oracle against golden vectors produced by the reference's own code
(tests/golden/make_golden.py).  These pin the oracle before it is trusted as
the checker of the CUDA kernels."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import golden_cpu, golden_meta, rel_err


@pytest.fixture(scope="module")
def g():
    return golden_cpu()


def test_rotation_matches_grid_sample(g):
    # FP32 grid_sample vs the FP64 restatement: FP32 rounding of the sample
    # coordinates only (values ~3)
    for i, th in enumerate(g["rot_theta"]):
        assert rel_err(O.rotate(g["rot_x"], th), g[f"rot_y{i}"]) < 2e-6, i


def test_rotation_non_square(g):
    assert rel_err(O.rotate(g["rot_hw_x"], 0.61), g["rot_hw_y"]) < 2e-6


def test_incident_scan(g):
    assert rel_err(O.incident_scan(g["mu_x"]), g["atten_x"]) < 1e-6


def test_cone_reference_layout(g):
    assert rel_err(O.cone_ref(g["cone_mu"], g["xrf_mask"]), g["cone_out"]) < 1e-12


def test_cone_beam_frame_equals_rot90_composition(g):
    # torch_xrf_atten_3D (position 'r'): exp(-rot90^-1(cone(rot90(mu_f))))
    res = O.cone_beam(g["mu_xrf"], g["xrf_mask"].astype(np.float32))
    assert rel_err(np.exp(-res), g["atten_xrf_r"]) < 1e-6


def test_cone_beam_left_detector_is_mirror(g):
    # detector on the left: the same path sum on the w-mirrored volume
    mu = g["mu_xrf"][..., ::-1]
    res = O.cone_beam(mu, g["xrf_mask"].astype(np.float32))[..., ::-1]
    assert rel_err(np.exp(-res), g["atten_xrf_l"]) < 1e-6


def test_rotated_pipeline(g):
    th = float(g["pipe_theta"])
    fr = O.rotate(g["atten_frac"], th)
    meta = golden_meta()["atten_param"]
    cs, rho, pix = meta["cs"], meta["rho"], meta["pix"]
    comps, elems = cs["elem_compound"], cs["elem_type"]
    cx = [float(np.float32(np.asarray(cs[f"{c}-x"]).reshape(-1)[0] * rho[c] * pix)) for c in comps]
    mux = np.stack([fr[j] * cx[j] for j in range(len(comps))])
    assert rel_err(O.incident_scan(mux), g["pipe_atten_x"]) < 2e-6
    muf = np.zeros_like(fr)
    for i, e in enumerate(elems):
        for j, c in enumerate(comps):
            muf[i] += fr[j] * float(np.float32(cs[f"{c}-{e}"] * rho[c] * pix))
    res = O.cone_beam(muf, g["xrf_mask"].astype(np.float32))
    assert rel_err(np.exp(-res), g["pipe_atten_xrf"]) < 2e-6


def test_oracle_matches_reference_cuda_kernels():
    """Pin the oracle against outputs of the reference's own CUDA extension
    (tests/golden/ref_gpu.npz, recorded by make_golden_refgpu.py)."""
    import os
    from tests.helpers import GOLDEN
    p = os.path.join(GOLDEN, "ref_gpu.npz")
    if not os.path.exists(p):
        pytest.skip("reference GPU fixtures not recorded")
    r = np.load(p)
    assert rel_err(O.cone_ref(r["cone_mu"], r["cone_mask"]), r["cone_out"]) < 1e-6
    assert rel_err(O.cone_ref(r["cone_mu"], r["cone_gmask"]), r["cone_gout"]) < 1e-6
    a, C, em, th, ratio = r["p_atten"], r["p_C"], r["p_em"], r["p_theta"], r["p_ratio"]
    assert rel_err(O.fwd_emission(a, C, em, th), r["p_fwd_batch"]) < 1e-6
    assert rel_err(O.bwd_emission(a, ratio, em, th), r["p_bwd_batch"]) < 1e-6
    assert rel_err(O.fwd_emission(a[:, 0], C[:, 0], em, th), r["p_fwd"]) < 1e-6
    assert rel_err(O.bwd_emission(a[:, 0], ratio[:, 0], em, th), r["p_bwd"]) < 1e-6
    C0 = np.ones_like(C)
    assert rel_err(O.mlem(C0, a, em, th, r["m_I"], 20, 1e-3, 0.01), r["m_beta"]) < 1e-5
    assert rel_err(O.mlem(C0, a, em, th, r["m_I"], 20, 0.0, 0.01), r["m_nobeta"]) < 1e-5
    assert rel_err(O.mlem(C0[:, 0], a[:, 0], em, th, r["m_I"][:, 0], 20, 1e-3, 0.01),
                   r["m_single"]) < 1e-5
