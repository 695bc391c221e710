"""Attenuation maps: rotation (FL/torch_image_util.py:13-114), incident scan
(FL/torch_functions.py:83-106), fluorescence cone (:110-176) and the fused
per-angle pipeline (FL/core.py:19-101), against the reference goldens and
the FP64 oracle."""
import math

import numpy as np
import pytest
import torch

from oracle import oracle as O
from fl_correction_b200 import _lib, core, torch_functions as TF, torch_image_util as TIU
from fl_correction_b200.detector_mask import generate_detector_mask
from tests.helpers import TOL_MAP, T, atten_param, golden_cpu, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    return golden_cpu()


def test_rotation_goldens(g):
    for i, th in enumerate(g["rot_theta"]):
        out = TIU.torch_rotate_image_nd(T(g["rot_x"]), torch.tensor(th, dtype=torch.float64))
        assert rel_err(out.cpu().numpy(), g[f"rot_y{i}"]) < 2e-6, i
    out = TIU.torch_rotate_image_nd(T(g["rot_hw_x"]), 0.61)
    assert rel_err(out.cpu().numpy(), g["rot_hw_y"]) < 2e-6


def test_rotation_oracle_random():
    rng = np.random.default_rng(0)
    x = rng.random((3, 4, 40, 40)).astype(np.float32)
    for th in rng.uniform(-math.pi, math.pi, 5):
        out = TIU.torch_rotate_image_nd(T(x), float(th)).cpu().numpy()
        assert rel_err(out, O.rotate(x, float(th))) < TOL_MAP


def test_rot90_goldens(g):
    x = torch.tensor(g["r90_x"])
    assert np.array_equal(TIU.torch_rot90_4D(x, 0, "clock").numpy(), g["r90_clock"])
    assert np.array_equal(TIU.torch_rot90_4D(x, 0, "c-clock").numpy(), g["r90_cclock"])


def test_xray_atten_golden(g):
    out = TF.torch_xray_atten_3D(T(g["atten_frac"]), atten_param())
    assert isinstance(out, np.ndarray)
    assert rel_err(out, g["atten_x"]) < TOL_MAP


def test_xrf_atten_goldens(g):
    p = atten_param()
    out = TF.torch_xrf_atten_3D(T(g["atten_frac"]), p, g["xrf_mask"], position_det="r")
    assert rel_err(out, g["atten_xrf_r"]) < TOL_MAP
    out = TF.torch_xrf_atten_3D(T(g["atten_frac"]), p, g["xrf_mask"], position_det="l")
    assert rel_err(out, g["atten_xrf_l"]) < TOL_MAP


def test_rotated_pipeline_goldens(g):
    p = atten_param()
    fr = TIU.torch_rotate_image_nd(T(g["atten_frac"]), float(g["pipe_theta"]))
    assert rel_err(TF.torch_xray_atten_3D(fr, p), g["pipe_atten_x"]) < TOL_MAP
    assert rel_err(TF.torch_xrf_atten_3D(fr, p, g["xrf_mask"]), g["pipe_atten_xrf"]) < TOL_MAP


def _pipeline_oracle(frac, angles, cx, cf, mask, incident):
    L = cf.shape[1]
    A = len(angles)
    S, N = frac.shape[1], frac.shape[-1]
    out = np.zeros((L, A, S, N, N))
    for a in range(A):
        fr = O.rotate(frac, np.float32(angles[a] / 180 * np.pi))
        mux = fr * cx[a][:, None, None, None]
        muf = np.einsum("ij,jshw->ishw", cf[a].astype(np.float64), fr)
        res = O.cone_beam(muf, mask.astype(np.float32))
        for i in range(L):
            if incident == "own":
                inc = O.incident_scan(mux[i:i + 1])[0]
            elif incident == "all":
                inc = O.incident_scan(1 - np.prod(1 - mux, axis=0, keepdims=True))[0]
            else:
                inc = 1.0
            out[i, a] = inc * np.exp(-res[i])
    return out


@pytest.mark.parametrize("incident", ["own", "all", "none"])
def test_atten_maps_pipeline(incident):
    rng = np.random.default_rng(1)
    n_ch, S, N, A, L = 3, 6, 24, 7, 2
    frac = (rng.random((n_ch, S, N, N)) * 0.8).astype(np.float32)
    angles = np.array([0, 17, 45, 90, 133.0, 180, 271])
    cx = rng.uniform(0.01, 0.05, (A, n_ch)).astype(np.float32)
    cf = rng.uniform(0.01, 0.05, (A, L, n_ch)).astype(np.float32)
    mask = generate_detector_mask(13.309, 13.309, N)
    ref = _pipeline_oracle(frac, angles, cx, cf, mask, incident)
    uv = core.mask_factors(mask, "cuda")
    out = core.atten_maps(T(frac), angles, cx, cf, uv, incident=incident).cpu().numpy()
    assert rel_err(out, ref) < TOL_MAP
    # the chunked two-stage form with events gives the same maps
    ev = []
    out2 = core.atten_maps(T(frac), angles, cx, cf, uv, incident=incident, chunk=3,
                           cone_events=ev).cpu().numpy()
    assert len(ev) == 3
    assert rel_err(out2, ref) < TOL_MAP


def test_incident_only_mode():
    rng = np.random.default_rng(2)
    frac = (rng.random((2, 4, 16, 16)) * 0.8).astype(np.float32)
    cx = rng.uniform(0.01, 0.05, (3, 2)).astype(np.float32)
    cf = np.zeros((3, 2, 2), np.float32)
    out = core.atten_maps(T(frac), [0, 30, 60], cx, cf, None, incident="own", xrf=False).cpu().numpy()
    for a, ang in enumerate([0, 30, 60]):
        fr = O.rotate(frac, np.float32(ang / 180 * np.pi))
        for i in range(2):
            ref = O.incident_scan(fr[i:i + 1] * cx[a, i])[0]
            assert rel_err(out[i, a], ref) < TOL_MAP


def test_core_api_against_per_angle_reference_composition():
    # FL/core.py:19-101 computes, per angle, rotate -> mu -> scan / cone
    rng = np.random.default_rng(3)
    N, S = 20, 5
    frac = (rng.random((2, S, N, N)) * 0.8).astype(np.float32)
    param = {"elem_type": ["Fe", "Ni"], "elem_compound": ["FeO", "NiO"], "pix": 2e-3,
             "rho": {"FeO": 5.0, "NiO": 6.0}, "em_cs": {"Fe": np.ones(4), "Ni": np.ones(4)},
             "cs": {"elem_type": ["Fe", "Ni"], "elem_compound": ["FeO", "NiO"],
                    "FeO-x": np.array([30.0, 31, 32, 33]), "NiO-x": np.array([25.0, 26, 27, 28]),
                    "FeO-Fe": 40.0, "FeO-Ni": 60.0, "NiO-Fe": 45.0, "NiO-Ni": 50.0}}
    angles = np.array([0.0, 33, 71, 152])
    mask = generate_detector_mask(13.309, 13.309, N)
    xrf = core.cal_xrf_atten_at_angles(T(frac), param, angles, mask).cpu().numpy()
    xray = core.cal_xray_atten_at_angles(T(frac), param, angles).cpu().numpy()
    tot = core.cal_atten_at_angles(T(frac), param, angles, mask).cpu().numpy()
    for a in range(4):
        fr = T(O.rotate(frac, np.float32(angles[a] / 180 * np.pi)))
        from fl_correction_b200.atten_util import extract_single_value_param
        p = extract_single_value_param(param, a)
        ref_x = TF.torch_xray_atten_3D(fr, p)
        ref_f = TF.torch_xrf_atten_3D(fr, p, mask)
        for i in range(2):
            assert rel_err(xray[i, a], ref_x[i]) < TOL_MAP
            assert rel_err(xrf[i, a], ref_f[i]) < TOL_MAP
            assert rel_err(tot[i, a], ref_x[i] * ref_f[i]) < TOL_MAP


def test_errors_for_unsupported_requests():
    x = torch.zeros((2, 3, 8, 8), device="cuda")
    with pytest.raises(NotImplementedError):
        TIU.torch_rotate_image_nd(x, 0.3, enable_crop=False)
    with pytest.raises(RuntimeError):
        TIU.torch_rot90_4D(torch.zeros((1, 3, 4, 5)), 0, "clock")


@pytest.mark.parametrize("n_ch,L", [(3, 2), (4, 3), (6, 4), (8, 1)])
def test_interleaved_stage_matches_planar(n_ch, L):
    # the stage reading a channel-interleaved copy of the fractions gives the
    # planar stage's incident terms and staged mu within the map tolerance (the
    # two builds of the kernel may fuse the multiply-adds of the rotated
    # coordinates differently, which moves a bilinear weight by an ulp)
    rng = np.random.default_rng(n_ch * 10 + L)
    S, N, A, a0, n_a = 5, 20, 6, 1, 4
    frac = T(rng.random((n_ch, S, N, N)).astype(np.float32))
    th = T(np.deg2rad(np.array([0, 17, 45, 90, 133.0, 271])).astype(np.float32))
    cx = T(rng.uniform(0.01, 0.05, (A, n_ch)).astype(np.float32))
    cf = T(rng.uniform(0.01, 0.05, (A, L, n_ch)).astype(np.float32))
    outs = []
    for ws_entry in (False, True):
        out = torch.zeros((L, A, S, N, N), device="cuda")
        mu = torch.zeros((n_a, L, S, N, N), device="cuda")
        for mode in (0, 1):
            if ws_entry:
                nb = _lib.query("flc_atten_stage_workspace_bytes", n_ch, S, N, N)
                ws = _lib.workspace(nb, "cuda")
                _lib.call("flc_atten_stage_ws", _lib.ptr(frac), _lib.ptr(th), _lib.ptr(cx),
                          _lib.ptr(cf), _lib.ptr(out), _lib.ptr(mu), n_ch, S, N, N, A, L, a0, n_a,
                          mode, 1, _lib.ptr(ws), nb, _lib.stream())
            else:
                _lib.call("flc_atten_stage", _lib.ptr(frac), _lib.ptr(th), _lib.ptr(cx),
                          _lib.ptr(cf), _lib.ptr(out), _lib.ptr(mu), n_ch, S, N, N, A, L, a0, n_a,
                          mode, 1, _lib.stream())
            outs.append((out.cpu().numpy().copy(), mu.cpu().numpy().copy()))
    for (o1, m1), (o2, m2) in zip(outs[:2], outs[2:]):
        assert rel_err(o2, o1) < TOL_MAP and rel_err(m2, m1) < TOL_MAP
