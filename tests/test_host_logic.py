"""Host-side logic that needs no GPU: parameter selection, coefficient
assembly, the bench's work counts, phantoms."""
import numpy as np
import pytest
import torch

import bench
from fl_correction_b200 import atten_util, core, phantoms, torch_functions
from fl_correction_b200.detector_mask import generate_detector_mask
from tests.helpers import atten_param, golden_cpu, golden_meta, rel_err


def _param_from_meta():
    m = golden_meta()["param"]
    cs = {k: (np.asarray(v) if isinstance(v, list) and k not in ("elem_type", "elem_compound") else v)
          for k, v in m["cs"].items()}
    return {"cs": cs, "rho": m["rho"], "pix": m["pix"], "elem_type": m["elem_type"],
            "elem_compound": m["elem_compound"],
            "em_cs": {k: np.asarray(v) for k, v in m["em_cs"].items()}}


def test_extract_single_value_param_matches_reference():
    param = _param_from_meta()
    for a, ref in enumerate(golden_meta()["param_selected"]):
        p = atten_util.extract_single_value_param(param, a)
        for k, v in ref["cs"].items():
            if k in ("elem_type", "elem_compound"):
                assert p["cs"][k] == v
            else:
                assert np.allclose(np.asarray(p["cs"][k]), np.asarray(v)), k
        for k, v in ref["em_cs"].items():
            assert np.allclose(np.asarray(p["em_cs"][k]), np.asarray(v)), k


def test_extract_em_cs_elem():
    param = _param_from_meta()
    assert np.allclose(atten_util.extract_em_cs_elem(param, "Ni"), golden_meta()["em_cs_elem_Ni"])


def test_mu_assembly_matches_reference():
    g = golden_cpu()
    p = atten_param()
    f = torch.tensor(g["atten_frac"])
    assert rel_err(torch_functions.torch_extract_3D_mu_xray(f, p).numpy(), g["mu_x"]) < 1e-7
    assert rel_err(torch_functions.torch_extract_3D_mu_xrf(f, p).numpy(), g["mu_xrf"]) < 1e-6


def test_atten_coefficients_layout():
    wl = phantoms.make_workload(0)
    cx, cf = core.atten_coefficients(wl.param, len(wl.angles))
    assert cx.shape == (60, 2) and cf.shape == (60, 1, 2)
    c = wl.param["elem_compound"][0]
    assert np.isclose(cx[3, 0], wl.param["cs"][f"{c}-x"][3] * wl.param["rho"][c] * wl.param["pix"])
    assert np.isclose(cx[0, 1], phantoms.MATRIX_MU * wl.param["pix"])


def test_cone_work_counts():
    m = generate_detector_mask(13.309, 13.309, 128)
    nnz, sep = bench.cone_work(m, 128, 128, 128)
    assert abs(nnz / 1.92e10 - 1) < 0.01
    assert abs(sep / 2.74e9 - 1) < 0.01


def test_mlem_bytes():
    assert abs(3 * bench.mlem_bytes_per_iter(120, 128, 128, 128) / 6.28e9 - 1) < 0.01


def test_pick_chunk():
    assert core.pick_chunk(128, 128, 128, 120, 3) == 10      # 256 MB of staged mu
    assert core.pick_chunk(64, 64, 64, 60, 1) == 60
    assert core.pick_chunk(8, 8, 8, 100000, 3, chunk=100000) == 65535 // 3


def test_phantoms_are_seeded():
    a = phantoms.make_workload(0).conc
    b = phantoms.make_workload(0).conc
    assert np.array_equal(a, b)
    assert a.min() > 0.04 and a.sum(axis=0).max() <= 0.9 + 1e-6   # mass fractions
    v = phantoms.voronoi_grains(24, np.random.default_rng(0), 2, n_seeds=8)
    assert v.shape == (2, 24, 24, 24) and v.max() <= 3.0


def test_optical_depth_in_range():
    wl = phantoms.make_workload(1)
    cx, cf = core.atten_coefficients(wl.param, 1)
    depth = (wl.conc.mean(axis=(1, 2, 3)) * cf[0, :, :3].max(axis=0)).max() * wl.N
    assert 0.1 < depth < 5


def test_assign_streams_balances_work():
    from fl_correction_b200.batch import assign_streams
    works = [100, 10, 90, 50, 40, 5, 5]
    g = assign_streams(works, 3)
    assert sorted(i for grp in g for i in grp) == list(range(len(works)))
    loads = [sum(works[i] for i in grp) for grp in g]
    assert max(loads) - min(loads) <= 20
    assert assign_streams([1, 2], 4) == [[1], [0]]


def test_batch_workloads_are_seeded_and_in_range():
    ws = phantoms.make_batch_workloads(6, sizes=(16, 24))
    ws2 = phantoms.make_batch_workloads(6, sizes=(16, 24))
    for a, b in zip(ws, ws2):
        assert a.name == b.name and np.array_equal(a.conc, b.conc)
        assert 1 <= len(a.elements) <= 3 and 60 <= len(a.angles) <= 180
        assert a.N in (16, 24) and 10.0 <= a.energy <= 16.0
