"""Reference-spectrum (XANES) incident cross section: the per-voxel mix of
reference spectra of FL/torch_functions.py:22-37 and
FL/cross_section_util.py:44-66, against goldens recorded from the reference's
own torch_xray_atten_3D with its update_dict_use_ref_at_angle rotation
(tests/golden/make_golden.py)."""
import numpy as np
import pytest

from fl_correction_b200.core import atten_coefficients, ref_coefficients
from tests.helpers import golden_cpu, golden_meta, rel_err


def _param():
    m = golden_meta()["xref"]
    p = m["param"]
    cs = {k: (np.asarray(v) if isinstance(v, list) and k not in ("elem_type", "elem_compound") else v)
          for k, v in p["cs"].items()}
    param = {"cs": cs, "rho": p["rho"], "pix": p["pix"], "elem_type": p["elem_type"],
             "elem_compound": p["elem_compound"],
             "em_cs": {k: np.asarray(v) for k, v in p["em_cs"].items()}}
    return param, m


def _mu_ref_numpy(fr_rot, ref_rot, spec, rho, pix):
    """The kernel's incident mu of the reference compound, in numpy FP64."""
    tot = ref_rot.astype(np.float64).sum(0) + 1e-12
    cs = sum(s * np.maximum(r / tot, 0.0) for s, r in zip(spec, ref_rot.astype(np.float64)))
    return fr_rot * cs * rho * pix


def test_ref_coefficients_select_per_angle():
    param, m = _param()
    A = len(m["angles_deg"])
    cr, ch = ref_coefficients(param, A, m["ref_comp"])
    assert ch == param["elem_compound"].index(m["ref_comp"])
    rho, pix = param["rho"][m["ref_comp"]], param["pix"]
    sel = np.array(m["selected_x_ref"]) * rho * pix
    assert np.allclose(cr[m["angle_id"]], sel, rtol=1e-6)


def test_reference_mix_formula_matches_reference_mu():
    # pins the formula the stage kernel evaluates against the reference's own
    # mu_x, on the reference-rotated inputs
    g = golden_cpu()
    param, m = _param()
    ch = param["elem_compound"].index(m["ref_comp"])
    rho, pix = param["rho"][m["ref_comp"]], param["pix"]
    import torch
    from oracle import oracle as O
    th = m["angles_deg"][m["angle_id"]] / 180.0 * np.pi
    fr_rot = O.rotate(g["xref_frac"], th)
    mu = _mu_ref_numpy(fr_rot[ch], g["xref_ref3d_rot"], m["selected_x_ref"], rho, pix)
    assert rel_err(mu, g["xref_mu_x"][ch]) < 2e-6
    # and the other channels are the scalar cross sections
    cx, _ = atten_coefficients(param, len(m["angles_deg"]), 3)
    for j in range(3):
        if j != ch:
            assert rel_err(fr_rot[j] * cx[m["angle_id"], j], g["xref_mu_x"][j]) < 2e-6


@pytest.mark.gpu
def test_stage_kernel_with_reference_volumes():
    import torch
    from fl_correction_b200.core import atten_maps, cal_xray_atten_at_angles
    g = golden_cpu()
    param, m = _param()
    dev = torch.device("cuda", 0)
    A = len(m["angles_deg"])
    a = m["angle_id"]
    cx, cf = atten_coefficients(param, A, 3)
    cr, ch = ref_coefficients(param, A, m["ref_comp"])
    frac = torch.tensor(g["xref_frac"], device=dev)
    ref3 = torch.tensor(g["xref_ref3d"], device=dev)
    out = atten_maps(frac, [m["angles_deg"][a]], cx[a:a + 1], cf[a:a + 1], None, incident="own",
                     xrf=False, ref=(ref3, cr[a:a + 1], ch))
    L = cf.shape[1]
    ref = g["xref_atten_x"][:L]
    assert rel_err(out[:, 0].cpu().numpy(), ref) < 1e-5
    # the reference's core function drops the reference volumes; apply_ref applies them
    d = {"use_ref": True, "ref_3D": g["xref_ref3d"], "ref_comp": m["ref_comp"]}
    plain = cal_xray_atten_at_angles(frac, param, m["angles_deg"], d)
    noref = atten_maps(frac, m["angles_deg"], cx, cf, None, incident="own", xrf=False)
    assert torch.equal(plain, noref)
    withref = cal_xray_atten_at_angles(frac, param, m["angles_deg"], d, apply_ref=True)
    assert rel_err(withref[:, a].cpu().numpy(), ref) < 1e-5


@pytest.mark.gpu
def test_torch_xray_atten_3D_with_reference_dict():
    import torch
    from fl_correction_b200.atten_util import extract_single_value_param, update_dict_use_ref_at_angle
    from fl_correction_b200.torch_functions import torch_xray_atten_3D
    from fl_correction_b200.torch_image_util import torch_rotate_image_nd
    g = golden_cpu()
    param, m = _param()
    dev = torch.device("cuda", 0)
    a = m["angle_id"]
    ang = m["angles_deg"][a]
    d = {"use_ref": True, "ref_3D": g["xref_ref3d"], "ref_comp": m["ref_comp"]}
    d_rot = update_dict_use_ref_at_angle(d, ang)
    assert rel_err(np.asarray(d_rot["ref_3D"]), g["xref_ref3d_rot"]) < 1e-5
    p_a = extract_single_value_param(param, a, d_rot)
    fr_rot = torch_rotate_image_nd(torch.tensor(g["xref_frac"], device=dev), ang / 180.0 * np.pi)
    out = torch_xray_atten_3D(fr_rot, p_a, d_rot)
    assert rel_err(out, g["xref_atten_x"]) < 1e-5
