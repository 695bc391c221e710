"""Per-angle parameter selection with the signatures of FL/atten_util.py.

Cross sections are plain numbers supplied by the caller (the reference gets
them from xraylib, FL/atten_util.py:14-39, which this package does not use).
"""
from copy import deepcopy

import numpy as np
import torch

__all__ = ["extract_single_value_param", "extract_em_cs_elem", "update_dict_use_ref_at_angle",
           "get_atten_coef"]


def get_atten_coef(elem_type, elem_compound, XEng_list, em_E):
    """Needs xraylib (FL/atten_util.py:14-39); raises ImportError when absent."""
    import xraylib  # noqa: F401  (deliberately unguarded)
    cs = {"elem_type": elem_type, "elem_compound": elem_compound, "x": XEng_list}
    for c in elem_compound:
        cs[f"{c}-x"] = np.array([xraylib.CS_Total_CP(c, e) for e in XEng_list])
        for e in elem_type:
            cs[f"{c}-{e}"] = xraylib.CS_Total_CP(c, em_E[e])
    return cs


def extract_em_cs_elem(param, elem, use_ref=False):
    """Emission cross sections of one element; with use_ref, an (n, n_ref)
    matrix from '<elem>_ref<k>' entries (FL/atten_util.py:63-76)."""
    em_cs_dict = param["em_cs"]
    em_cs = em_cs_dict[elem]
    n = len(em_cs)
    if use_ref:
        try:
            n_ref = em_cs_dict["n_ref"]
            em_cs = np.zeros((n, n_ref))
            for i in range(n_ref):
                em_cs[:, i] = em_cs_dict[f"{elem}_ref{i + 1}"]
        except Exception as err:  # the reference prints and returns the plain entry
            print(err)
            print(f"fail to extract em_cs for {elem} using reference")
    return em_cs


def update_dict_use_ref_at_angle(dict_use_ref, current_angle):
    """Copy of dict_use_ref with every reference volume of 'ref_3D' rotated by
    current_angle degrees (FL/atten_util.py:79-88), as the reference's rot3D
    does (scipy.ndimage.rotate, order 1, zero outside the slice;
    torch_image_util.rot3D_scipy on the device).  numpy in, float32 numpy
    out, as rot3D returns; a cuda tensor stays on its device."""
    d = deepcopy(dict_use_ref)
    if len(d) > 0 and d.get("use_ref", False):
        from .torch_image_util import rot3D_scipy
        refs = d["ref_3D"]
        for i in range(len(refs)):
            r = refs[i]
            if isinstance(r, torch.Tensor):
                refs[i] = rot3D_scipy(r, current_angle)
            else:
                t = torch.tensor(np.asarray(r, np.float32), device="cuda")
                refs[i] = rot3D_scipy(t, current_angle).cpu().numpy()
    return d


def _pick(v, idx):
    return v if len(v) == 1 else v[idx]


def extract_single_value_param(param, energy_angle_id, dict_use_ref={}):
    """param with every per-angle/per-energy array replaced by its entry at
    energy_angle_id (length-1 arrays kept as they are) (FL/atten_util.py:90-135)."""
    elem_type = param["elem_type"]
    elem_comp = param["elem_compound"]
    out = param.copy()
    cs = param["cs"]
    cs_sel = deepcopy(cs)
    for c in elem_comp:
        cs_sel[f"{c}-x"] = _pick(cs[f"{c}-x"], energy_angle_id)
    em = param["em_cs"]
    em_sel = deepcopy(em)
    for e in elem_type:
        em_sel[e] = _pick(em[e], energy_angle_id)
    if len(dict_use_ref) > 0 and dict_use_ref.get("use_ref", False):
        for k in cs_sel.keys():
            if "x_ref" in k:
                cs_sel[k] = cs[k][energy_angle_id]
        for k in em_sel.keys():
            if "x_ref" in k and "n_ref" not in k:
                em_sel[k] = em[k][energy_angle_id]
    out["cs"] = cs_sel
    out["em_cs"] = em_sel
    return out
