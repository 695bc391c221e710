"""Attenuation and projection front ends with the signatures of FL/torch_functions.py.

mu assembly follows FL/torch_functions.py:8-81; the incident scan, the cone
path sum and the projector run as native kernels.  As in the reference,
``torch_xray_atten_3D`` (flag_detach=True), ``torch_xrf_atten_3D`` and
``torch_3D_forward_projection`` return numpy arrays.
"""
import numpy as np
import torch

from . import _lib
from .cuda_lib.atten_cuda import cal_atten_cuda, forward_emission_batch, forward_emission
from .torch_image_util import torch_rotate_image_nd, torch_rot90_4D
from .detector_mask import factor_mask

__all__ = ["torch_extract_3D_mu_xray", "torch_extract_3D_mu_xrf", "torch_xray_atten_3D",
           "torch_xrf_atten_3D", "torch_3D_forward_projection", "coef_xray", "coef_xrf"]


def coef_xray(param_angle_energy, n_ch=None):
    """Per-channel incident coefficient cs[comp_j-x] * rho_j * pix as floats
    (FL/torch_functions.py:48).  Channels past the compound list keep the
    reference's mu = 1 (torch.ones_like at :39)."""
    cs = param_angle_energy["cs"]
    comps = cs["elem_compound"]
    rho, pix = param_angle_energy["rho"], param_angle_energy["pix"]
    vals = [float(np.asarray(cs[f"{c}-x"]).reshape(-1)[0]) * rho[c] * pix for c in comps]
    return vals


def coef_xrf(param_angle_energy):
    """coef[i][j] = cs[comp_j-elem_i] * rho_j * pix (FL/torch_functions.py:72-80)."""
    cs = param_angle_energy["cs"]
    comps, elems = cs["elem_compound"], cs["elem_type"]
    rho, pix = param_angle_energy["rho"], param_angle_energy["pix"]
    return [[float(cs[f"{c}-{e}"]) * rho[c] * pix for c in comps] for e in elems]


def torch_extract_3D_mu_xray(frac_4D, param_angle_energy, dict_use_ref_rotate={}):
    """mu_x[j] = frac[j] * cs[comp_j-x] * rho_j * pix; channels without a
    compound stay 1 (FL/torch_functions.py:8-52)."""
    if len(dict_use_ref_rotate) > 0 and dict_use_ref_rotate.get("use_ref", False):
        raise NotImplementedError("reference-spectrum cross sections are not implemented")
    mu_x = torch.ones_like(frac_4D)
    for j, cf in enumerate(coef_xray(param_angle_energy)):
        mu_x[j] = frac_4D[j] * torch.tensor(cf, dtype=frac_4D.dtype, device=frac_4D.device)
    return mu_x


def torch_extract_3D_mu_xrf(frac_4D, param_angle_energy):
    """mu_f[i] = sum_j frac[j] * cs[comp_j-elem_i] * rho_j * pix (FL/torch_functions.py:55-81)."""
    mu = torch.zeros_like(frac_4D)
    for i, row in enumerate(coef_xrf(param_angle_energy)):
        for j, cf in enumerate(row):
            mu[i] += frac_4D[j] * torch.tensor(cf, dtype=frac_4D.dtype, device=frac_4D.device)
    return mu


def torch_xray_atten_3D(frac_4D, param_angle_energy, dict_use_ref_rotate={}, flag_detach=True):
    """Incident attenuation prod_{h'>h}(1 - mu_x) per channel
    (FL/torch_functions.py:83-106), native scan."""
    mu_x = torch_extract_3D_mu_xray(frac_4D, param_angle_energy, dict_use_ref_rotate)
    _lib.require_cuda("torch_xray_atten_3D", mu_x)
    mu_x = mu_x.contiguous()
    out = torch.empty_like(mu_x)
    H, W = mu_x.shape[-2:]
    with torch.cuda.device(mu_x.device):
        _lib.call("flc_incident_scan", _lib.ptr(mu_x), _lib.ptr(out), mu_x.numel() // (H * W),
                  H, W, _lib.stream())
    if flag_detach:
        return out.detach().cpu().numpy()
    return out


def torch_xrf_atten_3D(frac_4D, param_angle_energy, detector_mask, detector_offset_angle=0,
                       position_det="r"):
    """Fluorescence attenuation exp(-cone(mu_f)) toward a detector on the
    right ('r') or left ('l') (FL/torch_functions.py:110-176).  The
    detector-offset branch of the reference (:134-166) is not implemented."""
    if abs(detector_offset_angle / 180.0 * np.pi) > 1e-2:
        raise NotImplementedError("detector_offset_angle != 0 is not implemented")
    mu_xrf = torch_extract_3D_mu_xrf(frac_4D, param_angle_energy)
    if position_det == "r":
        mu90 = torch_rot90_4D(mu_xrf, ax=0, mode="clock")
    elif position_det == "l":
        mu90 = torch_rot90_4D(mu_xrf, ax=0, mode="c-clock")
    else:
        raise ValueError("position_det must be 'r' or 'l'")
    mask = torch.as_tensor(np.asarray(detector_mask), dtype=torch.float32, device=frac_4D.device)
    res = cal_atten_cuda(mu90.to(torch.float32).contiguous(), mask)
    res = torch_rot90_4D(res, ax=0, mode="c-clock" if position_det == "r" else "clock")
    return torch.exp(-res).cpu().numpy()


def torch_3D_forward_projection(C, angle_list, em_cs, atten, mode="batch"):
    """Projection of C (R,S,H,W) at angle_list (degrees) through atten
    (A,S,H,W) with emission cs em_cs (A,R) (FL/torch_functions.py:220-244)."""
    dtype, device = C.dtype, C.device
    theta = torch.tensor(np.asarray(angle_list) / 180.0 * np.pi, dtype=dtype, device=device)
    em = torch.tensor(np.asarray(em_cs), dtype=dtype, device=device)
    at = torch.as_tensor(np.asarray(atten) if not isinstance(atten, torch.Tensor) else atten,
                         dtype=dtype, device=device)
    if mode == "batch":
        return forward_emission_batch(at, C, em, theta).cpu().numpy()
    n_sli = C.shape[1]
    prj = np.zeros((len(angle_list), n_sli, C.shape[-1]))
    for i in range(n_sli):
        prj[:, i] = forward_emission(at[:, i].contiguous(), C[:, i].contiguous(), em, theta).cpu().numpy()
    return prj
