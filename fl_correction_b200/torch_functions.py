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
           "torch_xrf_atten_3D", "torch_3D_forward_projection", "coef_xray", "coef_xrf",
           "compose_cs_incident_xray_with_reference", "offset_canvas",
           "torch_2D_xray_atten_with_ref", "torch_2D_xray_atten_with_ref_vectorize"]


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


def compose_cs_incident_xray_with_reference(ref_3D, ref_cs, ref_comp):
    """Per-voxel incident cross section sum_i spec_i * frac_i of the reference
    volumes ref_3D (n_ref, ...) (FL/cross_section_util.py:44-66), with
    frac_i = max(ref_i / (sum_k ref_k + 1e-12), 0), the fractions of
    FL.core.cal_frac(ref_3D, scale_range=[], enable_scale=False)
    (FL/core.py:159-205) without its Otsu-threshold mask: the reference masks
    with skimage's threshold_multiotsu and falls back to no mask when the
    threshold fails, which is the case this library reproduces.  FP64 on the
    device of ref_3D (numpy input: cuda)."""
    n_ref = int(ref_cs["n_ref"])
    if len(ref_3D) != n_ref:
        raise AssertionError("number of references and number of 3D stack in 'ref_3D' does not match")
    dev = ref_3D.device if isinstance(ref_3D, torch.Tensor) else torch.device("cuda")
    ref = torch.as_tensor(np.asarray(ref_3D) if not isinstance(ref_3D, torch.Tensor) else ref_3D,
                          dtype=torch.float64, device=dev)
    tot = ref.sum(dim=0) + 1e-12
    fr = torch.nan_to_num(ref / tot, nan=0.0, posinf=0.0, neginf=0.0).clamp_(min=0.0)
    spec = [float(np.asarray(ref_cs[f"{ref_comp}-x_ref{i + 1}"]).reshape(-1)[0]) for i in range(n_ref)]
    cs = torch.zeros_like(tot)
    for i in range(n_ref):
        cs += spec[i] * fr[i]
    return cs


def torch_extract_3D_mu_xray(frac_4D, param_angle_energy, dict_use_ref_rotate={}):
    """mu_x[j] = frac[j] * cs[comp_j-x] * rho_j * pix; channels without a
    compound stay 1 (FL/torch_functions.py:8-52).  With dict_use_ref_rotate
    ({'use_ref': True, 'ref_3D': (n_ref, S, H, W) already rotated,
    'ref_comp': compound}) the cross section of ref_comp is the per-voxel
    volume of compose_cs_incident_xray_with_reference (:22-37)."""
    use_ref = len(dict_use_ref_rotate) > 0 and dict_use_ref_rotate.get("use_ref", False)
    ref_comp = dict_use_ref_rotate.get("ref_comp") if use_ref else None
    if use_ref and ref_comp is None:
        raise AssertionError("need to provide 'ref_comp', e.g, 'LiNiO2'")
    mu_x = torch.ones_like(frac_4D)
    comps = param_angle_energy["cs"]["elem_compound"]
    for j, cf in enumerate(coef_xray(param_angle_energy)):
        if use_ref and comps[j] == ref_comp:
            cs3 = compose_cs_incident_xray_with_reference(dict_use_ref_rotate["ref_3D"],
                                                          param_angle_energy["cs"], ref_comp)
            coef = (cs3.to(frac_4D.device) * (param_angle_energy["rho"][ref_comp] *
                                              param_angle_energy["pix"])).to(frac_4D.dtype)
            mu_x[j] = frac_4D[j] * coef
        else:
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


def offset_canvas(H, W, phi):
    """Side of the square canvas that holds an H x W slice rotated by phi
    radians: the reference's _rotated_hw size (FL/torch_image_util.py:5-10)
    plus one pixel on each side -- so that no sample of the slice's window,
    rotated there and back, reaches the zero padding of the canvas edge --
    raised by one where needed so that the padding on each side is a whole
    number of pixels (the rotation centre then stays on the slice centre)."""
    c, s = abs(np.cos(phi)), abs(np.sin(phi))
    n = max(int(H * c + W * s + 0.5), int(W * c + H * s + 0.5), H, W) + 2
    if (n - H) % 2:
        n += 1
    return n


def _path_sum(mu, mask, position_det):
    """Cone path sum toward a detector on the right / left of the slice:
    rot90, cal_atten_cuda, rot90 back (FL/torch_functions.py:142-171)."""
    if position_det == "r":
        mu90 = torch_rot90_4D(mu, ax=0, mode="clock")
    elif position_det == "l":
        mu90 = torch_rot90_4D(mu, ax=0, mode="c-clock")
    else:
        raise ValueError("position_det must be 'r' or 'l'")
    res = cal_atten_cuda(mu90.to(torch.float32).contiguous(), mask)
    return torch_rot90_4D(res, ax=0, mode="c-clock" if position_det == "r" else "clock")


def torch_xrf_atten_3D(frac_4D, param_angle_energy, detector_mask, detector_offset_angle=0,
                       position_det="r"):
    """Fluorescence attenuation exp(-cone(mu_f)) toward a detector on the
    right ('r') or left ('l') (FL/torch_functions.py:110-176).

    detector_offset_angle (degrees, the detector at 90 - offset degrees to the
    beam) rotates mu_f counter-clockwise by the offset about the slice centre
    onto a zero-padded square canvas (offset_canvas) at the same pixel size,
    takes the cone path sum there, rotates the path sum back by -offset and
    crops the slice's own window.  The reference's branch (:134-166) differs:
    its expanded-canvas rotation (enable_crop=False) also magnifies the slice
    by the canvas ratio, because affine_grid maps normalised output
    coordinates onto normalised input coordinates; it rotates mu a second time
    by the offset after rot90 (:146); and its column crop start divides by
    -0.5 (:161), so the crop keeps the first W columns.  Those steps are not
    reproduced."""
    phi = float(np.float32(detector_offset_angle / 180.0 * np.pi))
    mu_xrf = torch_extract_3D_mu_xrf(frac_4D, param_angle_energy)
    mask = torch.as_tensor(np.asarray(detector_mask), dtype=torch.float32, device=frac_4D.device)
    if abs(phi) <= 1e-2:
        res = _path_sum(mu_xrf, mask, position_det)
    else:
        H, W = mu_xrf.shape[-2:]
        n = offset_canvas(H, W, phi)
        pr, pc = (n - H) // 2, (n - W) // 2
        mu_c = torch.nn.functional.pad(mu_xrf, (pc, n - W - pc, pr, n - H - pr))
        res_c = _path_sum(torch_rotate_image_nd(mu_c, phi), mask, position_det)
        res = torch_rotate_image_nd(res_c.contiguous(), -phi)[..., pr:pr + H, pc:pc + W]
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


def _xray_atten_with_ref(C, C_other, theta, cs_ref, rho, pix, variant):
    dev = _lib.require_cuda("torch_2D_xray_atten_with_ref", C, dtype=None)
    f32 = dict(dtype=torch.float32, device=dev)
    n_ref, H, W = C.shape
    th = torch.as_tensor(theta, **f32).reshape(-1).contiguous()
    A = th.numel()
    cs = torch.as_tensor(cs_ref, **f32).reshape(A, n_ref).contiguous()
    rh = torch.as_tensor(rho, **f32).expand(H, W).contiguous()
    Co = torch.as_tensor(C_other, **f32).expand(H, W).contiguous()
    Cc = C.detach().to(**f32).contiguous()
    out = torch.empty((A, H, W), **f32)
    nb = _lib.query("flc_xray_atten_ref2d_workspace_bytes")
    ws = _lib.workspace(nb, dev)
    _lib.call("flc_xray_atten_ref2d", _lib.ptr(Cc), _lib.ptr(Co), _lib.ptr(th), _lib.ptr(cs),
              _lib.ptr(rh), float(pix), _lib.ptr(out), n_ref, A, H, W, variant, _lib.ptr(ws), nb,
              _lib.stream(dev))
    return out.to(C.dtype)


def torch_2D_xray_atten_with_ref(C, C_other, theta_list, cs_ref, rho, pix):
    """Incident X-ray attenuation (n_angle, H, W) of one slice from reference
    volumes C (n_ref, H, W) (FL/torch_functions.py:181-215): C scaled by
    1 / (max(sum_j C_j + C_other) + 1e-9), rotated by theta_list (radians,
    grid_sample with align_corners=False), mu = sum_j cs_ref[a, j] * frac_j *
    rho * pix with rho (H, W) unrotated, and the exclusive product of
    max(1 - mu, 1e-6) over the rows below, last row 1.  One native call
    (flc_xray_atten_ref2d, variant 0); the result is not differentiable."""
    return _xray_atten_with_ref(C, C_other, theta_list, cs_ref, rho, pix, 0)


def torch_2D_xray_atten_with_ref_vectorize(C, C_other, theta, cs_ref, rho, pix):
    """FL/torch_functions.py:247-330 with its own numbers: scale 1 / (max +
    1e-8), rotation with align_corners=True, mu clipped at 0, floor 1e-8, and
    the reference's shifted cumulative product, which includes row h itself
    for h < H-1 (last row 1).  flc_xray_atten_ref2d, variant 1; the result
    is not differentiable."""
    return _xray_atten_with_ref(C, C_other, theta, cs_ref, rho, pix, 1)
