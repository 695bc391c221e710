"""Per-angle attenuation and re-projection with the signatures of FL/core.py.

The reference loops over angles in Python, rotating, assembling mu, running
the cone kernel and writing one TIFF per element per angle
(FL/core.py:19-101).  Here every angle of every element is produced by one
native call (flc_atten_maps) and kept on the device; ``fsave`` (default
None) optionally writes one ``.npy`` per element instead of per-angle TIFFs.
"""
import os

import ctypes

import numpy as np
import torch

from . import _lib
from .atten_util import extract_single_value_param
from .cuda_lib.atten_cuda import forward_emission_batch
from .detector_mask import factor_mask

__all__ = ["cal_frac", "atten_coefficients", "ref_coefficients", "mask_factors", "atten_maps", "pick_chunk", "cal_xrf_atten_at_angles",
           "cal_xray_atten_at_angles", "cal_total_atten_at_angles", "cal_atten_at_angles",
           "re_projection_cuda"]

INCIDENT_MODES = {"own": 0, "all": 1, "none": 2}


def atten_coefficients(param, n_angle, n_ch=None):
    """coef_x (A, n_ch) and coef_f (A, L, n_ch) as float32 numpy arrays,
    selecting per-angle cross sections like extract_single_value_param."""
    comps = param["elem_compound"]
    elems = param["elem_type"]
    n_ch = len(comps) if n_ch is None else n_ch
    cx = np.zeros((n_angle, n_ch), np.float32)
    cf = np.zeros((n_angle, len(elems), n_ch), np.float32)
    for a in range(n_angle):
        p = extract_single_value_param(param, a)
        cs, rho, pix = p["cs"], p["rho"], p["pix"]
        for j, c in enumerate(comps[:n_ch]):
            cx[a, j] = float(np.asarray(cs[f"{c}-x"]).reshape(-1)[0]) * rho[c] * pix
            for i, e in enumerate(elems):
                cf[a, i, j] = float(cs[f"{c}-{e}"]) * rho[c] * pix
    return cx, cf


def mask_factors(detector_mask, device):
    """Device copies (u, v) of the rank-one factors of each depth plane."""
    fac = factor_mask(detector_mask)
    if fac is None:
        raise ValueError("detector mask is not rank one per depth plane")
    u, v = fac
    return (torch.from_numpy(u).to(device).contiguous(), torch.from_numpy(v).to(device).contiguous(),
            tuple(np.shape(detector_mask)))


def atten_maps(frac_4D, angle_list, coef_x, coef_f, mask_uv=None, incident="own", xrf=True,
               out=None, chunk=0, workspace=None, cone_events=None, theta=None, ref=None):
    """Attenuation (L, A, S, H, W) for fractions frac_4D (n_ch, S, H, W) on the
    device: incident term (mode 'own' | 'all' | 'none') times exp(-cone).

    coef_x (A, n_ch), coef_f (A, L, n_ch): per-angle mu coefficients (numpy or
    device tensors).  mask_uv: (u, v, mask_shape) from mask_factors.
    cone_events: optional list; when given, the two pipeline stages are issued
    per angle chunk and (start, end, volumes) CUDA events of every cone launch
    are appended to it.  theta: optional device tensor of the angles in
    radians (float32), used instead of converting angle_list (no host copy,
    so the call can be captured in a CUDA graph).
    ref: optional (ref_3D, coef_ref, ref_ch) for a reference-spectrum incident
    cross section of compound ref_ch (the XANES case of
    FL/torch_functions.py:22-37): ref_3D (n_ref, S, H, W) raw reference
    volumes in the unrotated frame (rotated with the fractions), coef_ref
    (A, n_ref) the per-angle spectrum values cs[comp-x_ref{i+1}] * rho * pix
    (see ref_coefficients)."""
    _lib.require_cuda("atten_maps", frac_4D)
    dev = frac_4D.device
    frac = frac_4D.contiguous()
    n_ch, S, H, W = frac.shape
    if ref is not None:
        return _atten_maps_ref(frac, angle_list, coef_x, coef_f, mask_uv, incident, xrf, out,
                               chunk, workspace, cone_events, theta, ref)
    if theta is None:
        theta = torch.as_tensor(np.asarray(angle_list, dtype=np.float64) / 180.0 * np.pi,
                                dtype=torch.float32, device=dev)
    A = theta.numel()
    cx = torch.as_tensor(coef_x, dtype=torch.float32, device=dev).contiguous()
    cf = torch.as_tensor(coef_f, dtype=torch.float32, device=dev).contiguous()
    L = cf.shape[1]
    if out is None:
        out = torch.empty((L, A, S, H, W), dtype=torch.float32, device=dev)
    if xrf:
        u, v, (Mz, Mx, My) = mask_uv
    else:
        u = v = None
        Mz = Mx = My = 1
    chunk = pick_chunk(S, H, W, A, L, chunk)
    ws_bytes, mu_bytes, fft_bytes = atten_workspace_bytes(n_ch, S, H, W, A, L, chunk,
                                                          (Mz, Mx, My) if xrf else None)
    ws = workspace if workspace is not None and workspace.numel() >= ws_bytes else _lib.workspace(ws_bytes, dev)
    fft_ws = ctypes.c_void_p(ws.data_ptr() + mu_bytes) if fft_bytes else None
    # the channel-interleaved fractions sit at the end of the pipeline part
    frac4_bytes = int(_lib.query("flc_atten_stage_workspace_bytes", n_ch, S, H, W))
    frac4_ws = ctypes.c_void_p(ws.data_ptr() + mu_bytes - frac4_bytes)
    mode = INCIDENT_MODES[incident]
    with torch.cuda.device(dev):
        st = _lib.stream()
        if cone_events is None:
            _lib.call("flc_atten_maps", _lib.ptr(frac), _lib.ptr(theta), _lib.ptr(cx),
                      _lib.ptr(cf), _lib.ptr(u), _lib.ptr(v), _lib.ptr(out), n_ch, S, H, W, A, L,
                      Mz, Mx, My, mode, 0 if xrf else 1, chunk, _lib.ptr(ws), ws_bytes, st)
            return out
        # same two stages per angle chunk, with CUDA events around each cone launch
        for a0 in range(0, A, chunk):
            n_a = min(chunk, A - a0)
            _lib.call("flc_atten_stage_ws", _lib.ptr(frac), _lib.ptr(theta), _lib.ptr(cx),
                      _lib.ptr(cf), _lib.ptr(out), _lib.ptr(ws), n_ch, S, H, W, A, L, a0, n_a,
                      mode, 1 if xrf else 0, frac4_ws, frac4_bytes, st)
            if not xrf:
                continue
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.call("flc_cone_atten_apply_ws", _lib.ptr(ws), _lib.ptr(u), _lib.ptr(v),
                      _lib.ptr(out), n_a, L, S, H, W, A, a0, Mz, Mx, My, fft_ws, fft_bytes, st)
            e1.record()
            cone_events.append((e0, e1, n_a * L))
    return out


def _atten_maps_ref(frac, angle_list, coef_x, coef_f, mask_uv, incident, xrf, out, chunk,
                    workspace, cone_events, theta, ref):
    """atten_maps with reference volumes appended to the fractions
    (flc_atten_maps_ref)."""
    if cone_events is not None:
        raise ValueError("atten_maps: cone_events are not collected with reference volumes")
    ref_3D, coef_ref, ref_ch = ref
    dev = frac.device
    n_ch, S, H, W = frac.shape
    rv = torch.as_tensor(ref_3D, dtype=torch.float32, device=dev)
    if rv.dim() != 4 or tuple(rv.shape[1:]) != (S, H, W):
        raise ValueError("atten_maps: reference volumes must be (n_ref, S, H, W)")
    n_ref = rv.shape[0]
    allf = torch.cat([frac, rv]).contiguous()
    if theta is None:
        theta = torch.as_tensor(np.asarray(angle_list, dtype=np.float64) / 180.0 * np.pi,
                                dtype=torch.float32, device=dev)
    A = theta.numel()
    cx = torch.as_tensor(coef_x, dtype=torch.float32, device=dev).contiguous()
    cf = torch.as_tensor(coef_f, dtype=torch.float32, device=dev).contiguous()
    cr = torch.as_tensor(coef_ref, dtype=torch.float32, device=dev).reshape(A, n_ref).contiguous()
    L = cf.shape[1]
    if out is None:
        out = torch.empty((L, A, S, H, W), dtype=torch.float32, device=dev)
    if xrf:
        u, v, (Mz, Mx, My) = mask_uv
    else:
        u = v = None
        Mz = Mx = My = 1
    chunk = pick_chunk(S, H, W, A, L, chunk)
    ws_bytes, _, _ = atten_workspace_bytes(n_ch + n_ref, S, H, W, A, L, chunk,
                                           (Mz, Mx, My) if xrf else None)
    ws = workspace if workspace is not None and workspace.numel() >= ws_bytes else _lib.workspace(ws_bytes, dev)
    with torch.cuda.device(dev):
        _lib.call("flc_atten_maps_ref", _lib.ptr(allf), _lib.ptr(theta), _lib.ptr(cx),
                  _lib.ptr(cf), _lib.ptr(cr), _lib.ptr(u), _lib.ptr(v), _lib.ptr(out), n_ch, n_ref,
                  int(ref_ch), S, H, W, A, L, Mz, Mx, My, INCIDENT_MODES[incident],
                  0 if xrf else 1, chunk, _lib.ptr(ws), ws_bytes, _lib.stream())
    return out


def ref_coefficients(param, n_angle, ref_comp):
    """(A, n_ref) float32 spectrum values cs['<ref_comp>-x_ref<i+1>'] * rho *
    pix per angle (selected per angle like extract_single_value_param), and
    the channel of ref_comp."""
    cs = param["cs"]
    n_ref = int(cs["n_ref"])
    rho, pix = param["rho"][ref_comp], param["pix"]
    out = np.zeros((n_angle, n_ref), np.float32)
    for i in range(n_ref):
        v = np.asarray(cs[f"{ref_comp}-x_ref{i + 1}"], np.float64).reshape(-1)
        out[:, i] = (v if v.size > 1 else np.repeat(v, n_angle))[:n_angle] * rho * pix
    return out, list(param["elem_compound"]).index(ref_comp)


def atten_workspace_bytes(n_ch, S, H, W, A, L, chunk=0, mask_shape=None):
    """(total, pipeline, spectral-cone) workspace bytes of atten_maps for
    `chunk` angles per pass (0: the default chunk); the pipeline part holds
    the staged mu of one chunk and the channel-interleaved fractions.  mask_shape (Mz, Mx, My):
    the cone's mask, None for the incident term alone; the spectral-cone part
    is 0 where that form does not take the shape."""
    chunk = pick_chunk(S, H, W, A, L, chunk)
    mu_bytes = int(_lib.query("flc_atten_workspace_bytes", n_ch, S, H, W, A, L, chunk))
    fft_bytes = 0
    if mask_shape is not None:
        Mz, Mx, My = mask_shape
        fft_bytes = int(_lib.query("flc_cone_fft_workspace_bytes", chunk * L, S, H, W, Mz, Mx, My))
    return mu_bytes + fft_bytes, mu_bytes, fft_bytes


def pick_chunk(S, H, W, A, L, chunk=0):
    """Angles per pass of the attenuation pipeline (the native default when 0):
    about 256 MB of staged fluorescence mu, enough cone tiles per launch that
    the last wave of CTAs is a small fraction of the launch."""
    if chunk <= 0:
        chunk = max(1, (256 << 20) // (L * S * H * W * 4))
    chunk = min(chunk, A)
    return max(1, min(chunk, 65535 // L))


def _save(fsave, kind, param, maps):
    if fsave is None:
        return
    os.makedirs(fsave, exist_ok=True)
    for i, elem in enumerate(param["elem_type"]):
        np.save(os.path.join(fsave, f"atten_{kind}_{elem}.npy"), maps[i].cpu().numpy())


def cal_xrf_atten_at_angles(frac_4D, param, angle_list, detector_mask, detector_offset_angle=0,
                            position_det="r", dict_use_ref={}, fsave=None):
    """exp(-cone(mu_f)) at every angle for every element (FL/core.py:19-52):
    returns (L, A, S, H, W) on frac_4D's device."""
    # dict_use_ref does not enter the fluorescence mu (FL/torch_functions.py:55-81;
    # FL/core.py:36-47 only selects per-angle parameters with it)
    if abs(detector_offset_angle) > 1e-2 * 180 / np.pi or position_det != "r":
        # the per-angle path of the reference, on the native kernels
        # (offset semantics: torch_functions.torch_xrf_atten_3D)
        from .torch_functions import torch_xrf_atten_3D
        from .torch_image_util import torch_rotate_image_nd
        maps = []
        for a, ang in enumerate(angle_list):
            fr = torch_rotate_image_nd(frac_4D, float(ang) / 180.0 * np.pi)
            p = extract_single_value_param(param, a)
            att = torch_xrf_atten_3D(fr, p, detector_mask, detector_offset_angle, position_det)
            maps.append(torch.as_tensor(att[:len(param["elem_type"])], device=frac_4D.device))
        maps = torch.stack(maps, dim=1).contiguous()
        _save(fsave, "fl", param, maps)
        return maps
    cx, cf = atten_coefficients(param, len(angle_list), frac_4D.shape[0])
    maps = atten_maps(frac_4D, angle_list, cx, cf, mask_factors(detector_mask, frac_4D.device),
                      incident="none", xrf=True)
    _save(fsave, "fl", param, maps)
    return maps


def cal_xray_atten_at_angles(frac_4D, param, angle_list, dict_use_ref={}, fsave=None,
                             apply_ref=False):
    """Incident-beam attenuation at every angle (FL/core.py:55-81): element i
    uses channel i, as the reference writes atten_xray[i] for element i.

    The reference selects per-angle parameters with dict_use_ref but then
    calls torch_xray_atten_3D with an empty dict (FL/core.py:76-79), so its
    result does not depend on the reference volumes; that is the default here
    too.  apply_ref=True applies them as torch_xray_atten_3D does when it is
    given them (FL/torch_functions.py:22-37): the incident cross section of
    dict_use_ref['ref_comp'] becomes the per-voxel mix of the reference
    spectra, the reference volumes rotated with the fractions."""
    cx, cf = atten_coefficients(param, len(angle_list), frac_4D.shape[0])
    ref = None
    if apply_ref and len(dict_use_ref) > 0 and dict_use_ref.get("use_ref", False):
        cr, ch = ref_coefficients(param, len(angle_list), dict_use_ref["ref_comp"])
        ref = (dict_use_ref["ref_3D"], cr, ch)
    maps = atten_maps(frac_4D, angle_list, cx, cf, None, incident="own", xrf=False, ref=ref)
    _save(fsave, "xray", param, maps)
    return maps


def cal_total_atten_at_angles(fsave, param):
    """atten = atten_fl * atten_xray per element (FL/core.py:84-101), from the
    .npy files that the two functions above write into fsave."""
    out = {}
    for elem in param["elem_type"]:
        fl = np.load(os.path.join(fsave, f"atten_fl_{elem}.npy"))
        xr = np.load(os.path.join(fsave, f"atten_xray_{elem}.npy"))
        out[elem] = fl * xr
        np.save(os.path.join(fsave, f"atten_{elem}.npy"), out[elem])
    return out


def cal_atten_at_angles(frac_4D, param, angle_list, detector_mask, incident="own", out=None):
    """The total attenuation of FL/core.py:84-101 computed in one pass, without
    the intermediate files: (L, A, S, H, W)."""
    cx, cf = atten_coefficients(param, len(angle_list), frac_4D.shape[0])
    return atten_maps(frac_4D, angle_list, cx, cf, mask_factors(detector_mask, frac_4D.device),
                      incident=incident, xrf=True, out=out)


def re_projection_cuda(img3D, angle_list, param=None, rho_compound=1, atten_coef=None, elem="Ni",
                       use_ref=False, device="cuda"):
    """XRF projections of img3D ((S,H,W) or (R,S,H,W)) at angle_list (degrees)
    through atten_coef (A,S,H,W), emission cs from param (FL/core.py:104-156)."""
    n_angle = len(angle_list)
    if param is None:
        em = np.ones((n_angle, 1))
    else:
        pix = param["pix"]
        em_cs_dict = param["em_cs"]
        if use_ref:
            n_ref = img3D.shape[0]
            em = np.zeros([n_angle, n_ref])
            for i in range(n_ref):
                em[:, i] = em_cs_dict[f"{elem}_ref{i + 1}"] * pix
        else:
            em = np.asarray(em_cs_dict[elem]) * pix
            em = em.reshape((len(em), 1))
    img3D = img3D * rho_compound
    if isinstance(img3D, torch.Tensor):
        C = img3D.to(device=device, dtype=torch.float)
    else:
        C = torch.tensor(np.asarray(img3D), dtype=torch.float, device=device)
    if C.dim() == 3:
        C = C[None]
    n_ref, n_sli, H, W = C.shape
    if atten_coef is None:
        at = torch.ones(n_angle, n_sli, H, W, dtype=torch.float, device=device)
    else:
        at = torch.as_tensor(atten_coef, dtype=torch.float, device=device)
        if at.dim() == 3:
            at = at[:, None]
    theta = torch.tensor(np.asarray(angle_list) / 180.0 * np.pi, dtype=torch.float, device=device)
    em_t = torch.tensor(np.asarray(em), dtype=torch.float, device=device)
    return forward_emission_batch(at.contiguous(), C.contiguous(), em_t, theta).cpu().numpy()


def cal_frac(*args, scale_range=[0.02, 0.98], enable_scale=True, scale_limit=0.95, img_mask=None,
             out=None):
    """Fractions from concentration volumes, FL/core.py:159-205, on the device
    (flc_cal_frac): img (n, ...) -- one array/tensor, or several with the same
    shape -- summed over n; each channel divided by the sum (NaN, inf and
    negatives set to 0), clamped to its [scale_range] quantiles of positive
    values where it has more than 100, and scaled by sum / (its
    scale_limit-quantile) when enable_scale.  img_mask: the threshold mask
    (None: 1, the reference's value when its multi-Otsu threshold fails, as it
    does without scikit-image).  Returns {'frac', 'img_sum', 'img_mask'} with
    device tensors (float32)."""
    if len(args) == 1:
        img = args[0]
    else:
        img = torch.stack([torch.as_tensor(a) for a in args])
    img = torch.as_tensor(img if isinstance(img, torch.Tensor) else np.asarray(img, np.float32),
                          dtype=torch.float32)
    if not img.is_cuda:
        img = img.cuda()
    if img.dim() == 2:
        img = img[None]
    img = img.contiguous()
    n = img.shape[0]
    N = img[0].numel()
    dev = img.device
    mask = None
    if img_mask is not None:
        mask = torch.as_tensor(img_mask, dtype=torch.float32, device=dev).expand(img.shape[1:]).contiguous()
    frac = out if out is not None else torch.empty_like(img)
    isum = torch.empty(img.shape[1:], dtype=torch.float32, device=dev)
    nb = int(_lib.query("flc_cal_frac_workspace_bytes", n, N))
    ws = _lib.workspace(nb, dev)
    use = 1 if len(scale_range) else 0
    r0, r1 = (float(scale_range[0]), float(scale_range[1])) if use else (0.0, 1.0)
    with torch.cuda.device(dev):
        _lib.call("flc_cal_frac", _lib.ptr(img), _lib.ptr(mask), _lib.ptr(frac), _lib.ptr(isum), n, N,
                  use, r0, r1, 1 if enable_scale else 0, float(scale_limit), _lib.ptr(ws), nb,
                  _lib.stream())
    return {"frac": frac, "img_sum": isum, "img_mask": mask if mask is not None else 1}
