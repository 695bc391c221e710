"""Image rotation helpers with the signatures of FL/torch_image_util.py.

``torch_rotate_image_nd`` runs the native grid_sample-equivalent rotation
(bilinear, zero padding, align_corners=False, same-size output) for CUDA
tensors.  The rot90 helpers are pure index permutations (transpose + flip)
and stay as torch views/copies.
"""
import math

import torch

from . import _lib

__all__ = ["torch_rotate_image_nd", "torch_rot90_3D", "torch_rot90_4D", "rot3D_scipy"]


def _angle(theta):
    if isinstance(theta, torch.Tensor):
        return float(theta.detach().cpu().double())
    return float(theta)


def torch_rotate_image_nd(x, theta, enable_crop=True, align_corners=False, mode="bilinear",
                          padding_mode="zeros"):
    """Rotate (..., H, W) by theta radians counter-clockwise about the image
    centre (FL/torch_image_util.py:13-114).  Supports the configuration the
    hot path uses: enable_crop=True, bilinear, zero padding,
    align_corners=False; other settings raise NotImplementedError."""
    if not enable_crop or align_corners or mode != "bilinear" or padding_mode != "zeros":
        raise NotImplementedError("torch_rotate_image_nd: only enable_crop=True, bilinear, "
                                  "zeros padding, align_corners=False are implemented")
    if x.dim() < 2:
        raise ValueError("Input must have at least 2 dimensions")
    _lib.require_cuda("torch_rotate_image_nd", x)
    th = _angle(theta)
    # the reference builds an FP32 matrix from math.cos / math.sin
    c = float(torch.tensor(math.cos(th), dtype=torch.float32))
    s = float(torch.tensor(math.sin(th), dtype=torch.float32))
    H, W = x.shape[-2:]
    xc = x.contiguous()
    out = torch.empty_like(xc)
    with torch.cuda.device(x.device):
        _lib.call("flc_rotate", _lib.ptr(xc), _lib.ptr(out), xc.numel() // (H * W), H, W, c, s,
                  _lib.stream())
    return out


def rot3D_scipy(x, deg):
    """The reference's rot3D (FL/image_util.py:165-203; scipy.ndimage.rotate,
    order 1, reshape=False, mode='constant') of a CUDA tensor (..., H, W) by
    `deg` degrees counter-clockwise: grid_sample's sample points and weights,
    zero where the sample falls outside the slice (flc_rotate_ex, mode 1).
    NaN and inf become 0 first, as rot3D's rm_nan does; 0 degrees returns
    the cleaned input; a rotated result is clipped below at 0, as rot3D
    clips it.  (rot3D rotates in FP64 -- rm_nan returns float64 -- and at
    multiples of 90 degrees with order 0; here the FP32 bilinear rotation
    lands within FP32 rounding of both.)"""
    _lib.require_cuda("rot3D_scipy", x)
    xc = torch.nan_to_num(x.to(torch.float32), nan=0.0, posinf=0.0, neginf=0.0).contiguous()
    if float(deg) == 0.0:
        return xc
    th = float(deg) / 180.0 * math.pi
    c = float(torch.tensor(math.cos(th), dtype=torch.float32))
    s = float(torch.tensor(math.sin(th), dtype=torch.float32))
    H, W = xc.shape[-2:]
    out = torch.empty_like(xc)
    with torch.cuda.device(x.device):
        _lib.call("flc_rotate_ex", _lib.ptr(xc), _lib.ptr(out), xc.numel() // (H * W), H, W, c, s,
                  1, _lib.stream())
    return out.clamp_(min=0.0)


def torch_rot90_3D(img_raw, ax=0, mode="c-clock"):
    """90-degree rotation of a 3-D array about axis `ax` (FL/torch_image_util.py:117-147).
    'clock' is -90 degrees, 'c-clock' +90 degrees."""
    dims = {0: (1, 2), 1: (0, 2), 2: (0, 1)}[ax]
    img = img_raw.transpose(*dims)
    if mode == "clock":
        img = img.flip(dims=({0: 2, 1: 2, 2: 0}[ax],))
    elif mode == "c-clock":
        img = img.flip(dims=({0: 1, 1: 0, 2: 1}[ax],))
    return img.clone() if img.data_ptr() == img_raw.data_ptr() else img.contiguous()


def torch_rot90_4D(img4D, ax=0, mode="c-clock"):
    """torch_rot90_3D applied to every channel of (C, ., ., .) (FL/torch_image_util.py:150-155).
    Like the reference, the result keeps the input's shape, so the rotated
    axes must have equal length."""
    out = torch.stack([torch_rot90_3D(img4D[i], ax, mode) for i in range(img4D.shape[0])])
    if out.shape != img4D.shape:
        raise RuntimeError("torch_rot90_4D: rotated axes must have equal length")
    return out
