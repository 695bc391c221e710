"""Detector cone mask and its rank-one factorisation.

``generate_detector_mask`` reproduces FL/detector_mask.py:22-106: the
fluorescence collected by a rectangular detector from a point source is
modelled as a pyramid whose cross-section at depth j is the outer product of
two 1-D profiles (horizontal angle alfa, vertical angle theta), each cell
weighted by the fraction of it inside the cone; each depth plane is then
normalised by its sum and the result is squared-weighted (M_normal * Mask),
cut to (2*ceil(L*tan(theta/2))-1, L, 2*ceil(L*tan(alfa/2))-1) and laid out
as (slice, row=depth, col).  Angles are in degrees (full angles).

Because every depth plane is an outer product, the mask factors exactly into
u[depth][slice] * v[depth][col]; ``factor_mask`` returns those factors, which
the separable cone kernel consumes.
"""
import os

import numpy as np

__all__ = ["generate_detector_mask", "prep_detector_mask3D", "load_mask3D", "factor_mask",
           "detector_mask_device"]


def _profile(n_cells, depth, tan_a, cos_a, apex):
    """1-D cone profile (FL/detector_mask.py:109-151, g_mask): weight of cell
    I (0-based, cross axis) at depth J (0-based) for a cone of half-angle a
    whose apex row is `apex` (1-based).  tan_a / cos_a are FP32 values, the
    arithmetic is FP64 as in the reference's numba kernel."""
    i = np.arange(1, n_cells + 1, dtype=np.float64)[:, None]
    j = np.arange(1, depth + 1, dtype=np.float64)[None, :]
    t = float(tan_a)
    o = np.abs(apex - i)
    jt = j * t
    j1t = (j - 1) * t
    out = np.zeros((n_cells, depth))
    outside = o >= jt
    c2 = ~outside & (o < j1t) & (o + 1 > jt)
    c3 = ~outside & ~c2 & (o < jt) & (o + 1 > jt) & (o > j1t)
    c4 = ~outside & ~c2 & ~c3 & (o + 1 < jt) & (o < j1t) & (o + 1 > j1t)
    full = ~outside & ~c2 & ~c3 & ~c4
    fr_j1 = j1t - np.floor(j1t)
    fr_j = jt - np.floor(jt)
    v2 = 0.5 * (fr_j1 + fr_j) / float(cos_a)
    v3 = (0.5 * fr_j * (fr_j / t)) / float(cos_a)
    dd = np.ceil(j1t) - j1t
    v4 = (1.0 - 0.5 * dd * (dd / t)) / float(cos_a)
    vf = 1.0 / np.cos(np.arctan((apex - i) / j))
    out = np.where(c2, v2, out)
    out = np.where(c3, v3, out)
    out = np.where(c4, v4, out)
    out = np.where(full, vf, out)
    # the apex row is all ones except at depth 0 (FL/detector_mask.py:64-67)
    out[apex - 1, :] = 1.0
    out[apex - 1, 0] = 0.0
    return out


def _f32_of(fn, x):
    return np.float32(fn(np.float64(x)))


def generate_detector_mask(alfa0, theta0, leng0):
    """Cone mask, shape (2*N2_0-1, leng0, 2*N1_0-1), float64 (FL/detector_mask.py:22-106)."""
    alfa = np.float32(alfa0) / 2 / 180 * np.pi        # FP32, as in the reference
    theta = np.float32(theta0) / 2 / 180 * np.pi
    tan_a, tan_t = np.tan(alfa), np.tan(theta)
    n1_0 = int(np.ceil(leng0 * tan_a))
    n2_0 = int(np.ceil(leng0 * tan_t))
    leng = leng0 + 30
    n1 = int(np.ceil(leng * tan_a))
    n2 = int(np.ceil(leng * tan_t))
    s0, s1 = 2 * n1 - 1, 2 * n2 - 1
    # inside the profile the FP32 tan/cos are the correctly rounded values
    # (the numba kernel rounds the FP64 result), one ulp from numpy's tanf
    m1 = _profile(s0, leng, _f32_of(np.tan, alfa), _f32_of(np.cos, alfa), n1)
    m2 = _profile(s1, leng, _f32_of(np.tan, theta), _f32_of(np.cos, theta), n2)
    mask = m1[:, None, :] * m2[None, :, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        norm = mask / mask.sum(axis=(0, 1))[None, None, :]
    norm[~np.isfinite(norm)] = 0.0
    mask3d = norm * mask
    c0, c1 = s0 // 2, s1 // 2
    d0, d1 = (2 * n1_0 - 1) // 2, (2 * n2_0 - 1) // 2
    cut = mask3d[c0 - d0:c0 + d0 + 1, c1 - d1:c1 + d1 + 1, 0:leng0]
    cut = np.ascontiguousarray(np.transpose(cut, (1, 2, 0)))   # (slice, row, col)
    cut[np.isnan(cut)] = 0.0
    return cut


def factor_mask(mask, rtol=1e-6):
    """Split each depth plane mask[:, d, :] into u[d] (slices) x v[d] (cols).

    Returns (u, v) float32 arrays of shapes (Mx, Mz) and (Mx, My), or None if
    some plane is not rank one to relative tolerance `rtol`."""
    m = np.asarray(mask, dtype=np.float64)
    Mz, Mx, My = m.shape
    u = np.zeros((Mx, Mz))
    v = np.zeros((Mx, My))
    for d in range(Mx):
        p = m[:, d, :]
        k = np.argmax(np.abs(p))
        i, j = divmod(int(k), My)
        piv = p[i, j]
        if piv == 0.0:
            continue
        u[d] = p[:, j]
        v[d] = p[i, :] / piv
        if np.abs(np.outer(u[d], v[d]) - p).max() > rtol * abs(piv):
            return None
    return u.astype(np.float32), v.astype(np.float32)


def prep_detector_mask3D(alfa=15, beta=60, length_maximum=200, fn_save="mask3D.npz"):
    """Masks for every length from length_maximum down to 7
    (FL/detector_mask.py:12-19); cached as .npz instead of HDF5."""
    masks = {str(L): generate_detector_mask(alfa, beta, L) for L in range(length_maximum, 6, -1)}
    if fn_save:
        np.savez_compressed(fn_save, **masks)
    return masks


def load_mask3D(fn="mask3D.npz"):
    """Load a cache written by prep_detector_mask3D (FL/detector_mask.py:7-9)."""
    if not os.path.exists(fn):
        raise FileNotFoundError(fn)
    with np.load(fn) as z:
        return {k: z[k] for k in z.files}


def detector_mask_device(alfa0, theta0, leng0, device="cuda", dense=False):
    """The cone mask generated on the device (flc_detector_mask): returns
    (u, v, (Mz, Mx, My)) -- the FP32 rank-one factors of every depth plane,
    the form atten_maps and the cone kernels take (core.mask_factors gives the
    same tuple from a host mask) -- and, with dense=True, also the FP64 mask
    (Mz, Mx, My) that generate_detector_mask returns, as a device tensor."""
    import ctypes

    import torch

    from . import _lib
    Mz, Mx, My, nb = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_size_t()
    _lib.call("flc_detector_mask_shape", float(alfa0), float(theta0), int(leng0),
              ctypes.byref(Mz), ctypes.byref(Mx), ctypes.byref(My), ctypes.byref(nb))
    shape = (Mz.value, Mx.value, My.value)
    dev = torch.device(device)
    u = torch.empty((shape[1], shape[0]), dtype=torch.float32, device=dev)
    v = torch.empty((shape[1], shape[2]), dtype=torch.float32, device=dev)
    d = torch.empty(shape, dtype=torch.float64, device=dev) if dense else None
    scratch = torch.empty(max(1, nb.value // 8), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        _lib.call("flc_detector_mask", float(alfa0), float(theta0), int(leng0), _lib.ptr(u),
                  _lib.ptr(v), _lib.ptr(d), _lib.ptr(scratch), nb.value, _lib.stream())
    return (u, v, shape, d) if dense else (u, v, shape)
