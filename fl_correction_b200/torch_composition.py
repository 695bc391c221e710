"""The corrected projection written with plain torch operators, so that
torch autograd can differentiate it (FP64 in the gradient tests, FP32 as the
"plain way" of the gradient benchmark).  It is a comparison baseline, not a
product path: the product runs the native kernels.  Its steps restate the
reference's:

  rotation      F.affine_grid + F.grid_sample, zero padding, align_corners=False
                (FL/torch_image_util.py:13-114)
  incident      flip / cumprod / flip of (1 - mu_x)            (FL/torch_functions.py:95-102)
  cone          the correlation of atten_cuda_kernel.cu:10-57 in the unrotated frame,
                res[z,h,w] = sum mask[dz,dx,dy] mu[z+dz-hz, h-(dy-hy), w+dx], as conv3d
  projector     clamp to [0, N-1.001], floor, bilinear, summed along the beam
                (atten_cuda_kernel.cu:298-337)
"""
import math

import numpy as np
import torch
import torch.nn.functional as F


def _cs32(theta):
    return float(np.float32(math.cos(float(theta)))), float(np.float32(math.sin(float(theta))))


def rotate(x, theta):
    """x (n, S, H, W) -> rotated, as torch_rotate_image_nd (FP32 matrix entries)."""
    c, s = _cs32(theta)
    n, S, H, W = x.shape
    mat = torch.tensor([[c, -s, 0.0], [s, c, 0.0]], dtype=x.dtype, device=x.device)
    grid = F.affine_grid(mat[None].expand(n * S, 2, 3), (n * S, 1, H, W), align_corners=False)
    out = F.grid_sample(x.reshape(n * S, 1, H, W), grid, mode="bilinear", padding_mode="zeros",
                        align_corners=False)
    return out.reshape(n, S, H, W)


def exclusive_reverse_cumprod(f):
    """out[..., h, :] = prod_{h' > h} f[..., h', :] along dim -2."""
    g = torch.flip(f, [-2])
    c = torch.cumprod(g, dim=-2)
    ones = torch.ones_like(c[..., :1, :])
    return torch.flip(torch.cat([ones, c[..., :-1, :]], dim=-2), [-2])


def cone(mu, mask):
    """mu (K, S, H, W), mask (Mz, Mx, My) -> res (K, S, H, W).  A mask whose
    depth planes are rank one (the detector masks) runs as one pair of 1-D
    correlations per depth plane; any other mask as one dense conv3d."""
    Mz, Mx, My = mask.shape
    hz, hy = Mz // 2, My // 2
    K, S, H, W = mu.shape
    from fl_correction_b200.detector_mask import factor_mask
    fac = factor_mask(mask)
    if fac is None:
        k = torch.as_tensor(np.ascontiguousarray(np.transpose(mask, (0, 2, 1))[:, ::-1, :]),
                            dtype=mu.dtype, device=mu.device)     # [dz, My-1-dy, dx]
        x = F.pad(mu[:, None], (0, Mx - 1, hy, hy, hz, hz))
        return F.conv3d(x, k[None, None])[:, 0]
    # rank one per depth: the factors as FP64 products of the stored mask
    m = np.asarray(mask, np.float64)
    res = torch.zeros_like(mu)
    x = F.pad(mu, (0, Mx - 1))                                   # zero beyond the far face
    for d in range(min(Mx, W)):
        p = m[:, d, :]
        if not p.any():
            continue
        k = int(np.argmax(np.abs(p)))
        i, j = divmod(k, My)
        u = p[:, j]                                              # slice profile
        v = p[i, :] / p[i, j]                                    # column profile
        plane = x[..., d:d + W]
        # h - (dy - hy): correlate along h with the reversed column profile
        kv = torch.as_tensor(v[::-1].copy(), dtype=mu.dtype, device=mu.device)
        t = F.conv3d(F.pad(plane[:, None], (0, 0, hy, hy, 0, 0)), kv.view(1, 1, 1, My, 1))[:, 0]
        ku = torch.as_tensor(u.copy(), dtype=mu.dtype, device=mu.device)
        res = res + F.conv3d(F.pad(t[:, None], (0, 0, 0, 0, hz, hz)), ku.view(1, 1, Mz, 1, 1))[:, 0]
    return res


def project(att, C, em, theta):
    """att, C (S, H, W); em scalar -> Pf (S, W)."""
    S, H, W = att.shape
    c, s = math.cos(-float(np.float32(theta))), math.sin(-float(np.float32(theta)))
    cx, cy = (W - 1) / 2.0, (H - 1) / 2.0
    h = torch.arange(H, dtype=torch.float64, device=att.device)[:, None]
    w = torch.arange(W, dtype=torch.float64, device=att.device)[None, :]
    x = c * (h - cy) - s * (w - cx) + cy
    y = s * (h - cy) + c * (w - cx) + cx
    xc, yc = x.clamp(0, H - 1.001), y.clamp(0, W - 1.001)
    i0, j0 = torch.floor(xc), torch.floor(yc)
    fx, fy = (xc - i0).to(att.dtype), (yc - j0).to(att.dtype)
    i0, j0 = i0.long(), j0.long()
    Cf = C.reshape(S, H * W)
    v00 = Cf[:, i0 * W + j0]
    v01 = Cf[:, i0 * W + j0 + 1]
    v10 = Cf[:, (i0 + 1) * W + j0]
    v11 = Cf[:, (i0 + 1) * W + j0 + 1]
    val = (1 - fx) * (1 - fy) * v00 + (1 - fx) * fy * v01 + fx * (1 - fy) * v10 + fx * fy * v11
    return em * (att * val).sum(dim=1)


def xrf_project(frac, theta, cx, cf, mask, em, incident="own"):
    """frac (n_ch, S, H, W) tensor (the first L channels are C) -> Pf (L, A, S, W)."""
    L = cf.shape[1]
    out = []
    for a in range(len(theta)):
        fr = rotate(frac, theta[a])
        cxa = torch.as_tensor(cx[a], dtype=frac.dtype, device=frac.device)
        cfa = torch.as_tensor(cf[a], dtype=frac.dtype, device=frac.device)
        mux = fr * cxa[:, None, None, None]
        muf = torch.einsum("ij,jshw->ishw", cfa, fr)
        E = torch.exp(-cone(muf, mask))
        if incident == "own":
            inc = exclusive_reverse_cumprod(1 - mux[:L])
        elif incident == "all":
            inc = exclusive_reverse_cumprod(torch.prod(1 - mux, dim=0, keepdim=True)).expand(L, -1, -1, -1)
        else:
            inc = torch.ones_like(E)
        att = inc * E
        out.append(torch.stack([project(att[l], frac[l], float(em[l, a]), theta[a]) for l in range(L)]))
    return torch.stack(out, dim=1)
