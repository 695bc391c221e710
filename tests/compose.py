"""Independent compositions of the self-absorption-corrected MLEM (test
infrastructure, used by the parity tests and the parity leg of bench.py).

The reference runs the corrected loop as a script (FL/example/demo.py:244-336):
every k MLEM iterations it rebuilds the attenuation of every element at every
angle from the current estimate through FL/core.py:19-101 (rotate the
fractions, assemble mu, incident product, cone correlation, product of the
two terms) and then runs ``mlem_cuda_batch`` per element with that
attenuation held fixed.  ``recon.CorrectedMLEM`` does the same on the device.
The two functions here redo the whole schedule without any of this
repository's kernels:

* ``oracle_corrected_mlem``: every step in FP64 by the C oracle
  (oracle/flc_oracle.c), on the host;
* ``reference_corrected_mlem``: the reference's own composition in FP32 on
  the GPU -- the torch operators of FL/torch_functions.py:8-176 and
  FL/torch_image_util.py:13-155, restated here because the reference package
  does not import without xraylib, and the reference's own CUDA extension
  (``cal_atten_cuda`` and ``mlem_cuda_batch`` of FL/cuda_lib, built from its
  sources into oracle/_ref).

Both feed the estimate back as ``CorrectedMLEM`` does (``bounded_fractions``),
so the three results are comparable iteration for iteration.  Slices couple
only through the cone, so ``oracle_corrected_mlem`` can also run a slab of
slices with enough neighbouring planes for a given number of rebuilds.
"""
import math

import numpy as np

from oracle import oracle as O


def bounded_fractions(C):
    """The estimate as mass fractions, as CorrectedMLEM.recompute_attenuation
    feeds it back: clipped to [0, 1], then divided by the elements' total
    where that total exceeds 1.  numpy (L, ...) -> numpy."""
    f = np.clip(np.asarray(C, np.float64), 0.0, 1.0)
    tot = np.maximum(f.sum(axis=0, keepdims=True), 1.0)
    return f / tot


def _em_table(param, A):
    """(L, A) emission cross sections scaled by rho * pix (FL/torch_recon.py:83)."""
    return np.stack([np.broadcast_to(np.asarray(param["em_cs"][e], np.float64).reshape(-1), (A,))
                     * param["rho"][c] * param["pix"]
                     for e, c in zip(param["elem_type"], param["elem_compound"])])


def relative_errors(a, b, floor=1e-2):
    """Error of a against b: max|a-b|/max|b| (the parity measure of the tests)
    and the pointwise max |a-b|/|b| over the elements with |b| >= floor*max|b|."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = float(np.abs(b).max()) or 1.0
    keep = np.abs(b) >= floor * den
    pw = float((np.abs(a - b)[keep] / np.abs(b)[keep]).max()) if keep.any() else 0.0
    return {"max_abs_over_max": float(np.abs(a - b).max() / den),
            "pointwise_max_rel": pw, "pointwise_floor": floor}


# ---------------------------------------------------------------------------
# FP64 oracle composition
# ---------------------------------------------------------------------------
def oracle_atten(frac, theta, cx, cf, mask, z_range=None):
    """Attenuation (L, A, S, H, W) in FP64: per angle rotate, incident product
    of the element's own compound (FL/core.py:80-81), exp(-cone), product.
    z_range=(z0, z1) computes the cone for those output slices only (the
    other slices of the result are not valid)."""
    frac = np.asarray(frac, np.float64)
    L = cf.shape[1]
    n_ch, S, H, W = frac.shape
    A = len(theta)
    m32 = np.asarray(mask, np.float32)
    out = np.empty((L, A, S, H, W))
    for a in range(A):
        fr = O.rotate(frac, theta[a])
        mux = fr * np.asarray(cx[a], np.float64)[:, None, None, None]
        muf = np.einsum("ij,jshw->ishw", np.asarray(cf[a], np.float64), fr)
        if z_range is None:
            res = O.cone_beam(muf, m32)
        else:
            res = O.cone_beam_slab(muf, m32, z_range[0], z_range[1])
        out[:, a] = O.incident_scan(mux[:L]) * np.exp(-res)
    return out


def feedback_fractions(C, feedback, cal_frac_args=None):
    """The fractions fed back at a rebuild (numpy): 'bounded' as
    bounded_fractions, 'cal_frac' as the reference's cal_frac (the oracle's
    restatement, FL/core.py:159-205, threshold mask 1)."""
    if feedback == "cal_frac":
        kw = dict(scale_range=[0.02, 0.98], enable_scale=True, scale_limit=0.95)
        kw.update(cal_frac_args or {})
        return O.cal_frac(np.asarray(C, np.float32), **kw).astype(np.float64)
    return bounded_fractions(C)


def oracle_corrected_mlem(param, angles_deg, mask, I, fixed_frac, n_iter, recompute_every,
                          C0=None, beta=0.0, delta=0.01, z_range=None, feedback="bounded"):
    """Corrected MLEM in FP64 (host).  I (L, A, S, W); fixed_frac (n_ch-L, S,
    H, W) fractions of the non-element compounds.  With z_range=(z0, z1) the
    result is valid on those slices only: the inputs must then hold the slab
    [z0 - k*hz, z1 + k*hz) (hz = Mz // 2, k = number of rebuilds) clipped to
    the volume, with z_range relative to that slab."""
    from fl_correction_b200.core import atten_coefficients
    I = np.asarray(I, np.float64)
    L, A, S, W = I.shape
    H = W
    n_ch = L + fixed_frac.shape[0]
    cx, cf = atten_coefficients(param, A, n_ch)
    theta = (np.asarray(angles_deg, np.float64) / 180.0 * np.pi).astype(np.float32)
    em = _em_table(param, A)
    C = np.ones((L, S, H, W)) if C0 is None else np.asarray(C0, np.float64).copy()
    hz = np.shape(mask)[0] // 2
    done, k_done = 0, 0
    while done < n_iter:
        k = min(recompute_every, n_iter - done)
        if feedback != "bounded" and z_range is not None:
            raise ValueError("cal_frac's order statistics couple all slices: no slab form")
        frac = np.concatenate([feedback_fractions(C, feedback), np.asarray(fixed_frac, np.float64)])
        zr = None
        if z_range is not None:
            # rebuild on the slices later rebuilds still need
            n_left = math.ceil((n_iter - done) / recompute_every) - 1
            zr = (max(0, z_range[0] - n_left * hz), min(S, z_range[1] + n_left * hz))
        att = oracle_atten(frac, theta, cx, cf, mask, zr)
        for l in range(L):
            lo, hi = zr if zr is not None else (0, S)
            C[l:l + 1, lo:hi] = O.mlem(C[l:l + 1, lo:hi], att[l][:, lo:hi], em[l][:, None], theta,
                                       I[l][:, lo:hi], k, beta, delta)
        done += k
        k_done += 1
    return C


# ---------------------------------------------------------------------------
# The reference's own composition on the GPU (FP32)
# ---------------------------------------------------------------------------
def _rotate_nd(x, theta):
    """torch_rotate_image_nd (FL/torch_image_util.py:13-114), enable_crop:
    affine_grid with the FP32 matrix [[cos, -sin, 0], [sin, cos, 0]] of the
    FP64 angle, grid_sample bilinear, zero padding, align_corners=False."""
    import torch
    import torch.nn.functional as F
    H, W = x.shape[-2:]
    y = x.reshape(-1, 1, H, W)
    c, s = math.cos(theta), math.sin(theta)
    mat = torch.tensor([[c, -s, 0.0], [s, c, 0.0]], dtype=x.dtype, device=x.device)
    grid = F.affine_grid(mat[None].repeat(y.shape[0], 1, 1), (y.shape[0], 1, H, W),
                         align_corners=False)
    out = F.grid_sample(y, grid, mode="bilinear", padding_mode="zeros", align_corners=False)
    return out.reshape(x.shape)


def _rot90(x, mode):
    """torch_rot90_4D(ax=0) (FL/torch_image_util.py:117-155): per channel,
    transpose the last two axes, then flip the last ('clock') or the middle
    ('c-clock') one."""
    t = x.transpose(2, 3)
    return t.flip(3) if mode == "clock" else t.flip(2)


def reference_atten(ref, frac, theta64, cx, cf, mask):
    """Attenuation (L, A, S, H, W) by the reference's steps: per angle
    FL/core.py:43 rotation, torch_xray_atten_3D (FL/torch_functions.py:83-106;
    the element's own compound), torch_xrf_atten_3D (:110-176, detector on
    the right: rot90 clockwise, cal_atten_cuda, rot90 back, exp(-res)), and
    their product (FL/core.py:84-101)."""
    import torch
    L = cf.shape[1]
    n_ch, S, H, W = frac.shape
    A = len(theta64)
    dev = frac.device
    m = torch.as_tensor(np.asarray(mask, np.float32), device=dev)
    out = torch.empty((L, A, S, H, W), dtype=torch.float32, device=dev)
    for a in range(A):
        fr = _rotate_nd(frac, float(theta64[a]))
        for i in range(L):
            # mu_x of the element's own compound; exclusive reverse cumprod
            f = 1 - fr[i] * float(cx[a, i])
            inc = torch.ones_like(f)
            inc[:, :-1] = torch.cumprod(f.flip(1), dim=1)[:, :-1].flip(1)
            out[i, a] = inc
        muf = torch.zeros((L, S, H, W), dtype=torch.float32, device=dev)
        for i in range(L):
            for j in range(n_ch):
                muf[i] += fr[j] * float(cf[a, i, j])
        res = ref.cal_atten_cuda(_rot90(muf, "clock").contiguous(), m)
        out[:, a] *= torch.exp(-_rot90(res, "c-clock"))
    return out


def reference_corrected_mlem(ref, param, angles_deg, mask, I, fixed_frac, n_iter,
                             recompute_every, C0=None, beta=0.0, delta=0.01, feedback="bounded"):
    """Corrected MLEM through the reference's kernels (FP32, GPU).  I (L, A,
    S, W) device tensor; fixed_frac (n_ch-L, S, H, W) device tensor."""
    import torch
    from fl_correction_b200.core import atten_coefficients
    L, A, S, W = I.shape
    H = W
    dev = I.device
    n_ch = L + fixed_frac.shape[0]
    cx, cf = atten_coefficients(param, A, n_ch)
    th64 = np.asarray(angles_deg, np.float64) / 180.0 * np.pi
    theta = torch.tensor(th64, dtype=torch.float32, device=dev)
    em = torch.tensor(_em_table(param, A), dtype=torch.float32, device=dev)
    C = (torch.ones((L, S, H, W), dtype=torch.float32, device=dev) if C0 is None
         else C0.clone())
    done = 0
    while done < n_iter:
        k = min(recompute_every, n_iter - done)
        if feedback == "cal_frac":
            f = torch.tensor(feedback_fractions(C.cpu().numpy(), feedback), dtype=torch.float32,
                             device=dev)
        else:
            f = C.clamp(0.0, 1.0)
            f = f / f.sum(dim=0, keepdim=True).clamp(min=1.0)
        frac = torch.cat([f, fixed_frac]).contiguous()
        att = reference_atten(ref, frac, th64, cx, cf, mask)
        for l in range(L):
            C[l:l + 1] = ref.mlem_cuda_batch(C[l:l + 1].contiguous(), att[l].contiguous(),
                                             em[l][:, None].contiguous(), theta,
                                             I[l].contiguous(), k, beta, delta)
        done += k
        del att
    return C
