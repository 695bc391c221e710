"""numpy front end of the C oracle (``oracle/flc_oracle.c``).

TEST INFRASTRUCTURE ONLY: used by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py``.  Each wrapper names the reference
file:line that the C function restates.  Inputs are converted to float64;
angles stay float32 because the reference evaluates cos/sin of FP32 angles.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_i64 = ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def build():
    """Compile liboracle.so (make) if it is missing or stale."""
    so = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "flc_oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return so


def lib():
    global _LIB
    if _LIB is None:
        so = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(so):
            build()
        L = ctypes.CDLL(so)
        L.orc_max_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def set_threads(n):
    lib().orc_set_threads(ctypes.c_int(int(n)))


def max_threads():
    return int(lib().orc_max_threads())


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _pd(a):
    return a.ctypes.data_as(_dp)


def _pf(a):
    return a.ctypes.data_as(_fp)


def fp32_cos_sin(theta):
    """cos/sin as the reference builds its FP32 rotation matrix
    (FL/torch_image_util.py:77-85: math.cos/sin, then a float32 tensor)."""
    return float(np.float32(math.cos(float(theta)))), float(np.float32(math.sin(float(theta))))


def rotate(x, theta):
    """grid_sample rotation, FL/torch_image_util.py:13-114 (enable_crop=True)."""
    x = _d(x)
    H, W = x.shape[-2:]
    out = np.empty_like(x)
    c, s = fp32_cos_sin(theta)
    lib().orc_rotate(_pd(x), _pd(out), _i64(x.size // (H * W)), _i64(H), _i64(W),
                     ctypes.c_double(c), ctypes.c_double(s))
    return out


def rotate_adjoint(g, theta):
    g = _d(g)
    H, W = g.shape[-2:]
    out = np.empty_like(g)
    c, s = fp32_cos_sin(theta)
    lib().orc_rotate_adjoint(_pd(g), _pd(out), _i64(g.size // (H * W)), _i64(H), _i64(W),
                             ctypes.c_double(c), ctypes.c_double(s))
    return out


def incident_scan(mu):
    """Exclusive reverse product of (1-mu) along H, FL/torch_functions.py:95-102."""
    mu = _d(mu)
    H, W = mu.shape[-2:]
    out = np.empty_like(mu)
    lib().orc_incident_scan(_pd(mu), _pd(out), _i64(mu.size // (H * W)), _i64(H), _i64(W))
    return out


def cone_ref(mu, mask):
    """atten_kernel, FL/cuda_lib/atten_cuda_kernel.cu:10-57 (K,Z,X,Y layout)."""
    mu = _d(mu)
    mask = _d(mask)
    K, Z, X, Y = mu.shape
    Mz, Mx, My = mask.shape
    out = np.empty_like(mu)
    lib().orc_cone_ref(_pd(mu), _pd(mask), _pd(out), _i64(K), _i64(Z), _i64(X), _i64(Y),
                       _i64(Mz), _i64(Mx), _i64(My))
    return out


def cone_beam(mu, mask):
    """rot90 -> atten_kernel -> rot90^-1 (FL/torch_functions.py:142-171),
    evaluated directly in the unrotated frame; mu is (K,Z,H,W)."""
    mu = _d(mu)
    mask = _d(mask)
    K, Z, H, W = mu.shape
    Mz, Mx, My = mask.shape
    out = np.empty_like(mu)
    lib().orc_cone_beam(_pd(mu), _pd(mask), _pd(out), _i64(K), _i64(Z), _i64(H), _i64(W),
                        _i64(Mz), _i64(Mx), _i64(My))
    return out


def cone_beam_adjoint(g, mask):
    g = _d(g)
    mask = _d(mask)
    K, Z, H, W = g.shape
    Mz, Mx, My = mask.shape
    out = np.empty_like(g)
    lib().orc_cone_beam_adjoint(_pd(g), _pd(mask), _pd(out), _i64(K), _i64(Z), _i64(H), _i64(W),
                                _i64(Mz), _i64(Mx), _i64(My))
    return out


def _batchify(atten, C):
    atten = _d(atten)
    C = _d(C)
    if atten.ndim == 3:
        atten = atten[:, None]
    if C.ndim == 3:
        C = C[:, None]
    return atten, C


def fwd_emission(atten, C, em, theta):
    """forward_emission[_batch], atten_cuda_kernel.cu:91-142 / :298-337.
    atten (A,[B,]H,W), C (R,[B,]H,W), em (A,R), theta (A) radians -> (A,[B,]W)."""
    single = np.ndim(atten) == 3
    atten, C = _batchify(atten, C)
    A, B, H, W = atten.shape
    R = C.shape[0]
    em = _d(em).reshape(A, R)
    th = np.ascontiguousarray(theta, dtype=np.float32)
    Pf = np.empty((A, B, W))
    lib().orc_fwd_emission(_pd(atten), _pd(C), _pd(em), _pf(th), _pd(Pf),
                           _i64(A), _i64(B), _i64(R), _i64(H), _i64(W))
    return Pf[:, 0] if single else Pf


def bwd_emission(atten, ratio, em, theta):
    """backward_emission[_batch], atten_cuda_kernel.cu:177-231 / :390-446 -> (R,[B,]H,W)."""
    single = np.ndim(atten) == 3
    atten = _d(atten)
    ratio = _d(ratio)
    if single:
        atten = atten[:, None]
        ratio = ratio[:, None]
    A, B, H, W = atten.shape
    em = _d(em)
    R = em.shape[1]
    th = np.ascontiguousarray(theta, dtype=np.float32)
    out = np.empty((R, B, H, W))
    lib().orc_bwd_emission(_pd(atten), _pd(_d(ratio)), _pd(em), _pf(th), _pd(out),
                           _i64(A), _i64(B), _i64(R), _i64(H), _i64(W))
    return out[:, 0] if single else out


def fwd_emission_datten(gPf, C, em, theta):
    """d(sum gPf*Pf)/d(atten) for the batched projector."""
    C = _d(C)
    gPf = _d(gPf)
    R, B, H, W = C.shape
    A = gPf.shape[0]
    th = np.ascontiguousarray(theta, dtype=np.float32)
    out = np.empty((A, B, H, W))
    lib().orc_fwd_emission_datten(_pd(gPf), _pd(C), _pd(_d(em)), _pf(th), _pd(out),
                                  _i64(A), _i64(B), _i64(R), _i64(H), _i64(W))
    return out


def huber_grad(C, delta):
    """huber_grad[_batch], atten_cuda_kernel.cu:495-616."""
    C = _d(C)
    H, W = C.shape[-2:]
    g = np.empty_like(C)
    lib().orc_huber_grad(_pd(C), _pd(g), _i64(C.size // (H * W)), _i64(H), _i64(W),
                         ctypes.c_double(delta))
    return g


def mlem(C_init, atten, em, theta, I, n_iter, beta=1e-3, delta=0.01):
    """mlem_cuda[_batch], FL/cuda_lib/atten_cuda.cpp:244-345."""
    single = np.ndim(atten) == 3
    atten, C = _batchify(atten, C_init)
    I = _d(I)
    if single:
        I = I[:, None]
    A, B, H, W = atten.shape
    R = C.shape[0]
    C = C.copy()
    th = np.ascontiguousarray(theta, dtype=np.float32)
    lib().orc_mlem(_pd(C), _pd(atten), _pd(_d(em)), _pf(th), _pd(np.ascontiguousarray(I)),
                   _i64(n_iter), ctypes.c_double(beta), ctypes.c_double(delta),
                   _i64(A), _i64(B), _i64(R), _i64(H), _i64(W))
    return C[:, 0] if single else C


def cone_beam_slab(mu, mask, z0, z1):
    """cone_beam for output slices [z0, z1) only (others are zero)."""
    mu = _d(mu)
    mask = _d(mask)
    K, Z, H, W = mu.shape
    Mz, Mx, My = mask.shape
    out = np.zeros_like(mu)
    lib().orc_cone_beam_slab(_pd(mu), _pd(mask), _pd(out), _i64(K), _i64(Z), _i64(H), _i64(W),
                             _i64(Mz), _i64(Mx), _i64(My), _i64(z0), _i64(z1))
    return out


# ---------------------------------------------------------------------------
# Differentiable corrected projection (per-angle attenuation recomputed from
# the concentrations).  Forward: the composition FL/core.py:19-101 (rotate ->
# mu -> incident scan, cone) followed by the projector
# (atten_cuda_kernel.cu:298-337).  Adjoint: reverse mode of the same chain,
# composed from the adjoints above; pinned by finite differences in
# tests/test_oracle_adjoint.py (the reference has no such adjoint).
# ---------------------------------------------------------------------------
INCIDENT = {"own": 0, "all": 1, "none": 2}


def _xrf_angle(frac, theta, cx, cf, mask, incident):
    """Rotated fractions, incident term (L,S,H,W), exp(-cone) (L,S,H,W)."""
    L = cf.shape[0]
    fr = rotate(frac, theta)
    mux = fr * _d(cx)[:, None, None, None]
    muf = np.einsum("ij,jshw->ishw", _d(cf), fr)
    E = np.exp(-cone_beam(muf, mask))
    if incident == "own":
        inc = incident_scan(mux[:L])
    elif incident == "all":
        inc = np.repeat(incident_scan(1 - np.prod(1 - mux, axis=0, keepdims=True)), L, axis=0)
    else:
        inc = np.ones_like(E)
    return fr, mux, inc, E


def xrf_project(frac, theta, cx, cf, mask, em, incident="own"):
    """Pf (L, A, S, W) of C = frac[:L] through the attenuation of every angle.

    frac (n_ch,S,H,W); theta (A,) float32 radians; cx (A,n_ch); cf (A,L,n_ch);
    mask (Mz,Mx,My); em (L,A)."""
    frac = _d(frac)
    th = np.asarray(theta, np.float32)
    A = th.size
    L = np.shape(cf)[1]
    n_ch, S, H, W = frac.shape
    em = _d(em)
    Pf = np.zeros((L, A, S, W))
    for a in range(A):
        _, _, inc, E = _xrf_angle(frac, th[a], np.asarray(cx)[a], np.asarray(cf)[a], mask, incident)
        att = inc * E
        for l in range(L):
            Pf[l, a] = fwd_emission(att[l:l + 1], frac[l:l + 1], em[l, a].reshape(1, 1),
                                    th[a:a + 1])[0]
    return Pf


def _scan_adjoint(f, inc, dinc):
    """Reverse mode of inc[h-1] = f[h] * inc[h] (inc[H-1] = 1) along axis -2:
    returns d/df."""
    H = f.shape[-2]
    df = np.zeros_like(f)
    gbar = dinc[..., 0, :].copy()
    for h in range(1, H):
        df[..., h, :] = gbar * inc[..., h, :]
        gbar = dinc[..., h, :] + gbar * f[..., h, :]
    return df


def xrf_project_adjoint(frac, theta, cx, cf, mask, em, gPf, incident="own"):
    """dC (L, S, H, W) = d<gPf, xrf_project(frac)>/d frac[:L] (channels >= L
    are held fixed), through both the projector and the attenuation."""
    frac = _d(frac)
    th = np.asarray(theta, np.float32)
    A = th.size
    cx = np.asarray(cx)
    cf = np.asarray(cf)
    L = cf.shape[1]
    n_ch, S, H, W = frac.shape
    em = _d(em)
    gPf = _d(gPf)
    dC = np.zeros((L, S, H, W))
    for a in range(A):
        fr, mux, inc, E = _xrf_angle(frac, th[a], cx[a], cf[a], mask, incident)
        att = inc * E
        datt = np.zeros_like(att)
        for l in range(L):
            ema = em[l, a].reshape(1, 1)
            dC[l] += bwd_emission(att[l:l + 1], gPf[l, a][None], ema, th[a:a + 1])[0]
            datt[l] = fwd_emission_datten(gPf[l, a][None], frac[l:l + 1], ema, th[a:a + 1])[0]
        dinc = datt * E
        dres = -datt * att
        dmuf = cone_beam_adjoint(dres, mask)
        dmux = np.zeros_like(mux)
        if incident == "own":
            dmux[:L] = -_scan_adjoint(1 - mux[:L], inc, dinc)
        elif incident == "all":
            f = 1 - mux
            ftot = np.prod(f, axis=0, keepdims=True)
            dftot = _scan_adjoint(ftot, inc[:1], dinc.sum(axis=0, keepdims=True))
            for j in range(n_ch):
                others = np.prod(np.delete(f, j, axis=0), axis=0)
                dmux[j] = -dftot[0] * others
        dfr = dmux * cx[a][:, None, None, None] + np.einsum("ij,ishw->jshw", cf[a].astype(np.float64), dmuf)
        dC += rotate_adjoint(dfr[:L], th[a])
    return dC


def cal_frac(img, scale_range=(0.02, 0.98), enable_scale=True, scale_limit=0.95):
    """cal_frac, FL/core.py:159-205, with the threshold mask at its fallback
    value 1 (FL/core.py:177-179; the mask needs scikit-image): FP32 sums and
    ratios as numpy computes them on FP32 volumes.  Returns frac (float32)."""
    img = np.asarray(img, np.float32)
    s = np.sum(img, axis=0) + np.float32(1e-12)
    ss = np.sort(s[s > 0], axis=None)
    ratio = np.float32(1.0)
    if enable_scale and ss.size:
        ratio = s / ss[int(ss.size * scale_limit)]
    out = np.zeros(img.shape, np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        for i in range(img.shape[0]):
            t = img[i] / s
            t[~np.isfinite(t)] = 0
            t[t < 0] = 0
            if len(scale_range):
                ts = np.sort(t[t > 0])
                n = ts.size
                if n > 100:
                    ts = ts[int(n * scale_range[0]):int(n * scale_range[1])]
                    t[t >= ts[-1]] = ts[-1]
                    t[t <= ts[0]] = ts[0]
            out[i] = t * ratio
    return out


def _rotate_aspect(x, c, s, sxw, syh):
    """Bilinear rotation of (..., H, W) about the centre with grid_sample's
    zero-padded taps: out(h, w) samples x at ix = c dw - s dh sxw + cx,
    iy = s dw syh + c dh + cy (dw = w - cx, dh = h - cy)."""
    x = np.asarray(x, np.float64)
    H, W = x.shape[-2:]
    cx, cy = (W - 1) / 2.0, (H - 1) / 2.0
    dh, dw = np.meshgrid(np.arange(H) - cy, np.arange(W) - cx, indexing="ij")
    ix = c * dw - s * dh * sxw + cx
    iy = s * dw * syh + c * dh + cy
    x0, y0 = np.floor(ix).astype(np.int64), np.floor(iy).astype(np.int64)
    tx, ty = ix - x0, iy - y0
    out = np.zeros(x.shape)
    for dy, wy in ((0, 1 - ty), (1, ty)):
        for dx, wx in ((0, 1 - tx), (1, tx)):
            yy, xx = y0 + dy, x0 + dx
            ok = (yy >= 0) & (yy < H) & (xx >= 0) & (xx < W)
            v = x[..., np.clip(yy, 0, H - 1), np.clip(xx, 0, W - 1)]
            out += np.where(ok, v, 0.0) * wy * wx
    return out


def xray_atten_ref2d(C, C_other, theta, cs_ref, rho, pix, variant=0):
    """torch_2D_xray_atten_with_ref (variant 0, FL/torch_functions.py:181-215)
    and torch_2D_xray_atten_with_ref_vectorize (variant 1, :247-330) in FP64:
    C (n_ref, H, W), C_other (H, W), theta (A,) radians, cs_ref (A, n_ref),
    rho (H, W) -> (A, H, W).  Variant 0: scale eps 1e-9, align_corners=False
    rotation (aspect W/H), floor 1e-6, exclusive product of the rows below;
    variant 1: eps 1e-8, align_corners=True (aspect (W-1)/(H-1)), mu clipped
    at 0, floor 1e-8, product including row h for h < H-1; last row 1."""
    C = np.asarray(C, np.float64)
    n_ref, H, W = C.shape
    th = np.asarray(theta, np.float32).reshape(-1)
    cs = np.asarray(cs_ref, np.float64).reshape(len(th), n_ref)
    rho = np.broadcast_to(np.asarray(rho, np.float64), (H, W))
    eps = 1e-8 if variant == 1 else 1e-9
    frac = C / ((C.sum(axis=0) + np.asarray(C_other, np.float64)).max() + eps)
    if variant == 1:
        sxw, syh = (W - 1) / (H - 1), (H - 1) / (W - 1)
    else:
        sxw, syh = W / H, H / W
    out = np.ones((len(th), H, W))
    for a, t in enumerate(th):
        if variant == 1:
            c, s = float(np.cos(t)), float(np.sin(t))
        else:
            c, s = fp32_cos_sin(t)
        fr = _rotate_aspect(frac, c, s, sxw, syh)
        mu = np.einsum("j,jhw->hw", cs[a], fr) * rho * pix
        if variant == 1:
            mu = np.maximum(mu, 0.0)
        f = np.maximum(1.0 - mu, 1e-8 if variant == 1 else 1e-6)
        p = np.ones(W)
        for h in range(H - 1, -1, -1):
            if variant == 1:
                p = p * f[h]
                if h < H - 1:
                    out[a, h] = p
            else:
                if h < H - 1:
                    out[a, h] = p
                p = p * f[h]
    return out
