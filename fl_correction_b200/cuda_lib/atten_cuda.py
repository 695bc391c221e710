"""Drop-in for the reference's native module ``FL.cuda_lib.atten_cuda``.

Same function names, argument order, defaults and shapes as the pybind
module of FL/cuda_lib/atten_cuda.cpp:351-393; the work is done by the sm_100a
kernels of libflc.so through its C ABI, on torch's current stream.  Argument
errors raise RuntimeError like the reference's TORCH_CHECKs.
"""
import torch

from .. import _lib

__all__ = ["cal_atten_cuda", "forward_emission", "backward_emission", "forward_emission_batch",
           "backward_emission_batch", "mlem_cuda", "mlem_cuda_batch", "huber_grad",
           "huber_grad_batch"]


def _c(t):
    return t if t.is_contiguous() else t.contiguous()


# per device: (copy of the last mask, its factors u, v or None when it is not
# rank one per depth plane)
_MASK_FACTORS = {}


def _mask_factors(mask):
    """The rank-one factors of each depth plane of a float32 device mask,
    computed on the host once per distinct mask (a caller that passes the
    same mask every angle, as the reference's torch_xrf_atten_3D does, pays
    one device comparison per call), or None if some plane is not rank one."""
    from ..detector_mask import factor_mask
    key = (mask.device.index, tuple(mask.shape))
    hit = _MASK_FACTORS.get(key)
    if hit is not None and torch.equal(hit[0], mask):
        return hit[1]
    fac = factor_mask(mask.detach().cpu().numpy())
    uv = None if fac is None else tuple(torch.from_numpy(f).to(mask.device).contiguous()
                                        for f in fac)
    _MASK_FACTORS[key] = (mask.detach().clone(), uv)
    return uv


def cal_atten_cuda(mu, mask):
    """Cone-mask path sum (atten_cuda.cpp:12-28): mu (K,Z,X,Y), mask (Mz,Mx,My) -> (K,Z,X,Y).

    A mask that is rank one per depth plane (every mask generate_detector_mask
    builds) runs the separable forms with its factors cached and the spectral
    form's scratch taken from torch's allocator; any other mask, or a shape
    the separable kernels do not take, runs flc_cone_atten."""
    _lib.require_cuda("cal_atten_cuda", mu, mask)
    if mu.dim() != 4 or mask.dim() != 3:
        raise RuntimeError("cal_atten_cuda: mu must be (K,Z,X,Y) and mask (Mz,Mx,My)")
    mu, mask = _c(mu), _c(mask)
    out = torch.empty_like(mu)
    K, Z, X, Y = mu.shape
    Mz, Mx, My = mask.shape
    with torch.cuda.device(mu.device):
        uv = _mask_factors(mask) if mask.dtype == torch.float32 and K <= 65535 else None
        if uv is not None:
            nb = int(_lib.query("flc_cone_atten_workspace_bytes", K, Z, X, Y, Mz, Mx, My))
            ws = _lib.workspace(nb, mu.device) if nb else None
            try:
                _lib.call("flc_cone_atten_separable_ws", _lib.ptr(mu), _lib.ptr(uv[0]),
                          _lib.ptr(uv[1]), _lib.ptr(out), K, Z, X, Y, Mz, Mx, My, 0,
                          _lib.ptr(ws), nb, _lib.stream())
                return out
            except _lib.FlcError as e:
                if e.status != "FLC_ERR_UNSUPPORTED":
                    raise
        _lib.call("flc_cone_atten", _lib.ptr(mu), _lib.ptr(mask), _lib.ptr(out), K, Z, X, Y,
                  Mz, Mx, My, 0, _lib.stream())
    return out


def _proj_shapes(name, atten, C, em_cs, theta, batch):
    nd = 4 if batch else 3
    if atten.dim() != nd or C.dim() != nd:
        raise RuntimeError("%s: atten and C must be %dD" % (name, nd))
    if em_cs.dim() != 2 or theta.dim() != 1:
        raise RuntimeError("%s: em_cs must be (n_angle, n_ref) and theta (n_angle)" % name)
    A = atten.shape[0]
    R = C.shape[0]
    if em_cs.shape[0] != A or theta.shape[0] != A:
        raise RuntimeError("%s: n_angle mismatch" % name)
    if em_cs.shape[1] != R:
        raise RuntimeError("%s: n_ref mismatch" % name)
    if tuple(C.shape[1:]) != tuple(atten.shape[1:]):
        raise RuntimeError("%s: C and atten spatial shapes differ" % name)


def forward_emission_batch(atten, C, em_cs, theta):
    """Pf (A,B,W) from atten (A,B,H,W), C (R,B,H,W), em_cs (A,R), theta (A)
    (atten_cuda.cpp:142-182)."""
    _lib.require_cuda("forward_emission_batch", atten, C, em_cs, theta)
    _proj_shapes("forward_emission_batch", atten, C, em_cs, theta, True)
    atten, C, em_cs, theta = _c(atten), _c(C), _c(em_cs), _c(theta)
    A, B, H, W = atten.shape
    R = C.shape[0]
    Pf = torch.empty((A, B, W), dtype=atten.dtype, device=atten.device)
    with torch.cuda.device(atten.device):
        _lib.call("flc_fwd_emission", _lib.ptr(atten), _lib.ptr(C), _lib.ptr(em_cs),
                  _lib.ptr(theta), _lib.ptr(Pf), A, B, R, H, W, _lib.stream())
    return Pf


def backward_emission_batch(atten, ratio, em_cs, theta):
    """out (R,B,H,W), the exact transpose of forward_emission_batch applied to
    ratio (A,B,W) (atten_cuda.cpp:188-214)."""
    _lib.require_cuda("backward_emission_batch", atten, ratio, em_cs, theta)
    if atten.dim() != 4 or ratio.dim() != 3 or em_cs.dim() != 2 or theta.dim() != 1:
        raise RuntimeError("backward_emission_batch: expects atten (A,B,H,W), ratio (A,B,W), "
                           "em_cs (A,R), theta (A)")
    A, B, H, W = atten.shape
    if tuple(ratio.shape) != (A, B, W) or em_cs.shape[0] != A or theta.shape[0] != A:
        raise RuntimeError("backward_emission_batch: shape mismatch")
    atten, ratio, em_cs, theta = _c(atten), _c(ratio), _c(em_cs), _c(theta)
    R = em_cs.shape[1]
    out = torch.empty((R, B, H, W), dtype=atten.dtype, device=atten.device)
    with torch.cuda.device(atten.device):
        _lib.call("flc_bwd_emission", _lib.ptr(atten), _lib.ptr(ratio), _lib.ptr(em_cs),
                  _lib.ptr(theta), _lib.ptr(out), A, B, R, H, W, _lib.stream())
    return out


def forward_emission(atten, C, em_cs, theta):
    """Single slice (atten_cuda.cpp:82-108): atten (A,H,W), C (R,H,W) -> Pf (A,W)."""
    _lib.require_cuda("forward_emission", atten, C, em_cs, theta)
    _proj_shapes("forward_emission", atten, C, em_cs, theta, False)
    return forward_emission_batch(atten.unsqueeze(1), C.unsqueeze(1), em_cs, theta)[:, 0]


def backward_emission(atten, ratio, em_cs, theta):
    """Single slice (atten_cuda.cpp:113-135): ratio (A,W) -> (R,H,W)."""
    _lib.require_cuda("backward_emission", atten, ratio, em_cs, theta)
    if atten.dim() != 3 or ratio.dim() != 2:
        raise RuntimeError("backward_emission: expects atten (A,H,W) and ratio (A,W)")
    return backward_emission_batch(atten.unsqueeze(1), ratio.unsqueeze(1), em_cs, theta)[:, 0]


def huber_grad_batch(C, grad, delta):
    """In-place Huber gradient over the 4 in-plane neighbours
    (atten_cuda.cpp:228-238): C, grad (R,B,H,W)."""
    _lib.require_cuda("huber_grad_batch", C, grad)
    if C.shape != grad.shape or not grad.is_contiguous():
        raise RuntimeError("huber_grad_batch: grad must be a contiguous tensor shaped like C")
    C = _c(C)
    H, W = C.shape[-2:]
    with torch.cuda.device(C.device):
        _lib.call("flc_huber_grad", _lib.ptr(C), _lib.ptr(grad), C.numel() // (H * W), H, W,
                  float(delta), _lib.stream())


def huber_grad(C, grad, delta):
    """Single-slice form (atten_cuda.cpp:218-226): C, grad (R,H,W)."""
    huber_grad_batch(C, grad, delta)


def mlem_cuda_batch(C_init, atten, em_cs, theta, I, n_iter, beta=1e-3, delta=0.01):
    """MLEM with optional Huber term (atten_cuda.cpp:283-345): returns a new
    (R,B,H,W) tensor; C_init is not modified."""
    _lib.require_cuda("mlem_cuda_batch", C_init, atten, em_cs, theta, I)
    if C_init.dim() != 4 or atten.dim() != 4 or I.dim() != 3:
        raise RuntimeError("mlem_cuda_batch: C_init (R,B,H,W), atten (A,B,H,W), I (A,B,W)")
    _proj_shapes("mlem_cuda_batch", atten, C_init, em_cs, theta, True)
    A, B, H, W = atten.shape
    if tuple(I.shape) != (A, B, W):
        raise RuntimeError("mlem_cuda_batch: I must be (n_angle, B, W)")
    R = C_init.shape[0]
    C = C_init.clone(memory_format=torch.contiguous_format)
    atten, em_cs, theta, I = _c(atten), _c(em_cs), _c(theta), _c(I)
    ws_bytes = _lib.query("flc_mlem_workspace_bytes", A, B, R, H, W)
    ws = _lib.workspace(ws_bytes, atten.device)
    with torch.cuda.device(atten.device):
        _lib.call("flc_mlem", _lib.ptr(C), _lib.ptr(atten), _lib.ptr(em_cs), _lib.ptr(theta),
                  _lib.ptr(I), int(n_iter), float(beta), float(delta), A, B, R, H, W,
                  _lib.ptr(ws), ws_bytes, 1, _lib.stream())
    return C


def mlem_cuda(C_init, atten, em_cs, theta, I, n_iter, beta=1e-3, delta=0.01):
    """Single-slice MLEM (atten_cuda.cpp:244-281): C_init (R,H,W), atten (A,H,W), I (A,W)."""
    _lib.require_cuda("mlem_cuda", C_init, atten, em_cs, theta, I)
    if C_init.dim() != 3 or atten.dim() != 3 or I.dim() != 2:
        raise RuntimeError("mlem_cuda: C_init (R,H,W), atten (A,H,W), I (A,W)")
    return mlem_cuda_batch(C_init.unsqueeze(1), atten.unsqueeze(1), em_cs, theta,
                           I.unsqueeze(1), n_iter, beta, delta)[:, 0]
