"""ctypes binding of the native library ``libflc.so`` (C ABI in include/flc.h).

The library is loaded once; if it is missing or cannot be loaded every entry
point raises immediately -- there is no Python or CPU fallback.  Tensors are
passed as raw device pointers with 64-bit sizes and torch's current stream.
"""
import ctypes
import os

import torch

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libflc.so")

_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
_f32 = ctypes.c_float
_f64 = ctypes.c_double
_int = ctypes.c_int
_sz = ctypes.c_size_t

# name -> (restype, argtypes)
SIGNATURES = {
    "flc_status_string": (ctypes.c_char_p, [_int]),
    "flc_last_error": (ctypes.c_char_p, []),
    "flc_version": (ctypes.c_char_p, []),
    "flc_launch_count": (ctypes.c_uint64, []),
    "flc_device_status": (_int, [_int]),
    "flc_tune_set": (_int, [ctypes.c_char_p, _i64]),
    "flc_tune_get": (_i64, [ctypes.c_char_p]),
    "flc_cone_atten": (_int, [_vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _i64, _i64, _int, _vp]),
    "flc_cone_atten_separable": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _i64,
                                        _i64, _int, _vp]),
    "flc_fwd_emission": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _vp]),
    "flc_bwd_emission": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _vp]),
    "flc_huber_grad": (_int, [_vp, _vp, _i64, _i64, _i64, _f32, _vp]),
    "flc_mlem_workspace_bytes": (_sz, [_i64, _i64, _i64, _i64, _i64]),
    "flc_mlem": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _f64, _f64, _i64, _i64, _i64, _i64, _i64,
                        _vp, _sz, _int, _vp]),
    "flc_mlem_static": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _f64, _f64, _i64, _i64, _i64, _i64,
                               _i64, _vp]),
    "flc_atten_workspace_bytes": (_sz, [_i64, _i64, _i64, _i64, _i64, _i64, _i64]),
    "flc_atten_maps": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64,
                              _i64, _i64, _i64, _i64, _int, _int, _i64, _vp, _sz, _vp]),
    "flc_detector_mask_shape": (_int, [_f64, _f64, _i64, ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                                       ctypes.POINTER(_i64), ctypes.POINTER(_sz)]),
    "flc_detector_mask": (_int, [_f64, _f64, _i64, _vp, _vp, _vp, _vp, _sz, _vp]),
    "flc_cal_frac_workspace_bytes": (_sz, [_i64, _i64]),
    "flc_cal_frac": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _int, _f64, _f64, _int, _f64, _vp, _sz,
                            _vp]),
    "flc_mlem_multi_workspace_bytes": (_sz, [_i64, _vp, _vp, _i64, _i64, _i64]),
    "flc_mlem_multi": (_int, [_i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _f64,
                              _f64, _vp, _sz, _vp]),
    "flc_mlem_multi_sizes_workspace_bytes": (_sz, [_i64, _vp, _vp, _i64, _vp, _vp]),
    "flc_mlem_multi_sizes": (_int, [_i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _i64,
                                    _f64, _f64, _vp, _sz, _vp]),
    "flc_atten_maps_ref": (_int, [_vp] * 8 + [_i64] * 11 + [_int, _int, _i64, _vp, _sz, _vp]),
    "flc_atten_stage": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _i64,
                               _i64, _i64, _int, _int, _vp]),
    "flc_cone_atten_apply": (_int, [_vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _i64, _i64,
                                    _i64, _i64, _i64, _vp]),
    "flc_cone_fft_workspace_bytes": (_sz, [_i64] * 7),
    "flc_cone_atten_workspace_bytes": (_sz, [_i64] * 7),
    "flc_cone_atten_separable_ws": (_int, [_vp, _vp, _vp, _vp] + [_i64] * 7 + [_int, _vp, _sz, _vp]),
    "flc_atten_stage_workspace_bytes": (_sz, [_i64] * 4),
    "flc_atten_stage_ws": (_int, [_vp] * 6 + [_i64] * 8 + [_int, _int, _vp, _sz, _vp]),
    "flc_cone_atten_apply_ws": (_int, [_vp, _vp, _vp, _vp] + [_i64] * 10 + [_vp, _sz, _vp]),
    "flc_xrf_workspace_bytes": (_sz, [_i64, _i64, _i64, _i64, _i64, _i64, _i64]),
    "flc_xrf_workspace_bytes_ex": (_sz, [_i64] * 10),
    "flc_xrf_project": (_int, [_vp] * 8 + [_i64] * 9 + [_int, _i64, _vp, _sz, _vp]),
    "flc_xrf_project_adjoint": (_int, [_vp] * 11 + [_i64] * 9 + [_int, _i64, _vp, _sz, _vp]),
    "flc_rotate": (_int, [_vp, _vp, _i64, _i64, _i64, _f32, _f32, _vp]),
    "flc_incident_scan": (_int, [_vp, _vp, _i64, _i64, _i64, _vp]),
    "flc_rotate_ex": (_int, [_vp, _vp, _i64, _i64, _i64, _f32, _f32, _int, _vp]),
    "flc_xray_atten_ref2d_workspace_bytes": (_sz, []),
    "flc_xray_atten_ref2d": (_int, [_vp, _vp, _vp, _vp, _vp, _f32, _vp, _i64, _i64, _i64, _i64,
                                    _int, _vp, _sz, _vp]),
}

_LIB = None
_LOAD_ERROR = None


class FlcError(RuntimeError):
    """A native entry point returned a non-zero flc_status."""

    def __init__(self, name, status, message):
        self.status = status
        super().__init__("%s failed: %s: %s" % (name, status, message))


def load():
    """Load libflc.so (building it first if the sources are newer)."""
    global _LIB, _LOAD_ERROR
    if _LIB is not None:
        return _LIB
    if _LOAD_ERROR is not None:
        raise _LOAD_ERROR
    try:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
    except Exception as e:  # keep the first failure and re-raise it on every call
        _LOAD_ERROR = RuntimeError("fl_correction_b200: cannot load native library %s: %s"
                                   % (LIB_PATH, e))
        raise _LOAD_ERROR
    _LIB = lib
    return lib


def call(name, *args):
    """Call an flc_* entry point; raise FlcError on a non-zero status."""
    lib = load()
    st = getattr(lib, name)(*args)
    if st != 0:
        msg = lib.flc_last_error().decode(errors="replace")
        raise FlcError(name, lib.flc_status_string(st).decode(), msg)
    return st


def query(name, *args):
    return getattr(load(), name)(*args)


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream(device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def require_cuda(name, *tensors, dtype=torch.float32):
    """TORCH_CHECK-style argument checks of the reference (atten_cuda.cpp)."""
    dev = None
    for t in tensors:
        if not isinstance(t, torch.Tensor):
            raise TypeError("%s: expected a torch.Tensor, got %s" % (name, type(t).__name__))
        if not t.is_cuda:
            raise RuntimeError("%s: tensors must be CUDA tensors" % name)
        if dtype is not None and t.dtype != dtype:
            raise RuntimeError("%s: tensors must be %s (got %s)" % (name, dtype, t.dtype))
        if dev is None:
            dev = t.device
        elif t.device != dev:
            raise RuntimeError("%s: tensors must be on one device" % name)
    return dev


def workspace(nbytes, device):
    """A 256-byte aligned uint8 workspace from torch's caching allocator."""
    n = max(int(nbytes), 1) + 256
    buf = torch.empty(n, dtype=torch.uint8, device=device)
    off = (-buf.data_ptr()) % 256
    return buf[off:off + max(int(nbytes), 1)]


def ptr_array(tensors):
    """Host array of the device pointers of `tensors` (for the entry points
    that take one pointer per problem)."""
    arr = (ctypes.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])
    return ctypes.cast(arr, ctypes.c_void_p), arr


def i64_array(values):
    arr = (ctypes.c_int64 * len(values))(*[int(v) for v in values])
    return ctypes.cast(arr, ctypes.c_void_p), arr


def mlem_multi(Cs, attens, ems, thetas, Is, n_iter, beta, delta, ws=None):
    """flc_mlem_multi_sizes over the problems i: C (R, B, H, W) in place,
    atten (A, B, H, W), em (A, R), theta (A,), I (A, B, W); R shared, the
    other sizes per problem.  Returns the workspace `ws` (reusable for calls
    of the same shapes)."""
    P = len(Cs)
    R = Cs[0].shape[0]
    if any(c.shape[0] != R for c in Cs):
        raise ValueError("mlem_multi: every problem must have the same number of references")
    A = [a.shape[0] for a in attens]
    B = [a.shape[1] for a in attens]
    H = [a.shape[2] for a in attens]
    W = [a.shape[3] for a in attens]
    pa, ka = i64_array(A)
    pb, kb = i64_array(B)
    ph, kh = i64_array(H)
    pw, kw = i64_array(W)
    nb = query("flc_mlem_multi_sizes_workspace_bytes", P, pa, pb, R, ph, pw)
    if ws is None or ws.numel() < nb:
        ws = workspace(nb, Cs[0].device)
    keep = [ptr_array(x) for x in (Cs, attens, ems, thetas, Is)]
    with torch.cuda.device(Cs[0].device):
        call("flc_mlem_multi_sizes", P, *[k[0] for k in keep], pa, pb, R, ph, pw, int(n_iter),
             float(beta), float(delta), ptr(ws), nb, stream())
    del keep, ka, kb, kh, kw
    return ws
