"""Differentiable corrected projection with the attenuation recomputed from
the concentrations (gradient through mu as well as through the projector).

The reference's gradient reconstruction (FL/example/demo.py:413-475) holds
the attenuation fixed and differentiates only the projector
(FL/cuda_lib/autograd.py:5-77).  ``XRFProjector`` keeps the same forward
model -- per angle: rotate the fractions (FL/torch_image_util.py:13-114),
assemble mu, incident scan and cone path sum (FL/torch_functions.py:83-176),
project (atten_cuda_kernel.cu:298-337) -- but recomputes the attenuation of
each angle chunk inside one native call, and its backward is the
hand-written adjoint of the whole chain (flc_xrf_project_adjoint), so the
gradient also flows through the self-absorption.  Nothing of size
angles x volume is kept between forward and backward.
"""
import numpy as np
import torch

from . import _lib
from .core import INCIDENT_MODES, atten_coefficients, mask_factors

__all__ = ["XRFProjector", "XRFProjectFunction"]


class XRFProjector:
    """Pf = P(C) for C (L, S, H, W) -> (L, A, S, W), differentiable in C.

    param       reference-layout parameter dict (elem_type, elem_compound, cs,
                rho, pix, em_cs); compounds past the elements enter the
                attenuation with the fixed fractions ``fixed_frac``.
    angles_deg  (A,) projection angles in degrees.
    mask        cone mask (Mz, Mx, My), rank one per depth plane, odd Mz, My.
    incident    'own' | 'all' | 'none' (as core.atten_maps).
    chunk       angles per recomputation pass (0: about 8 GiB of scratch, at least one angle).
    """

    def __init__(self, param, angles_deg, mask, shape, fixed_frac=None, incident="own",
                 device="cuda", chunk=0):
        dev = torch.device(device)
        self.device = dev
        self.L = len(param["elem_type"])
        self.n_ch = len(param["elem_compound"])
        S, H, W = shape
        self.shape = (S, H, W)
        angles = np.asarray(angles_deg, np.float64)
        A = len(angles)
        self.A = A
        self.mode = INCIDENT_MODES[incident]
        cx, cf = atten_coefficients(param, A, self.n_ch)
        self.coef_x = torch.from_numpy(cx).to(dev)
        self.coef_f = torch.from_numpy(cf).to(dev)
        u, v, self.mask_shape = mask_factors(mask, dev)
        self.u, self.v = u, v
        # taps of every depth plane reversed, for the cone adjoint
        self.uf = torch.flip(u, dims=[1]).contiguous()
        self.vf = torch.flip(v, dims=[1]).contiguous()
        self.theta = torch.tensor(angles / 180.0 * np.pi, dtype=torch.float32, device=dev)
        em = np.stack([np.broadcast_to(np.asarray(param["em_cs"][e], np.float64).reshape(-1), (A,))
                       * param["rho"][c] * param["pix"]
                       for e, c in zip(param["elem_type"], param["elem_compound"])])
        self.em = torch.tensor(em, dtype=torch.float32, device=dev).contiguous()  # (L, A)
        self.frac = torch.zeros((self.n_ch, S, H, W), dtype=torch.float32, device=dev)
        if self.n_ch > self.L:
            ff = (fixed_frac if fixed_frac is not None
                  else np.ones((self.n_ch - self.L, S, H, W), np.float32))
            self.frac[self.L:] = torch.as_tensor(ff, dtype=torch.float32, device=dev)
        self.chunk = int(chunk)
        # with room for the interleaved fractions and the spectral cone's scratch
        self.ws_bytes = _lib.query("flc_xrf_workspace_bytes_ex", self.n_ch, S, H, W, A, self.L,
                                   self.chunk, *self.mask_shape)
        self.ws = _lib.workspace(self.ws_bytes, dev)

    def _args(self):
        S, H, W = self.shape
        Mz, Mx, My = self.mask_shape
        return (self.n_ch, S, H, W, self.A, self.L, Mz, Mx, My, self.mode, self.chunk,
                _lib.ptr(self.ws), self.ws_bytes)

    def _set(self, C):
        if tuple(C.shape) != (self.L,) + self.shape:
            raise ValueError("XRFProjector: C must be %s, got %s"
                             % ((self.L,) + self.shape, tuple(C.shape)))
        self.frac[:self.L].copy_(C.detach())

    def project(self, C):
        """Forward projections (L, A, S, W) (no autograd)."""
        _lib.require_cuda("XRFProjector.project", C)
        self._set(C)
        S, H, W = self.shape
        Pf = torch.empty((self.L, self.A, S, W), dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("flc_xrf_project", _lib.ptr(self.frac), _lib.ptr(self.theta),
                      _lib.ptr(self.coef_x), _lib.ptr(self.coef_f), _lib.ptr(self.u),
                      _lib.ptr(self.v), _lib.ptr(self.em), _lib.ptr(Pf), *self._args(),
                      _lib.stream())
        return Pf

    def adjoint(self, C, gPf):
        """d<gPf, P(C)>/dC (L, S, H, W), through projector and attenuation."""
        _lib.require_cuda("XRFProjector.adjoint", C, gPf)
        self._set(C)
        gPf = gPf.contiguous()
        dC = torch.empty((self.L,) + self.shape, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("flc_xrf_project_adjoint", _lib.ptr(self.frac), _lib.ptr(self.theta),
                      _lib.ptr(self.coef_x), _lib.ptr(self.coef_f), _lib.ptr(self.u),
                      _lib.ptr(self.v), _lib.ptr(self.uf), _lib.ptr(self.vf), _lib.ptr(self.em),
                      _lib.ptr(gPf), _lib.ptr(dC), *self._args(), _lib.stream())
        return dC

    def __call__(self, C):
        return XRFProjectFunction.apply(C, self)


class XRFProjectFunction(torch.autograd.Function):
    """autograd wrapper: forward flc_xrf_project, backward its adjoint."""

    @staticmethod
    def forward(ctx, C, proj):
        ctx.proj = proj
        ctx.save_for_backward(C)
        return proj.project(C)

    @staticmethod
    def backward(ctx, grad_out):
        (C,) = ctx.saved_tensors
        return ctx.proj.adjoint(C, grad_out), None
