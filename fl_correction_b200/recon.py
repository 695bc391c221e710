"""Self-absorption-corrected MLEM, device resident.

The reference's outer loop (FL/example/demo.py:244-336) recomputes the
attenuation maps from the current reconstruction through TIFF files
(FL/core.py:19-101), then runs ``mlem_cuda_batch`` per element
(FL/torch_recon.py:50-99) with the attenuation held fixed.  Here the whole
loop stays on one GPU: every ``recompute_every`` iterations the attenuation
of every element at every angle is rebuilt from the current concentrations
by one native call (rotation, mu assembly, incident scan, cone path sum), and
the MLEM iterations in between are native cluster launches.  Nothing is
copied to the host until the caller asks for the result.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .core import atten_coefficients, atten_maps, atten_workspace_bytes, cal_frac, mask_factors
from .detector_mask import generate_detector_mask

__all__ = ["CorrectedMLEM"]


class CorrectedMLEM:
    """Corrected MLEM for L elements on an (S, N, N) grid at A angles.

    param          reference-layout parameter dict (elem_type, elem_compound,
                   cs, rho, pix, em_cs); compounds past the elements (e.g. a
                   matrix) enter the attenuation with a fixed fraction.
    angles_deg     (A,) projection angles in degrees.
    mask           cone mask (Mz, Mx, My), e.g. generate_detector_mask(...).
    fixed_frac     (n_ch - L, S, N, N) fractions of the non-element compounds.
    incident       'own' (element i's incident term uses compound i, as
                   FL/core.py:80-81 does), 'all' (legacy product) or 'none'.
    feedback       how the estimate enters mu at each rebuild: 'bounded'
                   (default) clips to [0, 1] and scales voxels whose
                   elements' total exceeds 1 down to 1; 'cal_frac' runs the
                   reference's cal_frac on the device (FL/core.py:159-205, as
                   FL/example/demo.py:249-265 feeds the estimate back: per
                   element fraction of the total clamped to its
                   [scale_range] quantiles, times total / its scale_limit
                   quantile; threshold mask 1).  'bounded' keeps cal_frac's
                   non-negativity and replaces its quantile clamp and
                   percentile scaling by the mass-fraction bound.
    """

    def __init__(self, param, angles_deg, mask, shape, fixed_frac=None, incident="own",
                 beta=0.0, delta=0.01, device="cuda", chunk=0, bound_frac=True,
                 feedback="bounded", cal_frac_args=None, multi=False, concurrent=True):
        self.device = torch.device(device)
        # multi: the MLEM iterations of all elements in one persistent launch
        # each (flc_mlem_multi) instead of one flc_mlem call per element
        self.multi = multi
        # concurrent: the elements' flc_mlem calls (independent chains of
        # launches) on one stream each, joined back into the caller's stream,
        # so that one element's kernels fill the SMs another's leave idle
        self.concurrent = bool(concurrent)
        self._ws_multi = None
        self.bound_frac = bound_frac
        if feedback not in ("bounded", "cal_frac"):
            raise ValueError("feedback must be 'bounded' or 'cal_frac'")
        self.feedback = feedback
        self.cal_frac_args = dict(scale_range=[0.02, 0.98], enable_scale=True, scale_limit=0.95)
        self.cal_frac_args.update(cal_frac_args or {})
        self.param = param
        self.L = len(param["elem_type"])
        self.n_ch = len(param["elem_compound"])
        S, H, W = shape
        self.shape = (S, H, W)
        self.angles = np.asarray(angles_deg, np.float64)
        A = len(self.angles)
        self.A = A
        self.incident = incident
        self.beta, self.delta = float(beta), float(delta)
        cx, cf = atten_coefficients(param, A, self.n_ch)
        dev = self.device
        self.coef_x = torch.from_numpy(cx).to(dev)
        self.coef_f = torch.from_numpy(cf).to(dev)
        self.mask_uv = mask_factors(mask, dev)
        self.theta = torch.tensor(self.angles / 180.0 * np.pi, dtype=torch.float32, device=dev)
        # emission cs scaled by rho*pix per element (FL/torch_recon.py:83)
        em = np.stack([np.broadcast_to(np.asarray(param["em_cs"][e], np.float64).reshape(-1), (A,))
                       * param["rho"][c] * param["pix"]
                       for e, c in zip(param["elem_type"], param["elem_compound"])])
        self.em = torch.tensor(em[:, :, None], dtype=torch.float32, device=dev).contiguous()  # (L,A,1)
        self.frac = torch.zeros((self.n_ch, S, H, W), dtype=torch.float32, device=dev)
        if self.n_ch > self.L:
            ff = torch.as_tensor(fixed_frac if fixed_frac is not None
                                 else np.ones((self.n_ch - self.L, S, H, W), np.float32),
                                 dtype=torch.float32, device=dev)
            self.frac[self.L:] = ff
        self.atten = torch.empty((self.L, A, S, H, W), dtype=torch.float32, device=dev)
        ws, _, _ = atten_workspace_bytes(self.n_ch, S, H, W, A, self.L, chunk, self.mask_uv[2])
        self.chunk = chunk
        self.ws_atten = _lib.workspace(ws, dev)
        self.ws_mlem_bytes = _lib.query("flc_mlem_workspace_bytes", A, S, 1, H, W)
        self.ws_mlem = _lib.workspace(self.ws_mlem_bytes, dev)
        self._elem = None
        if self.concurrent and self.L > 1:
            # one stream and one MLEM workspace per element
            self._elem = [(torch.cuda.Stream(device=dev),
                           self.ws_mlem if l == 0 else _lib.workspace(self.ws_mlem_bytes, dev))
                          for l in range(self.L)]

    # -- building blocks -------------------------------------------------
    def recompute_attenuation(self, C, cone_events=None):
        """atten[l, a] from concentrations C (L, S, H, W) on the device.

        With feedback 'bounded' the estimate enters mu as mass fractions:
        clipped to [0, 1] and, where the elements' total exceeds 1, scaled
        down to a total of 1 (with bound_frac, the default); with 'cal_frac'
        as the reference's cal_frac makes them (FL/core.py:159-205).  Either
        way bounded fractions, not raw MLEM values, are fed back: without a
        bound, voxels that MLEM overshoots raise mu, which lowers the
        modelled signal there, which raises them further, and the outer loop
        diverges on absorbing samples."""
        f = self.frac[:self.L]
        if self.feedback == "cal_frac":
            cal_frac(C.contiguous(), out=f, **self.cal_frac_args)
        else:
            f.copy_(C)
        if self.feedback == "bounded" and self.bound_frac:
            f.clamp_(0.0, 1.0)
            tot = f.sum(dim=0, keepdim=True).clamp_(min=1.0)
            f.div_(tot)
        atten_maps(self.frac, self.angles, self.coef_x, self.coef_f, self.mask_uv,
                   incident=self.incident, xrf=True, out=self.atten, chunk=self.chunk,
                   workspace=self.ws_atten, cone_events=cone_events, theta=self.theta)
        return self.atten

    def mlem(self, C, I, n_iter, use_graph=0, mlem_events=None):
        """n_iter MLEM iterations per element with the current attenuation; C
        (L, S, H, W) is updated in place.  mlem_events: optional list receiving
        (start, end) CUDA events around each element's iterations (around all
        elements' when they run concurrently)."""
        S, H, W = self.shape
        if self.multi and use_graph == 0:
            if mlem_events is not None:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
            self._ws_multi = _lib.mlem_multi(
                [C[l:l + 1] for l in range(self.L)], [self.atten[l] for l in range(self.L)],
                [self.em[l] for l in range(self.L)], [self.theta] * self.L,
                [I[l] for l in range(self.L)], n_iter, self.beta, self.delta, self._ws_multi)
            if mlem_events is not None:
                e1.record()
                mlem_events.append((e0, e1, int(n_iter) * self.L))
            return C
        if self._elem is not None and use_graph == 0:
            with torch.cuda.device(self.device):
                main = torch.cuda.current_stream(self.device)
                if mlem_events is not None:
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(main)
                for l, (st, ws) in enumerate(self._elem):
                    st.wait_stream(main)
                    _lib.call("flc_mlem", _lib.ptr(C[l]), _lib.ptr(self.atten[l]),
                              _lib.ptr(self.em[l]), _lib.ptr(self.theta), _lib.ptr(I[l]),
                              int(n_iter), self.beta, self.delta, self.A, S, 1, H, W,
                              _lib.ptr(ws), self.ws_mlem_bytes, 0, ctypes.c_void_p(st.cuda_stream))
                for st, _ in self._elem:
                    main.wait_stream(st)
                if mlem_events is not None:
                    e1.record(main)
                    mlem_events.append((e0, e1, int(n_iter) * self.L))
            return C
        with torch.cuda.device(self.device):
            for l in range(self.L):
                if mlem_events is not None:
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                _lib.call("flc_mlem", _lib.ptr(C[l]), _lib.ptr(self.atten[l]), _lib.ptr(self.em[l]),
                          _lib.ptr(self.theta), _lib.ptr(I[l]), int(n_iter), self.beta, self.delta,
                          self.A, S, 1, H, W, _lib.ptr(self.ws_mlem), self.ws_mlem_bytes,
                          use_graph, _lib.stream())
                if mlem_events is not None:
                    e1.record()
                    mlem_events.append((e0, e1, int(n_iter)))
        return C

    def project(self, C):
        """Forward projections (L, A, S, W) of C through the current attenuation."""
        from .cuda_lib.atten_cuda import forward_emission_batch
        return torch.stack([forward_emission_batch(self.atten[l], C[l:l + 1].contiguous(),
                                                   self.em[l], self.theta)
                            for l in range(self.L)])

    # -- the corrected reconstruction --------------------------------------
    def run_into(self, C, I, n_iter=50, recompute_every=5, cone_events=None, mlem_events=None):
        """The corrected MLEM schedule on C (L, S, H, W) in place, starting from
        its current contents.  Allocates nothing and copies nothing to or from
        the host, so the whole schedule can be captured in a CUDA graph."""
        done = 0
        while done < n_iter:
            k = min(recompute_every, n_iter - done)
            self.recompute_attenuation(C, cone_events)
            self.mlem(C, I, k, mlem_events=mlem_events)
            done += k
        return C

    def run(self, I, C0=None, n_iter=50, recompute_every=5, cone_events=None, mlem_events=None):
        """Corrected MLEM: I (L, A, S, W) device projections; returns C (L, S, H, W).
        Attenuation is rebuilt from the current C before every block of
        `recompute_every` iterations (the first block uses C0).  The optional
        event lists collect per-kernel CUDA-event timings (see
        recompute_attenuation / mlem)."""
        S, H, W = self.shape
        if C0 is None:
            C = torch.ones((self.L, S, H, W), dtype=torch.float32, device=self.device)
        else:
            C = torch.as_tensor(C0, dtype=torch.float32, device=self.device).clone()
        return self.run_into(C, I.contiguous(), n_iter, recompute_every, cone_events, mlem_events)

    def run_host(self, I_host, C0_host=None, n_iter=50, recompute_every=5):
        """End-to-end form: host (pinned) projections in, host result out."""
        I = I_host.to(self.device, non_blocking=True)
        C0 = None if C0_host is None else C0_host.to(self.device, non_blocking=True)
        C = self.run(I, C0, n_iter, recompute_every)
        return C.to("cpu")


def default_mask(N, angle_deg):
    return generate_detector_mask(angle_deg, angle_deg, N)
