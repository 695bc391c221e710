"""MLEM drivers with the signatures of FL/torch_recon.py.

numpy in, numpy out, as in the reference: inputs are moved to the device,
em_cs is pre-scaled by rho * pix (FL/torch_recon.py:83), and the native
device-resident MLEM (flc_mlem) runs all iterations without host round trips.
"""
import numpy as np
import torch

from .cuda_lib.atten_cuda import mlem_cuda, mlem_cuda_batch

__all__ = ["torch_mlem_recon", "torch_mlem_recon_batch"]


def _em(em_cs, n_angle, n_ref, rho, pix):
    if em_cs is None:
        em_cs = np.ones((n_angle, n_ref))
    else:
        em_cs = np.asarray(em_cs)
        if em_cs.ndim == 1:
            em_cs = em_cs[:, np.newaxis]
    return em_cs * rho * pix


def torch_mlem_recon(C_init, prj_sli, angle_list, atten=None, em_cs=None, rho=1, pix=1,
                     n_iter=50, beta=1e-3, delta=0.01, device="cuda"):
    """Single-slice MLEM (FL/torch_recon.py:5-47): C_init (R,H,W), prj_sli (A,W)."""
    n_ref, H, W = np.shape(C_init)
    n_angle = len(angle_list)
    theta = torch.tensor(np.asarray(angle_list) / 180.0 * np.pi, dtype=torch.float, device=device)
    if atten is None:
        atten_t = torch.ones(n_angle, H, W, dtype=torch.float, device=device)
    else:
        atten_t = torch.tensor(np.asarray(atten), dtype=torch.float, device=device)
    em = torch.tensor(_em(em_cs, n_angle, n_ref, rho, pix), dtype=torch.float, device=device)
    C = torch.tensor(np.asarray(C_init), dtype=torch.float, device=device)
    I = torch.tensor(np.asarray(prj_sli), dtype=torch.float, device=device)
    return mlem_cuda(C, atten_t, em, theta, I, n_iter, beta, delta).cpu().numpy()


def torch_mlem_recon_batch(C_init, prjs, angle_list, atten=None, em_cs=None, rho=1, pix=1,
                           n_iter=50, beta=1e-3, delta=0.01, device="cuda"):
    """Batched MLEM (FL/torch_recon.py:50-99): C_init (R,S,H,W) or (R,H,W),
    prjs (A,S,W) or (A,W), atten (A,S,H,W) or (A,H,W)."""
    C_init = np.asarray(C_init)
    prjs = np.asarray(prjs)
    if C_init.ndim == 3:
        C_init = C_init[:, np.newaxis]
    if prjs.ndim == 2:
        prjs = prjs[:, np.newaxis]
    n_ref, n_sli, H, W = C_init.shape
    n_angle = len(angle_list)
    theta = torch.tensor(np.asarray(angle_list) / 180.0 * np.pi, dtype=torch.float, device=device)
    if atten is None:
        atten_t = torch.ones(n_angle, n_sli, H, W, dtype=torch.float, device=device)
    else:
        atten = np.asarray(atten)
        if atten.ndim == 3:
            atten = atten[:, np.newaxis]
        atten_t = torch.tensor(atten, dtype=torch.float, device=device)
    em = torch.tensor(_em(em_cs, n_angle, n_ref, rho, pix), dtype=torch.float, device=device)
    C = torch.tensor(C_init, dtype=torch.float, device=device)
    I = torch.tensor(prjs, dtype=torch.float, device=device)
    return mlem_cuda_batch(C, atten_t, em, theta, I, n_iter, beta, delta).cpu().numpy()
