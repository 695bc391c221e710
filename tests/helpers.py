"""Shared helpers for the tests.

Error measure used throughout (the parity bar of the port):
    rel_err(a, b) = max|a - b| / max|b|
i.e. the largest deviation relative to the reference's dynamic range.  Bars:
1e-5 for attenuation maps and projections, 1e-4 after 20 MLEM iterations.
"""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_MAP = 1e-5      # attenuation maps and projections
TOL_MLEM = 1e-4     # after 20 MLEM iterations


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, (a.shape, b.shape)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def golden_cpu():
    return np.load(os.path.join(GOLDEN, "ref_cpu.npz"))


def golden_meta():
    with open(os.path.join(GOLDEN, "ref_cpu.json")) as f:
        return json.load(f)


def atten_param():
    """The per-angle parameter dict used by the attenuation goldens."""
    m = golden_meta()["atten_param"]
    cs = dict(m["cs"])
    return {"cs": cs, "rho": m["rho"], "pix": m["pix"],
            "elem_type": cs["elem_type"], "elem_compound": cs["elem_compound"]}


def T(x, device="cuda"):
    import torch
    return torch.tensor(np.asarray(x), dtype=torch.float32, device=device)


def projector_case(rng, A, B, R, H, W, angles=None):
    atten = rng.random((A, B, H, W)).astype(np.float32)
    C = rng.random((R, B, H, W)).astype(np.float32)
    em = rng.uniform(0.5, 2.0, (A, R)).astype(np.float32)
    if angles is None:
        th = rng.uniform(-np.pi, np.pi, A).astype(np.float32)
    else:
        th = np.asarray(angles, np.float32)
    return atten, C, em, th
