"""Differentiable corrected projection (flc_xrf_project / _adjoint) against the
FP64 oracle composition of FL/core.py:19-101 and atten_cuda_kernel.cu:298-337,
whose adjoint is pinned by finite differences on the CPU."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from fl_correction_b200.detector_mask import generate_detector_mask
from fl_correction_b200.xrf import XRFProjector
from tests.helpers import TOL_MAP, T, rel_err

pytestmark = pytest.mark.gpu

# gradient bar: sums of up to A*H FP32 terms with atomics, relative to max|dC|
TOL_GRAD = 2e-5


def _param(L, n_ch, A, rng):
    comps = ["C%d" % j for j in range(n_ch)]
    elems = ["E%d" % i for i in range(L)]
    cs = {"elem_type": elems, "elem_compound": comps}
    for c in comps:
        cs[c + "-x"] = rng.uniform(20, 40, A)
        for e in elems:
            cs[c + "-" + e] = float(rng.uniform(30, 60))
    return {"elem_type": elems, "elem_compound": comps, "cs": cs, "pix": 4e-4,
            "rho": {c: float(rng.uniform(3, 6)) for c in comps},
            "em_cs": {e: rng.uniform(0.5, 2.0, A) for e in elems}}


def _case(seed, n_ch=3, L=2, S=5, N=24, A=7):
    rng = np.random.default_rng(seed)
    p = _param(L, n_ch, A, rng)
    angles = np.sort(rng.uniform(0, 360, A))
    mask = generate_detector_mask(13.309, 13.309, N)
    frac = (rng.random((n_ch, S, N, N)) * 0.8).astype(np.float32)
    return p, angles, mask, frac, rng


def _oracle_inputs(proj):
    return (proj.theta.cpu().numpy(), proj.coef_x.cpu().numpy(), proj.coef_f.cpu().numpy(),
            proj.em.cpu().numpy())


@pytest.mark.parametrize("incident", ["own", "all", "none"])
def test_forward_and_adjoint_match_oracle(incident):
    p, angles, mask, frac, rng = _case(11)
    S, N = frac.shape[1], frac.shape[-1]
    proj = XRFProjector(p, angles, mask, (S, N, N), fixed_frac=frac[2:], incident=incident)
    th, cx, cf, em = _oracle_inputs(proj)
    C = T(frac[:2])
    Pf = proj.project(C).cpu().numpy()
    ref = O.xrf_project(frac, th, cx, cf, mask, em, incident)
    assert rel_err(Pf, ref) < TOL_MAP
    g = rng.standard_normal(ref.shape).astype(np.float32)
    dC = proj.adjoint(C, T(g)).cpu().numpy()
    dref = O.xrf_project_adjoint(frac, th, cx, cf, mask, em, g, incident)
    assert rel_err(dC, dref) < TOL_GRAD


@pytest.mark.parametrize("rows", [1, 5, 7])
def test_adjoint_in_row_bands_matches_oracle(rows):
    # the rotation adjoint of a slice too large for shared memory runs in row
    # bands; forced here at 24^2 (one-row bands, four bands of 5 and one of 4,
    # bands of 7 with a short last one)
    from fl_correction_b200 import tune
    p, angles, mask, frac, rng = _case(14)
    S, N = frac.shape[1], frac.shape[-1]
    proj = XRFProjector(p, angles, mask, (S, N, N), fixed_frac=frac[2:])
    th, cx, cf, em = _oracle_inputs(proj)
    C = T(frac[:2])
    g = rng.standard_normal((2, len(angles), S, N)).astype(np.float32)
    old = tune.get_knob("xrf.band")
    tune.set_knob("xrf.band", rows)
    try:
        dC = proj.adjoint(C, T(g)).cpu().numpy()
    finally:
        tune.set_knob("xrf.band", old)
    dref = O.xrf_project_adjoint(frac, th, cx, cf, mask, em, g, "own")
    assert rel_err(dC, dref) < TOL_GRAD


def test_adjoint_of_large_slices_is_band_independent():
    # 256^2 slices do not fit in shared memory whole: the automatic bands and
    # bands of 32 rows give the same gradient up to summation order
    from fl_correction_b200 import tune
    p, angles, mask, frac, rng = _case(15, n_ch=2, L=1, S=2, N=256, A=6)
    S, N = frac.shape[1], frac.shape[-1]
    proj = XRFProjector(p, angles, mask, (S, N, N), fixed_frac=frac[1:])
    C = T(frac[:1])
    g = T(rng.standard_normal((1, 6, S, N)))
    auto = proj.adjoint(C, g)
    old = tune.get_knob("xrf.band")
    tune.set_knob("xrf.band", 32)
    try:
        b32 = proj.adjoint(C, g)
    finally:
        tune.set_knob("xrf.band", old)
    assert float(auto.abs().max()) > 0
    assert rel_err(b32.cpu().numpy(), auto.cpu().numpy()) < 1e-6


def test_chunked_recomputation_is_identical():
    p, angles, mask, frac, rng = _case(12, A=9)
    S, N = frac.shape[1], frac.shape[-1]
    C = T(frac[:2])
    full = XRFProjector(p, angles, mask, (S, N, N), fixed_frac=frac[2:])
    part = XRFProjector(p, angles, mask, (S, N, N), fixed_frac=frac[2:], chunk=2)
    assert part.ws_bytes < full.ws_bytes
    g = T(rng.standard_normal((2, 9, S, N)))
    assert torch.equal(full.project(C), part.project(C))
    assert rel_err(full.adjoint(C, g).cpu().numpy(), part.adjoint(C, g).cpu().numpy()) < 1e-6


def test_autograd_matches_adjoint():
    p, angles, mask, frac, rng = _case(13, n_ch=2, L=2, S=3, N=16, A=5)
    S, N = frac.shape[1], frac.shape[-1]
    proj = XRFProjector(p, angles, mask, (S, N, N))
    I = T(rng.random((2, 5, S, N)))
    C = T(frac).requires_grad_(True)
    loss = ((proj(C) - I) ** 2).sum()
    loss.backward()
    with torch.no_grad():
        want = proj.adjoint(C, 2 * (proj.project(C) - I))
    assert rel_err(C.grad.cpu().numpy(), want.cpu().numpy()) < 1e-6


def test_shape_errors():
    p, angles, mask, frac, _ = _case(14, n_ch=2, L=2, S=2, N=16, A=3)
    proj = XRFProjector(p, angles, mask, (2, 16, 16))
    with pytest.raises(ValueError):
        proj.project(torch.zeros((2, 3, 16, 16), device="cuda"))
    with pytest.raises(RuntimeError):
        proj.project(torch.zeros((2, 2, 16, 16)))
