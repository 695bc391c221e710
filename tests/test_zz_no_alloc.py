"""flc_mlem_static (MLEM with a static device scratch, no allocation) against
flc_mlem with a caller workspace.  Kept in a file collected last: it must
pass alone and after every other test in the same process."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O
from fl_correction_b200 import _lib
from tests.helpers import T, projector_case, rel_err


def test_oversized_problem_is_refused():
    # the size check comes before any CUDA call
    lib = _lib.load()
    p = ctypes.c_void_p(256)
    # 256 slices of 128^2: 3 x 16 MiB of images plus the projections, above 32 MiB
    assert lib.flc_mlem_static(p, p, p, p, p, 3, 1e-3, 0.01, 120, 256, 1, 128, 128, None) == 2
    assert b"static" in lib.flc_last_error()
    assert lib.flc_mlem_static(p, p, p, p, p, 3, 1e-3, 0.01, 0, 1, 1, 8, 8, None) == 1


@pytest.mark.gpu
def test_matches_workspace_entry_point_twice_in_a_row():
    rng = np.random.default_rng(21)
    A, B, R, H, W = 24, 3, 1, 48, 48
    atten, C, em, th = projector_case(rng, A, B, R, H, W)
    I = O.fwd_emission(atten, C, em, th) * rng.uniform(0.8, 1.2, (A, B, W))
    a, e, t, i = T(atten), T(em), T(th), T(I)
    ws_b = _lib.query("flc_mlem_workspace_bytes", A, B, R, H, W)
    ws = _lib.workspace(ws_b, "cuda")
    ref = T(np.ones_like(C))
    _lib.call("flc_mlem", _lib.ptr(ref), _lib.ptr(a), _lib.ptr(e), _lib.ptr(t), _lib.ptr(i), 10,
              1e-3, 0.01, A, B, R, H, W, _lib.ptr(ws), ws_b, 0, _lib.stream())
    for _ in range(2):
        out = T(np.ones_like(C))
        _lib.call("flc_mlem_static", _lib.ptr(out), _lib.ptr(a), _lib.ptr(e), _lib.ptr(t),
                  _lib.ptr(i), 10, 1e-3, 0.01, A, B, R, H, W, _lib.stream())
        torch.cuda.synchronize()
        # same iterations; border-frame pixels sum with shared atomics in run-dependent order
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < 1e-5
    assert rel_err(out.cpu().numpy(), O.mlem(np.ones_like(C), atten, em, th, I, 10)) < 1e-4
