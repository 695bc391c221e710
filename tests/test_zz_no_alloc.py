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

LIMIT = 32 << 20          # bytes of the static scratch
# flc_mlem_workspace_bytes is 3 images (R,B,H,W) + the projections (A,B,W):
# with R=1, B=512, H=W=64 that is 3 * 8 MiB + A * 128 KiB, so A = 64 needs
# exactly the limit and A = 65 one projection row more
AT_LIMIT = (64, 512, 1, 64, 64)
ABOVE_LIMIT = (65, 512, 1, 64, 64)


def test_workspace_sizes_of_the_limit_cases():
    assert _lib.query("flc_mlem_workspace_bytes", *AT_LIMIT) == LIMIT
    assert _lib.query("flc_mlem_workspace_bytes", *ABOVE_LIMIT) > LIMIT


def test_oversized_problem_is_refused():
    # the size check comes before any CUDA call, so dummy pointers are safe here
    lib = _lib.load()
    p = ctypes.c_void_p(256)
    # 256 slices of 128^2: 3 x 16 MiB of images plus the projections, above 32 MiB
    assert lib.flc_mlem_static(p, p, p, p, p, 3, 1e-3, 0.01, 120, 256, 1, 128, 128, None) == 2
    assert b"static" in lib.flc_last_error()
    # one projection row above the limit
    assert lib.flc_mlem_static(p, p, p, p, p, 3, 1e-3, 0.01, *ABOVE_LIMIT, None) == 2
    assert lib.flc_mlem_static(p, p, p, p, p, 3, 1e-3, 0.01, 0, 1, 1, 8, 8, None) == 1


def test_problem_at_the_limit_passes_the_size_check_without_a_gpu():
    # without a device the call stops at the device query, after the size
    # check, and launches nothing; on a GPU the same size runs for real in
    # test_problem_at_the_limit_runs below
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the real run covers this case")
    lib = _lib.load()
    p = ctypes.c_void_p(256)
    st = lib.flc_mlem_static(p, p, p, p, p, 3, 1e-3, 0.01, *AT_LIMIT, None)
    assert st not in (0, 1, 2), st


def _problem(rng, A, B, R, H, W, oracle_I=True):
    atten, C, em, th = projector_case(rng, A, B, R, H, W)
    if oracle_I:
        I = O.fwd_emission(atten, C, em, th) * rng.uniform(0.8, 1.2, (A, B, W))
    else:
        I = rng.uniform(0.5, 1.5, (A, B, W))
    return atten, C, em, th, I


def _run_workspace(a, e, t, i, C0, n_iter, sizes):
    ws_b = _lib.query("flc_mlem_workspace_bytes", *sizes)
    ws = _lib.workspace(ws_b, "cuda")
    ref = C0.clone()
    _lib.call("flc_mlem", _lib.ptr(ref), _lib.ptr(a), _lib.ptr(e), _lib.ptr(t), _lib.ptr(i),
              n_iter, 1e-3, 0.01, *sizes, _lib.ptr(ws), ws_b, 0, _lib.stream())
    return ref


@pytest.mark.gpu
def test_matches_workspace_entry_point_twice_in_a_row():
    rng = np.random.default_rng(21)
    sizes = (24, 3, 1, 48, 48)
    atten, C, em, th, I = _problem(rng, *sizes)
    a, e, t, i = T(atten), T(em), T(th), T(I)
    C0 = T(np.ones_like(C))
    ref = _run_workspace(a, e, t, i, C0, 10, sizes)
    outs = [C0.clone(), C0.clone()]
    torch.cuda.synchronize()
    free = []
    for out in outs:
        _lib.call("flc_mlem_static", _lib.ptr(out), _lib.ptr(a), _lib.ptr(e), _lib.ptr(t),
                  _lib.ptr(i), 10, 1e-3, 0.01, *sizes, _lib.stream())
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        # same iterations; border-frame pixels sum with shared atomics in run-dependent order
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < 1e-5
    # the first call may commit the array; the second allocates nothing
    assert free[1] == free[0], free
    assert rel_err(outs[1].cpu().numpy(), O.mlem(np.ones_like(C), atten, em, th, I, 10)) < 1e-4


@pytest.mark.gpu
def test_problem_at_the_limit_runs():
    rng = np.random.default_rng(22)
    atten, C, em, th, I = _problem(rng, *AT_LIMIT, oracle_I=False)
    a, e, t, i = T(atten), T(em), T(th), T(I)
    C0 = T(np.ones_like(C))
    ref = _run_workspace(a, e, t, i, C0, 2, AT_LIMIT)
    out = C0.clone()
    _lib.call("flc_mlem_static", _lib.ptr(out), _lib.ptr(a), _lib.ptr(e), _lib.ptr(t),
              _lib.ptr(i), 2, 1e-3, 0.01, *AT_LIMIT, _lib.stream())
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < 1e-5
