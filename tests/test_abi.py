"""The C ABI: every entry point declared in include/flc.h is exported by
libflc.so, and argument validation answers with a status code (these calls
never reach the GPU)."""
import ctypes
import os
import re

import pytest

from fl_correction_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "flc.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"FLC_API\s+[\w\s\*]+?\b(flc_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert len(names) >= 15
    for n in ("flc_cone_atten", "flc_fwd_emission", "flc_bwd_emission", "flc_mlem",
              "flc_atten_maps", "flc_huber_grad"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    assert set(declared()) <= set(_lib.SIGNATURES)


def test_status_strings_and_version():
    lib = _lib.load()
    assert lib.flc_status_string(0) == b"FLC_OK"
    assert lib.flc_status_string(4) == b"FLC_ERR_WORKSPACE"
    assert lib.flc_status_string(99) == b"FLC_ERR_UNKNOWN"
    assert b"sm_100a" in lib.flc_version()


@pytest.mark.parametrize("name,args", [
    ("flc_fwd_emission", (None, None, None, None, None, 1, 1, 1, 4, 4, None)),
    ("flc_bwd_emission", (None, None, None, None, None, 1, 1, 1, 4, 4, None)),
    ("flc_cone_atten", (None, None, None, 1, 1, 1, 1, 1, 1, 1, 0, None)),
    ("flc_huber_grad", (None, None, 1, 4, 4, 0.01, None)),
    ("flc_rotate", (None, None, 1, 4, 4, 1.0, 0.0, None)),
    ("flc_incident_scan", (None, None, 1, 4, 4, None)),
])
def test_null_pointers_are_rejected(name, args):
    lib = _lib.load()
    assert getattr(lib, name)(*args) == 1          # FLC_ERR_INVALID_ARG
    assert b"null pointer" in lib.flc_last_error()


def test_bad_sizes_are_rejected():
    lib = _lib.load()
    p = ctypes.c_void_p(16)   # never dereferenced: validation fails first
    assert lib.flc_fwd_emission(p, p, p, p, p, 4, 2, 1, 1, 8, None) == 1      # H < 2
    assert lib.flc_fwd_emission(p, p, p, p, p, 4, 2, 9, 8, 8, None) == 1      # R > 8
    assert lib.flc_mlem(p, p, p, p, p, 5, 1e-3, 0.01, 4, 2, 1, 8, 8, None, 0, 0, None) == 1
    ws = ctypes.c_void_p(256 * 7)
    assert lib.flc_mlem(p, p, p, p, p, 5, 1e-3, 0.01, 4, 2, 1, 8, 8, ws, 16, 0, None) == 4
    assert lib.flc_mlem(p, p, p, p, p, 5, 1e-3, 0.01, 4, 2, 1, 8, 8, ctypes.c_void_p(300),
                        1 << 30, 0, None) == 3
    assert lib.flc_atten_maps(p, p, p, p, p, p, p, 3, 4, 8, 6, 5, 2, 3, 8, 3, 0, 0, 0, p,
                              1 << 30, None) == 1                         # H != W


def test_workspace_queries():
    lib = _lib.load()
    assert lib.flc_mlem_workspace_bytes(120, 128, 1, 128, 128) >= 3 * 4 * 128 ** 3
    assert lib.flc_mlem_workspace_bytes(0, 1, 1, 1, 1) == 0
    assert lib.flc_atten_workspace_bytes(4, 128, 128, 128, 120, 3, 2) >= 2 * 3 * 4 * 128 ** 3
    # the pipeline part: the staged mu of a chunk, then the channel-interleaved
    # fractions (one float4 per pixel per four channels)
    v = 128 ** 3
    assert lib.flc_atten_stage_workspace_bytes(4, 128, 128, 128) == 16 * v
    assert lib.flc_atten_stage_workspace_bytes(5, 128, 128, 128) == 32 * v
    assert lib.flc_atten_stage_workspace_bytes(9, 128, 128, 128) == 0      # more than 8 channels
    assert lib.flc_atten_workspace_bytes(4, 128, 128, 128, 120, 3, 2) == 2 * 3 * 4 * v + 16 * v
    # the extended adjoint workspace holds the base one and the interleaved fractions
    base = lib.flc_xrf_workspace_bytes(4, 96, 96, 96, 90, 3, 0)
    assert lib.flc_xrf_workspace_bytes_ex(4, 96, 96, 96, 90, 3, 0, 25, 96, 25) >= base + 16 * 96 ** 3


def test_cpu_tensors_fail_loudly():
    import torch
    from fl_correction_b200.cuda_lib import atten_cuda
    x = torch.zeros(2, 3, 4, 4)
    with pytest.raises(RuntimeError, match="CUDA"):
        atten_cuda.cal_atten_cuda(x, torch.zeros(3, 3, 3))
    with pytest.raises(RuntimeError, match="CUDA"):
        atten_cuda.forward_emission_batch(x, x, torch.ones(2, 2), torch.zeros(2))


def test_tuning_knobs_round_trip():
    lib = _lib.load()
    for name in (b"proj.cluster", b"proj.apc", b"cone.variant", b"atten.chunk", b"proj.bwd",
                 b"cone.test_wait_limit", b"cone.test_skip_load", b"proj.legacy", b"proj.band",
                 b"xrf.band"):
        old = lib.flc_tune_get(name)
        assert old >= 0
        assert lib.flc_tune_set(name, 3) == 0
        assert lib.flc_tune_get(name) == 3
        assert lib.flc_tune_set(name, old) == 0
    assert lib.flc_tune_get(b"no.such.knob") == -1
    assert lib.flc_tune_set(b"no.such.knob", 1) == 1
    assert b"unknown knob" in lib.flc_last_error()
    assert lib.flc_tune_set(b"proj.cluster", -1) == 1


def test_xrf_argument_checks():
    lib = _lib.load()
    p = ctypes.c_void_p(256)
    assert lib.flc_xrf_workspace_bytes(3, 4, 16, 16, 10, 2, 0) > 0
    assert lib.flc_xrf_workspace_bytes(3, 4, 16, 16, 10, 2, 2) < lib.flc_xrf_workspace_bytes(
        3, 4, 16, 16, 10, 2, 10)
    # even cone extent in slices is rejected before anything runs
    assert lib.flc_xrf_project(p, p, p, p, p, p, p, p, 3, 4, 16, 16, 10, 2, 4, 16, 3, 0, 0, p,
                               1 << 30, None) == 1
    assert lib.flc_xrf_project(p, p, p, p, p, p, p, p, 3, 4, 16, 12, 10, 2, 3, 16, 3, 0, 0, p,
                               1 << 30, None) == 1                      # H != W
    assert lib.flc_xrf_project_adjoint(p, p, p, p, p, p, p, p, p, None, p, 3, 4, 16, 16, 10, 2,
                                       3, 16, 3, 0, 0, p, 1 << 30, None) == 1


def test_multi_workspace_holds_tables_per_slice_width():
    # per slice width two problem tables and a counter, then the problems'
    # buffers: two problems of different widths need one more width group's
    # tables than the same two problems at one width with the same buffer bytes
    import ctypes
    lib = _lib.load()
    arr = lambda *v: (ctypes.c_int64 * len(v))(*v)
    A, B, R = arr(8, 8), arr(4, 4), 1
    # widths 32 + 48 (one group each) against 40 + 40 (one group): the same
    # image bytes per problem pair (32 + 48 = 2 x 40 columns at one height)
    two = lib.flc_mlem_multi_sizes_workspace_bytes(2, A, B, R, arr(40, 40), arr(32, 48))
    one = lib.flc_mlem_multi_sizes_workspace_bytes(2, A, B, R, arr(40, 40), arr(40, 40))
    assert two > one
    three = lib.flc_mlem_multi_sizes_workspace_bytes(3, arr(8, 8, 8), arr(4, 4, 4), R,
                                                     arr(40, 40, 40), arr(32, 48, 32))
    # the third problem shares the first one's width: no new tables, only its
    # sensitivity and second C buffer (4 x 40 x 32 floats each) and its ratio
    # (8 x 4 x 32 floats)
    assert three - two == 2 * 4 * 40 * 32 * 4 + 8 * 4 * 32 * 4
    # a width group's tables hold at least 64 problem entries each
    assert two - one >= 2 * 64 * 8 * 8
    assert lib.flc_mlem_multi_sizes_workspace_bytes(0, A, B, R, arr(40, 40), arr(40, 40)) == 0
