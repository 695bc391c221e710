"""Cone path sum parity: cal_atten_cuda (atten_cuda_kernel.cu:10-86) through
the C ABI against the FP64 oracle, separable and general paths."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from fl_correction_b200 import _lib
from fl_correction_b200.cuda_lib import atten_cuda as AC
from fl_correction_b200.detector_mask import factor_mask, generate_detector_mask
from tests.helpers import TOL_MAP, T, golden_cpu, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("K,Z,X,Y,L", [(2, 9, 20, 20, 20), (1, 16, 32, 32, 32), (3, 5, 16, 12, 16),
                                       (1, 40, 24, 30, 24), (1, 64, 64, 64, 64)])
def test_separable_matches_oracle(K, Z, X, Y, L):
    rng = np.random.default_rng(K * 100 + Z)
    mask = generate_detector_mask(13.309, 13.309, L).astype(np.float32)
    mu = (rng.random((K, Z, X, Y)) * 0.05).astype(np.float32)
    out = AC.cal_atten_cuda(T(mu), T(mask)).cpu().numpy()
    assert rel_err(out, O.cone_ref(mu, mask)) < TOL_MAP


def test_wide_mask_and_uneven_angles():
    rng = np.random.default_rng(3)
    mask = generate_detector_mask(15.0, 60.0, 12).astype(np.float32)   # (13, 12, 3)
    mu = rng.random((2, 11, 14, 18)).astype(np.float32)
    out = AC.cal_atten_cuda(T(mu), T(mask)).cpu().numpy()
    assert rel_err(out, O.cone_ref(mu, mask)) < TOL_MAP


def test_general_mask_matches_oracle():
    rng = np.random.default_rng(4)
    mask = rng.random((5, 7, 3)).astype(np.float32)
    mask[mask < 0.3] = 0
    mu = rng.random((2, 9, 20, 21)).astype(np.float32)
    out = AC.cal_atten_cuda(T(mu), T(mask)).cpu().numpy()
    assert rel_err(out, O.cone_ref(mu, mask)) < TOL_MAP


def test_forced_general_equals_separable():
    rng = np.random.default_rng(5)
    mask = generate_detector_mask(13.309, 13.309, 16).astype(np.float32)
    mu = rng.random((1, 12, 16, 16)).astype(np.float32)
    sep = AC.cal_atten_cuda(T(mu), T(mask))
    gen = torch.empty_like(sep)
    m, x = T(mask), T(mu)
    _lib.call("flc_cone_atten", _lib.ptr(x), _lib.ptr(m), _lib.ptr(gen), 1, 12, 16, 16, 3, 16, 3,
              1, _lib.stream())
    assert rel_err(gen.cpu().numpy(), sep.cpu().numpy()) < 1e-6


def test_window_wider_than_a_block():
    # the reference kernel launches one thread per column, so Y > 1024 fails there
    rng = np.random.default_rng(6)
    mask = generate_detector_mask(13.309, 13.309, 8).astype(np.float32)
    mu = rng.random((1, 3, 8, 1100)).astype(np.float32)
    out = AC.cal_atten_cuda(T(mu), T(mask)).cpu().numpy()
    assert rel_err(out, O.cone_ref(mu, mask)) < TOL_MAP


def test_golden_correlation():
    g = golden_cpu()
    out = AC.cal_atten_cuda(T(g["cone_mu"]), T(g["xrf_mask"])).cpu().numpy()
    assert rel_err(out, g["cone_out"]) < TOL_MAP


def test_separable_entry_point_modes():
    rng = np.random.default_rng(7)
    mask = generate_detector_mask(13.309, 13.309, 20)
    u, v = factor_mask(mask)
    mu = (rng.random((2, 7, 20, 20)) * 0.1).astype(np.float32)
    ref = O.cone_ref(mu, mask.astype(np.float32))
    x, U, V = T(mu), T(u), T(v)
    for mode, expect in ((0, ref), (1, np.exp(-ref))):
        out = torch.empty_like(x)
        _lib.call("flc_cone_atten_separable", _lib.ptr(x), _lib.ptr(U), _lib.ptr(V), _lib.ptr(out),
                  2, 7, 20, 20, mask.shape[0], mask.shape[1], mask.shape[2], mode, _lib.stream())
        assert rel_err(out.cpu().numpy(), expect) < TOL_MAP


def test_benchmark_size_slab():
    # 128-wide slices with the 128-deep mask, 12 of the 128 slices
    rng = np.random.default_rng(8)
    mask = generate_detector_mask(13.309, 13.309, 128).astype(np.float32)
    mu = (rng.random((1, 12, 128, 128)) * 0.01).astype(np.float32)
    out = AC.cal_atten_cuda(T(mu), T(mask)).cpu().numpy()
    assert rel_err(out, O.cone_ref(mu, mask)) < TOL_MAP


@pytest.mark.parametrize("K,Z,X,Y,L", [(2, 9, 20, 20, 20), (3, 64, 64, 64, 64), (1, 128, 128, 128, 128),
                                       (2, 40, 36, 44, 36), (1, 160, 24, 32, 24)])
def test_pipelined_and_plain_kernels_agree(K, Z, X, Y, L):
    rng = np.random.default_rng(Z + X)
    mask = generate_detector_mask(13.309, 13.309, L)
    u, v = factor_mask(mask)
    mu = (rng.random((K, Z, X, Y)) * 0.02).astype(np.float32)
    x, U, V = T(mu), T(u), T(v)
    outs = []
    for flag in (0, 16):                       # 16 = FLC_CONE_PLAIN_KERNEL
        out = torch.empty_like(x)
        _lib.call("flc_cone_atten_separable", _lib.ptr(x), _lib.ptr(U), _lib.ptr(V), _lib.ptr(out),
                  K, Z, X, Y, mask.shape[0], mask.shape[1], mask.shape[2], flag, _lib.stream())
        outs.append(out.cpu().numpy())
    assert _lib.query("flc_device_status", 1) == 0
    assert rel_err(outs[0], outs[1]) < 1e-6
    if Z * X * Y <= 64 ** 3:
        assert rel_err(outs[0], O.cone_ref(mu, mask.astype(np.float32))) < TOL_MAP


@pytest.mark.parametrize("Z,n_mask,angle", [(192, 192, 19.0), (256, 256, 13.309)])
def test_tall_volume_with_wide_mask(Z, n_mask, angle):
    # slice counts and mask extents of the 192^3 and 256^3 workloads: the
    # pipelined kernel streams each depth's filters through a small ring
    rng = np.random.default_rng(Z)
    mask = generate_detector_mask(angle, angle, n_mask)
    u, v = factor_mask(mask)
    K, X, Y = 1, 24, 32
    mu = (rng.random((K, Z, X, Y)) * 0.02).astype(np.float32)
    x, U, V = T(mu), T(u), T(v)
    out = torch.empty_like(x)
    _lib.call("flc_cone_atten_separable", _lib.ptr(x), _lib.ptr(U), _lib.ptr(V), _lib.ptr(out),
              K, Z, X, Y, mask.shape[0], mask.shape[1], mask.shape[2], 0, _lib.stream())
    assert _lib.query("flc_device_status", 1) == 0
    assert rel_err(out.cpu().numpy(), O.cone_ref(mu, mask.astype(np.float32))) < TOL_MAP


@pytest.mark.parametrize("n_a,L,S,N,mask_args", [
    (2, 3, 9, 20, (13.309, 13.309, 20)),
    (1, 2, 16, 31, (13.309, 13.309, 31)),     # odd planes: radix-3/5 padding
    (2, 1, 5, 12, (15.0, 60.0, 12)),          # mask taller (13) than the volume (5)
    (1, 1, 7, 2, (13.309, 13.309, 2)),        # 2 x 2 planes
    (1, 2, 6, 40, (19.0, 19.0, 60)),          # mask deeper (60) than the volume (40)
])
def test_spectral_cone_matches_oracle(n_a, L, S, N, mask_args):
    # the spectral form (2-D FFTs of the depth planes, per-frequency depth
    # correlation, inverse FFTs) and the plain direct kernel, both through the
    # beam-layout entry point, against the FP64 path sum of the staged mu
    from fl_correction_b200 import tune
    rng = np.random.default_rng(S * 100 + N)
    mask = generate_detector_mask(*mask_args)
    u, v = factor_mask(mask)
    Mz, Mx, My = mask.shape
    A, a0 = n_a + 1, 1
    mu = (rng.random((n_a, L, S, N, N)) * 0.05).astype(np.float32)   # (n_a, L, S, W, H)
    base = rng.uniform(0.5, 1.0, (L, A, S, N, N)).astype(np.float32)
    nb = _lib.query("flc_cone_fft_workspace_bytes", n_a * L, S, N, N, Mz, Mx, My)
    assert nb > 0
    ws = _lib.workspace(nb, "cuda")
    x, U, V = T(mu), T(u), T(v)
    outs = {}
    old = tune.get_knob("cone.variant")
    try:
        # 4: spectral, 5: spectral with the split (two-pass) plane transforms, 3: direct
        for variant in (4, 5, 3):
            tune.set_knob("cone.variant", variant)
            out = T(base)
            _lib.call("flc_cone_atten_apply_ws", _lib.ptr(x), _lib.ptr(U), _lib.ptr(V),
                      _lib.ptr(out), n_a, L, S, N, N, A, a0, Mz, Mx, My,
                      _lib.ptr(ws) if variant != 3 else None, nb, _lib.stream())
            outs[variant] = out.cpu().numpy()
    finally:
        tune.set_knob("cone.variant", old)
    res = O.cone_ref(mu.reshape(n_a * L, S, N, N), mask)   # cone frame (Z=S, X=W, Y=H)
    exp = base.astype(np.float64)
    for al in range(n_a):
        for l in range(L):
            r = res[al * L + l]
            exp[l, a0 + al] *= np.exp(-r[:, :, ::-1].transpose(0, 2, 1))
    assert rel_err(outs[4], exp) < TOL_MAP
    assert rel_err(outs[5], exp) < TOL_MAP
    assert rel_err(outs[3], exp) < TOL_MAP
    assert np.array_equal(outs[4][:, 0], base[:, 0])   # angles outside the chunk untouched
    assert np.array_equal(outs[5][:, 0], base[:, 0])


def test_spectral_cone_large_planes_split():
    """200 x 200 planes (216^2 padded) do not fit one CTA's shared memory
    twice: the spectral form runs its plane transforms in two passes by
    itself.  cal_atten_cuda (reference layout) against the oracle and the
    direct kernel."""
    from fl_correction_b200 import tune
    from fl_correction_b200.cuda_lib import atten_cuda as AC
    rng = np.random.default_rng(21)
    mask = generate_detector_mask(13.309, 13.309, 6).astype(np.float32)
    mu = (rng.random((1, 200, 6, 200)) * 0.05).astype(np.float32)    # (K, Z, X, Y)
    Mz, Mx, My = mask.shape
    assert _lib.query("flc_cone_fft_workspace_bytes", 1, 200, 6, 200, Mz, Mx, My) > 0
    got = AC.cal_atten_cuda(T(mu), T(mask)).cpu().numpy()
    old = tune.get_knob("cone.variant")
    try:
        tune.set_knob("cone.variant", 3)
        direct = AC.cal_atten_cuda(T(mu), T(mask)).cpu().numpy()
    finally:
        tune.set_knob("cone.variant", old)
    ref = O.cone_ref(mu, mask)
    assert rel_err(got, ref) < TOL_MAP
    assert rel_err(direct, ref) < TOL_MAP


def test_spectral_cone_benchmark_size():
    # 128^2 planes with the 29 x 128 x 29 mask: spectral form against the
    # pipelined direct kernel (the FP64 sum at this size takes minutes)
    from fl_correction_b200 import tune
    rng = np.random.default_rng(12)
    mask = generate_detector_mask(13.309, 13.309, 128)
    u, v = factor_mask(mask)
    Mz, Mx, My = mask.shape
    n_a, L, S, N, A = 1, 2, 10, 128, 1
    mu = (rng.random((n_a, L, S, N, N)) * 0.01).astype(np.float32)
    nb = _lib.query("flc_cone_fft_workspace_bytes", n_a * L, S, N, N, Mz, Mx, My)
    ws = _lib.workspace(nb, "cuda")
    x, U, V = T(mu), T(u), T(v)
    outs = []
    old = tune.get_knob("cone.variant")
    try:
        for variant in (4, 1):
            tune.set_knob("cone.variant", variant)
            out = torch.ones((L, A, S, N, N), device="cuda")
            _lib.call("flc_cone_atten_apply_ws", _lib.ptr(x), _lib.ptr(U), _lib.ptr(V),
                      _lib.ptr(out), n_a, L, S, N, N, A, 0, Mz, Mx, My, _lib.ptr(ws), nb,
                      _lib.stream())
            outs.append(out.cpu().numpy())
    finally:
        tune.set_knob("cone.variant", old)
    assert _lib.query("flc_device_status", 1) == 0
    assert rel_err(outs[0], outs[1]) < 2e-6


def test_spectral_cone_full_planes_against_oracle():
    """128^2 planes, the benchmark's (29, 128, 29) mask (every depth of the
    128-deep correlation), 6 slices: the spectral form against the FP64
    oracle (a few seconds of the oracle's threads)."""
    from fl_correction_b200 import tune
    rng = np.random.default_rng(13)
    mask = generate_detector_mask(13.309, 13.309, 128)
    u, v = factor_mask(mask)
    Mz, Mx, My = mask.shape
    n_a, L, S, N, A = 1, 1, 6, 128, 1
    mu = (rng.random((n_a, L, S, N, N)) * 0.01).astype(np.float32)
    mu[..., 40:90, 30:70] += 0.02
    nb = _lib.query("flc_cone_fft_workspace_bytes", n_a * L, S, N, N, Mz, Mx, My)
    ws = _lib.workspace(nb, "cuda")
    x, U, V = T(mu), T(u), T(v)           # held until the kernels have run
    old = tune.get_knob("cone.variant")
    try:
        tune.set_knob("cone.variant", 4)
        out = torch.ones((L, A, S, N, N), device="cuda")
        _lib.call("flc_cone_atten_apply_ws", _lib.ptr(x), _lib.ptr(U), _lib.ptr(V),
                  _lib.ptr(out), n_a, L, S, N, N, A, 0, Mz, Mx, My, _lib.ptr(ws), nb,
                  _lib.stream())
        got = out.cpu().numpy()
    finally:
        tune.set_knob("cone.variant", old)
    O.set_threads(O.max_threads())
    res = O.cone_ref(mu.reshape(n_a * L, S, N, N), mask)          # cone frame (Z=S, X=W, Y=H)
    exp = np.exp(-res[0][:, :, ::-1].transpose(0, 2, 1))
    assert rel_err(got[0, 0], exp) < TOL_MAP
    # the path sum itself where it is large enough to carry digits (exp(-res) is
    # within rounding of 1 wherever res is tiny)
    r_got = -np.log(np.clip(got[0, 0].astype(np.float64), 1e-30, None))
    r_ref = res[0][:, :, ::-1].transpose(0, 2, 1)
    big = r_ref > 1e-3 * r_ref.max()
    assert np.abs(r_got - r_ref)[big].max() <= 1e-4 * r_ref.max()


def test_bounded_wait_runs_out_and_reports_timeout():
    """The direct cone's bounded TMA waits: with the test hooks the first
    staged plane's load is never issued and the wait gives up after a few
    thousand polls.  The kernel waits for its other loads, stops, and leaves
    FLC_ERR_TIMEOUT for flc_device_status; the context stays usable."""
    lib = _lib.load()
    rng = np.random.default_rng(5)
    K, Z, X, Y = 1, 16, 16, 16
    mask = generate_detector_mask(13.309, 13.309, X)
    u, v = factor_mask(mask)
    mu = (rng.random((K, Z, X, Y)) * 0.02).astype(np.float32)
    x, U, V = T(mu), T(u), T(v)
    out = torch.empty_like(x)

    def run():
        _lib.call("flc_cone_atten_separable", _lib.ptr(x), _lib.ptr(U), _lib.ptr(V),
                  _lib.ptr(out), K, Z, X, Y, *mask.shape, 0, _lib.stream())
        torch.cuda.synchronize()

    assert lib.flc_device_status(1) == 0
    try:
        assert lib.flc_tune_set(b"cone.test_wait_limit", 4000) == 0
        assert lib.flc_tune_set(b"cone.test_skip_load", 1) == 0
        run()
    finally:
        lib.flc_tune_set(b"cone.test_skip_load", 0)
        lib.flc_tune_set(b"cone.test_wait_limit", 0)
    assert lib.flc_device_status(1) == 6            # FLC_ERR_TIMEOUT, then cleared
    assert lib.flc_device_status(0) == 0
    run()                                           # the same call works again
    assert lib.flc_device_status(1) == 0
    assert rel_err(out.cpu().numpy(), O.cone_ref(mu, mask.astype(np.float32))) < TOL_MAP


def test_cached_mask_factors_follow_the_mask():
    # cal_atten_cuda factors a mask once and reuses the factors while the same
    # mask comes back: the cached path against flc_cone_atten (which reads and
    # factors the mask on every call), then after the mask changes in place,
    # then with a mask that is not rank one (the general gather)
    rng = np.random.default_rng(12)
    mu = T((rng.random((3, 20, 24, 20)) * 0.05).astype(np.float32))
    mask = T(generate_detector_mask(13.309, 13.309, 24).astype(np.float32))

    def direct(m):
        out = torch.empty_like(mu)
        _lib.call("flc_cone_atten", _lib.ptr(mu), _lib.ptr(m), _lib.ptr(out), *mu.shape,
                  *m.shape, 0, _lib.stream())
        return out

    for _ in range(2):
        got = AC.cal_atten_cuda(mu, mask)
        assert rel_err(got.cpu().numpy(), direct(mask).cpu().numpy()) < 1e-6
    mask.mul_(0.5)
    got = AC.cal_atten_cuda(mu, mask)
    assert rel_err(got.cpu().numpy(), O.cone_ref(mu.cpu().numpy(), mask.cpu().numpy())) < TOL_MAP
    mask[0, 3, 1] += 0.7        # no longer rank one in that depth plane
    got = AC.cal_atten_cuda(mu, mask)
    assert rel_err(got.cpu().numpy(), O.cone_ref(mu.cpu().numpy(), mask.cpu().numpy())) < TOL_MAP
