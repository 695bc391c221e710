"""The spectral cone's mathematics in FP64 numpy, against the oracle (CPU).

The CUDA spectral cone (fl_correction_b200/csrc/flc_cone_fft.cu) rests on
three facts checked here without a GPU:
  * the padded lengths (smallest even 2,3,5-smooth >= plane + mask half-width)
    make the circular correlation equal to the zero-padded path sum of
    atten_cuda_kernel.cu:10-57 on the output range;
  * with G_d = Uf_d (x) Vf_d from the rank-one mask factors, the depth sum is a
    per-frequency correlation along x;
  * the Stockham recurrence the kernels use (butterfly j reads j + r*N/R,
    twiddles e^{-2 pi i (j mod Ns) r / (Ns R)}, writes (j div Ns)*Ns*R +
    (j mod Ns) + r*Ns) and the packing of two real rows into one complex
    transform reproduce the DFT.
"""
import numpy as np
import pytest

from oracle import oracle as O


def smooth_even(n):
    m = n + (n & 1)
    while True:
        k = m
        for r in (2, 3, 5):
            while k % r == 0:
                k //= r
        if k == 1:
            return m
        m += 2


def radices(n):
    """The kernels' passes: 2^e in 8s and 4s (fewest passes, 4 on ties),
    3^f in 9s and a 3, then 5s."""
    rs = []
    e = f = 0
    while n % 2 == 0:
        n //= 2
        e += 1
    while n % 3 == 0:
        n //= 3
        f += 1
    while e > 0:
        t = 3 if (e >= 3 and e != 4) else (2 if e >= 2 else 1)
        rs.append(1 << t)
        e -= t
    while f >= 2:
        rs.append(9)
        f -= 2
    if f == 1:
        rs.append(3)
    while n % 5 == 0:
        rs.append(5)
        n //= 5
    assert n == 1
    return rs


def _dft(v, sg):
    R = v.shape[-1]
    return v @ np.exp(sg * 2j * np.pi * np.outer(np.arange(R), np.arange(R)) / R).T


def dft8_kernel_form(v, sg):
    """dft_small<8>: 2-point DFTs of (n, n+4), odd outputs turned by
    e^{sg i pi n/4}, 4-point DFTs over n; output k1 + 2 k2."""
    e = v[..., :4] + v[..., 4:]
    o = (v[..., :4] - v[..., 4:]) * np.exp(sg * 1j * np.pi * np.arange(4) / 4)
    out = np.empty_like(v)
    out[..., 0::2] = _dft(e, sg)
    out[..., 1::2] = _dft(o, sg)
    return out


def dft9_kernel_form(v, sg):
    """dft_small<9>: 3-point DFTs over n1 of x[3 n1 + n2], turned by
    e^{sg 2 pi i n2 k1 / 9}, 3-point DFTs over n2; output k1 + 3 k2."""
    y = np.stack([_dft(v[..., [n2, n2 + 3, n2 + 6]], sg) for n2 in range(3)], -2)  # [n2][k1]
    y = y * np.exp(sg * 2j * np.pi * np.outer(np.arange(3), np.arange(3)) / 9)
    out = np.empty_like(v)
    for k1 in range(3):
        out[..., k1::3] = _dft(y[..., :, k1], sg)
    return out


@pytest.mark.parametrize("sg", [-1, 1])
def test_radix8_and_radix9_butterflies(sg):
    rng = np.random.default_rng(8 + sg)
    for R, form in ((8, dft8_kernel_form), (9, dft9_kernel_form)):
        v = rng.random((4, R)) + 1j * rng.random((4, R))
        assert np.abs(form(v, sg) - _dft(v, sg)).max() < 1e-12


def test_pass_counts():
    assert radices(144) == [4, 4, 9]
    assert radices(216) == [8, 9, 3]
    assert radices(288) == [8, 4, 9]
    assert radices(160) == [8, 4, 5]


def stockham(x, sign=-1):
    """The kernels' pass order and index formulas, on the last axis."""
    N = x.shape[-1]
    tw = np.exp(-2j * np.pi * np.arange(N) / N)
    if sign > 0:
        tw = np.conj(tw)
    a = np.array(x, dtype=np.complex128)
    Ns = 1
    for R in radices(N):
        M = N // R
        step = N // (Ns * R)
        b = np.empty_like(a)
        dft = np.exp(sign * 2j * np.pi * np.outer(np.arange(R), np.arange(R)) / R)
        for j in range(M):
            jm = j % Ns
            v = np.stack([a[..., j + r * M] * (tw[jm * r * step] if r else 1.0) for r in range(R)], -1)
            y = v @ dft.T
            base = (j - jm) * R + jm
            for r in range(R):
                b[..., base + r * Ns] = y[..., r]
        a = b
        Ns *= R
    return a


@pytest.mark.parametrize("n", [2, 4, 6, 8, 12, 18, 20, 36, 50, 72, 144, 160, 216, 288])
def test_stockham_recurrence_is_the_dft(n):
    rng = np.random.default_rng(n)
    x = rng.random((3, n)) + 1j * rng.random((3, n))
    assert np.abs(stockham(x) - np.fft.fft(x)).max() < 1e-10 * n
    assert np.abs(stockham(x, +1) - n * np.fft.ifft(x)).max() < 1e-10 * n


def test_two_real_rows_per_complex_transform():
    # forward: Xa = (Z_k + conj Z_{-k}) / 2, Xb = (Z_k - conj Z_{-k}) / (2i);
    # inverse: IFFT(Xa + i Xb) = xa + i xb for Hermitian half spectra
    rng = np.random.default_rng(1)
    n = 36
    xa, xb = rng.random(n), rng.random(n)
    Z = stockham(xa + 1j * xb)
    Zn = Z[(-np.arange(n)) % n]
    Xa, Xb = (Z + np.conj(Zn)) / 2, (Z - np.conj(Zn)) / 2j
    assert np.allclose(Xa, np.fft.fft(xa)) and np.allclose(Xb, np.fft.fft(xb))
    half = n // 2
    ha, hb = Xa[:half + 1], Xb[:half + 1]
    k = np.arange(n)
    up = k > half
    kk = np.where(up, n - k, k)
    fa = np.where(up, np.conj(ha[kk]), ha[kk])
    fb = np.where(up, np.conj(hb[kk]), hb[kk])
    r = stockham(fa + 1j * fb, +1) / n
    assert np.allclose(r.real, xa) and np.allclose(r.imag, xb)


def spectral_cone(mu, u, v):
    """res (K, Z, X, Y) of the separable mask u[d][dz] v[d][dy], the way the
    kernels compute it, in FP64."""
    K, Z, X, Y = mu.shape
    Mx, Mz = u.shape
    My = v.shape[1]
    hz, hy = Mz // 2, My // 2
    Nz = smooth_even(Z + max(1, hz, Mz - 1 - hz))
    Ny = smooth_even(Y + max(hy, My - 1 - hy))
    Nyh = Ny // 2 + 1
    kz = np.arange(Nz)[None, :, None]
    ky = np.arange(Nyh)[None, :, None]
    Uf = (u[:, None, :] * np.exp(2j * np.pi * kz * (np.arange(Mz) - hz)[None, None, :] / Nz)).sum(-1)
    Vf = (v[:, None, :] * np.exp(2j * np.pi * ky * (np.arange(My) - hy)[None, None, :] / Ny)).sum(-1)
    G = Uf[:, :, None] * Vf[:, None, :]
    out = np.empty_like(mu)
    for k in range(K):
        P = np.zeros((X, Nz, Nyh), complex)
        for p in range(X):
            plane = np.zeros((Nz, Ny))
            plane[:Z, :Y] = mu[k, :, p, :]
            P[p] = np.fft.rfft2(plane)
        for x in range(X):
            R = sum(G[d] * P[x + d] for d in range(min(Mx, X - x)))
            out[k, :, x, :] = np.fft.irfft2(R, s=(Nz, Ny))[:Z, :Y]
    return out


@pytest.mark.parametrize("Z,X,Y,Mz,Mx,My", [(20, 12, 28, 7, 5, 9), (16, 9, 16, 6, 9, 4),
                                            (5, 10, 12, 13, 12, 3), (7, 2, 2, 1, 2, 1),
                                            (9, 6, 11, 5, 14, 5)])
def test_spectral_cone_equals_the_path_sum(Z, X, Y, Mz, Mx, My):
    # even mask extents, masks taller / deeper than the volume, 2 x 2 planes
    rng = np.random.default_rng(Z * 31 + X)
    mu = rng.random((2, Z, X, Y))
    u, v = rng.random((Mx, Mz)), rng.random((Mx, My))
    mask = u.T[:, :, None] * v[None, :, :]          # (Mz, Mx, My)
    ref = O.cone_ref(mu, mask)
    got = spectral_cone(mu, u, v)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
