// Spectral cone path sum (sm_100a).
//
// The separable cone (atten_cuda_kernel.cu:10-57 for a mask whose every depth
// plane is an outer product u[d] (x) v[d], FL/detector_mask.py) is, for each
// target depth plane x, a sum over depths d of 2-D correlations of the source
// plane p = x + d with the depth-d mask plane:
//   res[z,x,y] = sum_d sum_dz sum_dy u[d][dz] v[d][dy] mu[z+dz-hz, x+d, y+dy-hy].
// Each 2-D correlation is a pointwise product in the Fourier domain of the
// (z, y) plane, so with P_p = FFT2(mu plane p), zero-padded to Nz x Ny, and
// G_d(kz,ky) = Uf_d(kz) Vf_d(ky), Uf_d(kz) = sum_dz u[d][dz] e^{+2 pi i kz (dz-hz)/Nz}
// (Vf likewise), the whole depth sum is, per frequency, a 1-D correlation
// along x:  R_x(k) = sum_d G_d(k) P_{x+d}(k),  res_x = IFFT2(R_x) cropped.
// Nz >= Z + max(hz, Mz-1-hz) (and Ny likewise) keeps the circular
// correlation equal to the zero-padded one on the output range.
//
// Per 128^3 volume with a 29 x 128 x 29 mask this is ~0.35 G FMAs of
// correlation plus the transforms, against ~2.7 G FMAs for the direct
// separable sum.  The arithmetic is FP32 (twiddles and filter spectra are
// rounded from FP64); the result agrees with the FP64 oracle to ~1e-6 of
// its largest value.
//
// Kernels, in launch order:
//   fft_filter_kernel : G (Mx x Nz x Nyh) and the twiddle tables, FP64 -> FP32
//   fft_fwd_kernel    : one CTA per (volume, plane): rows (two real rows per
//                       complex FFT), then columns; writes P
//   fft_corr_kernel   : one CTA per (volume, 16 frequencies): R_x for all x,
//                       written over P in place
//   fft_inv_kernel    : one CTA per (volume, plane x): columns, then rows
//                       (two real rows per complex FFT); writes res or
//                       exp(-res) in the reference layout
//   fft_apply_kernel  : beam layout modes: exp(-res) multiplied (or stored)
//                       into out[l][a][z][Y-1-y][x] through a tiled transpose
// Planes whose padded transform does not fit one CTA's shared memory twice
// (beyond about 150^2) replace fft_fwd_kernel by fft_fwd_rows_kernel +
// fft_cols_kernel and fft_inv_kernel by fft_cols_kernel + fft_inv_rows_kernel:
// the same transforms in two passes through the spectra buffer.
// All transforms are Stockham autosort passes (radix 4, 2, 3, 5) over the
// sequences held in shared memory, ping-ponging between two buffers.

#include <algorithm>

#include "flc_common.cuh"

namespace flc {
namespace {

constexpr int kFftThreads = 1024;
constexpr int kCorrK = 16;       // frequencies per correlation CTA, one per lane of each half-warp
constexpr int kCorrWarps = 8;
constexpr int kMaxStages = 16;
constexpr int kLoadBatch = 4;    // global loads per thread issued before their shared stores

struct Radices {
    int n;               // transform length
    int nst;             // passes
    int r[kMaxStages];   // radix of each pass
};

struct FftGeom {
    int Z, X, Y, Mz, Mx, My;
    int Nz, Ny, Nyh, NP;   // padded sizes; NP = Nz * Nyh spectrum points per plane
    Radices rz, ry;
    int split;             // 1: plane transforms in two passes through the spectra buffer
};

// Split transforms (planes too large for one CTA's shared memory): a row CTA
// transforms kRowPairs pairs of rows, a column CTA kColK columns.
constexpr int kRowPairs = 16;
constexpr int kColK = 16;
constexpr int kSplitThreads = 512;

// Paired FP32 arithmetic: sm_100 executes an FMA on both FP32 halves of a
// 64-bit register pair in one instruction (PTX fma.rn.f32x2), each half
// rounded as the scalar FMA would round it.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pk2(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void upk2(f32x2 r, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
// A complex value in shared memory as a register pair (one 8-byte load).
__device__ __forceinline__ f32x2 ld2(const float2* p) {
    return *reinterpret_cast<const f32x2*>(p);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// i * sg * z for sg = +-1
__device__ __forceinline__ float2 rot_i(float2 z, float sg) { return make_float2(-sg * z.y, sg * z.x); }

// y[k] = sum_r v[r] e^{sg 2 pi i r k / R}, in place.
template <int R>
__device__ __forceinline__ void dft_small(float2 (&v)[R], float sg) {
    if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = make_float2(a.x + b.x, a.y + b.y);
        v[1] = make_float2(a.x - b.x, a.y - b.y);
    } else if constexpr (R == 4) {
        const float2 s02 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
        const float2 d02 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
        const float2 s13 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
        const float2 w13 = rot_i(make_float2(v[1].x - v[3].x, v[1].y - v[3].y), sg);
        v[0] = make_float2(s02.x + s13.x, s02.y + s13.y);
        v[2] = make_float2(s02.x - s13.x, s02.y - s13.y);
        v[1] = make_float2(d02.x + w13.x, d02.y + w13.y);
        v[3] = make_float2(d02.x - w13.x, d02.y - w13.y);
    } else if constexpr (R == 3) {
        const float c3 = -0.5f, s3 = 0.866025403784438647f;  // cos, sin of 2 pi / 3
        const float2 a = make_float2(v[1].x + v[2].x, v[1].y + v[2].y);
        const float2 t = make_float2(fmaf(c3, a.x, v[0].x), fmaf(c3, a.y, v[0].y));
        const float2 u = rot_i(make_float2(s3 * (v[1].x - v[2].x), s3 * (v[1].y - v[2].y)), sg);
        v[0] = make_float2(v[0].x + a.x, v[0].y + a.y);
        v[1] = make_float2(t.x + u.x, t.y + u.y);
        v[2] = make_float2(t.x - u.x, t.y - u.y);
    } else if constexpr (R == 8) {
        // 8 = 2 x 4: pairs (n, n+4) by 2-point DFTs, the odd outputs turned by
        // e^{sg i pi n / 4}, then 4-point DFTs over n; output k1 + 2 k2
        constexpr float h = 0.7071067811865476f;   // sqrt(1/2)
        float2 e[4], o[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            e[n] = make_float2(v[n].x + v[n + 4].x, v[n].y + v[n + 4].y);
            o[n] = make_float2(v[n].x - v[n + 4].x, v[n].y - v[n + 4].y);
        }
        o[1] = make_float2(h * (o[1].x - sg * o[1].y), h * (o[1].y + sg * o[1].x));
        o[2] = rot_i(o[2], sg);
        o[3] = make_float2(h * (-o[3].x - sg * o[3].y), h * (-o[3].y + sg * o[3].x));
        dft_small<4>(e, sg);
        dft_small<4>(o, sg);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[2 * k] = e[k];
            v[2 * k + 1] = o[k];
        }
    } else if constexpr (R == 9) {
        // 9 = 3 x 3: 3-point DFTs over n1 of x[3 n1 + n2], turned by
        // e^{sg 2 pi i n2 k1 / 9}, then 3-point DFTs over n2; output k1 + 3 k2
        constexpr float c1 = 0.766044443118978f, s1 = 0.6427876096865393f;    // 2 pi / 9
        constexpr float c2 = 0.17364817766693041f, s2 = 0.984807753012208f;   // 4 pi / 9
        constexpr float c4 = -0.9396926207859083f, s4 = 0.3420201433256689f;  // 8 pi / 9
        float2 y[3][3];   // y[n2][k1]
#pragma unroll
        for (int n2 = 0; n2 < 3; ++n2) {
            float2 t[3] = {v[n2], v[n2 + 3], v[n2 + 6]};
            dft_small<3>(t, sg);
#pragma unroll
            for (int k1 = 0; k1 < 3; ++k1) y[n2][k1] = t[k1];
        }
        auto turn = [&](float2 z, float c, float sn) {
            const float ss = sg * sn;
            return make_float2(c * z.x - ss * z.y, c * z.y + ss * z.x);
        };
        y[1][1] = turn(y[1][1], c1, s1);
        y[1][2] = turn(y[1][2], c2, s2);
        y[2][1] = turn(y[2][1], c2, s2);
        y[2][2] = turn(y[2][2], c4, s4);
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) {
            float2 t[3] = {y[0][k1], y[1][k1], y[2][k1]};
            dft_small<3>(t, sg);
#pragma unroll
            for (int k2 = 0; k2 < 3; ++k2) v[k1 + 3 * k2] = t[k2];
        }
    } else {  // R == 5
        const float c1 = 0.309016994374947424f, c2 = -0.809016994374947424f;  // cos 2pi/5, 4pi/5
        const float s1 = 0.951056516295153572f, s2 = 0.587785252292473129f;   // sin 2pi/5, 4pi/5
        const float2 a1 = make_float2(v[1].x + v[4].x, v[1].y + v[4].y);
        const float2 b1 = make_float2(v[1].x - v[4].x, v[1].y - v[4].y);
        const float2 a2 = make_float2(v[2].x + v[3].x, v[2].y + v[3].y);
        const float2 b2 = make_float2(v[2].x - v[3].x, v[2].y - v[3].y);
        const float2 t1 = make_float2(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
        const float2 t2 = make_float2(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
        const float2 u1 = rot_i(make_float2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), sg);
        const float2 u2 = rot_i(make_float2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), sg);
        v[0] = make_float2(v[0].x + a1.x + a2.x, v[0].y + a1.y + a2.y);
        v[1] = make_float2(t1.x + u1.x, t1.y + u1.y);
        v[4] = make_float2(t1.x - u1.x, t1.y - u1.y);
        v[2] = make_float2(t2.x + u2.x, t2.y + u2.y);
        v[3] = make_float2(t2.x - u2.x, t2.y - u2.y);
    }
}

// One Stockham pass of radix R over a batch of `nseq` sequences of length N
// (element i of sequence s at s*ss + i*es): butterfly j reads elements
// j + r*N/R, multiplies by the twiddles e^{sg 2 pi i (j mod Ns) r / (Ns R)},
// takes the R-point DFT and writes elements (j div Ns)*Ns*R + (j mod Ns) + r*Ns.
// tw[m] = e^{-2 pi i m / N}; sg = +1 uses its conjugate.  seq_fast: adjacent
// threads take adjacent sequences (columns) rather than adjacent butterflies.
// floor(a / b) for 0 <= a < 2^22, b >= 1, from b's reciprocal: (a + 1/2) / b
// stays at least 1/(2b) from an integer, far more than the rounding error.
__device__ __forceinline__ int div_small(int a, float rb) {
    return (int)(((float)a + 0.5f) * rb);
}

template <int R>
__device__ void fft_pass(const float2* in, float2* out, int N, int Ns, int nseq, int ss, int es,
                         const float2* tw, float sg, bool seq_fast) {
    const int M = N / R;
    const int step = N / (Ns * R);
    const int total = nseq * M;
    const float r_nseq = 1.f / (float)nseq, r_M = 1.f / (float)M, r_Ns = 1.f / (float)Ns;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        int s, j;
        if (seq_fast) {
            j = div_small(idx, r_nseq);
            s = idx - j * nseq;
        } else {
            s = div_small(idx, r_M);
            j = idx - s * M;
        }
        const float2* src = in + s * ss;
        const int jm = j - div_small(j, r_Ns) * Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[(j + r * M) * es];
#pragma unroll
        for (int r = 1; r < R; ++r) {
            float2 t = tw[jm * r * step];
            t.y *= -sg;   // tw holds e^{-i..}: sg = -1 keeps it, +1 conjugates
            v[r] = cmul(v[r], t);
        }
        dft_small<R>(v, sg);
        float2* dst = out + s * ss;
        const int base = (j - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[(base + r * Ns) * es] = v[r];
    }
}

// Full transform of the batch; the input is in `a`, `b` is scratch of the
// same size.  Returns the buffer holding the result.
__device__ float2* fft_batch(float2* a, float2* b, const Radices& rad, int nseq, int ss, int es,
                             const float2* tw, float sg, bool seq_fast) {
    int Ns = 1;
    for (int st = 0; st < rad.nst; ++st) {
        const int R = rad.r[st];
        if (R == 4) fft_pass<4>(a, b, rad.n, Ns, nseq, ss, es, tw, sg, seq_fast);
        else if (R == 8) fft_pass<8>(a, b, rad.n, Ns, nseq, ss, es, tw, sg, seq_fast);
        else if (R == 9) fft_pass<9>(a, b, rad.n, Ns, nseq, ss, es, tw, sg, seq_fast);
        else if (R == 2) fft_pass<2>(a, b, rad.n, Ns, nseq, ss, es, tw, sg, seq_fast);
        else if (R == 3) fft_pass<3>(a, b, rad.n, Ns, nseq, ss, es, tw, sg, seq_fast);
        else fft_pass<5>(a, b, rad.n, Ns, nseq, ss, es, tw, sg, seq_fast);
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

// e^{sg 2 pi i m / n} in FP64, m reduced modulo n first.
__device__ __forceinline__ double2 unit_root(int64_t m, int n, double sg) {
    m %= n;
    if (m < 0) m += n;
    double s, c;
    sincospi(2.0 * (double)m / (double)n, &s, &c);
    return make_double2(c, sg * s);
}

// Block d < Mx: G[d][kz][ky] = Uf_d(kz) Vf_d(ky).  Block Mx: twiddle tables
// Tz[m] = e^{-2 pi i m / Nz}, Ty[m] = e^{-2 pi i m / Ny}.
__global__ void __launch_bounds__(256)
fft_filter_kernel(const float* __restrict__ U, const float* __restrict__ V, float2* __restrict__ G,
                  float2* __restrict__ Tz, float2* __restrict__ Ty, FftGeom g) {
    extern __shared__ double2 sd[];   // Uf[Nz] | Vf[Nyh]
    const int d = blockIdx.x;
    if (d == g.Mx) {
        for (int m = threadIdx.x; m < g.Nz; m += blockDim.x) {
            const double2 t = unit_root(m, g.Nz, -1.0);
            Tz[m] = make_float2((float)t.x, (float)t.y);
        }
        for (int m = threadIdx.x; m < g.Ny; m += blockDim.x) {
            const double2 t = unit_root(m, g.Ny, -1.0);
            Ty[m] = make_float2((float)t.x, (float)t.y);
        }
        return;
    }
    double2* Uf = sd;
    double2* Vf = sd + g.Nz;
    const int hz = g.Mz / 2, hy = g.My / 2;
    for (int k = threadIdx.x; k < g.Nz + g.Nyh; k += blockDim.x) {
        const bool zk = k < g.Nz;
        const int kk = zk ? k : k - g.Nz;
        const int n = zk ? g.Nz : g.Ny, M = zk ? g.Mz : g.My, h = zk ? hz : hy;
        const float* w = zk ? U + (int64_t)d * g.Mz : V + (int64_t)d * g.My;
        double re = 0.0, im = 0.0;
        for (int t = 0; t < M; ++t) {
            const double wt = (double)__ldg(w + t);
            if (wt == 0.0) continue;
            const double2 e = unit_root((int64_t)kk * (t - h), n, 1.0);
            re += wt * e.x;
            im += wt * e.y;
        }
        sd[k] = make_double2(re, im);
    }
    __syncthreads();
    float2* Gd = G + (int64_t)d * g.NP;
    for (int i = threadIdx.x; i < g.NP; i += blockDim.x) {
        const int kz = i / g.Nyh, ky = i - kz * g.Nyh;
        const double2 a = Uf[kz], b = Vf[ky];
        Gd[i] = make_float2((float)(a.x * b.x - a.y * b.y), (float)(a.x * b.y + a.y * b.x));
    }
}

// Forward transform of source plane p of volume v (grid (X, Vn)).
__global__ void __launch_bounds__(kFftThreads, 1)
fft_fwd_kernel(const float* __restrict__ mu, const float2* __restrict__ Tzg,
               const float2* __restrict__ Tyg, float2* __restrict__ S, FftGeom g) {
    extern __shared__ __align__(16) float2 sm[];
    float2* A = sm;
    float2* B = A + g.NP;
    float2* Tz = B + g.NP;
    float2* Ty = Tz + g.Nz;
    const int p = blockIdx.x, v = blockIdx.y;
    const int Z = g.Z, X = g.X, Y = g.Y, Ny = g.Ny, Nyh = g.Nyh;
    const float rNy = 1.f / (float)Ny, rNyh = 1.f / (float)Nyh;
    for (int m = threadIdx.x; m < g.Nz; m += blockDim.x) Tz[m] = Tzg[m];
    for (int m = threadIdx.x; m < Ny; m += blockDim.x) Ty[m] = Tyg[m];
    // rows 2q, 2q+1 as the real and imaginary parts of sequence q (in B)
    const int npairs = (Z + 1) / 2;
    const float* src = mu + (int64_t)v * Z * X * Y + (int64_t)p * Y;
    const int64_t zs = (int64_t)X * Y;
    // kLoadBatch elements per thread in flight before their shared stores
    const int nrow = npairs * Ny;
    for (int i0 = threadIdx.x; i0 < nrow; i0 += kLoadBatch * blockDim.x) {
        float2 t[kLoadBatch];
#pragma unroll
        for (int b = 0; b < kLoadBatch; ++b) {
            const int i = i0 + b * blockDim.x;
            const int q = div_small(i, rNy), y = i - q * Ny;
            const int za = 2 * q, zb = za + 1;
            const bool in = i < nrow && y < Y;
            t[b] = make_float2(in ? __ldg(src + za * zs + y) : 0.f,
                               (in && zb < Z) ? __ldg(src + zb * zs + y) : 0.f);
        }
#pragma unroll
        for (int b = 0; b < kLoadBatch; ++b) {
            const int i = i0 + b * blockDim.x;
            if (i < nrow) B[i] = t[b];
        }
    }
    __syncthreads();
    float2* R1 = fft_batch(B, A, g.ry, npairs, Ny, 1, Ty, -1.f, false);
    float2* O = R1 == A ? B : A;
    // unpack the two real rows' half spectra: Xa = (Zk + conj Zn)/2,
    // Xb = (Zk - conj Zn)/(2i), Zn = Z[(Ny - k) mod Ny]; rows >= Z are zero
    for (int i = threadIdx.x; i < g.NP; i += blockDim.x) {
        const int z = div_small(i, rNyh), k = i - z * Nyh;
        float2 o = make_float2(0.f, 0.f);
        if (z < Z) {
            const float2* Zq = R1 + (z >> 1) * Ny;
            const float2 zk = Zq[k], zn = Zq[k == 0 ? 0 : Ny - k];
            o = (z & 1) ? make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x))
                        : make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
        }
        O[i] = o;
    }
    __syncthreads();
    float2* R2 = fft_batch(O, R1, g.rz, Nyh, 1, Nyh, Tz, -1.f, true);
    float2* dst = S + ((int64_t)v * X + p) * g.NP;
    for (int i = threadIdx.x; i < g.NP; i += blockDim.x) dst[i] = R2[i];
}

// ---------------------------------------------------------------------------
// Split transforms.  The one-CTA-per-plane kernels above hold a padded plane
// twice in shared memory, which caps the plane near 150^2.  For larger planes
// the same 2-D transforms run in two passes through the spectra buffer S
// (layout [v][x][kz][ky], as the one-pass kernels write it): row CTAs
// transform kRowPairs pairs of rows along y and write the unpacked half
// spectra, column CTAs transform kColK columns along z in place; the inverse
// runs columns first, then rows.  The arithmetic per sequence is the one-pass
// kernels' (the same passes, twiddles and packing), so the results agree.
// ---------------------------------------------------------------------------

// Forward, rows: grid (X, Vn, ceil(npairs / kRowPairs)).  Rows 2q, 2q+1 of
// source plane p as one complex sequence, transformed and unpacked into rows
// z of S; the CTAs of the first row batch also zero the rows Z .. Nz-1.
__global__ void __launch_bounds__(kSplitThreads)
fft_fwd_rows_kernel(const float* __restrict__ mu, const float2* __restrict__ Tyg,
                    float2* __restrict__ S, FftGeom g) {
    extern __shared__ __align__(16) float2 sm[];
    const int Ny = g.Ny, Nyh = g.Nyh, Z = g.Z, X = g.X, Y = g.Y;
    float2* A = sm;
    float2* B = A + kRowPairs * Ny;
    float2* Ty = B + kRowPairs * Ny;
    const int p = blockIdx.x, v = blockIdx.y;
    const int npairs = (Z + 1) / 2;
    const int q0 = blockIdx.z * kRowPairs, nq = min(kRowPairs, npairs - q0);
    const float rNy = 1.f / (float)Ny, rNyh = 1.f / (float)Nyh;
    for (int m = threadIdx.x; m < Ny; m += blockDim.x) Ty[m] = Tyg[m];
    const float* src = mu + (int64_t)v * Z * X * Y + (int64_t)p * Y;
    const int64_t zs = (int64_t)X * Y;
    for (int i = threadIdx.x; i < nq * Ny; i += blockDim.x) {
        const int qq = div_small(i, rNy), y = i - qq * Ny;
        const int za = 2 * (q0 + qq), zb = za + 1;
        const bool in = y < Y;
        B[i] = make_float2(in ? __ldg(src + za * zs + y) : 0.f,
                           (in && zb < Z) ? __ldg(src + zb * zs + y) : 0.f);
    }
    __syncthreads();
    const float2* R1 = fft_batch(B, A, g.ry, nq, Ny, 1, Ty, -1.f, false);
    float2* dst = S + ((int64_t)v * X + p) * g.NP;
    const int z0 = 2 * q0, z1 = min(Z, 2 * (q0 + nq));
    for (int i = threadIdx.x; i < (z1 - z0) * Nyh; i += blockDim.x) {
        const int zz = div_small(i, rNyh), k = i - zz * Nyh;
        const int z = z0 + zz;
        const float2* Zq = R1 + ((z >> 1) - q0) * Ny;
        const float2 zk = Zq[k], zn = Zq[k == 0 ? 0 : Ny - k];
        dst[(int64_t)z * Nyh + k] = (z & 1) ? make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x))
                                            : make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
    }
    if (blockIdx.z == 0)
        for (int i = Z * Nyh + threadIdx.x; i < g.NP; i += blockDim.x) dst[i] = make_float2(0.f, 0.f);
}

// Columns along z, in place in S (grid (X, Vn, ceil(Nyh / kColK))); sg = -1
// forward, +1 inverse.
__global__ void __launch_bounds__(kSplitThreads)
fft_cols_kernel(float2* __restrict__ S, const float2* __restrict__ Tzg, float sg, FftGeom g) {
    extern __shared__ __align__(16) float2 sm[];
    const int Nz = g.Nz, Nyh = g.Nyh;
    const int sp = Nz + 1;                 // odd sequence pitch: the transposing
                                           // accesses spread over the banks
    float2* A = sm;
    float2* B = A + kColK * sp;
    float2* Tz = B + kColK * sp;
    const int p = blockIdx.x, v = blockIdx.y;
    const int k0 = blockIdx.z * kColK, nk = min(kColK, Nyh - k0);
    for (int m = threadIdx.x; m < Nz; m += blockDim.x) Tz[m] = Tzg[m];
    float2* pl = S + ((int64_t)v * g.X + p) * g.NP;
    // element (z, kk) of the batch at A[kk * sp + z]; loads run along ky
    for (int i = threadIdx.x; i < Nz * nk; i += blockDim.x) {
        const int z = i / nk, kk = i - z * nk;
        A[kk * sp + z] = pl[(int64_t)z * Nyh + k0 + kk];
    }
    __syncthreads();
    const float2* R = fft_batch(A, B, g.rz, nk, sp, 1, Tz, sg, false);
    for (int i = threadIdx.x; i < Nz * nk; i += blockDim.x) {
        const int z = i / nk, kk = i - z * nk;
        pl[(int64_t)z * Nyh + k0 + kk] = R[kk * sp + z];
    }
}

// Inverse, rows: grid (X, Vn, ceil(npairs / kRowPairs)).  Rows 2q, 2q+1 of
// plane x's (z, ky) half spectra as one Hermitian-extended complex sequence,
// transformed along y; writes res (mode 0) or exp(-res) (mode 1) in the
// reference layout.
__global__ void __launch_bounds__(kSplitThreads)
fft_inv_rows_kernel(const float2* __restrict__ S, const float2* __restrict__ Tyg,
                    float* __restrict__ out, int mode, FftGeom g) {
    extern __shared__ __align__(16) float2 sm[];
    const int Ny = g.Ny, Nyh = g.Nyh, Z = g.Z, X = g.X, Y = g.Y;
    float2* A = sm;
    float2* B = A + kRowPairs * Ny;
    float2* Ty = B + kRowPairs * Ny;
    const int x = blockIdx.x, v = blockIdx.y;
    const int npairs = (Z + 1) / 2;
    const int q0 = blockIdx.z * kRowPairs, nq = min(kRowPairs, npairs - q0);
    const float rNy = 1.f / (float)Ny;
    for (int m = threadIdx.x; m < Ny; m += blockDim.x) Ty[m] = Tyg[m];
    const float2* R1 = S + ((int64_t)v * X + x) * g.NP;
    const int half = Ny / 2;
    for (int i = threadIdx.x; i < nq * Ny; i += blockDim.x) {
        const int qq = div_small(i, rNy), k = i - qq * Ny;
        const int za = 2 * (q0 + qq), zb = za + 1;
        const bool up = k > half;
        const int kk = up ? Ny - k : k;
        float2 a = R1[(int64_t)za * Nyh + kk];
        float2 b = zb < Z ? R1[(int64_t)zb * Nyh + kk] : make_float2(0.f, 0.f);
        if (kk == 0 || kk == half) { a.y = 0.f; b.y = 0.f; }
        if (up) { a.y = -a.y; b.y = -b.y; }
        A[i] = make_float2(a.x - b.y, a.y + b.x);
    }
    __syncthreads();
    const float2* R2 = fft_batch(A, B, g.ry, nq, Ny, 1, Ty, 1.f, false);
    const float scale = 1.f / ((float)g.Nz * (float)Ny);
    float* ov = out + (int64_t)v * Z * X * Y + (int64_t)x * Y;
    const int z0 = 2 * q0, z1 = min(Z, 2 * (q0 + nq));
    for (int i = threadIdx.x; i < (z1 - z0) * Y; i += blockDim.x) {
        const int zz = div_small(i, 1.f / (float)Y), y = i - zz * Y;
        const int z = z0 + zz;
        const float2 c = R2[((z >> 1) - q0) * Ny + y];
        const float r = ((z & 1) ? c.y : c.x) * scale;
        ov[(int64_t)z * X * Y + y] = mode == 1 ? expf(-r) : r;
    }
}

// R_x(k) = sum_{d < min(Mx, X - x)} G_d(k) P_{x+d}(k), over P in place
// (grid (ceil(NP / 16), Vn), kCorrWarps warps).  The two half-warps take the
// same 16 frequencies (one per lane) and split each group's depth range, so
// a CTA needs half the shared memory of one frequency per lane and four CTAs
// fit an SM; a shuffle adds the two halves' sums at the end.  A warp owns
// groups of 8 consecutive x, paired first with last so that every warp sums
// about the same number of depths.  P rows past X and G rows past Mx are
// zero in shared memory, so the blocks of 8 depths need no edge tests.
__global__ void __launch_bounds__(kCorrWarps * 32, 3)
fft_corr_kernel(float2* __restrict__ S, const float2* __restrict__ G, FftGeom g) {
    extern __shared__ __align__(16) float2 sc[];
    const int X = g.X, Mx = g.Mx;
    const int prow = X + Mx + 16, grow = Mx + 8;
    float2* sP = sc;                           // [prow][16]
    float2* sG = sP + (size_t)prow * kCorrK;   // [grow][16]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int half = lane >> 4, l16 = lane & 15;
    const int k = blockIdx.x * kCorrK + l16;
    const bool kin = k < g.NP;
    float2* Sv = S + (int64_t)blockIdx.y * X * g.NP;
    // a warp loads two rows per step, one per half
    for (int r0 = 2 * warp; r0 < prow + grow; r0 += kLoadBatch * 2 * kCorrWarps) {
        float2 t[kLoadBatch];
#pragma unroll
        for (int b = 0; b < kLoadBatch; ++b) {
            const int r = r0 + b * 2 * kCorrWarps + half;
            const bool p = r < prow;
            const int rr = p ? r : r - prow;
            t[b] = (kin && (p ? rr < X : rr < Mx))
                       ? (p ? Sv[(int64_t)rr * g.NP + k] : __ldg(G + (int64_t)rr * g.NP + k))
                       : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int b = 0; b < kLoadBatch; ++b) {
            const int r = r0 + b * 2 * kCorrWarps + half;
            if (r < prow + grow) sc[r * kCorrK + l16] = t[b];   // sG follows sP
        }
    }
    __syncthreads();
    const int nxg = (X + 7) / 8;
    for (int gi = warp; gi < (nxg + 1) / 2; gi += kCorrWarps) {
        for (int side = 0; side < 2; ++side) {
            const int grp = side ? nxg - 1 - gi : gi;
            if (side && grp == gi) break;
            const int x0 = 8 * grp;
            const int dmax = min(Mx, X - x0);
            // half 0: depths [0, dsplit), half 1: [dsplit, dmax); dsplit is a
            // multiple of 8 near dmax / 2
            const int dsplit = ((dmax + 15) / 16) * 8;
            const int dlo = half ? dsplit : 0, dhi = half ? dmax : dsplit;
            // acc[t] = sum_e G[d0+e] * P[x0+t+d0+e] in two paired sums:
            // pr[t] = sum G.x * (P.x, P.y), qi[t] = sum G.y * (P.x, P.y), one
            // paired FMA each per depth (the complex product is
            // (pr.x - qi.y, pr.y + qi.x), formed once at the end)
            f32x2 pr[8], qi[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) pr[t] = qi[t] = pk2(0.f, 0.f);
            f32x2 lo[8], hi[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) lo[i] = ld2(sP + (x0 + dlo + i) * kCorrK + l16);
#define FLC_CMAC2(W)                                \
    pr[t] = fma2(gx, W, pr[t]);                     \
    qi[t] = fma2(gy, W, qi[t]);
            for (int d0 = dlo; d0 < dhi; d0 += 16) {
#pragma unroll
                for (int i = 0; i < 8; ++i) hi[i] = ld2(sP + (x0 + d0 + 8 + i) * kCorrK + l16);
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const float2 gv = sG[(d0 + e) * kCorrK + l16];
                    const f32x2 gx = pk2(gv.x, gv.x), gy = pk2(gv.y, gv.y);
#pragma unroll
                    for (int t = 0; t < 8; ++t) {
                        if (t + e < 8) { FLC_CMAC2(lo[t + e]) }
                        else { FLC_CMAC2(hi[t + e - 8]) }
                    }
                }
                if (d0 + 8 >= dhi) break;
#pragma unroll
                for (int i = 0; i < 8; ++i) lo[i] = ld2(sP + (x0 + d0 + 16 + i) * kCorrK + l16);
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const float2 gv = sG[(d0 + 8 + e) * kCorrK + l16];
                    const f32x2 gx = pk2(gv.x, gv.x), gy = pk2(gv.y, gv.y);
#pragma unroll
                    for (int t = 0; t < 8; ++t) {
                        if (t + e < 8) { FLC_CMAC2(hi[t + e]) }
                        else { FLC_CMAC2(lo[t + e - 8]) }
                    }
                }
            }
#undef FLC_CMAC2
            float2 acc[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                float px, py, qx, qy;
                upk2(pr[t], px, py);
                upk2(qi[t], qx, qy);
                acc[t] = make_float2(px - qy, py + qx);
            }
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                acc[t].x += __shfl_xor_sync(0xffffffffu, acc[t].x, 16);
                acc[t].y += __shfl_xor_sync(0xffffffffu, acc[t].y, 16);
            }
            if (kin && half == 0) {
#pragma unroll
                for (int t = 0; t < 8; ++t)
                    if (x0 + t < X) Sv[(int64_t)(x0 + t) * g.NP + k] = acc[t];
            }
        }
    }
}

// Inverse transform of R_x (grid (X, Vn)); writes res (mode 0), exp(-res)
// (mode 1) into out in the reference layout (v, z, x, y), or res into `res`
// for the beam-layout modes.
__global__ void __launch_bounds__(kFftThreads, 1)
fft_inv_kernel(const float2* __restrict__ S, const float2* __restrict__ Tzg,
               const float2* __restrict__ Tyg, float* __restrict__ out, int mode, FftGeom g) {
    extern __shared__ __align__(16) float2 sm[];
    float2* A = sm;
    float2* B = A + g.NP;
    float2* Tz = B + g.NP;
    float2* Ty = Tz + g.Nz;
    const int x = blockIdx.x, v = blockIdx.y;
    const int Z = g.Z, X = g.X, Y = g.Y, Ny = g.Ny, Nyh = g.Nyh;
    const float rNy = 1.f / (float)Ny;
    for (int m = threadIdx.x; m < g.Nz; m += blockDim.x) Tz[m] = Tzg[m];
    for (int m = threadIdx.x; m < Ny; m += blockDim.x) Ty[m] = Tyg[m];
    const float2* src = S + ((int64_t)v * X + x) * g.NP;
    for (int i0 = threadIdx.x; i0 < g.NP; i0 += kLoadBatch * blockDim.x) {
        float2 t[kLoadBatch];
#pragma unroll
        for (int b = 0; b < kLoadBatch; ++b) {
            const int i = i0 + b * blockDim.x;
            t[b] = i < g.NP ? __ldg(src + i) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int b = 0; b < kLoadBatch; ++b) {
            const int i = i0 + b * blockDim.x;
            if (i < g.NP) A[i] = t[b];
        }
    }
    __syncthreads();
    float2* R1 = fft_batch(A, B, g.rz, Nyh, 1, Nyh, Tz, 1.f, true);
    float2* O = R1 == A ? B : A;
    // rows 2q, 2q+1 of the (z, ky) half spectra as one full complex sequence
    // Xa + i Xb (Hermitian extension; the imaginary parts of the k = 0 and
    // k = Ny/2 bins of a real row are dropped)
    const int npairs = (Z + 1) / 2;
    const int half = Ny / 2;
    for (int i = threadIdx.x; i < npairs * Ny; i += blockDim.x) {
        const int q = div_small(i, rNy), k = i - q * Ny;
        const int za = 2 * q, zb = za + 1;
        const bool up = k > half;
        const int kk = up ? Ny - k : k;
        float2 a = R1[za * Nyh + kk];
        float2 b = zb < Z ? R1[zb * Nyh + kk] : make_float2(0.f, 0.f);
        if (kk == 0 || kk == half) { a.y = 0.f; b.y = 0.f; }
        if (up) { a.y = -a.y; b.y = -b.y; }
        O[i] = make_float2(a.x - b.y, a.y + b.x);
    }
    __syncthreads();
    float2* R2 = fft_batch(O, R1, g.ry, npairs, Ny, 1, Ty, 1.f, false);
    const float scale = 1.f / ((float)g.Nz * (float)Ny);
    float* ov = out + (int64_t)v * Z * X * Y + (int64_t)x * Y;
    for (int i = threadIdx.x; i < Z * Y; i += blockDim.x) {
        const int z = div_small(i, 1.f / (float)Y), y = i - z * Y;
        const float2 c = R2[(z >> 1) * Ny + y];
        const float r = ((z & 1) ? c.y : c.x) * scale;
        ov[(int64_t)z * X * Y + y] = mode == 1 ? expf(-r) : r;
    }
}

// Beam layout: out[l][a_base + al][z][Y-1-y][x] (*)= exp(-res[v][z][x][y]),
// v = al * L + l (mode 2 multiplies, 3 stores).  Grid (ceil(Y/32),
// ceil(X/32), Vn * Z), block (32, 8).
__global__ void fft_apply_kernel(const float* __restrict__ res, float* __restrict__ out, int mode,
                                 int L, int a_base, int64_t out_a_stride, int64_t out_l_stride,
                                 FftGeom g) {
    __shared__ float tile[32][33];
    const int Z = g.Z, X = g.X, Y = g.Y;
    const int vz = blockIdx.z;
    const int v = vz / Z, z = vz - v * Z;
    const int y0 = blockIdx.x * 32, x0 = blockIdx.y * 32;
    const float* rp = res + ((int64_t)v * Z + z) * X * Y;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int x = x0 + i, y = y0 + threadIdx.x;
        tile[i][threadIdx.x] = (x < X && y < Y) ? __ldg(rp + (int64_t)x * Y + y) : 0.f;
    }
    __syncthreads();
    const int al = v / L, l = v - al * L;
    float* ob = out + l * out_l_stride + (int64_t)(a_base + al) * out_a_stride;
    // the block's rows of the attenuation are loaded together before any is
    // stored (blockDim.y = 8: four rows per thread), so the read-modify-write
    // keeps four loads in flight
    constexpr int kRows = 4;
    const int x = x0 + threadIdx.x;
    float prev[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        const int y = y0 + threadIdx.y + r * 8;
        prev[r] = (mode == 2 && y < Y && x < X)
                      ? ob[((int64_t)z * Y + (Y - 1 - y)) * X + x] : 1.f;
    }
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
        const int i = threadIdx.y + r * 8, y = y0 + i;
        if (y >= Y || x >= X) continue;
        ob[((int64_t)z * Y + (Y - 1 - y)) * X + x] = prev[r] * expf(-tile[threadIdx.x][i]);
    }
}

// Smallest even n >= need whose only prime factors are 2, 3 and 5.
int smooth_even(int need) {
    for (int n = need + (need & 1);; n += 2) {
        int k = n;
        for (int r : {2, 3, 5})
            while (k % r == 0) k /= r;
        if (k == 1) return n;
    }
}

// The passes of a length-n transform: the factor 2^e in passes of 8 and 4
// (fewest passes, radix 4 where the count ties), 3^f in 9s and a 3, then 5s.
// Every pass is one read and one write of the sequences in shared memory
// with a barrier, so fewer, larger butterflies shorten the latency-bound
// transforms (144 = 4 x 4 x 9: three passes instead of four).
Radices radices(int n) {
    Radices r{};
    r.n = n;
    int k = n, e = 0, f = 0;
    while (k % 2 == 0) { k /= 2; ++e; }
    while (k % 3 == 0) { k /= 3; ++f; }
    while (e > 0 && r.nst < kMaxStages) {
        const int t = (e >= 3 && e != 4) ? 3 : (e >= 2 ? 2 : 1);
        r.r[r.nst++] = 1 << t;
        e -= t;
    }
    while (f >= 2 && r.nst < kMaxStages) { r.r[r.nst++] = 9; f -= 2; }
    if (f == 1 && r.nst < kMaxStages) r.r[r.nst++] = 3;
    while (k % 5 == 0 && r.nst < kMaxStages) { r.r[r.nst++] = 5; k /= 5; }
    return r;
}

size_t plane_smem(const FftGeom& g) {
    return sizeof(float2) * (2 * (size_t)g.NP + g.Nz + g.Ny);
}

size_t rows_smem(const FftGeom& g) {
    return sizeof(float2) * (2 * (size_t)kRowPairs * g.Ny + g.Ny);
}

size_t cols_smem(const FftGeom& g) {
    return sizeof(float2) * (2 * (size_t)kColK * (g.Nz + 1) + g.Nz);
}

size_t corr_smem(const FftGeom& g) {
    return sizeof(float2) * kCorrK * ((size_t)(g.X + g.Mx + 16) + (g.Mx + 8));
}

size_t al256(size_t n) { return (n + 255) & ~(size_t)255; }

bool fft_geom(int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My, FftGeom* g) {
    if (Z < 1 || X < 1 || Y < 1 || Mz < 1 || Mx < 1 || My < 1) return false;
    if (Z > 4096 || Y > 4096 || X > 65535 || Mx > 4096) return false;
    const int hz = (int)Mz / 2, hy = (int)My / 2;
    g->Z = (int)Z; g->X = (int)X; g->Y = (int)Y;
    g->Mz = (int)Mz; g->Mx = (int)Mx; g->My = (int)My;
    g->Nz = smooth_even((int)Z + std::max(1, std::max(hz, (int)Mz - 1 - hz)));
    g->Ny = smooth_even((int)Y + std::max(hy, (int)My - 1 - hy));
    g->Nyh = g->Ny / 2 + 1;
    g->NP = g->Nz * g->Nyh;
    g->rz = radices(g->Nz);
    g->ry = radices(g->Ny);
    const size_t cap = (size_t)max_smem_optin();
    if (corr_smem(*g) > cap) return false;
    g->split = plane_smem(*g) > cap || tune(kTuneConeVariant) == 5;
    return !g->split || (rows_smem(*g) <= cap && cols_smem(*g) <= cap);
}

struct FftWs {
    float2 *G, *Tz, *Ty, *S;
    float* res;
    size_t bytes;
};

FftWs fft_ws(const FftGeom& g, int64_t Vn, int mode, char* base) {
    FftWs w{};
    size_t off = 0;
    auto take = [&](size_t n) { char* p = base ? base + off : nullptr; off += al256(n); return p; };
    w.G = (float2*)take(sizeof(float2) * (size_t)g.Mx * g.NP);
    w.Tz = (float2*)take(sizeof(float2) * g.Nz);
    w.Ty = (float2*)take(sizeof(float2) * g.Ny);
    w.S = (float2*)take(sizeof(float2) * (size_t)Vn * g.X * g.NP);
    w.res = mode >= 2 ? (float*)take(sizeof(float) * (size_t)Vn * g.Z * g.X * g.Y) : nullptr;
    w.bytes = off;
    return w;
}

}  // namespace

// Scratch bytes of the spectral cone for Vn volumes, 0 if the shape does not
// fit it (the caller then uses the direct kernels).
size_t cone_fft_ws_bytes(int64_t Vn, int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx,
                         int64_t My, int mode) {
    FftGeom g;
    if (!fft_geom(Z, X, Y, Mz, Mx, My, &g)) return 0;
    return fft_ws(g, Vn, mode, nullptr).bytes;
}

// Spectral cone path sum; modes as cone_sep_launch (0 res, 1 exp(-res) in the
// reference layout; 2 multiply / 3 store exp(-res) in the beam layout).
// FLC_ERR_UNSUPPORTED (nothing launched) when the shape does not fit or the
// workspace is too small.
int cone_fft_launch(const float* mu, const float* U, const float* Vw, float* out, int64_t Vn,
                    int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My, int mode,
                    int L, int a_base, int64_t out_a_stride, int64_t out_l_stride,
                    void* workspace, size_t ws_bytes, cudaStream_t st) {
    FftGeom g;
    if (!workspace || Vn < 1 || Vn > 65535 || !fft_geom(Z, X, Y, Mz, Mx, My, &g))
        return FLC_ERR_UNSUPPORTED;
    if (mode >= 2 && Vn * Z > 65535) return FLC_ERR_UNSUPPORTED;   // apply grid's z extent
    if (((uintptr_t)workspace & 255) != 0) return FLC_ERR_UNSUPPORTED;
    FftWs w = fft_ws(g, Vn, mode, (char*)workspace);
    if (w.bytes > ws_bytes) return FLC_ERR_UNSUPPORTED;
    const size_t fsm = sizeof(double2) * (size_t)(g.Nz + g.Nyh);
    fft_filter_kernel<<<(unsigned)(g.Mx + 1), 256, fsm, st>>>(U, Vw, w.G, w.Tz, w.Ty, g);
    FLC_TRY(check_launch("fft_filter_kernel"));
    const size_t psm = plane_smem(g), rsm = rows_smem(g), csm_t = cols_smem(g);
    const unsigned nrb = (unsigned)ceil_div((g.Z + 1) / 2, kRowPairs);
    const unsigned ncb = (unsigned)ceil_div(g.Nyh, kColK);
    if (g.split) {
        FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)fft_fwd_rows_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsm));
        FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)fft_inv_rows_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsm));
        FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)fft_cols_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm_t));
        fft_fwd_rows_kernel<<<dim3((unsigned)g.X, (unsigned)Vn, nrb), kSplitThreads, rsm, st>>>(
            mu, w.Ty, w.S, g);
        FLC_TRY(check_launch("fft_fwd_rows_kernel"));
        fft_cols_kernel<<<dim3((unsigned)g.X, (unsigned)Vn, ncb), kSplitThreads, csm_t, st>>>(
            w.S, w.Tz, -1.f, g);
        FLC_TRY(check_launch("fft_cols_kernel"));
    } else {
        FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)fft_fwd_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
        FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)fft_inv_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
        fft_fwd_kernel<<<dim3((unsigned)g.X, (unsigned)Vn), kFftThreads, psm, st>>>(mu, w.Tz, w.Ty,
                                                                                   w.S, g);
        FLC_TRY(check_launch("fft_fwd_kernel"));
    }
    const size_t csm = corr_smem(g);
    FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)fft_corr_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm));
    fft_corr_kernel<<<dim3((unsigned)ceil_div(g.NP, kCorrK), (unsigned)Vn), kCorrWarps * 32, csm,
                      st>>>(w.S, w.G, g);
    FLC_TRY(check_launch("fft_corr_kernel"));
    if (g.split) {
        fft_cols_kernel<<<dim3((unsigned)g.X, (unsigned)Vn, ncb), kSplitThreads, csm_t, st>>>(
            w.S, w.Tz, 1.f, g);
        FLC_TRY(check_launch("fft_cols_kernel"));
        fft_inv_rows_kernel<<<dim3((unsigned)g.X, (unsigned)Vn, nrb), kSplitThreads, rsm, st>>>(
            w.S, w.Ty, mode >= 2 ? w.res : out, mode >= 2 ? 0 : mode, g);
        FLC_TRY(check_launch("fft_inv_rows_kernel"));
    } else {
        fft_inv_kernel<<<dim3((unsigned)g.X, (unsigned)Vn), kFftThreads, psm, st>>>(
            w.S, w.Tz, w.Ty, mode >= 2 ? w.res : out, mode >= 2 ? 0 : mode, g);
        FLC_TRY(check_launch("fft_inv_kernel"));
    }
    if (mode >= 2) {
        dim3 grid((unsigned)ceil_div(g.Y, 32), (unsigned)ceil_div(g.X, 32), (unsigned)(Vn * g.Z));
        fft_apply_kernel<<<grid, dim3(32, 8), 0, st>>>(w.res, out, mode, L, a_base, out_a_stride,
                                                       out_l_stride, g);
        FLC_TRY(check_launch("fft_apply_kernel"));
    }
    return FLC_OK;
}

}  // namespace flc
