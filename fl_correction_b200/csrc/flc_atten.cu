// Per-angle attenuation maps for sm_100a: rotation (grid_sample semantics),
// mu assembly, incident-beam exclusive product scan, and the fluorescence
// cone-mask path sum (general and separable forms).
//
// Reference path (per angle, FL/core.py:19-101):
//   frac_rot = torch_rotate_image_nd(frac, theta)           FL/torch_image_util.py:13-114
//   mu_x[j]  = frac_rot[j] * cs[comp_j-x] * rho_j * pix     FL/torch_functions.py:39-51
//   atten_x  = exclusive reverse cumprod of (1 - mu_x) on H FL/torch_functions.py:95-102
//   mu_f[i]  = sum_j frac_rot[j] * cs[comp_j-elem_i]*rho_j*pix   :71-80
//   res      = rot90^-1(atten_kernel(rot90(mu_f), mask))    :142-171, atten_cuda_kernel.cu:10-57
//   atten[i] = atten_x[i] * exp(-res[i])                    :174, FL/core.py:99
// Here one kernel rotates every channel, assembles both mu's, runs the scan
// along the beam in registers and writes the incident term straight into the
// output, plus mu_f in the layout the cone kernel streams (the reference's
// rot90 frame, where a detector-depth plane is a set of contiguous rows).  The
// cone kernel then multiplies exp(-res) into the same output.

#include <math.h>
#include <string.h>

#include <vector>

#include "flc_common.cuh"
#include "flc_geom.cuh"

namespace flc {
namespace {

// ---------------------------------------------------------------------------
// grid_sample rotation: out(h,w) samples the input at
//   ix = c*(w-cx) - s*(h-cy)*(W/H) + cx,  iy = s*(w-cx)*(H/W) + c*(h-cy) + cy
// (affine_grid with [[c,-s,0],[s,c,0]], align_corners=False, unnormalised),
// bilinear, zero padding outside the image.
// ---------------------------------------------------------------------------
// RotGeom / rot_sample live in flc_geom.cuh, shared with the adjoint kernels.

__global__ void rotate_kernel(const float* __restrict__ x, float* __restrict__ out, int64_t N,
                              int H, int W, RotGeom g, int scipy_mode) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    int h = blockIdx.y;
    if (w >= W) return;
    for (int64_t n = blockIdx.z; n < N; n += gridDim.z) {
        const float* img = x + n * H * W;
        out[(n * H + h) * W + w] = scipy_mode ? rot_sample_scipy(img, H, W, g, h, w)
                                              : rot_sample(img, H, W, g, h, w);
    }
}

__global__ void incident_scan_kernel(const float* __restrict__ mu, float* __restrict__ out,
                                     int64_t N, int H, int W) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * W) return;
    int64_t n = i / W;
    int w = (int)(i - n * W);
    const float* m = mu + n * H * W + w;
    float* o = out + n * H * W + w;
    float p = 1.f;
    for (int h = H - 1; h >= 0; --h) {
        o[(int64_t)h * W] = p;
        p *= 1.f - m[(int64_t)h * W];
    }
}

// ---------------------------------------------------------------------------
// Fused per-angle stage: grid (S, A_chunk), block W threads (one per detector
// column).  Walks the beam from h = H-1 to 0:
//   out[i][a][s][h][w] = incident term (exclusive product, mode-dependent)
//   mu_ref[a][i][s][x=w][y=H-1-h] = mu_f[i]
// A thread's mu_f values of consecutive beam steps are consecutive y of its
// own row x of mu_ref: it keeps kRun of them in registers and stores them as
// whole 32-byte sectors (two float4), so the stage needs no shared-memory
// transpose and no barriers, and the kRun beam steps of a group, unrolled,
// issue their rotation loads together.
// ---------------------------------------------------------------------------
constexpr int kMaxCh = 8;
constexpr int kMaxL = 8;
constexpr int kRun = 8;

struct StageCoef {
    float cx[kMaxCh];
    float cf[kMaxL][kMaxCh];
    float cref[kMaxCh];
};

// Reference-spectrum incident cross section (FL/torch_functions.py:22-37 with
// FL/cross_section_util.py:44-66): channels [n_ch, n_ch + n) of the rotated
// fractions are raw reference volumes; the incident coefficient of channel
// ch becomes, per voxel, sum_i coef[a][i] * max(ref_i / (sum_k ref_k +
// 1e-12), 0) -- the reference fractions of cal_frac (FL/core.py:159-205)
// with enable_scale off and no threshold mask -- times the spectrum value
// cs[comp-x_ref{i+1}] * rho * pix in coef (A, n).  ch < 0: not used.
struct RefSpec {
    const float* coef;
    int ch;
    int n;
};

// Channel-interleaved copy of the fractions: frac4[s][h][w][q] holds channels
// 4q .. 4q+3 of pixel (s, h, w) (zero past n_ch), so that one bilinear tap of
// every channel is G = ceil(n_ch / 4) 16-byte loads instead of n_ch scattered
// 4-byte ones.
__global__ void frac_interleave_kernel(const float* __restrict__ frac, float4* __restrict__ frac4,
                                       int n_ch, int64_t n_pix, int G) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pix) return;
    for (int q = 0; q < G; ++q) {
        float c[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int j = 4 * q + k;
            c[k] = j < n_ch ? __ldg(frac + (int64_t)j * n_pix + i) : 0.f;
        }
        frac4[i * G + q] = make_float4(c[0], c[1], c[2], c[3]);
    }
}

// rot_sample_tap (flc_geom.cuh) of the 4G channels of an interleaved slice at
// once: the same taps, weights and operations per channel.
template <int G>
__device__ __forceinline__ void rot_sample_all(const float4* __restrict__ img, int H, int W,
                                               const RotGeom& g, int h, int w, float (&fr)[kMaxCh],
                                               int scipy_from = kMaxCh) {
    const RotTap t = rot_tap(g, h, w);
    const int x0 = t.x0, y0 = t.y0;
    const bool xin0 = x0 >= 0 && x0 < W, xin1 = x0 + 1 >= 0 && x0 + 1 < W;
    const bool yin0 = y0 >= 0 && y0 < H, yin1 = y0 + 1 >= 0 && y0 + 1 < H;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < G; ++q) {
        const float4 v00 = (yin0 && xin0) ? __ldg(img + ((int64_t)y0 * W + x0) * G + q) : z4;
        const float4 v01 = (yin0 && xin1) ? __ldg(img + ((int64_t)y0 * W + x0 + 1) * G + q) : z4;
        const float4 v10 = (yin1 && xin0) ? __ldg(img + ((int64_t)(y0 + 1) * W + x0) * G + q) : z4;
        const float4 v11 = (yin1 && xin1) ? __ldg(img + ((int64_t)(y0 + 1) * W + x0 + 1) * G + q) : z4;
        const float a00[4] = {v00.x, v00.y, v00.z, v00.w}, a01[4] = {v01.x, v01.y, v01.z, v01.w};
        const float a10[4] = {v10.x, v10.y, v10.z, v10.w}, a11[4] = {v11.x, v11.y, v11.z, v11.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float top = fmaf(t.tx, a01[k] - a00[k], a00[k]);
            const float bot = fmaf(t.tx, a11[k] - a10[k], a10[k]);
            fr[4 * q + k] = fmaf(t.ty, bot - top, top);
        }
    }
#pragma unroll
    for (int j = 4 * G; j < kMaxCh; ++j) fr[j] = 0.f;
    // channels from scipy_from on take the reference's scipy rotation rule
    if (!t.inside) {
#pragma unroll
        for (int j = 0; j < kMaxCh; ++j)
            if (j >= scipy_from) fr[j] = 0.f;
    }
}

// LM: lines held in registers (>= L).  G > 0: the rotation reads the
// interleaved copy frac4 (G float4 per pixel); G == 0: the planar frac.
template <int LM, int G>
__global__ void atten_stage_kernel(const float* __restrict__ frac, const float4* __restrict__ frac4,
                                   const float* __restrict__ theta,
                                   const float* __restrict__ coef_x,
                                   const float* __restrict__ coef_f, float* __restrict__ out,
                                   float* __restrict__ mu_ref, int n_ch, int S, int H, int W,
                                   int L, int64_t out_a_stride, int64_t out_l_stride, int a_base,
                                   int incident_mode, int write_mu, int out_a0, RefSpec ref) {
    __shared__ StageCoef cf;
    const int s = blockIdx.x;
    const int al = blockIdx.y;
    const int a = a_base + al;
    const int w = threadIdx.x;
    for (int t = threadIdx.x; t < kMaxCh * (kMaxL + 2); t += blockDim.x) {
        int j = t % kMaxCh, i = t / kMaxCh;
        if (i == kMaxL + 1)
            cf.cref[j] = j < ref.n ? ref.coef[(int64_t)a * ref.n + j] : 0.f;
        else if (i == kMaxL)
            cf.cx[j] = j < n_ch ? coef_x[(int64_t)a * n_ch + j] : 0.f;
        else
            cf.cf[i][j] = (i < L && j < n_ch) ? coef_f[((int64_t)a * L + i) * n_ch + j] : 0.f;
    }
    __syncthreads();
    const int n_tot = n_ch + ref.n;       // channels sampled (compounds, then references)
    if (w >= W) return;
    // the reference rounds math.cos / math.sin of the angle to an FP32 matrix
    const double th = (double)theta[a];
    const RotGeom g = rot_geom((float)cos(th), (float)sin(th), H, W);
    float prod[LM];
#pragma unroll
    for (int i = 0; i < LM; ++i) prod[i] = 1.f;
    const int64_t HW = (int64_t)H * W;
    float* outw = out + (int64_t)(out_a0 + al) * out_a_stride + s * HW + w;
    // mu_ref row x = w of each line; whole-sector stores need H % 4 == 0
    float* murow = mu_ref + ((int64_t)al * L * S + s) * HW + (int64_t)w * H;
    const int64_t mu_l = (int64_t)S * HW;
    const bool vec = (H & 3) == 0;
    for (int y0 = 0; y0 < H; y0 += kRun) {
        const int n = min(kRun, H - y0);
        float mb[LM][kRun];
#pragma unroll
        for (int r = 0; r < kRun; ++r) {
            if (r >= n) break;
            const int h = H - 1 - (y0 + r);
            float fr[kMaxCh];
            // the reference volumes rotate as the reference's rot3D does
            // (FL/atten_util.py:79-88): scipy's boundary rule
            if constexpr (G > 0) {
                rot_sample_all<G>(frac4 + (int64_t)s * HW * G, H, W, g, h, w, fr, n_ch);
            } else {
#pragma unroll
                for (int j = 0; j < kMaxCh; ++j)
                    fr[j] = j < n_ch ? rot_sample(frac + ((int64_t)j * S + s) * HW, H, W, g, h, w)
                          : j < n_tot ? rot_sample_scipy(frac + ((int64_t)j * S + s) * HW, H, W, g, h, w)
                                      : 0.f;
            }
            // the reference-spectrum coefficient of channel ref.ch at this voxel
            // (the rotated reference volumes clipped below at 0, as rot3D
            // clips them)
            float cxr = 0.f;
            if (ref.ch >= 0) {
                float tot = 1e-12f;
#pragma unroll
                for (int j = 0; j < kMaxCh; ++j)
                    if (j >= n_ch && j < n_tot) tot += fmaxf(fr[j], 0.f);
#pragma unroll
                for (int j = 0; j < kMaxCh; ++j)
                    if (j >= n_ch && j < n_tot) cxr += cf.cref[j - n_ch] * (fmaxf(fr[j], 0.f) / tot);
            }
            // incident term: write the exclusive product, then fold in this voxel
            if (incident_mode != 2) {
#pragma unroll
                for (int i = 0; i < LM; ++i)
                    if (i < L) outw[i * out_l_stride + (int64_t)h * W] = prod[i];
                if (incident_mode == 0) {
#pragma unroll
                    for (int i = 0; i < LM; ++i)
                        if (i < L) prod[i] *= 1.f - fr[i] * (i == ref.ch ? cxr : cf.cx[i]);
                } else {
                    float f = 1.f;
#pragma unroll
                    for (int j = 0; j < kMaxCh; ++j)
                        if (j < n_ch) f *= 1.f - fr[j] * (j == ref.ch ? cxr : cf.cx[j]);
#pragma unroll
                    for (int i = 0; i < LM; ++i) prod[i] *= f;
                }
            } else {
#pragma unroll
                for (int i = 0; i < LM; ++i)
                    if (i < L) outw[i * out_l_stride + (int64_t)h * W] = 1.f;
            }
#pragma unroll
            for (int i = 0; i < LM; ++i) {
                float m = 0.f;
#pragma unroll
                for (int j = 0; j < kMaxCh; ++j)
                    if (j < n_ch) m += fr[j] * cf.cf[i][j];
                mb[i][r] = m;
            }
        }
        if (!write_mu) continue;
#pragma unroll
        for (int i = 0; i < LM; ++i) {
            if (i >= L) break;
            float* dst = murow + i * mu_l + y0;
            if (vec && n == kRun) {
                reinterpret_cast<float4*>(dst)[0] = make_float4(mb[i][0], mb[i][1], mb[i][2], mb[i][3]);
                reinterpret_cast<float4*>(dst)[1] = make_float4(mb[i][4], mb[i][5], mb[i][6], mb[i][7]);
            } else {
#pragma unroll
                for (int r = 0; r < kRun; ++r)
                    if (r < n) dst[r] = mb[i][r];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Cone path sum, general mask: thread per output, loop over the non-zero taps
// (dz, dx, dy, weight) listed by the host.  Reference layout (K,Z,X,Y).
// ---------------------------------------------------------------------------
struct ConeTap {
    int dz, dx, dy;
    float w;
};

__global__ void cone_general_kernel(const float* __restrict__ mu, const ConeTap* __restrict__ taps,
                                    int ntaps, float* __restrict__ out, int64_t KZ, int Z, int X, int Y) {
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    int x = blockIdx.y;
    if (y >= Y) return;
    for (int64_t kz = blockIdx.z; kz < KZ; kz += gridDim.z) {
        int z = (int)(kz % Z);
        const float* base = mu + (kz - z) * X * Y;
        float acc = 0.f;
        for (int t = 0; t < ntaps; ++t) {
            ConeTap tp = taps[t];
            int zz = z + tp.dz, xx = x + tp.dx, yy = y + tp.dy;
            if (zz < 0 || zz >= Z || xx >= X || yy < 0 || yy >= Y) continue;
            acc = fmaf(__ldg(base + ((int64_t)zz * X + xx) * Y + yy), tp.w, acc);
        }
        out[(kz * X + x) * Y + y] = acc;
    }
}

// ---------------------------------------------------------------------------
// Cone path sum, separable mask (mask[dz,dx,dy] = u[dx][dz] * v[dx][dy]).
// Reference layout (V, Z, X, Y): depth axis X (towards the detector), window
// axes Z (centred) and Y (centred).  For target depth x and source plane
// p = x + d:   res[z,x,y] += sum_dz u_d[dz] sum_dy v_d[dy] mu[z+dz-hz, p, y+dy-hy].
// CTA tile: every z, TY window columns y0.., XB consecutive targets x0...
// For each source plane p the CTA loads mu[:, p, y0-hy : y0+TY+hy) once and,
// for each of the XB targets it feeds (d = p - x), runs the y filter then the
// z filter, accumulating in registers.  Thread t owns window column
// (t % TY) and 8 consecutive z for all XB targets.
// ---------------------------------------------------------------------------
constexpr int kTY = 16;
constexpr int kXB = 8;
constexpr int kZB = 8;

struct SepDims {
    int Z, X, Y, Mz, Mx, My;
    int hz, hy;
    int PS;   // smem pitch of a plane row (window axis), floats
    int PZ;   // smem pitch of an X-filtered column (z axis, zero padded), floats
    int MzP, MyP;  // tap counts padded to a multiple of 4
};

__host__ __device__ inline int pad4(int n) { return (n + 3) & ~3; }
__host__ __device__ inline int pitch4mod32(int n) {
    while ((n & 31) != 4) ++n;
    return n;
}

// mode 0: out = res (reference layout); 1: out = exp(-res) (reference layout);
// 2: beam layout multiply: out_beam[l][a][z][h=Y-1-y][w=x] *= exp(-res),
//    volume v = a_local * L + l.
__global__ void __launch_bounds__(512)
cone_sep_kernel(const float* __restrict__ mu, const float* __restrict__ U,
                const float* __restrict__ Vw, float* __restrict__ out, SepDims d, int mode,
                int L, int a_base, int64_t out_a_stride, int64_t out_l_stride) {
    extern __shared__ __align__(16) float sm[];
    const int Z = d.Z, X = d.X, Y = d.Y;
    float* sS = sm;                                  // [Z][PS]
    float* sX = sS + Z * d.PS;                       // [kXB][kTY][PZ]
    float* sU = sX + kXB * kTY * d.PZ;               // [kXB][MzP]
    float* sV = sU + kXB * d.MzP;                    // [kXB][MyP]
    __shared__ int s_lo_y[kXB], s_hi_y[kXB], s_lo_z[kXB], s_hi_z[kXB], s_act[kXB];

    const int v = blockIdx.z;
    const int y0 = blockIdx.x * kTY;
    const int x0 = blockIdx.y * kXB;
    const float* mu_v = mu + (int64_t)v * Z * X * Y;
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;
    const int t = tid % kTY;          // window column owned in the z filter
    const int zb = tid / kTY;         // z block owned in the z filter
    const int zs = zb * kZB;

    float acc[kXB][kZB];
#pragma unroll
    for (int j = 0; j < kXB; ++j)
#pragma unroll
        for (int q = 0; q < kZB; ++q) acc[j][q] = 0.f;

    // zero the z padding of the X buffer once (rows outside [hz, hz+Z) stay 0)
    for (int i = tid; i < kXB * kTY * d.PZ; i += nthr) sX[i] = 0.f;

    const int p_end = min(X, x0 + kXB - 1 + d.Mx);
    for (int p = x0; p < p_end; ++p) {
        __syncthreads();
        // ---- load plane p window rows: sS[z][c] = mu[z][p][y0 - hy + c] ----
        const int W_in = kTY + d.MyP + 4;
        for (int i = tid; i < Z * W_in; i += nthr) {
            int z = i / W_in, c = i - z * W_in;
            int y = y0 - d.hy + c;
            float val = 0.f;
            if (y >= 0 && y < Y && c < kTY + d.My - 1) val = __ldg(mu_v + ((int64_t)z * X + p) * Y + y);
            sS[z * d.PS + c] = val;
        }
        // ---- filters of the targets this plane feeds ----
        if (tid < kXB) {
            int dd = p - (x0 + tid);
            int act = (dd >= 0 && dd < d.Mx && x0 + tid < X) ? 1 : 0;
            s_act[tid] = act;
            int lo_y = d.My, hi_y = 0, lo_z = d.Mz, hi_z = 0;
            for (int k = 0; k < d.MyP; ++k) {
                float wv = (act && k < d.My) ? Vw[dd * d.My + k] : 0.f;
                sV[tid * d.MyP + k] = wv;
                if (wv != 0.f) { lo_y = min(lo_y, k); hi_y = max(hi_y, k + 1); }
            }
            for (int k = 0; k < d.MzP; ++k) {
                float wu = (act && k < d.Mz) ? U[dd * d.Mz + k] : 0.f;
                sU[tid * d.MzP + k] = wu;
                if (wu != 0.f) { lo_z = min(lo_z, k); hi_z = max(hi_z, k + 1); }
            }
            if (hi_y <= lo_y || hi_z <= lo_z) s_act[tid] = 0;
            s_lo_y[tid] = lo_y & ~3;
            s_hi_y[tid] = hi_y;
            s_lo_z[tid] = lo_z & ~3;
            s_hi_z[tid] = hi_z;
        }
        __syncthreads();
        // ---- y filter: X[j][t][hz+z] = sum_k v_j[k] * S[z][t+k] ----
        for (int pair = tid; pair < kXB * Z; pair += nthr) {
            int j = pair / Z, z = pair - j * Z;
            if (!s_act[j]) continue;
            float xa[kTY];
#pragma unroll
            for (int q = 0; q < kTY; ++q) xa[q] = 0.f;
            const float* row = sS + z * d.PS;
            const float* vw = sV + j * d.MyP;
            for (int k0 = s_lo_y[j]; k0 < s_hi_y[j]; k0 += 4) {
                float4 wv = *reinterpret_cast<const float4*>(vw + k0);
                float win[kTY + 4];
#pragma unroll
                for (int q = 0; q < (kTY + 4) / 4; ++q) {
                    float4 f = *reinterpret_cast<const float4*>(row + k0 + 4 * q);
                    win[4 * q] = f.x; win[4 * q + 1] = f.y; win[4 * q + 2] = f.z; win[4 * q + 3] = f.w;
                }
#pragma unroll
                for (int q = 0; q < kTY; ++q) {
                    xa[q] = fmaf(wv.x, win[q], xa[q]);
                    xa[q] = fmaf(wv.y, win[q + 1], xa[q]);
                    xa[q] = fmaf(wv.z, win[q + 2], xa[q]);
                    xa[q] = fmaf(wv.w, win[q + 3], xa[q]);
                }
            }
            float* xo = sX + (j * kTY) * d.PZ + d.hz + z;
#pragma unroll
            for (int q = 0; q < kTY; ++q) xo[q * d.PZ] = xa[q];
        }
        __syncthreads();
        // ---- z filter: acc[j][q] += sum_k u_j[k] * X[j][t][zs+q+k] ----
        if (zs < Z) {
#pragma unroll
            for (int j = 0; j < kXB; ++j) {
                if (!s_act[j]) continue;
                const float* col = sX + (j * kTY + t) * d.PZ + zs;
                const float* uw = sU + j * d.MzP;
                for (int k0 = s_lo_z[j]; k0 < s_hi_z[j]; k0 += 4) {
                    float4 wu = *reinterpret_cast<const float4*>(uw + k0);
                    float win[kZB + 4];
#pragma unroll
                    for (int q = 0; q < (kZB + 4) / 4; ++q) {
                        float4 f = *reinterpret_cast<const float4*>(col + k0 + 4 * q);
                        win[4 * q] = f.x; win[4 * q + 1] = f.y; win[4 * q + 2] = f.z; win[4 * q + 3] = f.w;
                    }
#pragma unroll
                    for (int q = 0; q < kZB; ++q) {
                        acc[j][q] = fmaf(wu.x, win[q], acc[j][q]);
                        acc[j][q] = fmaf(wu.y, win[q + 1], acc[j][q]);
                        acc[j][q] = fmaf(wu.z, win[q + 2], acc[j][q]);
                        acc[j][q] = fmaf(wu.w, win[q + 3], acc[j][q]);
                    }
                }
            }
        }
    }
    // ---- epilogue ----
    const int y = y0 + t;
    if (zs >= Z || y >= Y) return;
    if (mode >= 2) {
        // beam layout: 2 multiplies exp(-res) in, 3 stores exp(-res)
        const int al = v / L, l = v - al * L;
        float* ob = out + l * out_l_stride + (int64_t)(a_base + al) * out_a_stride;
        const int h = Y - 1 - y;
#pragma unroll
        for (int q = 0; q < kZB; ++q) {
            int z = zs + q;
            if (z >= Z) break;
            float* o = ob + ((int64_t)z * Y + h) * X + x0;
#pragma unroll
            for (int j = 0; j < kXB; ++j) {
                if (x0 + j >= X) continue;
                const float e = expf(-acc[j][q]);
                if (mode == 2) o[j] *= e; else o[j] = e;
            }
        }
    } else {
        float* ov = out + (int64_t)v * Z * X * Y;
#pragma unroll
        for (int q = 0; q < kZB; ++q) {
            int z = zs + q;
            if (z >= Z) break;
#pragma unroll
            for (int j = 0; j < kXB; ++j) {
                if (x0 + j >= X) continue;
                float r = acc[j][q];
                ov[((int64_t)z * X + x0 + j) * Y + y] = mode == 1 ? expf(-r) : r;
            }
        }
    }
}

SepDims sep_dims(int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My) {
    SepDims d;
    d.Z = (int)Z; d.X = (int)X; d.Y = (int)Y;
    d.Mz = (int)Mz; d.Mx = (int)Mx; d.My = (int)My;
    d.hz = (int)Mz / 2; d.hy = (int)My / 2;
    d.MzP = pad4((int)Mz);
    d.MyP = pad4((int)My);
    d.PS = pitch4mod32(kTY + d.MyP + 4);
    d.PZ = pitch4mod32((int)Z + 2 * d.hz + d.MzP + 12);
    return d;
}

size_t sep_smem(const SepDims& d) {
    return sizeof(float) * ((size_t)d.Z * d.PS + (size_t)kXB * kTY * d.PZ + kXB * (d.MzP + d.MyP));
}

int sep_threads(int Z) { return kTY * ((Z + kZB - 1) / kZB); }
constexpr int kSepMaxThreads = 512;

}  // namespace

// TMA-pipelined separable kernel (flc_cone.cu); FLC_ERR_UNSUPPORTED when the
// shape does not fit it.
int cone_tma_launch(const float* mu, const float* U, const float* Vw, float* out, int64_t Vn,
                    int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My, int mode,
                    int L, int a_base, int64_t out_a_stride, int64_t out_l_stride, cudaStream_t st);

// Spectral form (flc_cone_fft.cu).
size_t cone_fft_ws_bytes(int64_t Vn, int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx,
                         int64_t My, int mode);
int cone_fft_launch(const float* mu, const float* U, const float* Vw, float* out, int64_t Vn,
                    int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My, int mode,
                    int L, int a_base, int64_t out_a_stride, int64_t out_l_stride,
                    void* workspace, size_t ws_bytes, cudaStream_t st);

// Separable cone path sum.  `mode` (0/1/2, see cone_sep_kernel) may carry
// kConePlain to select the plain kernel below even where the pipelined one fits.
int cone_sep_launch(const float* mu, const float* U, const float* Vw, float* out, int64_t Vn,
                    int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My, int mode,
                    int L, int a_base, int64_t out_a_stride, int64_t out_l_stride,
                    cudaStream_t st) {
    if (!(mode & kConePlain)) {
        int r = cone_tma_launch(mu, U, Vw, out, Vn, Z, X, Y, Mz, Mx, My, mode, L, a_base,
                                out_a_stride, out_l_stride, st);
        if (r != FLC_ERR_UNSUPPORTED) return r;
        clear_error();
    }
    mode &= ~kConePlain;
    SepDims d = sep_dims(Z, X, Y, Mz, Mx, My);
    size_t smem = sep_smem(d);
    int threads = sep_threads((int)Z);
    if (threads > kSepMaxThreads || smem > (size_t)max_smem_optin()) {
        set_error("separable cone: Z=%lld Mz=%lld My=%lld needs %d threads / %zu B shared memory",
                  (long long)Z, (long long)Mz, (long long)My, threads, smem);
        return FLC_ERR_UNSUPPORTED;
    }
    FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)cone_sep_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)ceil_div(Y, kTY), (unsigned)ceil_div(X, kXB), (unsigned)Vn);
    cone_sep_kernel<<<grid, threads, smem, st>>>(mu, U, Vw, out, d, mode, L, a_base, out_a_stride,
                                                 out_l_stride);
    return check_launch("cone_sep_kernel");
}

// Cone path sum with scratch for the spectral form: the spectral kernels run
// when the "cone.variant" knob allows them (0 automatic, 4 spectral, 5
// spectral with split plane transforms) and the shape and scratch fit;
// otherwise cone_sep_launch.
int cone_launch_ws(const float* mu, const float* U, const float* Vw, float* out, int64_t Vn,
                   int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My, int mode,
                   int L, int a_base, int64_t out_a_stride, int64_t out_l_stride, void* ws,
                   size_t ws_bytes, cudaStream_t st) {
    const int64_t var = tune(kTuneConeVariant);
    if (ws && (var == 0 || var == 4 || var == 5)) {
        int r = cone_fft_launch(mu, U, Vw, out, Vn, Z, X, Y, Mz, Mx, My, mode, L, a_base,
                                out_a_stride, out_l_stride, ws, ws_bytes, st);
        if (r != FLC_ERR_UNSUPPORTED) return r;
        clear_error();
    }
    return cone_sep_launch(mu, U, Vw, out, Vn, Z, X, Y, Mz, Mx, My, mode, L, a_base, out_a_stride,
                           out_l_stride, st);
}

namespace {

// Splits each depth plane of a host mask into u (Mz) x v (My) if it is rank
// one to FP32 precision.  Returns false otherwise.
bool factor_mask(const std::vector<float>& m, int64_t Mz, int64_t Mx, int64_t My,
                 std::vector<float>& U, std::vector<float>& V) {
    U.assign(Mx * Mz, 0.f);
    V.assign(Mx * My, 0.f);
    for (int64_t dx = 0; dx < Mx; ++dx) {
        double best = 0.0;
        int64_t bi = 0, bj = 0;
        for (int64_t i = 0; i < Mz; ++i)
            for (int64_t j = 0; j < My; ++j) {
                double a = fabs((double)m[(i * Mx + dx) * My + j]);
                if (a > best) { best = a; bi = i; bj = j; }
            }
        if (best == 0.0) continue;
        double piv = m[(bi * Mx + dx) * My + bj];
        for (int64_t i = 0; i < Mz; ++i) U[dx * Mz + i] = m[(i * Mx + dx) * My + bj];
        for (int64_t j = 0; j < My; ++j) V[dx * My + j] = (float)(m[(bi * Mx + dx) * My + j] / piv);
        for (int64_t i = 0; i < Mz; ++i)
            for (int64_t j = 0; j < My; ++j) {
                double e = fabs((double)U[dx * Mz + i] * V[dx * My + j] - m[(i * Mx + dx) * My + j]);
                if (e > 1e-6 * best) return false;
            }
    }
    return true;
}

}  // namespace

int rotate_launch(const float* x, float* out, int64_t N, int64_t H, int64_t W, float c, float s,
                  cudaStream_t st, int scipy_mode = 0) {
    RotGeom g = rot_geom(c, s, (int)H, (int)W);
    dim3 grid((unsigned)ceil_div(W, 128), (unsigned)H, (unsigned)(N < 65535 ? N : 65535));
    rotate_kernel<<<grid, 128, 0, st>>>(x, out, N, (int)H, (int)W, g, scipy_mode);
    return check_launch("rotate_kernel");
}

namespace {

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

int64_t pick_chunk(int64_t S, int64_t H, int64_t W, int64_t A, int64_t L, int64_t chunk) {
    if (chunk <= 0) chunk = tune(kTuneAttenChunk);
    if (chunk <= 0) {
        int64_t vol = L * S * H * W * (int64_t)sizeof(float);
        chunk = (256LL << 20) / (vol > 0 ? vol : 1);
        if (chunk < 1) chunk = 1;
    }
    if (chunk > A) chunk = A;
    if (chunk * L > 65535) chunk = 65535 / L;
    return chunk < 1 ? 1 : chunk;
}

}  // namespace

int frac_groups(int64_t n_ch) { return (int)((n_ch + 3) / 4); }

size_t frac4_bytes(int64_t n_ch, int64_t S, int64_t H, int64_t W) {
    return align256(sizeof(float4) * frac_groups(n_ch) * S * H * W);
}

// Workspace of the attenuation pipeline: the staged mu of one chunk, then the
// channel-interleaved fractions.
size_t atten_ws_bytes(int64_t n_ch, int64_t S, int64_t H, int64_t W, int64_t A, int64_t L,
                      int64_t chunk) {
    chunk = pick_chunk(S, H, W, A, L, chunk);
    return align256(sizeof(float) * chunk * L * S * H * W) + frac4_bytes(n_ch, S, H, W);
}

int frac_interleave_launch(const float* frac, float4* frac4, int64_t n_ch, int64_t S, int64_t H,
                           int64_t W, cudaStream_t st) {
    const int64_t n = S * H * W;
    frac_interleave_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(frac, frac4, (int)n_ch, n,
                                                                       frac_groups(n_ch));
    return check_launch("frac_interleave_kernel");
}

// frac4: the channel-interleaved copy (frac_interleave_launch) or nullptr
// for the planar frac.
int atten_stage_launch_ref(const float* frac, const float* theta, const float* coef_x,
                           const float* coef_f, float* out, float* mu_ref, int n_ch, int S, int H,
                           int W, int L, int64_t out_a_stride, int64_t out_l_stride, int a_base,
                           int n_a, int incident_mode, int write_mu, cudaStream_t st, int out_a0,
                           const float4* frac4, RefSpec ref) {
    const int threads = (W + 31) & ~31;
    using K = void (*)(const float*, const float4*, const float*, const float*, const float*,
                       float*, float*, int, int, int, int, int, int64_t, int64_t, int, int, int,
                       int, RefSpec);
    K kern;
    const int G = frac4 ? frac_groups(n_ch + ref.n) : 0;
    if (G == 1)
        kern = L <= 1 ? atten_stage_kernel<1, 1> : L <= 2 ? atten_stage_kernel<2, 1>
             : L <= 4 ? atten_stage_kernel<4, 1> : atten_stage_kernel<8, 1>;
    else if (G == 2)
        kern = L <= 1 ? atten_stage_kernel<1, 2> : L <= 2 ? atten_stage_kernel<2, 2>
             : L <= 4 ? atten_stage_kernel<4, 2> : atten_stage_kernel<8, 2>;
    else
        kern = L <= 1 ? atten_stage_kernel<1, 0> : L <= 2 ? atten_stage_kernel<2, 0>
             : L <= 4 ? atten_stage_kernel<4, 0> : atten_stage_kernel<8, 0>;
    kern<<<dim3((unsigned)S, (unsigned)n_a), threads, 0, st>>>(
        frac, frac4, theta, coef_x, coef_f, out, mu_ref, n_ch, S, H, W, L, out_a_stride,
        out_l_stride, a_base, incident_mode, write_mu, out_a0 < 0 ? a_base : out_a0, ref);
    return check_launch("atten_stage_kernel");
}

int atten_stage_launch(const float* frac, const float* theta, const float* coef_x,
                       const float* coef_f, float* out, float* mu_ref, int n_ch, int S, int H,
                       int W, int L, int64_t out_a_stride, int64_t out_l_stride, int a_base,
                       int n_a, int incident_mode, int write_mu, cudaStream_t st, int out_a0,
                       const float4* frac4) {
    return atten_stage_launch_ref(frac, theta, coef_x, coef_f, out, mu_ref, n_ch, S, H, W, L,
                                  out_a_stride, out_l_stride, a_base, n_a, incident_mode,
                                  write_mu, st, out_a0, frac4, RefSpec{nullptr, -1, 0});
}

int atten_maps_launch(const float* frac, const float* theta, const float* coef_x,
                      const float* coef_f, const float* u, const float* v, float* out,
                      int64_t n_ch, int64_t S, int64_t H, int64_t W, int64_t A, int64_t L,
                      int64_t Mz, int64_t Mx, int64_t My, int incident_mode, int xrf_mode,
                      int64_t chunk, void* workspace, size_t ws_bytes, cudaStream_t st,
                      RefSpec ref = RefSpec{nullptr, -1, 0}) {
    chunk = pick_chunk(S, H, W, A, L, chunk);
    float* mu_ref = (float*)workspace;
    // the interleaved fractions (compounds, then reference volumes) follow the
    // staged mu; the spectral cone's scratch is whatever the workspace holds
    // past both
    const int64_t n_tot = n_ch + ref.n;
    const size_t pipe_bytes = atten_ws_bytes(n_tot, S, H, W, A, L, chunk);
    float4* frac4 = (float4*)((char*)workspace + (pipe_bytes - frac4_bytes(n_tot, S, H, W)));
    void* fft_ws = ws_bytes > pipe_bytes ? (char*)workspace + pipe_bytes : nullptr;
    const size_t fft_bytes = ws_bytes > pipe_bytes ? ws_bytes - pipe_bytes : 0;
    FLC_TRY(frac_interleave_launch(frac, frac4, n_tot, S, H, W, st));
    const int64_t out_a = S * H * W, out_l = A * S * H * W;
    for (int64_t a0 = 0; a0 < A; a0 += chunk) {
        int n_a = (int)(A - a0 < chunk ? A - a0 : chunk);
        FLC_TRY(atten_stage_launch_ref(frac, theta, coef_x, coef_f, out, mu_ref, (int)n_ch,
                                       (int)S, (int)H, (int)W, (int)L, out_a, out_l, (int)a0, n_a,
                                       incident_mode, xrf_mode == 0, st, -1, frac4, ref));
        if (xrf_mode != 0) continue;
        // reference frame of the cone: (Z=S, X=W, Y=H)
        FLC_TRY(cone_launch_ws(mu_ref, u, v, out, (int64_t)n_a * L, S, W, H, Mz, Mx, My, 2,
                               (int)L, (int)a0, out_a, out_l, fft_ws, fft_bytes, st));
    }
    return FLC_OK;
}

}  // namespace flc

using namespace flc;

extern "C" int flc_rotate(const float* x, float* out, int64_t N, int64_t H, int64_t W,
                          float cos_t, float sin_t, void* stream) {
    clear_error();
    FLC_REQUIRE(x && out, "flc_rotate: null pointer argument");
    FLC_REQUIRE(N >= 1 && H >= 1 && W >= 1, "flc_rotate: sizes must be positive");
    return rotate_launch(x, out, N, H, W, cos_t, sin_t, as_stream(stream));
}

extern "C" int flc_rotate_ex(const float* x, float* out, int64_t N, int64_t H, int64_t W,
                             float cos_t, float sin_t, int mode, void* stream) {
    clear_error();
    FLC_REQUIRE(x && out, "flc_rotate_ex: null pointer argument");
    FLC_REQUIRE(N >= 1 && H >= 1 && W >= 1, "flc_rotate_ex: sizes must be positive");
    FLC_REQUIRE(mode == 0 || mode == 1, "flc_rotate_ex: mode must be 0 or 1");
    return rotate_launch(x, out, N, H, W, cos_t, sin_t, as_stream(stream), mode);
}

extern "C" int flc_incident_scan(const float* mu, float* out, int64_t N, int64_t H, int64_t W,
                                 void* stream) {
    clear_error();
    FLC_REQUIRE(mu && out, "flc_incident_scan: null pointer argument");
    FLC_REQUIRE(N >= 1 && H >= 1 && W >= 1, "flc_incident_scan: sizes must be positive");
    int64_t n = N * W;
    incident_scan_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, as_stream(stream)>>>(mu, out, N,
                                                                                   (int)H, (int)W);
    return check_launch("incident_scan_kernel");
}

extern "C" int flc_cone_atten_separable(const float* mu, const float* u, const float* v,
                                        float* out, int64_t K, int64_t Z, int64_t X, int64_t Y,
                                        int64_t Mz, int64_t Mx, int64_t My, int mode,
                                        void* stream) {
    clear_error();
    FLC_REQUIRE(mu && u && v && out, "flc_cone_atten_separable: null pointer argument");
    FLC_REQUIRE(K >= 1 && Z >= 1 && X >= 1 && Y >= 1 && Mz >= 1 && Mx >= 1 && My >= 1,
                "flc_cone_atten_separable: sizes must be positive");
    FLC_REQUIRE((mode & ~FLC_CONE_PLAIN_KERNEL) == 0 || (mode & ~FLC_CONE_PLAIN_KERNEL) == 1,
                "flc_cone_atten_separable: mode must be 0 or 1 (optionally | FLC_CONE_PLAIN_KERNEL)");
    if (mode & FLC_CONE_PLAIN_KERNEL) mode = (mode & ~FLC_CONE_PLAIN_KERNEL) | kConePlain;
    FLC_REQUIRE(K <= 65535, "flc_cone_atten_separable: K must be <= 65535");
    return cone_sep_launch(mu, u, v, out, K, Z, X, Y, Mz, Mx, My, mode, 1, 0, 0, 0,
                           as_stream(stream));
}

extern "C" size_t flc_cone_atten_workspace_bytes(int64_t K, int64_t Z, int64_t X, int64_t Y,
                                                 int64_t Mz, int64_t Mx, int64_t My) {
    if (K < 1 || Z < 1 || X < 1 || Y < 1 || Mz < 1 || Mx < 1 || My < 1) return 0;
    return cone_fft_ws_bytes(K, Z, X, Y, Mz, Mx, My, 0);
}

extern "C" int flc_cone_atten_separable_ws(const float* mu, const float* u, const float* v,
                                           float* out, int64_t K, int64_t Z, int64_t X,
                                           int64_t Y, int64_t Mz, int64_t Mx, int64_t My,
                                           int mode, void* workspace, size_t workspace_bytes,
                                           void* stream) {
    clear_error();
    FLC_REQUIRE(mu && u && v && out, "flc_cone_atten_separable_ws: null pointer argument");
    FLC_REQUIRE(K >= 1 && Z >= 1 && X >= 1 && Y >= 1 && Mz >= 1 && Mx >= 1 && My >= 1,
                "flc_cone_atten_separable_ws: sizes must be positive");
    FLC_REQUIRE(mode == 0 || mode == 1, "flc_cone_atten_separable_ws: mode must be 0 or 1");
    FLC_REQUIRE(K <= 65535, "flc_cone_atten_separable_ws: K must be <= 65535");
    if (workspace && ((uintptr_t)workspace & 255) != 0) {
        set_error("flc_cone_atten_separable_ws: workspace must be 256-byte aligned");
        return FLC_ERR_ALIGNMENT;
    }
    return cone_launch_ws(mu, u, v, out, K, Z, X, Y, Mz, Mx, My, mode, 1, 0, 0, 0, workspace,
                          workspace ? workspace_bytes : 0, as_stream(stream));
}

extern "C" int flc_cone_atten(const float* mu, const float* mask, float* out, int64_t K,
                              int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My,
                              int flags, void* stream) {
    clear_error();
    FLC_REQUIRE(mu && mask && out, "flc_cone_atten: null pointer argument");
    FLC_REQUIRE(K >= 1 && Z >= 1 && X >= 1 && Y >= 1 && Mz >= 1 && Mx >= 1 && My >= 1,
                "flc_cone_atten: sizes must be positive");
    FLC_REQUIRE(K * Z <= 2147483647LL && X <= 65535, "flc_cone_atten: volume too large");
    cudaStream_t st = as_stream(stream);
    std::vector<float> hm((size_t)(Mz * Mx * My));
    FLC_TRY_CUDA(cudaMemcpyAsync(hm.data(), mask, sizeof(float) * hm.size(), cudaMemcpyDeviceToHost, st));
    FLC_TRY_CUDA(cudaStreamSynchronize(st));
    std::vector<float> U, V;
    bool sep = !(flags & FLC_CONE_FORCE_GENERAL) && factor_mask(hm, Mz, Mx, My, U, V) &&
               K <= 65535 && sep_threads((int)Z) <= kSepMaxThreads &&
               sep_smem(sep_dims(Z, X, Y, Mz, Mx, My)) <= (size_t)max_smem_optin();
    if (sep) {
        // the factors, then (256-byte aligned) the spectral form's scratch
        // where the shape takes it
        float* dbuf = nullptr;
        const size_t fbytes = align256(sizeof(float) * (U.size() + V.size()));
        const size_t fft_bytes = cone_fft_ws_bytes(K, Z, X, Y, Mz, Mx, My, 0);
        const size_t bytes = fbytes + (fft_bytes ? fft_bytes + 256 : 0);
        FLC_TRY_CUDA(cudaMallocAsync((void**)&dbuf, bytes, st));
        int s = FLC_OK;
        cudaError_t e = cudaMemcpyAsync(dbuf, U.data(), sizeof(float) * U.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dbuf + U.size(), V.data(), sizeof(float) * V.size(), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) s = cuda_fail(e, "cudaMemcpyAsync");
        void* fft_ws = nullptr;
        if (fft_bytes) {
            const uintptr_t p = ((uintptr_t)dbuf + fbytes + 255) & ~(uintptr_t)255;
            fft_ws = (void*)p;
        }
        if (s == FLC_OK)
            s = cone_launch_ws(mu, dbuf, dbuf + U.size(), out, K, Z, X, Y, Mz, Mx, My, 0, 1, 0, 0,
                               0, fft_ws, fft_bytes, st);
        cudaFreeAsync(dbuf, st);
        // the host vectors are read by the copies above before they return
        cudaStreamSynchronize(st);
        return s;
    }
    std::vector<ConeTap> taps;
    for (int64_t dz = 0; dz < Mz; ++dz)
        for (int64_t dx = 0; dx < Mx; ++dx)
            for (int64_t dy = 0; dy < My; ++dy) {
                float w = hm[(dz * Mx + dx) * My + dy];
                if (w != 0.f) taps.push_back({(int)(dz - Mz / 2), (int)dx, (int)(dy - My / 2), w});
            }
    if (taps.empty()) {
        FLC_TRY_CUDA(cudaMemsetAsync(out, 0, sizeof(float) * K * Z * X * Y, st));
        return FLC_OK;
    }
    ConeTap* dt = nullptr;
    FLC_TRY_CUDA(cudaMallocAsync((void**)&dt, sizeof(ConeTap) * taps.size(), st));
    int s = FLC_OK;
    cudaError_t e = cudaMemcpyAsync(dt, taps.data(), sizeof(ConeTap) * taps.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) s = cuda_fail(e, "cudaMemcpyAsync");
    if (s == FLC_OK) {
        dim3 grid((unsigned)ceil_div(Y, 128), (unsigned)X, (unsigned)(K * Z < 65535 ? K * Z : 65535));
        cone_general_kernel<<<grid, 128, 0, st>>>(mu, dt, (int)taps.size(), out, K * Z, (int)Z,
                                                  (int)X, (int)Y);
        s = check_launch("cone_general_kernel");
    }
    cudaFreeAsync(dt, st);
    cudaStreamSynchronize(st);
    return s;
}

extern "C" size_t flc_atten_workspace_bytes(int64_t n_ch, int64_t S, int64_t H, int64_t W,
                                            int64_t A, int64_t L, int64_t chunk) {
    if (n_ch < 1 || S < 1 || H < 1 || W < 1 || A < 1 || L < 1) return 0;
    return atten_ws_bytes(n_ch, S, H, W, A, L, chunk);
}

extern "C" int flc_atten_maps(const float* frac, const float* theta, const float* coef_x,
                              const float* coef_f, const float* u, const float* v, float* out,
                              int64_t n_ch, int64_t S, int64_t H, int64_t W, int64_t A, int64_t L,
                              int64_t Mz, int64_t Mx, int64_t My, int incident_mode, int xrf_mode,
                              int64_t chunk, void* workspace, size_t workspace_bytes,
                              void* stream) {
    clear_error();
    FLC_REQUIRE(frac && theta && coef_x && coef_f && out && workspace,
                "flc_atten_maps: null pointer argument");
    FLC_REQUIRE(xrf_mode != 0 || (u && v), "flc_atten_maps: mask factors required");
    FLC_REQUIRE(n_ch >= 1 && n_ch <= kMaxCh, "flc_atten_maps: 1 <= n_ch <= %d", kMaxCh);
    FLC_REQUIRE(L >= 1 && L <= kMaxL, "flc_atten_maps: 1 <= L <= %d", kMaxL);
    FLC_REQUIRE(S >= 1 && S <= 65535 && A >= 1 && A <= 65535, "flc_atten_maps: S, A in [1, 65535]");
    FLC_REQUIRE(H == W && H >= 2 && W <= 1024,
                "flc_atten_maps: needs square slices H == W in [2, 1024] (the reference's rot90 "
                "does too)");
    FLC_REQUIRE(incident_mode >= 0 && incident_mode <= 2 && (xrf_mode == 0 || xrf_mode == 1),
                "flc_atten_maps: bad mode");
    FLC_REQUIRE(xrf_mode != 0 || (Mz >= 1 && Mx >= 1 && My >= 1), "flc_atten_maps: bad mask size");
    if (((uintptr_t)workspace & 255) != 0) {
        set_error("flc_atten_maps: workspace must be 256-byte aligned");
        return FLC_ERR_ALIGNMENT;
    }
    size_t need = atten_ws_bytes(n_ch, S, H, W, A, L, chunk);
    if (workspace_bytes < need) {
        set_error("flc_atten_maps: workspace of %zu bytes is smaller than the %zu required",
                  workspace_bytes, need);
        return FLC_ERR_WORKSPACE;
    }
    return atten_maps_launch(frac, theta, coef_x, coef_f, u, v, out, n_ch, S, H, W, A, L, Mz, Mx,
                             My, incident_mode, xrf_mode, chunk, workspace, workspace_bytes,
                             as_stream(stream));
}

extern "C" int flc_atten_maps_ref(const float* frac, const float* theta, const float* coef_x,
                                  const float* coef_f, const float* coef_ref, const float* u,
                                  const float* v, float* out, int64_t n_ch, int64_t n_ref,
                                  int64_t ref_ch, int64_t S, int64_t H, int64_t W, int64_t A,
                                  int64_t L, int64_t Mz, int64_t Mx, int64_t My,
                                  int incident_mode, int xrf_mode, int64_t chunk, void* workspace,
                                  size_t workspace_bytes, void* stream) {
    clear_error();
    FLC_REQUIRE(frac && theta && coef_x && coef_f && out && workspace,
                "flc_atten_maps_ref: null pointer argument");
    FLC_REQUIRE(xrf_mode != 0 || (u && v), "flc_atten_maps_ref: mask factors required");
    FLC_REQUIRE(n_ref >= 0 && n_ch >= 1 && n_ch + n_ref <= kMaxCh,
                "flc_atten_maps_ref: 1 <= n_ch and n_ch + n_ref <= %d", kMaxCh);
    FLC_REQUIRE(n_ref == 0 || (coef_ref && ref_ch >= 0 && ref_ch < n_ch),
                "flc_atten_maps_ref: with references, coef_ref is required and 0 <= ref_ch < n_ch");
    FLC_REQUIRE(L >= 1 && L <= kMaxL, "flc_atten_maps_ref: 1 <= L <= %d", kMaxL);
    FLC_REQUIRE(S >= 1 && S <= 65535 && A >= 1 && A <= 65535,
                "flc_atten_maps_ref: S, A in [1, 65535]");
    FLC_REQUIRE(H == W && H >= 2 && W <= 1024,
                "flc_atten_maps_ref: needs square slices H == W in [2, 1024]");
    FLC_REQUIRE(incident_mode >= 0 && incident_mode <= 2 && (xrf_mode == 0 || xrf_mode == 1),
                "flc_atten_maps_ref: bad mode");
    FLC_REQUIRE(xrf_mode != 0 || (Mz >= 1 && Mx >= 1 && My >= 1),
                "flc_atten_maps_ref: bad mask size");
    if (((uintptr_t)workspace & 255) != 0) {
        set_error("flc_atten_maps_ref: workspace must be 256-byte aligned");
        return FLC_ERR_ALIGNMENT;
    }
    size_t need = atten_ws_bytes(n_ch + n_ref, S, H, W, A, L, chunk);
    if (workspace_bytes < need) {
        set_error("flc_atten_maps_ref: workspace of %zu bytes is smaller than the %zu required",
                  workspace_bytes, need);
        return FLC_ERR_WORKSPACE;
    }
    RefSpec ref{n_ref > 0 ? coef_ref : nullptr, n_ref > 0 ? (int)ref_ch : -1, (int)n_ref};
    return atten_maps_launch(frac, theta, coef_x, coef_f, u, v, out, n_ch, S, H, W, A, L, Mz, Mx,
                             My, incident_mode, xrf_mode, chunk, workspace, workspace_bytes,
                             as_stream(stream), ref);
}

extern "C" int flc_atten_stage(const float* frac, const float* theta, const float* coef_x,
                               const float* coef_f, float* out, float* mu_ref, int64_t n_ch,
                               int64_t S, int64_t H, int64_t W, int64_t A, int64_t L,
                               int64_t a0, int64_t n_a, int incident_mode, int write_mu,
                               void* stream) {
    clear_error();
    FLC_REQUIRE(frac && theta && coef_x && coef_f && out && (mu_ref || !write_mu),
                "flc_atten_stage: null pointer argument");
    FLC_REQUIRE(n_ch >= 1 && n_ch <= kMaxCh && L >= 1 && L <= kMaxL,
                "flc_atten_stage: 1 <= n_ch <= %d, 1 <= L <= %d", kMaxCh, kMaxL);
    FLC_REQUIRE(H == W && H >= 2 && W <= 1024 && S >= 1 && S <= 65535,
                "flc_atten_stage: needs square slices, 2 <= H == W <= 1024");
    FLC_REQUIRE(a0 >= 0 && n_a >= 1 && a0 + n_a <= A && n_a <= 65535,
                "flc_atten_stage: angle range [a0, a0+n_a) outside [0, A)");
    FLC_REQUIRE(incident_mode >= 0 && incident_mode <= 2, "flc_atten_stage: bad incident_mode");
    return atten_stage_launch(frac, theta, coef_x, coef_f, out, mu_ref, (int)n_ch, (int)S, (int)H,
                              (int)W, (int)L, S * H * W, A * S * H * W, (int)a0, (int)n_a,
                              incident_mode, write_mu, as_stream(stream), -1, nullptr);
}

extern "C" size_t flc_atten_stage_workspace_bytes(int64_t n_ch, int64_t S, int64_t H,
                                                  int64_t W) {
    if (n_ch < 1 || n_ch > kMaxCh || S < 1 || H < 1 || W < 1) return 0;
    return frac4_bytes(n_ch, S, H, W);
}

extern "C" int flc_atten_stage_ws(const float* frac, const float* theta, const float* coef_x,
                                  const float* coef_f, float* out, float* mu_ref, int64_t n_ch,
                                  int64_t S, int64_t H, int64_t W, int64_t A, int64_t L,
                                  int64_t a0, int64_t n_a, int incident_mode, int write_mu,
                                  void* workspace, size_t workspace_bytes, void* stream) {
    clear_error();
    FLC_REQUIRE(frac && theta && coef_x && coef_f && out && (mu_ref || !write_mu) && workspace,
                "flc_atten_stage_ws: null pointer argument");
    FLC_REQUIRE(n_ch >= 1 && n_ch <= kMaxCh && L >= 1 && L <= kMaxL,
                "flc_atten_stage_ws: 1 <= n_ch <= %d, 1 <= L <= %d", kMaxCh, kMaxL);
    FLC_REQUIRE(H == W && H >= 2 && W <= 1024 && S >= 1 && S <= 65535,
                "flc_atten_stage_ws: needs square slices, 2 <= H == W <= 1024");
    FLC_REQUIRE(a0 >= 0 && n_a >= 1 && a0 + n_a <= A && n_a <= 65535,
                "flc_atten_stage_ws: angle range [a0, a0+n_a) outside [0, A)");
    FLC_REQUIRE(incident_mode >= 0 && incident_mode <= 2, "flc_atten_stage_ws: bad incident_mode");
    if (((uintptr_t)workspace & 255) != 0) {
        set_error("flc_atten_stage_ws: workspace must be 256-byte aligned");
        return FLC_ERR_ALIGNMENT;
    }
    const size_t need = frac4_bytes(n_ch, S, H, W);
    if (workspace_bytes < need) {
        set_error("flc_atten_stage_ws: workspace of %zu bytes is smaller than the %zu required",
                  workspace_bytes, need);
        return FLC_ERR_WORKSPACE;
    }
    cudaStream_t st = as_stream(stream);
    float4* frac4 = (float4*)workspace;
    FLC_TRY(frac_interleave_launch(frac, frac4, n_ch, S, H, W, st));
    return atten_stage_launch(frac, theta, coef_x, coef_f, out, mu_ref, (int)n_ch, (int)S, (int)H,
                              (int)W, (int)L, S * H * W, A * S * H * W, (int)a0, (int)n_a,
                              incident_mode, write_mu, st, -1, frac4);
}

extern "C" int flc_cone_atten_apply(const float* mu_ref, const float* u, const float* v,
                                    float* atten, int64_t n_a, int64_t L, int64_t S, int64_t H,
                                    int64_t W, int64_t A, int64_t a0, int64_t Mz, int64_t Mx,
                                    int64_t My, void* stream) {
    clear_error();
    FLC_REQUIRE(mu_ref && u && v && atten, "flc_cone_atten_apply: null pointer argument");
    FLC_REQUIRE(H == W && H >= 2 && S >= 1 && L >= 1 && n_a >= 1 && a0 >= 0 && a0 + n_a <= A,
                "flc_cone_atten_apply: bad sizes");
    FLC_REQUIRE(n_a * L <= 65535 && Mz >= 1 && Mx >= 1 && My >= 1,
                "flc_cone_atten_apply: bad sizes");
    return cone_sep_launch(mu_ref, u, v, atten, n_a * L, S, W, H, Mz, Mx, My, 2, (int)L, (int)a0,
                           S * H * W, A * S * H * W, as_stream(stream));
}

extern "C" size_t flc_cone_fft_workspace_bytes(int64_t n_vol, int64_t S, int64_t H, int64_t W,
                                               int64_t Mz, int64_t Mx, int64_t My) {
    if (n_vol < 1 || S < 1 || H < 1 || W < 1 || Mz < 1 || Mx < 1 || My < 1) return 0;
    // cone frame (Z = S, X = W, Y = H), beam-layout output
    return cone_fft_ws_bytes(n_vol, S, W, H, Mz, Mx, My, 2);
}

extern "C" int flc_cone_atten_apply_ws(const float* mu_ref, const float* u, const float* v,
                                       float* atten, int64_t n_a, int64_t L, int64_t S, int64_t H,
                                       int64_t W, int64_t A, int64_t a0, int64_t Mz, int64_t Mx,
                                       int64_t My, void* workspace, size_t workspace_bytes,
                                       void* stream) {
    clear_error();
    FLC_REQUIRE(mu_ref && u && v && atten, "flc_cone_atten_apply_ws: null pointer argument");
    FLC_REQUIRE(H == W && H >= 2 && S >= 1 && L >= 1 && n_a >= 1 && a0 >= 0 && a0 + n_a <= A,
                "flc_cone_atten_apply_ws: bad sizes");
    FLC_REQUIRE(n_a * L <= 65535 && Mz >= 1 && Mx >= 1 && My >= 1,
                "flc_cone_atten_apply_ws: bad sizes");
    if (workspace && ((uintptr_t)workspace & 255) != 0) {
        set_error("flc_cone_atten_apply_ws: workspace must be 256-byte aligned");
        return FLC_ERR_ALIGNMENT;
    }
    return cone_launch_ws(mu_ref, u, v, atten, n_a * L, S, W, H, Mz, Mx, My, 2, (int)L, (int)a0,
                          S * H * W, A * S * H * W, workspace, workspace_bytes,
                          as_stream(stream));
}

extern "C" int flc_device_status(int reset) {
    clear_error();
    return cone_device_status(reset);
}
