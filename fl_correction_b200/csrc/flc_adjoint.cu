// Self-absorption-corrected XRF projection with the attenuation recomputed
// per angle chunk, and its hand-written adjoint (sm_100a).
//
// Forward model, per element l and angle a (the composition of
// FL/core.py:19-101, FL/torch_functions.py:8-176 and the projector of
// FL/cuda_lib/atten_cuda_kernel.cu:298-337):
//   fr_j   = rotate(frac_j, theta_a)                      (grid_sample, zero pad)
//   inc_l  = prod_{h'>h} (1 - cx_l fr_l)                  (own compound; or all)
//   E_l    = exp(-cone(sum_j cf_lj fr_j))
//   Pf_l,a = sum_h inc_l E_l em_l,a bilerp(C_l, theta_a)  with C_l = frac_l
// The reference holds the attenuation fixed and differentiates the projector
// in C only (FL/cuda_lib/autograd.py:5-77).  The adjoint here also carries
// the gradient through the attenuation, i.e. through mu, back to C:
//   G        = dL/dPf * em * bilerp(C)                     (d Pf / d atten)
//   dres     = -G * atten,  dinc = G * E
//   dmu_f    = cone^T(dres)          (the cone with flipped taps, depth reversed)
//   dmu_x    = reverse-mode of the exclusive product scan
//   dfr_j    = cx_j dmu_x_j + sum_l cf_lj dmu_f_l
//   dC_l    += rotate^T(dfr_l) + P_a^T[atten](dL/dPf)     (direct term)
// Nothing of size A x volume is stored: each chunk of angles is recomputed in
// the backward pass (so 256^3 x 180-angle problems fit in HBM).

#include <cooperative_groups.h>

#include <algorithm>

#include "flc_common.cuh"
#include "flc_geom.cuh"

namespace flc {
namespace cg = cooperative_groups;

int atten_stage_launch(const float* frac, const float* theta, const float* coef_x,
                       const float* coef_f, float* out, float* mu_ref, int n_ch, int S, int H,
                       int W, int L, int64_t out_a_stride, int64_t out_l_stride, int a_base,
                       int n_a, int incident_mode, int write_mu, cudaStream_t st, int out_a0,
                       const float4* frac4);
int cone_launch_ws(const float* mu, const float* U, const float* Vw, float* out, int64_t Vn,
                   int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My, int mode,
                   int L, int a_base, int64_t out_a_stride, int64_t out_l_stride, void* ws,
                   size_t ws_bytes, cudaStream_t st);
size_t cone_fft_ws_bytes(int64_t Vn, int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx,
                         int64_t My, int mode);
size_t frac4_bytes(int64_t n_ch, int64_t S, int64_t H, int64_t W);
int frac_interleave_launch(const float* frac, float4* frac4, int64_t n_ch, int64_t S, int64_t H,
                           int64_t W, cudaStream_t st);
int fwd_emission_launch(const float* atten, const float* C, const float* em, const float* theta,
                        float* Pf, const float* I, int64_t A, int64_t B, int64_t R, int64_t H,
                        int64_t W, cudaStream_t st);
int bwd_emission_launch(const float* atten, const float* ratio, const float* em,
                        const float* theta, float* out, int64_t A, int64_t B, int64_t R,
                        int64_t H, int64_t W, float clamp_min, cudaStream_t st);

namespace {

constexpr int kMaxCh = 8;
constexpr int kMaxL = 8;

__global__ void mul_kernel(const float* __restrict__ a, const float* __restrict__ b,
                           float* __restrict__ o, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = a[i] * b[i];
}

__global__ void add_kernel(float* __restrict__ y, const float* __restrict__ x, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
}

// G = dL/dPf * em * bilerp(C) per sample; writes dinc = G*E (beam layout) and
// dres = -G*atten in the depth-reversed reference layout that the cone
// adjoint streams: dres_rev[al*L + l][s][W-1-w][H-1-h].
// grid (ceil(W/32)*ceil(H/32), S, n_a*L), block (32, 8).
__global__ void xrf_g_kernel(const float* __restrict__ C, const float* __restrict__ theta,
                             const float* __restrict__ em, const float* __restrict__ gPf,
                             const float* __restrict__ ATT, const float* __restrict__ E,
                             float* __restrict__ dinc, float* __restrict__ dres_rev, int L, int A,
                             int a0, int n_a, int S, int H, int W) {
    __shared__ float T[32][33];
    const int nbw = (W + 31) >> 5;
    const int w0 = (blockIdx.x % nbw) * 32, h0 = (blockIdx.x / nbw) * 32;
    const int s = blockIdx.y;
    const int l = blockIdx.z % L;
    const int al = blockIdx.z / L;
    const int a = a0 + al;
    const Geo g = make_geo(theta[a], H, W);
    const float* Cl = C + ((int64_t)l * S + s) * H * W;
    const float gem = em[(int64_t)l * A + a];
    const float* gp = gPf + (((int64_t)l * A + a) * S + s) * W;
    const int64_t base = (((int64_t)l * n_a + al) * S + s) * H * W;
    for (int k = 0; k < 32; k += 8) {
        const int hl = threadIdx.y + k, h = h0 + hl, w = w0 + threadIdx.x;
        float dr = 0.f;
        if (h < H && w < W) {
            const Smp sm = sample(g, h, w);
            const float Gv = gp[w] * gem * bilerp(Cl, W, sm);
            const int64_t o = base + (int64_t)h * W + w;
            dinc[o] = Gv * E[o];
            dr = -Gv * ATT[o];
        }
        T[hl][threadIdx.x] = dr;
    }
    __syncthreads();
    const int64_t vbase = (((int64_t)al * L + l) * S + s) * W;
    for (int k = 0; k < 32; k += 8) {
        const int wl = threadIdx.y + k, hl = threadIdx.x;
        const int w = w0 + wl, h = h0 + hl;
        if (h < H && w < W) dres_rev[(vbase + (W - 1 - w)) * H + (H - 1 - h)] = T[hl][wl];
    }
}

// Reverse mode of the per-angle stage (rotation, mu assembly, incident scan),
// one thread per detector column walking the beam from h = 0 upward:
//   gbar[h] = dinc[h] + gbar[h-1] * f[h],  df[h] = gbar[h-1] * inc[h]
// (the adjoint of inc[h-1] = f[h] * inc[h]), then
//   dfr_j = cx_j * dmu_x_j + sum_l cf_lj * dmu_f_l
// stored per sample, D[j][al][s][h][w] (channels j < L), for
// rot_adjoint_splat_kernel to spread back onto the unrotated grid.
// grid (S, n_a), block = W rounded to 32.
__global__ void xrf_stage_adjoint_kernel(const float* __restrict__ frac,
                                         const float* __restrict__ theta,
                                         const float* __restrict__ coef_x,
                                         const float* __restrict__ coef_f,
                                         const float* __restrict__ INC,
                                         const float* __restrict__ dinc,
                                         const float* __restrict__ dmu_rev, float* __restrict__ D,
                                         int n_ch, int S, int H, int W, int L, int a0, int n_a,
                                         int incident_mode) {
    __shared__ float cx[kMaxCh];
    __shared__ float cf[kMaxL][kMaxCh];
    const int s = blockIdx.x, al = blockIdx.y, a = a0 + al, w = threadIdx.x;
    for (int t = threadIdx.x; t < kMaxCh * (kMaxL + 1); t += blockDim.x) {
        int j = t % kMaxCh, i = t / kMaxCh;
        if (i == kMaxL)
            cx[j] = j < n_ch ? coef_x[(int64_t)a * n_ch + j] : 0.f;
        else
            cf[i][j] = (i < L && j < n_ch) ? coef_f[((int64_t)a * L + i) * n_ch + j] : 0.f;
    }
    __syncthreads();
    if (w >= W) return;
    const double th = (double)theta[a];
    const RotGeom g = rot_geom((float)cos(th), (float)sin(th), H, W);
    const int64_t HW = (int64_t)H * W;
    float gbar[kMaxL];
#pragma unroll
    for (int l = 0; l < kMaxL; ++l) gbar[l] = 0.f;
    for (int h = 0; h < H; ++h) {
        const RotTap tp = rot_tap(g, h, w);
        float fr[kMaxCh];
#pragma unroll
        for (int j = 0; j < kMaxCh; ++j)
            fr[j] = j < n_ch ? rot_sample_tap(frac + ((int64_t)j * S + s) * HW, H, W, tp) : 0.f;
        float dmux[kMaxCh];
#pragma unroll
        for (int j = 0; j < kMaxCh; ++j) dmux[j] = 0.f;
        if (incident_mode == 0) {
#pragma unroll
            for (int l = 0; l < kMaxL; ++l) {
                if (l >= L) break;
                const int64_t o = (((int64_t)l * n_a + al) * S + s) * HW + (int64_t)h * W + w;
                const float f = 1.f - fr[l] * cx[l];
                const float df = h > 0 ? gbar[l] * INC[o] : 0.f;
                gbar[l] = h > 0 ? fmaf(gbar[l], f, dinc[o]) : dinc[o];
                dmux[l] = -df;
            }
        } else if (incident_mode == 1) {
            // one recursion on the summed adjoint: every element sees the same f
            float ftot = 1.f, dsum = 0.f;
#pragma unroll
            for (int j = 0; j < kMaxCh; ++j)
                if (j < n_ch) ftot *= 1.f - fr[j] * cx[j];
            for (int l = 0; l < L; ++l)
                dsum += dinc[(((int64_t)l * n_a + al) * S + s) * HW + (int64_t)h * W + w];
            const float inc = INC[(((int64_t)0 * n_a + al) * S + s) * HW + (int64_t)h * W + w];
            const float df = h > 0 ? gbar[0] * inc : 0.f;
            gbar[0] = h > 0 ? fmaf(gbar[0], ftot, dsum) : dsum;
#pragma unroll
            for (int j = 0; j < kMaxCh; ++j) {
                if (j >= n_ch) break;
                float others = 1.f;
#pragma unroll
                for (int k = 0; k < kMaxCh; ++k)
                    if (k < n_ch && k != j) others *= 1.f - fr[k] * cx[k];
                dmux[j] = -df * others;
            }
        }
        // fluorescence mu gradient of every line at this sample
        float dmuf[kMaxL];
#pragma unroll
        for (int l = 0; l < kMaxL; ++l) {
            dmuf[l] = 0.f;
            if (l < L)
                dmuf[l] = __ldg(dmu_rev + ((((int64_t)al * L + l) * S + s) * W + (W - 1 - w)) * H +
                                (H - 1 - h));
        }
        // only the concentration channels (j < L) carry a gradient
#pragma unroll
        for (int j = 0; j < kMaxL; ++j) {
            if (j >= L) break;
            float d = cx[j] * dmux[j];
#pragma unroll
            for (int l = 0; l < kMaxL; ++l)
                if (l < L) d = fmaf(cf[l][j], dmuf[l], d);
            D[(((int64_t)j * n_a + al) * S + s) * HW + (int64_t)h * W + w] = d;
        }
    }
}

// The same reverse stage for the own-compound incident scan (incident_mode
// 0), where line l's scan uses only its own compound channel l, so the lines'
// reverse scans are independent: one thread per (detector column w, line j)
// walks the beam for line j, samples only channel j's rotated fraction and
// writes D[j] -- the same operations in the same order as the kernel above.
// The cone adjoint's output, stored reversed and transposed
// ([al][l][s][W-1-w][H-1-h]), is staged through shared memory kAdjRows rows
// at a time, so that its loads are whole sectors.  grid (L, S, n_a): the L
// lines of one (slice, angle) are adjacent and share those rows through L2.
// block = W rounded to 32 (up to 1024; wider slices take the kernel above).
constexpr int kAdjRows = 8;

size_t stage_adjoint_own_smem(int64_t L, int64_t W) {
    return sizeof(float) * (size_t)L * kAdjRows * (size_t)(W + 1);
}

constexpr int kAdjOwnMaxThreads = 1024;

__global__ void __launch_bounds__(kAdjOwnMaxThreads)
xrf_stage_adjoint_own_kernel(const float* __restrict__ frac, const float* __restrict__ theta,
                             const float* __restrict__ coef_x, const float* __restrict__ coef_f,
                             const float* __restrict__ INC, const float* __restrict__ dinc,
                             const float* __restrict__ dmu_rev, float* __restrict__ D, int n_ch,
                             int S, int H, int W, int L, int a0, int n_a) {
    extern __shared__ float sdm[];          // [L][kAdjRows][W + 1]
    const int j = blockIdx.x, s = blockIdx.y, al = blockIdx.z, a = a0 + al, w = threadIdx.x;
    const int P = W + 1;
    const float cxj = __ldg(coef_x + (int64_t)a * n_ch + j);
    float cfj[kMaxL];
#pragma unroll
    for (int l = 0; l < kMaxL; ++l)
        cfj[l] = l < L ? __ldg(coef_f + ((int64_t)a * L + l) * n_ch + j) : 0.f;
    const double th = (double)theta[a];
    const RotGeom g = rot_geom((float)cos(th), (float)sin(th), H, W);
    const int64_t HW = (int64_t)H * W;
    const float* fj = frac + ((int64_t)j * S + s) * HW;
    const int64_t o0 = (((int64_t)j * n_a + al) * S + s) * HW;
    float gbar = 0.f;
    for (int h0 = 0; h0 < H; h0 += kAdjRows) {
        const int nr = min(kAdjRows, H - h0);
        __syncthreads();   // the previous rows have been read
        // dmu of rows h0 .. h0+nr-1: for each (line, column) nr consecutive
        // floats of the transposed layout
        for (int t = threadIdx.x; t < L * W * nr; t += blockDim.x) {
            const int lx = t / nr, r = t - lx * nr;
            const int l = lx / W, x = lx - l * W;
            sdm[(l * kAdjRows + r) * P + (W - 1 - x)] =
                __ldg(dmu_rev + ((((int64_t)al * L + l) * S + s) * W + x) * H + (H - 1 - h0 - r));
        }
        __syncthreads();
        if (w >= W) continue;
        // (issuing all eight rows' loads before the recursion needs 128
        // registers and measured slower: 7.8 against 5.3 ms per 4-angle call
        // at 256 slices of 256^2)
        for (int r = 0; r < nr; ++r) {
            const int h = h0 + r;
            const RotTap tp = rot_tap(g, h, w);
            const float fr = rot_sample_tap(fj, H, W, tp);
            const int64_t o = o0 + (int64_t)h * W + w;
            const float f = 1.f - fr * cxj;
            const float di = dinc[o];
            const float df = h > 0 ? gbar * INC[o] : 0.f;
            gbar = h > 0 ? fmaf(gbar, f, di) : di;
            float d = cxj * -df;
#pragma unroll
            for (int l = 0; l < kMaxL; ++l)
                if (l < L) d = fmaf(cfj[l], sdm[(l * kAdjRows + r) * P + w], d);
            D[o] = d;
        }
    }
}

// The rotation adjoint without global atomics: D[j][al][s] (the per-sample
// gradient of the rotated fractions, one angle of the chunk) spread onto the
// unrotated grid with the rotation's own taps (rot_tap: the points and
// weights the forward sampled; taps outside the slice are dropped, as the
// forward's zero padding reads 0 there), summed over the chunk's angles and
// added to dC[j][s].  grid (G, S x bands, L), cluster (G, 1, 1): CTA g of (s, j)
// splats angles g, g + G, ... into a shared-memory image of the slice; the
// cluster adds its images over DSMEM.  The rotation of a square slice is an
// isometry, so the sample points of columns three apart, and of same-parity
// segments (>= 2 samples) of one column, are three or more apart and their
// 2x2 tap boxes are disjoint: six phases per angle ((w mod 3) x segment
// parity) update the image with plain read-modify-writes.
constexpr int kRotAdjThreads = 512;
constexpr int kRotAdjBatch = 8;   // samples whose loads are issued together

__global__ void __launch_bounds__(kRotAdjThreads)
rot_adjoint_splat_kernel(const float* __restrict__ D, const float* __restrict__ theta,
                         float* __restrict__ dC, int S, int H, int W, int a0, int n_a, int seg,
                         int hb) {
    extern __shared__ __align__(16) float simg[];
    cg::cluster_group cluster = cg::this_cluster();
    const int G = (int)cluster.num_blocks(), rank = (int)cluster.block_rank();
    // a slice too large for shared memory is split into bands of hb rows: the
    // CTA of band b applies only the taps that fall on its rows (every tap row
    // belongs to one band, so the bands' sums are exact)
    const int nband = (H + hb - 1) / hb;
    const int s = blockIdx.y / nband, band = blockIdx.y - s * nband, j = blockIdx.z;
    const int r0 = band * hb, r1 = min(H, r0 + hb);
    const int pitch = slice_pitch(W);
    const int64_t HW = (int64_t)H * W;
    for (int i = threadIdx.x; i < (r1 - r0) * pitch; i += blockDim.x) simg[i] = 0.f;
    __syncthreads();
    const int nseg = (H + seg - 1) / seg;
    for (int al = rank; al < n_a; al += G) {
        const double th = (double)theta[a0 + al];
        const RotGeom g = rot_geom((float)cos(th), (float)sin(th), H, W);
        const float* d = D + (((int64_t)j * n_a + al) * S + s) * HW;
        for (int ph = 0; ph < 6; ++ph) {
            const int pw = ph >> 1, ps = ph & 1;
            const int nw = (W - pw + 2) / 3, nsp = (nseg - ps + 1) / 2;
            for (int it = threadIdx.x; it < nw * nsp; it += blockDim.x) {
                const int k = it / nw, cw = it - k * nw;
                const int w = pw + 3 * cw;
                const int h0 = (ps + 2 * k) * seg, h1 = min(H, h0 + seg);
                int hs = h0, he = h1;
                if (nband > 1) {
                    // the sample row iy is linear in h along a column: keep the
                    // samples whose iy lies within a row of [r0 - 1, r1), a
                    // superset of those with a tap in the band
                    const float ya = rot_tap_y(g, h0, w);
                    const float lo = (float)r0 - 2.f, hi = (float)r1 + 1.f;
                    if (fabsf(g.c) > 1e-6f) {
                        float ha = (lo - ya) / g.c, hz = (hi - ya) / g.c;
                        if (ha > hz) { const float t = ha; ha = hz; hz = t; }
                        ha = fmaxf(ha, -1.f);
                        hz = fminf(hz, (float)(h1 - h0));
                        hs = h0 + (int)floorf(ha);
                        he = h0 + (int)ceilf(hz) + 1;
                        hs = max(hs, h0);
                        he = min(he, h1);
                    } else if (ya < lo || ya > hi) {
                        continue;
                    }
                }
                for (int hq = hs; hq < he; hq += kRotAdjBatch) {
                    float vb[kRotAdjBatch];
#pragma unroll
                    for (int u = 0; u < kRotAdjBatch; ++u)
                        vb[u] = hq + u < he ? __ldg(d + (int64_t)(hq + u) * W + w) : 0.f;
#pragma unroll
                    for (int u = 0; u < kRotAdjBatch; ++u) {
                    const float v = vb[u];
                    if (v == 0.f) continue;
                    const int h = hq + u;
                    const RotTap t = rot_tap(g, h, w);
                    const int x0 = t.x0, y0 = t.y0;
                    const bool xin0 = x0 >= 0 && x0 < W, xin1 = x0 + 1 >= 0 && x0 + 1 < W;
                    const bool yin0 = y0 >= r0 && y0 < r1, yin1 = y0 + 1 >= r0 && y0 + 1 < r1;
                    const float a = v * (1.f - t.ty), b = v * t.ty;
                    if (yin0) {
                        float* p = simg + (y0 - r0) * pitch + x0;
                        if (xin0) p[0] += a * (1.f - t.tx);
                        if (xin1) p[1] += a * t.tx;
                    }
                    if (yin1) {
                        float* p = simg + (y0 + 1 - r0) * pitch + x0;
                        if (xin0) p[0] += b * (1.f - t.tx);
                        if (xin1) p[1] += b * t.tx;
                    }
                    }
                }
            }
            __syncthreads();
        }
    }
    cluster.sync();
    const int64_t nb = (int64_t)(r1 - r0) * W;
    const int64_t share = (nb + G - 1) / G;
    const int64_t i0 = rank * share, i1 = min(nb, i0 + share);
    float* out = dC + ((int64_t)j * S + s) * HW + (int64_t)r0 * W;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const int h = (int)(i / W), w = (int)(i - (int64_t)h * W);
        float sum = 0.f;
        for (int q = 0; q < G; ++q) sum += cluster.map_shared_rank(simg, q)[h * pitch + w];
        out[i] += sum;
    }
    cluster.sync();
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

struct XrfBufs {
    float *INC, *E, *ATT, *DINC, *MU, *DRES, *DMU, *TMP;
};

size_t xrf_layout(int64_t S, int64_t H, int64_t W, int64_t L, int64_t chunk, char* base,
                  XrfBufs* b) {
    const size_t vol = align256(sizeof(float) * (size_t)L * chunk * S * H * W);
    const size_t one = align256(sizeof(float) * (size_t)S * H * W);
    if (b) {
        float** p[7] = {&b->INC, &b->E, &b->ATT, &b->DINC, &b->MU, &b->DRES, &b->DMU};
        for (int i = 0; i < 7; ++i) *p[i] = (float*)(base + i * vol);
        b->TMP = (float*)(base + 7 * vol);
    }
    return 7 * vol + one;
}

int64_t xrf_chunk(int64_t S, int64_t H, int64_t W, int64_t A, int64_t L, int64_t chunk) {
    if (chunk <= 0) {
        // about 8 GiB of per-chunk scratch: larger chunks fill the GPU better
        // (one Adam step at 256^3 x 4 lines x 180 angles: 2.85 s with one
        // angle per chunk, 2.59 s with four)
        int64_t per_angle = 7 * L * S * H * W * (int64_t)sizeof(float);
        chunk = (8LL << 30) / (per_angle > 0 ? per_angle : 1);
        if (chunk < 1) chunk = 1;
    }
    if (chunk > A) chunk = A;
    if (chunk * L > 65535) chunk = 65535 / L;
    return chunk < 1 ? 1 : chunk;
}

// Rotation adjoint of one angle chunk: cluster size G (angles split over the
// cluster) chosen so that S x L x G CTAs fill the GPU, at most 8 and at most
// the chunk's angles.
int rot_adjoint_launch(const float* D, const float* theta, float* dC, int64_t S, int64_t H,
                       int64_t W, int64_t L, int a0, int n_a, cudaStream_t st) {
    // bands of rows: the whole slice where it fits in shared memory, else the
    // fewest even bands that do
    const size_t row_bytes = sizeof(float) * (size_t)slice_pitch((int)W);
    int64_t nband = 1;
    while (ceil_div(H, nband) * row_bytes > (size_t)max_smem_optin() && nband < H) ++nband;
    if (int64_t t = tune(kTuneXrfBand)) nband = std::max(nband, ceil_div(H, std::min(t, H)));
    const int hb = (int)ceil_div(H, nband);
    nband = ceil_div(H, hb);
    const size_t smem = row_bytes * (size_t)hb;
    if (smem > (size_t)max_smem_optin()) {
        set_error("xrf adjoint: a row of %lld columns does not fit in shared memory", (long long)W);
        return FLC_ERR_UNSUPPORTED;
    }
    const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(8, (size_t)smem_per_sm() / (smem + 1024)));
    int G = (int)ceil_div((int64_t)sm_count() * per_sm, S * nband * L);
    G = std::max(1, std::min(G, std::min(8, n_a)));
    int seg = 2;
    const int64_t nw = (W + 2) / 3;
    while (seg < H && nw * (((H + seg - 1) / seg + 1) / 2) > kRotAdjThreads) ++seg;
    const void* fn = (const void*)rot_adjoint_splat_kernel;
    FLC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FLC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)G, (unsigned)(S * nband), (unsigned)L);
    cfg.blockDim = dim3(kRotAdjThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int iS = (int)S, iH = (int)H, iW = (int)W;
    FLC_TRY_CUDA(cudaLaunchKernelEx(&cfg, rot_adjoint_splat_kernel, D, theta, dC, iS, iH, iW, a0,
                                    n_a, seg, hb));
    count_launches(1);
    return FLC_OK;
}

int check_xrf_args(int64_t n_ch, int64_t S, int64_t H, int64_t W, int64_t A, int64_t L,
                   int64_t Mz, int64_t Mx, int64_t My, int incident_mode) {
    FLC_REQUIRE(n_ch >= 1 && n_ch <= kMaxCh && L >= 1 && L <= kMaxL && L <= n_ch,
                "xrf: need 1 <= L <= n_ch <= %d", kMaxCh);
    FLC_REQUIRE(H == W && H >= 2 && W <= 1024 && S >= 1 && S <= 65535 && A >= 1,
                "xrf: needs square slices 2 <= H == W <= 1024");
    FLC_REQUIRE(Mz >= 1 && Mx >= 1 && My >= 1 && (Mz & 1) && (My & 1),
                "xrf: the cone mask needs odd slice/column extents (got %lld x %lld)",
                (long long)Mz, (long long)My);
    FLC_REQUIRE(incident_mode >= 0 && incident_mode <= 2, "xrf: bad incident_mode");
    return FLC_OK;
}

}  // namespace

size_t xrf_ws_bytes(int64_t S, int64_t H, int64_t W, int64_t A, int64_t L, int64_t chunk) {
    return xrf_layout(S, H, W, L, xrf_chunk(S, H, W, A, L, chunk), nullptr, nullptr);
}

namespace {

// Optional scratch past the base layout: the channel-interleaved fractions
// (the stage's taps in 16-byte loads), then the spectral cone's scratch.
// Either is left out (nullptr / 0) when the workspace is too small for it;
// the planar stage and the direct cone kernels then run.
struct XrfExtra {
    float4* frac4;
    void* fft;
    size_t fft_bytes;
};

XrfExtra xrf_extra(char* ws, size_t ws_bytes, size_t base, int64_t n_ch, int64_t S, int64_t H,
                   int64_t W) {
    XrfExtra x{nullptr, nullptr, 0};
    const size_t f4 = frac4_bytes(n_ch, S, H, W);
    if (ws_bytes >= base + f4) {
        x.frac4 = (float4*)(ws + base);
        x.fft = ws + base + f4;
        x.fft_bytes = ws_bytes - base - f4;
    }
    return x;
}

}  // namespace

}  // namespace flc

using namespace flc;

extern "C" size_t flc_xrf_workspace_bytes(int64_t n_ch, int64_t S, int64_t H, int64_t W, int64_t A,
                                          int64_t L, int64_t chunk) {
    if (n_ch < 1 || S < 1 || H < 1 || W < 1 || A < 1 || L < 1) return 0;
    return xrf_ws_bytes(S, H, W, A, L, chunk);
}

extern "C" size_t flc_xrf_workspace_bytes_ex(int64_t n_ch, int64_t S, int64_t H, int64_t W,
                                             int64_t A, int64_t L, int64_t chunk, int64_t Mz,
                                             int64_t Mx, int64_t My) {
    if (n_ch < 1 || n_ch > kMaxCh || S < 1 || H < 1 || W < 1 || A < 1 || L < 1 || Mz < 1 ||
        Mx < 1 || My < 1)
        return 0;
    const int64_t c = xrf_chunk(S, H, W, A, L, chunk);
    // cone frame (Z = S, X = W, Y = H); the beam-layout modes need the most
    return xrf_ws_bytes(S, H, W, A, L, chunk) + frac4_bytes(n_ch, S, H, W) +
           cone_fft_ws_bytes(c * L, S, W, H, Mz, Mx, My, 2);
}

extern "C" int flc_xrf_project(const float* frac, const float* theta, const float* coef_x,
                               const float* coef_f, const float* u, const float* v,
                               const float* em, float* Pf, int64_t n_ch, int64_t S, int64_t H,
                               int64_t W, int64_t A, int64_t L, int64_t Mz, int64_t Mx,
                               int64_t My, int incident_mode, int64_t chunk, void* workspace,
                               size_t workspace_bytes, void* stream) {
    clear_error();
    FLC_REQUIRE(frac && theta && coef_x && coef_f && u && v && em && Pf && workspace,
                "flc_xrf_project: null pointer argument");
    FLC_TRY(check_xrf_args(n_ch, S, H, W, A, L, Mz, Mx, My, incident_mode));
    chunk = xrf_chunk(S, H, W, A, L, chunk);
    size_t need = xrf_layout(S, H, W, L, chunk, nullptr, nullptr);
    if (workspace_bytes < need || ((uintptr_t)workspace & 255)) {
        set_error("flc_xrf_project: need a 256-byte aligned workspace of %zu bytes", need);
        return workspace_bytes < need ? FLC_ERR_WORKSPACE : FLC_ERR_ALIGNMENT;
    }
    cudaStream_t st = as_stream(stream);
    XrfBufs b;
    xrf_layout(S, H, W, L, chunk, (char*)workspace, &b);
    const XrfExtra x = xrf_extra((char*)workspace, workspace_bytes, need, n_ch, S, H, W);
    if (x.frac4) FLC_TRY(frac_interleave_launch(frac, x.frac4, n_ch, S, H, W, st));
    const int64_t vol = S * H * W;
    for (int64_t a0 = 0; a0 < A; a0 += chunk) {
        const int n_a = (int)(A - a0 < chunk ? A - a0 : chunk);
        // incident term straight into ATT, fluorescence mu into MU
        FLC_TRY(atten_stage_launch(frac, theta, coef_x, coef_f, b.ATT, b.MU, (int)n_ch, (int)S,
                                   (int)H, (int)W, (int)L, vol, (int64_t)n_a * vol, (int)a0, n_a,
                                   incident_mode, 1, st, 0, x.frac4));
        FLC_TRY(cone_launch_ws(b.MU, u, v, b.ATT, (int64_t)n_a * L, S, W, H, Mz, Mx, My, 2,
                               (int)L, 0, vol, (int64_t)n_a * vol, x.fft, x.fft_bytes, st));
        for (int64_t l = 0; l < L; ++l)
            FLC_TRY(fwd_emission_launch(b.ATT + l * n_a * vol, frac + l * vol, em + l * A + a0,
                                        theta + a0, Pf + (l * A + a0) * S * W, nullptr, n_a, S, 1,
                                        H, W, st));
    }
    return FLC_OK;
}

extern "C" int flc_xrf_project_adjoint(const float* frac, const float* theta, const float* coef_x,
                                       const float* coef_f, const float* u, const float* v,
                                       const float* uf, const float* vf, const float* em,
                                       const float* gPf, float* dC, int64_t n_ch, int64_t S,
                                       int64_t H, int64_t W, int64_t A, int64_t L, int64_t Mz,
                                       int64_t Mx, int64_t My, int incident_mode, int64_t chunk,
                                       void* workspace, size_t workspace_bytes, void* stream) {
    clear_error();
    FLC_REQUIRE(frac && theta && coef_x && coef_f && u && v && uf && vf && em && gPf && dC &&
                    workspace,
                "flc_xrf_project_adjoint: null pointer argument");
    FLC_TRY(check_xrf_args(n_ch, S, H, W, A, L, Mz, Mx, My, incident_mode));
    chunk = xrf_chunk(S, H, W, A, L, chunk);
    size_t need = xrf_layout(S, H, W, L, chunk, nullptr, nullptr);
    if (workspace_bytes < need || ((uintptr_t)workspace & 255)) {
        set_error("flc_xrf_project_adjoint: need a 256-byte aligned workspace of %zu bytes", need);
        return workspace_bytes < need ? FLC_ERR_WORKSPACE : FLC_ERR_ALIGNMENT;
    }
    cudaStream_t st = as_stream(stream);
    XrfBufs b;
    xrf_layout(S, H, W, L, chunk, (char*)workspace, &b);
    const XrfExtra x = xrf_extra((char*)workspace, workspace_bytes, need, n_ch, S, H, W);
    if (x.frac4) FLC_TRY(frac_interleave_launch(frac, x.frac4, n_ch, S, H, W, st));
    const int64_t vol = S * H * W;
    FLC_TRY_CUDA(cudaMemsetAsync(dC, 0, sizeof(float) * L * vol, st));
    for (int64_t a0 = 0; a0 < A; a0 += chunk) {
        const int n_a = (int)(A - a0 < chunk ? A - a0 : chunk);
        const int64_t nv = (int64_t)n_a * L * vol;
        // recompute the chunk: INC, E = exp(-cone), ATT = INC * E
        FLC_TRY(atten_stage_launch(frac, theta, coef_x, coef_f, b.INC, b.MU, (int)n_ch, (int)S,
                                   (int)H, (int)W, (int)L, vol, (int64_t)n_a * vol, (int)a0, n_a,
                                   incident_mode, 1, st, 0, x.frac4));
        FLC_TRY(cone_launch_ws(b.MU, u, v, b.E, (int64_t)n_a * L, S, W, H, Mz, Mx, My, 3, (int)L,
                               0, vol, (int64_t)n_a * vol, x.fft, x.fft_bytes, st));
        mul_kernel<<<(unsigned)ceil_div(nv, 256), 256, 0, st>>>(b.INC, b.E, b.ATT, nv);
        FLC_TRY(check_launch("mul_kernel"));
        // direct term: P^T[atten](dL/dPf) per element
        for (int64_t l = 0; l < L; ++l) {
            FLC_TRY(bwd_emission_launch(b.ATT + l * n_a * vol, gPf + (l * A + a0) * S * W,
                                        em + l * A + a0, theta + a0, b.TMP, n_a, S, 1, H, W, 0.f,
                                        st));
            add_kernel<<<(unsigned)ceil_div(vol, 256), 256, 0, st>>>(dC + l * vol, b.TMP, vol);
            FLC_TRY(check_launch("add_kernel"));
        }
        // through the attenuation
        dim3 gg((unsigned)(ceil_div(W, 32) * ceil_div(H, 32)), (unsigned)S, (unsigned)(n_a * L));
        xrf_g_kernel<<<gg, dim3(32, 8), 0, st>>>(frac, theta, em, gPf, b.ATT, b.E, b.DINC, b.DRES,
                                                  (int)L, (int)A, (int)a0, n_a, (int)S, (int)H,
                                                  (int)W);
        FLC_TRY(check_launch("xrf_g_kernel"));
        FLC_TRY(cone_launch_ws(b.DRES, uf, vf, b.DMU, (int64_t)n_a * L, S, W, H, Mz, Mx, My, 0,
                               1, 0, 0, 0, x.fft, x.fft_bytes, st));
        const int threads = (int)((W + 31) & ~31);
        // the per-sample gradient of the rotated fractions into ATT (free
        // again), then its rotation adjoint into dC
        const size_t own_smem = stage_adjoint_own_smem(L, W);
        if (incident_mode == 0 && threads <= kAdjOwnMaxThreads &&
            own_smem <= (size_t)max_smem_optin()) {
            if (own_smem > 48 * 1024)
                FLC_TRY_CUDA(cudaFuncSetAttribute(xrf_stage_adjoint_own_kernel,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)own_smem));
            xrf_stage_adjoint_own_kernel<<<dim3((unsigned)L, (unsigned)S, (unsigned)n_a), threads,
                                           own_smem, st>>>(
                frac, theta, coef_x, coef_f, b.INC, b.DINC, b.DMU, b.ATT, (int)n_ch, (int)S,
                (int)H, (int)W, (int)L, (int)a0, n_a);
            FLC_TRY(check_launch("xrf_stage_adjoint_own_kernel"));
        } else {
            xrf_stage_adjoint_kernel<<<dim3((unsigned)S, (unsigned)n_a), threads, 0, st>>>(
                frac, theta, coef_x, coef_f, b.INC, b.DINC, b.DMU, b.ATT, (int)n_ch, (int)S,
                (int)H, (int)W, (int)L, (int)a0, n_a, incident_mode);
            FLC_TRY(check_launch("xrf_stage_adjoint_kernel"));
        }
        FLC_TRY(rot_adjoint_launch(b.ATT, theta, dC, S, H, W, L, (int)a0, n_a, st));
    }
    return FLC_OK;
}
