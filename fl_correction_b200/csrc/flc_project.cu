// Attenuated emission projector (forward / exact-transpose backward), the
// Huber term and the device-resident MLEM iteration, for sm_100a.
//
// Reference semantics: FL/cuda_lib/atten_cuda_kernel.cu:91-446,495-616 and
// FL/cuda_lib/atten_cuda.cpp:82-345.  The reference scatters with one global
// atomicAdd per sample (forward) and four per sample per reference
// (backward).  Here one CTA owns one slice b and a group of angles:
//  * the slice of C is staged once in shared memory (row pitch == 9 mod 32,
//    which spreads the rotated bilinear taps of a warp over the banks);
//  * per angle the atten tile (H x W, contiguous) is copied into shared memory
//    with coalesced 128-bit loads, issued one angle ahead into registers so
//    the copy overlaps the previous angle's work;
//  * the forward sums each detector column along the beam in registers and
//    combines a fixed number of partial sums in a fixed order (no atomics,
//    deterministic);
//  * the backward splats the exact transpose into a shared-memory image of the
//    slice in nine phases: samples whose (h, w) agree modulo 3 sit >= 3 apart
//    on the rotated lattice, so their 2x2 footprints are disjoint and plain
//    read-modify-writes cannot race.  Samples clamped to the edge (they land
//    only on the border frame: rows 0, H-2, H-1, columns 0, W-2, W-1) go with
//    shared atomics into separate frame buffers, folded into the image after
//    the last angle; samples clamped in both coordinates all land on one of
//    the four corners and are summed in registers.  Every lane of a warp runs
//    the same code for unclamped samples (no divergent border path), and
//    each thread issues two footprints' loads before their stores;
//  * the CTAs of one slice form a thread-block cluster and reduce their images
//    through distributed shared memory in rank order;
//  * one MLEM iteration (forward, ratio, backward, Huber, update, clamp) is a
//    single cluster launch that reads each atten tile from HBM once.

#include <cooperative_groups.h>

#include <mutex>
#include <vector>

#include "flc_common.cuh"
#include "flc_geom.cuh"

namespace cg = cooperative_groups;

namespace flc {
namespace {

constexpr int kThreads = 512;
constexpr int kMaxCluster = 8;
constexpr int kMaxR = 8;
constexpr int kTileRegs = 8;   // float4 per thread prefetched for the next tile


// Partial sums per detector column: enough (w, part) items to fill the CTA.
__host__ __device__ inline int col_parts(int W, int H) {
    int p = (2 * kThreads + W - 1) / W;
    if (p > 16) p = 16;
    if (p > H) p = H;
    return p < 1 ? 1 : p;
}

// Sample geometry (Geo, sample, ...) lives in flc_geom.cuh, shared with the adjoints.

// ---------------------------------------------------------------------------
// Tile staging: copy n floats (16-byte aligned when vec) from global into a
// register set (issue) and later into shared memory (commit).
// ---------------------------------------------------------------------------
struct TileRegs {
    float4 r[kTileRegs];
};

__device__ __forceinline__ void tile_issue(TileRegs& t, const float* __restrict__ src, int n) {
    const int n4 = n >> 2;
#pragma unroll
    for (int k = 0; k < kTileRegs; ++k) {
        int i = threadIdx.x + k * blockDim.x;
        if (i < n4) t.r[k] = __ldg(reinterpret_cast<const float4*>(src) + i);
    }
}

__device__ __forceinline__ void tile_commit(const TileRegs& t, const float* __restrict__ src,
                                            float* dst, int n) {
    const int n4 = n >> 2;
#pragma unroll
    for (int k = 0; k < kTileRegs; ++k) {
        int i = threadIdx.x + k * blockDim.x;
        if (i < n4) reinterpret_cast<float4*>(dst)[i] = t.r[k];
    }
    // tiles larger than the register set, and the n % 4 tail, are copied directly
    for (int i = kTileRegs * blockDim.x + threadIdx.x; i < n4; i += blockDim.x)
        reinterpret_cast<float4*>(dst)[i] = __ldg(reinterpret_cast<const float4*>(src) + i);
    for (int i = (n4 << 2) + threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}

// Plain staged copy (used when the tile start is not 16-byte aligned).
__device__ __forceinline__ void tile_copy(const float* __restrict__ src, float* dst, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}

// Loads R slices C[r, b] (H x W, row stride W) into smem with row pitch `pitch`.
__device__ void stage_slice(float* sC, const float* __restrict__ C, int R, int B, int b,
                            int H, int W, int pitch) {
    for (int r = 0; r < R; ++r) {
        const float* src = C + ((int64_t)r * B + b) * (int64_t)H * W;
        float* dst = sC + (int64_t)r * H * pitch;
        for (int i = threadIdx.x; i < H * W; i += blockDim.x) {
            int h = i / W, w = i - h * W;
            dst[h * pitch + w] = __ldg(src + i);
        }
    }
}

// ---------------------------------------------------------------------------
// Forward of one (angle, slice): spart[p][w] = sum over beam steps h of part
// p of atten[h][w] * sum_r em_r * bilerp(C_r).
// ---------------------------------------------------------------------------
__device__ void forward_angle(const float* sA, const float* sC, int img_stride, int pitch,
                              const float* em_a, int R, const Geo& g, int H, int W, int parts,
                              float* spart) {
    const int hper = (H + parts - 1) / parts;
    for (int item = threadIdx.x; item < parts * W; item += blockDim.x) {
        const int part = item / W, w = item - part * W;
        const int h0 = part * hper, h1 = min(H, h0 + hper);
        const float bx = col_bx(g, w), by = col_by(g, w);
        float acc0 = 0.f, acc1 = 0.f;
        int h = h0;
        float hf = (float)h0 - g.cy;
        for (; h + 1 < h1; h += 2, hf += 2.f) {
            Smp s0 = sample_xy(g, fmaf(g.c, hf, bx), fmaf(g.s, hf, by));
            Smp s1 = sample_xy(g, fmaf(g.c, hf + 1.f, bx), fmaf(g.s, hf + 1.f, by));
            float v0 = 0.f, v1 = 0.f;
            for (int r = 0; r < R; ++r) {
                const float* p0 = sC + r * img_stride + s0.i0 * pitch + s0.j0;
                const float* p1 = sC + r * img_stride + s1.i0 * pitch + s1.j0;
                float t0 = fmaf(s0.fy, p0[1] - p0[0], p0[0]);
                float b0 = fmaf(s0.fy, p0[pitch + 1] - p0[pitch], p0[pitch]);
                float t1 = fmaf(s1.fy, p1[1] - p1[0], p1[0]);
                float b1 = fmaf(s1.fy, p1[pitch + 1] - p1[pitch], p1[pitch]);
                v0 = fmaf(em_a[r], fmaf(s0.fx, b0 - t0, t0), v0);
                v1 = fmaf(em_a[r], fmaf(s1.fx, b1 - t1, t1), v1);
            }
            acc0 = fmaf(sA[h * W + w], v0, acc0);
            acc1 = fmaf(sA[(h + 1) * W + w], v1, acc1);
        }
        if (h < h1) {
            Smp s0 = sample_xy(g, fmaf(g.c, hf, bx), fmaf(g.s, hf, by));
            float v0 = 0.f;
            for (int r = 0; r < R; ++r) {
                const float* p0 = sC + r * img_stride + s0.i0 * pitch + s0.j0;
                float t0 = fmaf(s0.fy, p0[1] - p0[0], p0[0]);
                float b0 = fmaf(s0.fy, p0[pitch + 1] - p0[pitch], p0[pitch]);
                v0 = fmaf(em_a[r], fmaf(s0.fx, b0 - t0, t0), v0);
            }
            acc0 = fmaf(sA[h * W + w], v0, acc0);
        }
        spart[part * W + w] = acc0 + acc1;
    }
}

// Corner sums of samples clamped in both coordinates, in registers for the
// first kCornerR references: v[r][k], k = 2*xhigh + yhigh.  (Indexed with
// compile-time constants only, so they stay in registers.)
constexpr int kCornerR = 2;
struct Corners {
    float v[kCornerR][4];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int r = 0; r < kCornerR; ++r)
#pragma unroll
            for (int k = 0; k < 4; ++k) v[r][k] = 0.f;
    }
    __device__ __forceinline__ void add(int r, int k, float x) {
#pragma unroll
        for (int rr = 0; rr < kCornerR; ++rr)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) v[rr][kk] += (rr == r && kk == k) ? x : 0.f;
    }
};

// Samples clamped to the image border (atten_cuda_kernel.cu:116-133) land
// only on the border frame: a row clamp on row 0 (x < 0, weight 1) or rows
// ih = H-2, ih+1 (x > rmax, weights 1-fxh, fxh); a column clamp likewise on
// columns 0 or W-2, W-1.  They are collected, with shared atomics, in frame
// buffers kept apart from the slice image so that the unclamped samples can
// update the image with plain read-modify-writes.  The split of a high clamp
// between its two rows (columns) is the same constant for every sample, so a
// clamped sample only adds its weights along the edge, (1-fy, fy) at j0, j0+1
// (rows) or (1-fx, fx) at i0, i0+1 (columns), into a low or a high buffer:
//   row part    [r][slot][j], slot 0: row 0, 1: rows H-2, H-1   (R x 2 x W)
//   column part [r][slot][i], slot 0: col 0, 1: cols W-2, W-1   (R x 2 x H)
// `ncopy` (1 to kMaxFrameCopies) such frames, one per group of warps
// (warp % ncopy), spread the atomics on one edge pixel over several
// addresses.  They are added into the image once, after the last angle
// (fold_frame), the high slots split by (1 - fxh, fxh) and (1 - fyh, fyh).
constexpr int kMaxFrameCopies = 4;

__host__ __device__ inline int frame_floats(int R, int H, int W, int ncopy) {
    return ncopy * 2 * R * (H + W);
}

// Adds v, spread over the pixels of corner class k (2*xhigh + yhigh), into
// the row part of one reference's frame.
__device__ __forceinline__ void corner_add(float* srow, int W, const Geo& g, int k, float v) {
    const bool xh = k >= 2, yh = k & 1;
    const int j0 = yh ? g.jh : 0;
    const float fy = yh ? g.fyh : 0.f;
    float* b = srow + (xh ? W : 0) + j0;
    atomicAdd(b, v * (1.f - fy));
    if (fy != 0.f) atomicAdd(b + 1, v * fy);
}

// Bilinear footprint of one sample on the clamped grid.
struct Foot {
    int off;                 // i0 * pitch + j0
    int i0, j0;
    float w00, w01, w10, w11;
    float fx, fy;            // bilinear fractions on the clamped grid
    float av;                // atten * ratio
    int kind;                // bits: 1 x < 0, 2 x > rmax, 4 y < 0, 8 y > cmax
};

__device__ __forceinline__ Foot footprint(const Geo& g, const float* sA, const float* sratio,
                                          int W, int pitch, int h, int w) {
    Foot f;
    f.av = sratio ? sA[h * W + w] * sratio[w] : sA[h * W + w];
    const float hf = (float)h - g.cy;
    const float x = fmaf(g.c, hf, col_bx(g, w)), y = fmaf(g.s, hf, col_by(g, w));
    const float xc = fminf(fmaxf(x, 0.f), g.rmax), yc = fminf(fmaxf(y, 0.f), g.cmax);
    float fx, fy;
    f.i0 = ffloor(xc, fx);
    f.j0 = ffloor(yc, fy);
    f.fx = fx;
    f.fy = fy;
    f.off = f.i0 * pitch + f.j0;
    f.w00 = (1.f - fy) * (1.f - fx);
    f.w01 = fy * (1.f - fx);
    f.w10 = (1.f - fy) * fx;
    f.w11 = fy * fx;
    f.kind = (x < 0.f ? 1 : 0) | (x > g.rmax ? 2 : 0) | (y < 0.f ? 4 : 0) | (y > g.cmax ? 8 : 0);
    return f;
}

// Contribution v of a clamped sample of reference r into the frame buffers
// (or, clamped in both coordinates, r < kCornerR and REG -- the reference
// count is a compile-time constant -- the corner registers).  A corner
// handled here takes the row path: its clamped fraction fx is 0 or fxh.
template <bool REG>
__device__ __forceinline__ void frame_add(const Foot& f, float v, float* srow, float* scol, int H,
                                          int W, Corners& cs, int r) {
    const bool rowc = (f.kind & 3) != 0;
    const bool corner = rowc && (f.kind & 12) != 0;
    if (REG && corner && r < kCornerR) {
        cs.add(r, ((f.kind & 2) ? 2 : 0) + ((f.kind & 8) ? 1 : 0), v);
    } else {
        float* base = rowc ? srow + (2 * r + ((f.kind & 1) ? 0 : 1)) * W + f.j0
                           : scol + (2 * r + ((f.kind & 4) ? 0 : 1)) * H + f.i0;
        const float t = rowc ? f.fy : f.fx;
        atomicAdd(base, v * (1.f - t));
        if (t != 0.f) atomicAdd(base + 1, v * t);
    }
}

// Backward of one (angle, slice): sacc_r += em_r * atten * ratio[w] * bilinear
// weights, the exact transpose of forward_angle.  Nine phases, separated by
// barriers: the unclamped samples of a phase have disjoint footprints and
// update the image with plain read-modify-writes; clamped ones go to the
// frame buffers.  Each thread takes its items two at a time and issues both
// footprints' loads before either's stores (legal: they are disjoint), and
// every lane of a warp runs the same code except for the clamped samples.
// RC > 0: exactly RC references (unrolled); RC == 0: R at run time.
template <int RC>
__device__ void backward_angle(const float* sA, const float* sratio, float* sacc, float* srow,
                               float* scol, int img_stride, int pitch, const float* em_a, int Rrt,
                               const Geo& g, int H, int W, Corners& cs) {
    const int R = RC > 0 ? RC : Rrt;
    const int nthr = blockDim.x;
    const float tq = (float)threadIdx.x + 0.5f, nq = (float)nthr + 0.5f;
    for (int ph = 0; ph < 3; ++ph) {
        for (int pw = 0; pw < 3; ++pw) {
            const int nh = (H - ph + 2) / 3, nw = (W - pw + 2) / 3;
            // item it = hh * nw + ww walks by nthr: advance (hh, ww) without
            // division.  floor((t + 1/2) / nw) in FP32 is exact for t < 2^22
            // (the quotient stays >= 1/(2 nw) from an integer).  A phase can be
            // empty (H or W <= 2): skip to the barrier.
            int hh = nh, ww = 0, dh = 0, dw = 0;
            if (nh > 0 && nw > 0) {
                const float inv = 1.f / (float)nw;
                hh = (int)(tq * inv);
                ww = (int)threadIdx.x - hh * nw;
                dh = (int)(nq * inv);
                dw = nthr - dh * nw;
            }
            while (hh < nh) {
                int hb = hh + dh, wb = ww + dw;
                if (wb >= nw) { wb -= nw; ++hb; }
                const bool has_b = hb < nh;
                const Foot fa = footprint(g, sA, sratio, W, pitch, ph + 3 * hh, pw + 3 * ww);
                const Foot fb = footprint(g, sA, sratio, W, pitch, has_b ? ph + 3 * hb : ph,
                                          has_b ? pw + 3 * wb : pw);
                const bool pa = fa.kind == 0, pb = has_b && fb.kind == 0;
#pragma unroll
                for (int r = 0; r < (RC > 0 ? RC : R); ++r) {
                    const float em = em_a[r];
                    float* img = sacc + r * img_stride;
                    float* qa = img + fa.off;
                    float* qb = img + fb.off;
                    float a00 = 0.f, a01 = 0.f, a10 = 0.f, a11 = 0.f;
                    float b00 = 0.f, b01 = 0.f, b10 = 0.f, b11 = 0.f;
                    if (pa) { a00 = qa[0]; a01 = qa[1]; a10 = qa[pitch]; a11 = qa[pitch + 1]; }
                    if (pb) { b00 = qb[0]; b01 = qb[1]; b10 = qb[pitch]; b11 = qb[pitch + 1]; }
                    const float va = em * fa.av, vb = em * fb.av;
                    if (pa) {
                        qa[0] = fmaf(va, fa.w00, a00);
                        qa[1] = fmaf(va, fa.w01, a01);
                        qa[pitch] = fmaf(va, fa.w10, a10);
                        qa[pitch + 1] = fmaf(va, fa.w11, a11);
                    }
                    if (pb) {
                        qb[0] = fmaf(vb, fb.w00, b00);
                        qb[1] = fmaf(vb, fb.w01, b01);
                        qb[pitch] = fmaf(vb, fb.w10, b10);
                        qb[pitch + 1] = fmaf(vb, fb.w11, b11);
                    }
                    if (!pa) frame_add<(RC > 0)>(fa, va, srow, scol, H, W, cs, r);
                    if (has_b && !pb) frame_add<(RC > 0)>(fb, vb, srow, scol, H, W, cs, r);
                }
                hh = hb + dh;
                ww = wb + dw;
                if (ww >= nw) { ww -= nw; ++hh; }
            }
            __syncthreads();
        }
    }
}

// Backward of one (angle, slice) by column segments (the "proj.bwd" = 4
// variant).  A detector column is a straight line of samples in the image;
// lines three columns apart, and pieces of one line one segment apart, are
// at least three pixels apart (seg >= 2), so their 2 x 2 footprints are
// disjoint.  Six phases -- (w mod 3) x (segment parity) -- each give every
// thread about one segment of `seg` consecutive samples of one column (the
// host picks seg so that one round of items fills the CTA), walked in order: the
// overlapping footprints of consecutive samples are updated by the same
// thread, one after the other, with plain read-modify-writes.  Clamped
// samples go to the frame buffers as in the nine-phase form.
template <int RC>
__device__ void backward_angle_seg(const float* sA, const float* sratio, float* sacc, float* srow,
                                   float* scol, int img_stride, int pitch, const float* em_a,
                                   int Rrt, const Geo& g, int H, int W, Corners& cs, int seg) {
    const int R = RC > 0 ? RC : Rrt;
    const int nseg = (H + seg - 1) / seg;
    for (int pw = 0; pw < 3; ++pw) {
        const int nw = (W - pw + 2) / 3;
        for (int ps = 0; ps < 2; ++ps) {
            const int nsp = (nseg - ps + 1) / 2;   // segments of this parity
            const int items = nw * nsp;
            for (int it = threadIdx.x; it < items; it += blockDim.x) {
                const int k = it / nw, cw = it - k * nw;   // a warp spans columns
                const int w = pw + 3 * cw;
                const int h0 = (ps + 2 * k) * seg, h1 = min(H, h0 + seg);
                for (int h = h0; h < h1; ++h) {
                    const Foot f = footprint(g, sA, sratio, W, pitch, h, w);
#pragma unroll
                    for (int r = 0; r < (RC > 0 ? RC : R); ++r) {
                        const float v = em_a[r] * f.av;
                        if (f.kind == 0) {
                            float* q = sacc + r * img_stride + f.off;
                            q[0] = fmaf(v, f.w00, q[0]);
                            q[1] = fmaf(v, f.w01, q[1]);
                            q[pitch] = fmaf(v, f.w10, q[pitch]);
                            q[pitch + 1] = fmaf(v, f.w11, q[pitch + 1]);
                        } else {
                            frame_add<(RC > 0)>(f, v, srow, scol, H, W, cs, r);
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Backward of one (angle, slice) with shared-memory atomics instead of
// phases (the "proj.bwd" = 1 variant): every thread takes samples it = t,
// t + nthr, ... (a warp covers a run of consecutive columns of one beam row)
// and adds its four bilinear weights with atomicAdd; no barrier inside the
// angle.  Samples clamped in both coordinates pile onto a corner and are
// summed in registers (compile-time reference count) or added like the rest.
// Float atomics on shared memory are read-modify-write loops on this part,
// and neighbouring lanes hit neighbouring cells, so the nine-phase form is
// the default; this one stays for the autotuner.
template <int RC>
__device__ void backward_angle_atomic(const float* sA, const float* sratio, float* sacc,
                                      int img_stride, int pitch, const float* em_a, int Rrt,
                                      const Geo& g, int H, int W, Corners& cs, int dh, int dw,
                                      int h0, int w0) {
    const int R = RC > 0 ? RC : Rrt;
    int h = h0, w = w0;
    while (h < H) {
        const Foot f = footprint(g, sA, sratio, W, pitch, h, w);
        const bool corner = (f.kind & 3) && (f.kind & 12);
#pragma unroll
        for (int r = 0; r < (RC > 0 ? RC : R); ++r) {
            const float v = em_a[r] * f.av;
            if (RC > 0 && corner && r < kCornerR) {
                cs.add(r, ((f.kind & 2) ? 2 : 0) + ((f.kind & 8) ? 1 : 0), v);
                continue;
            }
            float* q = sacc + r * img_stride + f.off;
            if (f.w00 != 0.f) atomicAdd(q, v * f.w00);
            if (f.w01 != 0.f) atomicAdd(q + 1, v * f.w01);
            if (f.w10 != 0.f) atomicAdd(q + pitch, v * f.w10);
            if (f.w11 != 0.f) atomicAdd(q + pitch + 1, v * f.w11);
        }
        h += dh;
        w += dw;
        if (w >= W) { w -= W; ++h; }
    }
}

// Backward of one (angle, slice) in gather form, one reference (the
// "proj.bwd" = 3 variant).  sQ holds the staged atten tile; it is scaled in
// place by ratio[w] * em.  Every thread owns pixels p = t, t + nthr, ... of
// the slice image and sums, over the 3 x 3 beam-frame samples around the
// pixel's inverse image, the unclamped samples whose footprint covers it with
// the forward's own weights (1 - |x - i|)(1 - |y - j|) -- the sample point and
// the unclamped test are computed exactly as the forward computes them.  The
// owner adds the sum into the image: no atomics, no phases.  The clamped
// samples (they land on the border frame only) are then walked once and go
// to the frame buffers or the corner registers.
__device__ void backward_angle_gather(float* sQ, const float* sratio, float em, float* sacc,
                                      float* srow, float* scol, int pitch, const Geo& g, int H,
                                      int W, Corners& cs, int dh, int dw, int h0, int w0) {
    int h = h0, w = w0;
    while (h < H) {
        sQ[h * W + w] *= sratio[w] * em;
        h += dh;
        w += dw;
        if (w >= W) { w -= W; ++h; }
    }
    __syncthreads();
    // inverse of x = c(h-cy) - s(w-cx) + cy, y = s(h-cy) + c(w-cx) + cx
    int i = h0, j = w0;
    while (i < H) {
        const float xi = (float)i - g.cy, yj = (float)j - g.cx;
        const int hr = __float2int_rn(fmaf(g.c, xi, fmaf(g.s, yj, g.cy)));
        const int wr = __float2int_rn(fmaf(-g.s, xi, fmaf(g.c, yj, g.cx)));
        float val = 0.f;
#pragma unroll
        for (int a = -1; a <= 1; ++a) {
            const int hh = hr + a;
            const float hf = (float)hh - g.cy;
            const bool hin = (unsigned)hh < (unsigned)H;
#pragma unroll
            for (int b = -1; b <= 1; ++b) {
                const int ww = wr + b;
                const float x = fmaf(g.c, hf, col_bx(g, ww)), y = fmaf(g.s, hf, col_by(g, ww));
                const float wx = 1.f - fabsf(x - (float)i), wy = 1.f - fabsf(y - (float)j);
                const bool ok = hin && (unsigned)ww < (unsigned)W && x >= 0.f && x <= g.rmax &&
                                y >= 0.f && y <= g.cmax && wx > 0.f && wy > 0.f;
                if (ok) val = fmaf(wx * wy, sQ[hh * W + ww], val);
            }
        }
        sacc[i * pitch + j] += val;
        i += dh;
        j += dw;
        if (j >= W) { j -= W; ++i; }
    }
    h = h0;
    w = w0;
    while (h < H) {
        const float hf = (float)h - g.cy;
        const float x = fmaf(g.c, hf, col_bx(g, w)), y = fmaf(g.s, hf, col_by(g, w));
        if (!(x >= 0.f && x <= g.rmax && y >= 0.f && y <= g.cmax)) {
            const Foot f = footprint(g, sQ, nullptr, W, pitch, h, w);
            frame_add<true>(f, f.av, srow, scol, H, W, cs, 0);
        }
        h += dh;
        w += dw;
        if (w >= W) { w -= W; ++h; }
    }
}

// Adds the register corner sums into the row buffers: warp-reduce, then one
// atomic per warp and pixel.
__device__ void flush_corners(Corners& cs, float* srow, const Geo& g, int R, int W) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int r = 0; r < kCornerR; ++r) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float v = cs.v[r][k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (r < R && lane == 0 && v != 0.f) corner_add(srow + r * 2 * W, W, g, k, v);
        }
    }
}

// After the last angle: corners into the row buffers, then every copy of the
// frame into the image (one thread per column / row, slots in order, so a
// coinciding row or column -- H or W == 2 -- is still summed correctly).
__device__ void fold_frame(Corners& cs, float* sacc, float* sframe, int ncopy, int img_stride,
                           int pitch, int R, int H, int W) {
    // every thread passes the barriers below (callers have finished all angles)
    __syncthreads();
    const Geo g0 = make_geo(0.f, H, W);
    flush_corners(cs, sframe, g0, R, W);
    __syncthreads();
    const int copy = 2 * R * (H + W);
    for (int t = threadIdx.x; t < R * W; t += blockDim.x) {
        const int r = t / W, j = t - r * W;
        float lo = 0.f, hi = 0.f;
        for (int c = 0; c < ncopy; ++c) {
            lo += sframe[c * copy + 2 * r * W + j];
            hi += sframe[c * copy + 2 * r * W + W + j];
        }
        float* img = sacc + r * img_stride + j;
        img[0] += lo;
        img[(H - 2) * pitch] += hi * (1.f - g0.fxh);
        img[(H - 1) * pitch] += hi * g0.fxh;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < R * H; t += blockDim.x) {
        const int r = t / H, i = t - r * H;
        float lo = 0.f, hi = 0.f;
        for (int c = 0; c < ncopy; ++c) {
            lo += sframe[c * copy + 2 * R * W + 2 * r * H + i];
            hi += sframe[c * copy + 2 * R * W + 2 * r * H + H + i];
        }
        float* img = sacc + r * img_stride + i * pitch;
        img[0] += lo;
        img[W - 2] += hi * (1.f - g0.fyh);
        img[W - 1] += hi * g0.fyh;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Forward projection: grid (angle groups, B); optional MLEM ratio epilogue.
// ---------------------------------------------------------------------------
// stage_tile: atten tiles are copied to shared memory (else read from global);
// stage_c: the C slice is staged (else read from global with pitch W).
__global__ void __launch_bounds__(kThreads, 1)
proj_fwd_kernel(const float* __restrict__ atten, const float* __restrict__ C,
                const float* __restrict__ em, const float* __restrict__ theta,
                float* __restrict__ Pf, const float* __restrict__ I, int A, int B, int R,
                int H, int W, int apc, int stage_tile, int stage_c) {
    extern __shared__ __align__(16) float smem[];
    const int b = blockIdx.y;
    const int a0 = blockIdx.x * apc, a1 = min(A, a0 + apc);
    const int pitch = stage_c ? slice_pitch(W) : W;
    const int parts = col_parts(W, H);
    const int HW = H * W;
    const int img_stride = stage_c ? H * pitch : B * HW;
    float* sA = smem;                                        // [H*W] (16-byte aligned)
    float* sC = sA + (stage_tile ? ((HW + 3) & ~3) : 0);     // [R][H][pitch]
    float* spart = sC + (stage_c ? R * img_stride : 0);      // [parts][W]
    float* sem = spart + parts * W;                          // [R]
    const float* Cb = stage_c ? sC : C + (int64_t)b * HW;
    const bool vec = stage_tile && ((HW & 3) == 0) && (((uintptr_t)atten & 15) == 0);
    if (stage_c) stage_slice(sC, C, R, B, b, H, W, pitch);
    TileRegs tr;
    if (a0 < a1 && vec) tile_issue(tr, atten + ((int64_t)a0 * B + b) * HW, HW);
    for (int a = a0; a < a1; ++a) {
        const float* src = atten + ((int64_t)a * B + b) * HW;
        __syncthreads();  // previous angle done with sA / spart
        if (vec) tile_commit(tr, src, sA, HW);
        else if (stage_tile) tile_copy(src, sA, HW);
        if (threadIdx.x < R) sem[threadIdx.x] = em[a * R + threadIdx.x];
        __syncthreads();
        if (a + 1 < a1 && vec) tile_issue(tr, atten + ((int64_t)(a + 1) * B + b) * HW, HW);
        const Geo g = make_geo(theta[a], H, W);
        forward_angle(stage_tile ? sA : src, Cb, img_stride, pitch, sem, R, g, H, W, parts, spart);
        __syncthreads();
        for (int w = threadIdx.x; w < W; w += blockDim.x) {
            float s = 0.f;
            for (int p = 0; p < parts; ++p) s += spart[p * W + w];
            int64_t o = ((int64_t)a * B + b) * W + w;
            if (I) s = I[o] / fmaxf(s, 1e-6f);
            Pf[o] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// Cluster reduction of the G images (rank order) for this CTA's share of the
// slice; `fn(i, r, h, w, back)` consumes each reduced pixel.
// ---------------------------------------------------------------------------
template <class Fn>
__device__ void cluster_reduce(cg::cluster_group& cluster, float* sacc, int R, int H, int W,
                               int pitch, Fn fn) {
    const int G = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int img_stride = H * pitch;
    const int64_t n = (int64_t)R * H * W;
    const int64_t share = (n + G - 1) / G;
    const int64_t i0 = rank * share, i1 = min(n, i0 + share);
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const int r = (int)(i / ((int64_t)H * W));
        const int rem = (int)(i - (int64_t)r * H * W);
        const int h = rem / W, w = rem - h * W;
        const int off = r * img_stride + h * pitch + w;
        float s = 0.f;
        for (int q = 0; q < G; ++q) s += cluster.map_shared_rank(sacc, q)[off];
        fn(r, h, w, s);
    }
}

// ---------------------------------------------------------------------------
// Backward projection: grid (G, B), cluster (G, 1, 1).  CTA g of slice b
// splats angles [g*apc, (g+1)*apc).  ratio == nullptr means ratio = 1
// (sensitivity); clamp_min > 0 applies max(out, clamp_min).
// ---------------------------------------------------------------------------
template <int RC>
__global__ void __launch_bounds__(kThreads, 1)
proj_bwd_kernel(const float* __restrict__ atten, const float* __restrict__ ratio,
                const float* __restrict__ em, const float* __restrict__ theta,
                float* __restrict__ out, int A, int B, int R, int H, int W, int apc,
                float clamp_min, int stage_tile, int bwd_mode, int ncopy, int seg) {
    extern __shared__ __align__(16) float smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int b = blockIdx.y;
    const int a0 = blockIdx.x * apc, a1 = min(A, a0 + apc);
    const int pitch = slice_pitch(W);
    const int HW = H * W;
    const int img_stride = H * pitch;
    float* sA = smem;
    float* sacc = sA + (stage_tile ? ((HW + 3) & ~3) : 0);
    float* sframe = sacc + R * img_stride;                   // ncopy x [R][2][W + H]
    float* srow = sframe + ((threadIdx.x >> 5) % ncopy) * 2 * R * (H + W);
    float* scol = srow + 2 * R * W;
    float* sratio = sframe + frame_floats(R, H, W, ncopy);
    float* sem = sratio + W;
    const bool vec = stage_tile && ((HW & 3) == 0) && (((uintptr_t)atten & 15) == 0);
    for (int i = threadIdx.x; i < R * img_stride + frame_floats(R, H, W, ncopy); i += blockDim.x)
        sacc[i] = 0.f;
    const int wk_dh = blockDim.x / W, wk_dw = blockDim.x - wk_dh * W;
    const int wk_h0 = threadIdx.x / W, wk_w0 = threadIdx.x - wk_h0 * W;
    Corners cs;
    cs.zero();
    TileRegs tr;
    if (a0 < a1 && vec) tile_issue(tr, atten + ((int64_t)a0 * B + b) * HW, HW);
    for (int a = a0; a < a1; ++a) {
        const float* src = atten + ((int64_t)a * B + b) * HW;
        __syncthreads();
        if (vec) tile_commit(tr, src, sA, HW);
        else if (stage_tile) tile_copy(src, sA, HW);
        if (threadIdx.x < R) sem[threadIdx.x] = em[a * R + threadIdx.x];
        for (int w = threadIdx.x; w < W; w += blockDim.x)
            sratio[w] = ratio ? ratio[((int64_t)a * B + b) * W + w] : 1.f;
        __syncthreads();
        if (a + 1 < a1 && vec) tile_issue(tr, atten + ((int64_t)(a + 1) * B + b) * HW, HW);
        if (RC == 1 && bwd_mode == 3 && stage_tile)
            backward_angle_gather(sA, sratio, sem[0], sacc, srow, scol, pitch,
                                  make_geo(theta[a], H, W), H, W, cs, wk_dh, wk_dw, wk_h0, wk_w0);
        else if (bwd_mode == 4)
            backward_angle_seg<RC>(stage_tile ? sA : src, sratio, sacc, srow, scol, img_stride,
                                   pitch, sem, R, make_geo(theta[a], H, W), H, W, cs, seg);
        else if (bwd_mode != 1)
            backward_angle<RC>(stage_tile ? sA : src, sratio, sacc, srow, scol, img_stride, pitch,
                               sem, R, make_geo(theta[a], H, W), H, W, cs);
        else
            backward_angle_atomic<RC>(stage_tile ? sA : src, sratio, sacc, img_stride, pitch, sem,
                                      R, make_geo(theta[a], H, W), H, W, cs, wk_dh, wk_dw, wk_h0,
                                      wk_w0);
    }
    fold_frame(cs, sacc, sframe, ncopy, img_stride, pitch, R, H, W);
    cluster.sync();
    cluster_reduce(cluster, sacc, R, H, W, pitch, [&](int r, int h, int w, float s) {
        if (clamp_min > 0.f) s = fmaxf(s, clamp_min);
        out[(((int64_t)r * B + b) * H + h) * W + w] = s;
    });
    cluster.sync();
}

// ---------------------------------------------------------------------------
// One fused MLEM iteration (grid (G, B), cluster (G,1,1)):
//   Pf = max(P C, 1e-6); ratio = I / Pf; back = P^T ratio;
//   C' = C*back / (sens + beta*huber(C))  (or C*back/sens), C' = max(C', 0)
// as atten_cuda.cpp:321-342.  Reads C from Cin, writes Cout (ping-pong: the
// Huber term needs the old neighbours).
// ---------------------------------------------------------------------------
template <int RC>
__global__ void __launch_bounds__(kThreads, 1)
mlem_iter_kernel(const float* __restrict__ atten, const float* __restrict__ em,
                 const float* __restrict__ theta, const float* __restrict__ I,
                 const float* __restrict__ sens, const float* __restrict__ Cin,
                 float* __restrict__ Cout, int A, int B, int R, int H, int W, int apc,
                 float beta, float delta, int bwd_mode, int ncopy, int seg) {
    extern __shared__ __align__(16) float smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int b = blockIdx.y;
    const int a0 = blockIdx.x * apc, a1 = min(A, a0 + apc);
    const int pitch = slice_pitch(W);
    const int parts = col_parts(W, H);
    const int HW = H * W;
    const int img_stride = H * pitch;
    float* sA = smem;
    float* sC = sA + ((HW + 3) & ~3);
    float* sacc = sC + R * img_stride;
    float* sframe = sacc + R * img_stride;                   // ncopy x [R][2][W + H]
    float* srow = sframe + ((threadIdx.x >> 5) % ncopy) * 2 * R * (H + W);
    float* scol = srow + 2 * R * W;
    float* spart = sframe + frame_floats(R, H, W, ncopy);
    float* sratio = spart + parts * W;
    float* sem = sratio + W;
    const bool vec = ((HW & 3) == 0) && (((uintptr_t)atten & 15) == 0);
    stage_slice(sC, Cin, R, B, b, H, W, pitch);
    for (int i = threadIdx.x; i < R * img_stride + frame_floats(R, H, W, ncopy); i += blockDim.x)
        sacc[i] = 0.f;
    const int wk_dh = blockDim.x / W, wk_dw = blockDim.x - wk_dh * W;
    const int wk_h0 = threadIdx.x / W, wk_w0 = threadIdx.x - wk_h0 * W;
    Corners cs;
    cs.zero();
    TileRegs tr;
    if (a0 < a1 && vec) tile_issue(tr, atten + ((int64_t)a0 * B + b) * HW, HW);
    for (int a = a0; a < a1; ++a) {
        const float* src = atten + ((int64_t)a * B + b) * HW;
        __syncthreads();
        if (vec) tile_commit(tr, src, sA, HW); else tile_copy(src, sA, HW);
        if (threadIdx.x < R) sem[threadIdx.x] = em[a * R + threadIdx.x];
        __syncthreads();
        if (a + 1 < a1 && vec) tile_issue(tr, atten + ((int64_t)(a + 1) * B + b) * HW, HW);
        const Geo g = make_geo(theta[a], H, W);
        forward_angle(sA, sC, img_stride, pitch, sem, R, g, H, W, parts, spart);
        __syncthreads();
        for (int w = threadIdx.x; w < W; w += blockDim.x) {
            float s = 0.f;
            for (int p = 0; p < parts; ++p) s += spart[p * W + w];
            sratio[w] = I[((int64_t)a * B + b) * W + w] / fmaxf(s, 1e-6f);
        }
        __syncthreads();
        if (RC == 1 && bwd_mode == 3)
            backward_angle_gather(sA, sratio, sem[0], sacc, srow, scol, pitch, g, H, W, cs, wk_dh,
                                  wk_dw, wk_h0, wk_w0);
        else if (bwd_mode == 4)
            backward_angle_seg<RC>(sA, sratio, sacc, srow, scol, img_stride, pitch, sem, R, g, H, W,
                                   cs, seg);
        else if (bwd_mode != 1)
            backward_angle<RC>(sA, sratio, sacc, srow, scol, img_stride, pitch, sem, R, g, H, W,
                               cs);
        else
            backward_angle_atomic<RC>(sA, sratio, sacc, img_stride, pitch, sem, R, g, H, W, cs,
                                      wk_dh, wk_dw, wk_h0, wk_w0);
    }
    fold_frame(cs, sacc, sframe, ncopy, img_stride, pitch, R, H, W);
    cluster.sync();
    cluster_reduce(cluster, sacc, R, H, W, pitch, [&](int r, int h, int w, float back) {
        const float* img = sC + r * img_stride;
        const float cp = img[h * pitch + w];
        const int64_t gi = (((int64_t)r * B + b) * H + h) * W + w;
        float den = sens[gi];
        if (beta > 0.f) {
            float hg = 0.f;
            if (h > 0) { float d = cp - img[(h - 1) * pitch + w]; hg += fabsf(d) <= delta ? d : copysignf(delta, d); }
            if (h + 1 < H) { float d = cp - img[(h + 1) * pitch + w]; hg += fabsf(d) <= delta ? d : copysignf(delta, d); }
            if (w > 0) { float d = cp - img[h * pitch + w - 1]; hg += fabsf(d) <= delta ? d : copysignf(delta, d); }
            if (w + 1 < W) { float d = cp - img[h * pitch + w + 1]; hg += fabsf(d) <= delta ? d : copysignf(delta, d); }
            den = __fadd_rn(den, __fmul_rn(beta, hg));
        }
        Cout[gi] = fmaxf(__fmul_rn(cp, back) / den, 0.f);
    });
    cluster.sync();
}

// ===========================================================================
// The lean projector kernels (default): forward (+ MLEM ratio) and backward
// (+ sensitivity clamp or MLEM update), each sized so that three CTAs share
// an SM -- one slice image in shared memory per CTA, no attenuation tile --
// so that one CTA's barriers and shared-memory latencies are covered by the
// other two.  An MLEM iteration is the two launches; the attenuation is read
// by each (the bytes the reference's forward and backward calls read).
// ===========================================================================
constexpr int kT2 = 256;      // threads per CTA of the lean kernels
constexpr int kFwdU = 8;      // attenuation loads issued together in the forward
constexpr int kSegU = 8;      // ... and in a backward segment walk

// Partial column sums of one (angle, slice) for the lean kernels: work item =
// (column w, part p); the thread sums atten(h, w) * sum_r em_r bilerp(C_r)
// over the part's rows of column w into sp[p][w].  A warp's loads of atten
// run along w (coalesced); batch j of kFwdU rows is loaded while batch j - 1
// is computed.  em_a: the angle's R emission values (RC == 1: unused, the
// caller scales the column sums).
template <int RC, int WC>
__device__ __forceinline__ void fwd_angle2(const float* __restrict__ at, const float* sC, int img,
                                           int pitch, const float* __restrict__ em_a, int R,
                                           const Geo& g, int H, int Wrt, int parts, float* sp) {
    const int W = WC > 0 ? WC : Wrt;       // a compile-time width makes the row strides immediates
    const int hper = (H + parts - 1) / parts;
    const int nitems = parts * W;
    for (int item = threadIdx.x; item < nitems; item += blockDim.x) {
        const int part = item / W, w = item - part * W;
        const int h0 = part * hper, n = min(H, h0 + hper) - h0;
        if (n <= 0) {                      // a part past the last row
            sp[part * W + w] = 0.f;
            continue;
        }
        const float bx = col_bx(g, w), by = col_by(g, w);
        const float* ap = at + (int64_t)h0 * W + w;
        float acc = 0.f;
        float hf = (float)h0 - g.cy;
        // rows past the part have weight 0
        float cur[kFwdU], nxt[kFwdU];
#pragma unroll
        for (int k = 0; k < kFwdU; ++k) cur[k] = k < n ? __ldg(ap + (int64_t)k * W) : 0.f;
        auto walk = [&]() {
#pragma unroll
            for (int k = 0; k < kFwdU; ++k) {
                const Smp s = sample_xy(g, fmaf(g.c, hf, bx), fmaf(g.s, hf, by));
                hf += 1.f;
                float v;
                if (RC == 1) {
                    v = bilerp(sC, pitch, s);
                } else {
                    v = 0.f;
                    for (int r = 0; r < R; ++r)
                        v = fmaf(__ldg(em_a + r), bilerp(sC + r * img, pitch, s), v);
                }
                acc = fmaf(cur[k], v, acc);
            }
#pragma unroll
            for (int k = 0; k < kFwdU; ++k) cur[k] = nxt[k];
        };
        int j = 0;
        // the next batch lies inside the part: its loads need no bound
        for (; j + 2 * kFwdU <= n; j += kFwdU) {
            const float* an = ap + (int64_t)(j + kFwdU) * W;
#pragma unroll
            for (int k = 0; k < kFwdU; ++k) nxt[k] = __ldg(an + (int64_t)k * W);
            walk();
        }
        for (; j < n; j += kFwdU) {
#pragma unroll
            for (int k = 0; k < kFwdU; ++k) {
                const int r = j + kFwdU + k;
                nxt[k] = r < n ? __ldg(ap + (int64_t)r * W) : 0.f;
            }
            walk();
        }
        sp[part * W + w] = acc;
    }
}

// Column sums of the partials (fixed order) -> Pf, or the MLEM ratio
// I / max(Pf, 1e-6) when I != nullptr (atten_cuda.cpp:326-329).
__device__ __forceinline__ void fwd_finish(const float* sp, int parts, int W, float scale,
                                           const float* __restrict__ I, float* __restrict__ out,
                                           int64_t row) {
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        float s = 0.f;
        for (int p = 0; p < parts; ++p) s += sp[p * W + w];
        s *= scale;
        const int64_t o = row * W + w;
        if (I) s = I[o] / fmaxf(s, 1e-6f);
        out[o] = s;
    }
}

// Forward: grid (angle groups, B).  The CTA stages slice b of C (R images,
// row pitch == 9 mod 32) and walks its angles (fwd_angle2).  The partial sums
// are double buffered, so an angle costs one barrier.  I != nullptr: out =
// I / max(Pf, 1e-6) (the MLEM ratio), else out = Pf.
template <int RC, int WC>
__global__ void __launch_bounds__(kT2, 3)
proj_fwd2_kernel(const float* __restrict__ atten, const float* __restrict__ C,
                 const float* __restrict__ em, const float* __restrict__ theta,
                 float* __restrict__ out, const float* __restrict__ I, int A, int B, int Rrt,
                 int H, int Wrt, int apc, int parts) {
    extern __shared__ __align__(16) float smem[];
    const int W = WC > 0 ? WC : Wrt;
    const int R = RC > 0 ? RC : Rrt;
    const int b = blockIdx.y;
    const int a0 = blockIdx.x * apc, a1 = min(A, a0 + apc);
    const int pitch = slice_pitch(W);
    const int img = H * pitch;
    float* sC = smem;                      // [R][H][pitch]
    float* spart = sC + R * img;           // [2][parts][W]
    stage_slice(sC, C, R, B, b, H, W, pitch);
    __syncthreads();
    for (int a = a0; a < a1; ++a) {
        const Geo g = make_geo(theta[a], H, W);
        float* sp = spart + (a & 1) * parts * W;
        fwd_angle2<RC, WC>(atten + ((int64_t)a * B + b) * H * W, sC, img, pitch,
                           em + (int64_t)a * R, R, g, H, W, parts, sp);
        __syncthreads();
        fwd_finish(sp, parts, W, RC == 1 ? __ldg(em + (int64_t)a * R) : 1.f, I, out,
                   (int64_t)a * B + b);
        // the next angle writes the other partial buffer; the one after it
        // writes this buffer again only past the next barrier
    }
}

// The per-angle weights q[r][w] = ratio(a, b, w) * em(a, r) of the backward
// (ratio == nullptr: ratio = 1, the sensitivity P^T 1).
__device__ __forceinline__ void stage_q(float* sq, const float* __restrict__ ratio,
                                        const float* __restrict__ em, int a, int b, int B, int R,
                                        int W) {
    for (int i = threadIdx.x; i < R * W; i += blockDim.x) {
        const int r = i / W, w = i - r * W;
        const float rq = ratio ? __ldg(ratio + ((int64_t)a * B + b) * W + w) : 1.f;
        sq[i] = rq * __ldg(em + (int64_t)a * R + r);
    }
}

// Splats samples h0 <= h < h1 of column w (one angle) into sacc: unclamped
// samples with plain read-modify-writes (the caller's phases keep concurrent
// footprints disjoint), clamped ones into the frame buffers.  The segment's
// attenuation values are loaded kSegU at a time before any of them is used.
// (Taking the clamped samples out of the phases -- into the threads a phase
// leaves idle, or into a pass over all threads after each angle -- measured
// slower: 2.53 and 1.92 ms against 1.56 ms for the backward of 120 angles x
// 128 slices of 128^2; without any clamped samples it would run 1.22 ms.
// Adding every footprint on the border frame with shared atomics straight
// into the image, without frame buffers, measured 1.79 against 1.40 ms: the
// clamped samples crowd onto a few border pixels.
// Splitting each segment into its clamped ends and a clamp-free run between
// them -- exact, since the sample coordinates are monotone along a column --
// measured 2.10 ms against 1.40: three short runs per segment of 13 samples
// break up the batched loads.)
template <int RC, int WC>
__device__ __forceinline__ void bwd_segment(const float* __restrict__ at, const float* q,
                                            float* sacc, float* srow, float* scol, int img,
                                            int pitch, int R, const Geo& g, int H, int Wrt, int w,
                                            int h0, int h1, Corners& cs) {
    const int W = WC > 0 ? WC : Wrt;       // a compile-time width makes the row strides immediates
    const float bx = col_bx(g, w), by = col_by(g, w);
    const float q0 = q[w];
    const float* ap = at + (int64_t)h0 * W + w;
    const int n = h1 - h0;
    float hf = (float)h0 - g.cy;
    for (int j = 0; j < n; j += kSegU) {
        float av[kSegU];
        const float* aj = ap + (int64_t)j * W;
        if (j + kSegU <= n) {
#pragma unroll
            for (int k = 0; k < kSegU; ++k) av[k] = __ldg(aj + (int64_t)k * W);
        } else {
#pragma unroll
            for (int k = 0; k < kSegU; ++k) av[k] = j + k < n ? __ldg(aj + (int64_t)k * W) : 0.f;
        }
#pragma unroll
        for (int k = 0; k < kSegU; ++k) {
            if (j + k >= n) break;
            const float x = fmaf(g.c, hf, bx), y = fmaf(g.s, hf, by);
            hf += 1.f;
            const float xc = fminf(fmaxf(x, 0.f), g.rmax), yc = fminf(fmaxf(y, 0.f), g.cmax);
            float fx, fy;
            const int i0 = ffloor(xc, fx), j0 = ffloor(yc, fy);
            if (x == xc && y == yc) {
                if (RC == 1) {
                    const float v = av[k] * q0;
                    const float ra = v * fx, rb = v - ra;     // row i0+1, row i0
                    const float a1 = ra * fy, b1 = rb * fy;   // their column j0+1 parts
                    float* p = sacc + i0 * pitch + j0;
                    const float p0 = p[0], p1 = p[1], p2 = p[pitch], p3 = p[pitch + 1];
                    p[0] = p0 + (rb - b1);
                    p[1] = p1 + b1;
                    p[pitch] = p2 + (ra - a1);
                    p[pitch + 1] = p3 + a1;
                } else {
                    for (int r = 0; r < R; ++r) {
                        const float v = av[k] * q[r * W + w];
                        const float ra = v * fx, rb = v - ra;
                        const float a1 = ra * fy, b1 = rb * fy;
                        float* p = sacc + r * img + i0 * pitch + j0;
                        p[0] += rb - b1;
                        p[1] += b1;
                        p[pitch] += ra - a1;
                        p[pitch + 1] += a1;
                    }
                }
            } else {
                Foot f;
                f.i0 = i0;
                f.j0 = j0;
                f.fx = fx;
                f.fy = fy;
                f.kind = (x < 0.f ? 1 : 0) | (x > g.rmax ? 2 : 0) | (y < 0.f ? 4 : 0) |
                         (y > g.cmax ? 8 : 0);
                if (RC == 1) {
                    frame_add<false>(f, av[k] * q0, srow, scol, H, W, cs, 0);
                } else {
                    for (int r = 0; r < R; ++r)
                        frame_add<false>(f, av[k] * q[r * W + w], srow, scol, H, W, cs, r);
                }
            }
        }
    }
}

// Splats angles [a0, a1) of slice b into this CTA's shared-memory image of
// the slice (zeroed first) in six phases per angle ((w mod 3) x (segment
// parity), column segments of `seg` samples; see backward_angle_seg), with
// the clamped samples in the frame buffers, which are folded into the image
// at the end.  q = ratio * em of each angle is staged during the previous
// angle's last phase (ratio == nullptr: 1).
template <int RC, int WC>
__device__ void bwd_splat_angles(const float* __restrict__ atten, const float* __restrict__ ratio,
                                 const float* __restrict__ em, const float* __restrict__ theta,
                                 float* sacc, float* sframe, float* sq, int ncopy, int a0, int a1,
                                 int b, int B, int R, int H, int Wrt, int seg) {
    const int W = WC > 0 ? WC : Wrt;
    const int pitch = slice_pitch(W);
    const int img = H * pitch;
    float* srow = sframe + ((threadIdx.x >> 5) % ncopy) * 2 * R * (H + W);
    float* scol = srow + 2 * R * W;
    for (int i = threadIdx.x; i < R * img; i += blockDim.x) sacc[i] = 0.f;
    for (int i = threadIdx.x; i < frame_floats(R, H, W, ncopy); i += blockDim.x) sframe[i] = 0.f;
    if (a0 < a1) stage_q(sq + (a0 & 1) * R * W, ratio, em, a0, b, B, R, W);
    __syncthreads();
    Corners cs;
    cs.zero();
    const int nseg = (H + seg - 1) / seg;
    for (int a = a0; a < a1; ++a) {
        const Geo g = make_geo(theta[a], H, W);
        const float* at = atten + ((int64_t)a * B + b) * H * W;
        const float* q = sq + (a & 1) * R * W;
        for (int ph = 0; ph < 6; ++ph) {
            const int pw = ph >> 1, ps = ph & 1;
            const int nw = (W - pw + 2) / 3, nsp = (nseg - ps + 1) / 2;
            const int items = nw * nsp;
            // (dynamic fetching of the items by warps, with shorter segments,
            // measured slower here: 1.49-1.58 against 1.45 ms; the band
            // kernel, whose line windows differ in length, uses it.  Three
            // phases per angle -- every segment of a column class at once,
            // the two samples at each inner segment end added with shared
            // atomics -- measured 1.463 against 1.474 ms with the same
            // per-sample test in both: the barriers are not what bounds it)
            for (int it = threadIdx.x; it < items; it += blockDim.x) {
                const int k = it / nw, cw = it - k * nw;
                const int h0 = (ps + 2 * k) * seg;
                bwd_segment<RC, WC>(at, q, sacc, srow, scol, img, pitch, R, g, H, W, pw + 3 * cw,
                                    h0, min(H, h0 + seg), cs);
            }
            // the other q buffer was last read in the previous angle
            if (ph == 5 && a + 1 < a1) stage_q(sq + ((a + 1) & 1) * R * W, ratio, em, a + 1, b, B, R, W);
            __syncthreads();
        }
    }
    fold_frame(cs, sacc, sframe, ncopy, img, pitch, R, H, W);
}

// Epilogue of a reduced back-projection pixel s of (r, b, h, w):
//   mode 0: out = s, or max(s, clamp_min) when clamp_min > 0;
//   mode 1: MLEM update out = max(Cin*s / (sens + beta*huber(Cin)), 0)
//           (atten_cuda.cpp:331-341), Cin and sens (R,B,H,W) in global memory.
__device__ __forceinline__ void bwd_epilogue(int mode, float* __restrict__ out,
                                             const float* __restrict__ Cin,
                                             const float* __restrict__ sens, float clamp_min,
                                             float beta, float delta, int r, int b, int B, int H,
                                             int W, int h, int w, float s) {
    const int64_t gi = (((int64_t)r * B + b) * H + h) * W + w;
    if (mode == 0) {
        out[gi] = clamp_min > 0.f ? fmaxf(s, clamp_min) : s;
        return;
    }
    const float* ci = Cin + ((int64_t)r * B + b) * H * W;
    const float cp = ci[h * W + w];
    float den = sens[gi];
    if (beta > 0.f) {
        float hg = 0.f;
        if (h > 0) { float d = cp - ci[(h - 1) * W + w]; hg += fabsf(d) <= delta ? d : copysignf(delta, d); }
        if (h + 1 < H) { float d = cp - ci[(h + 1) * W + w]; hg += fabsf(d) <= delta ? d : copysignf(delta, d); }
        if (w > 0) { float d = cp - ci[h * W + w - 1]; hg += fabsf(d) <= delta ? d : copysignf(delta, d); }
        if (w + 1 < W) { float d = cp - ci[h * W + w + 1]; hg += fabsf(d) <= delta ? d : copysignf(delta, d); }
        den = __fadd_rn(den, __fmul_rn(beta, hg));
    }
    out[gi] = fmaxf(__fmul_rn(cp, s) / den, 0.f);
}

// Backward with an epilogue: grid (G, B), cluster (G, 1, 1).  CTA g of slice b
// splats angles [g*apc, (g+1)*apc) (bwd_splat_angles); the cluster then sums
// its G images over DSMEM in rank order and applies bwd_epilogue.
template <int RC, int WC>
__global__ void __launch_bounds__(kT2, 3)
proj_bwd2_kernel(const float* __restrict__ atten, const float* __restrict__ ratio,
                 const float* __restrict__ em, const float* __restrict__ theta,
                 float* __restrict__ out, const float* __restrict__ Cin,
                 const float* __restrict__ sens, int A, int B, int Rrt, int H, int Wrt, int apc,
                 int seg, int ncopy, float clamp_min, int mode, float beta, float delta) {
    extern __shared__ __align__(16) float smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int R = RC > 0 ? RC : Rrt;
    const int W = WC > 0 ? WC : Wrt;
    const int b = blockIdx.y;
    const int a0 = blockIdx.x * apc, a1 = min(A, a0 + apc);
    const int pitch = slice_pitch(W);
    float* sacc = smem;                                     // [R][H][pitch]
    float* sframe = sacc + R * H * pitch;                   // ncopy x [R][2][W + H]
    float* sq = sframe + frame_floats(R, H, W, ncopy);      // [2][R][W]
    bwd_splat_angles<RC, WC>(atten, ratio, em, theta, sacc, sframe, sq, ncopy, a0, a1, b, B, R, H,
                             W, seg);
    cluster.sync();
    cluster_reduce(cluster, sacc, R, H, W, pitch, [&](int r, int h, int w, float s) {
        bwd_epilogue(mode, out, Cin, sens, clamp_min, beta, delta, r, b, B, H, W, h, w, s);
    });
    cluster.sync();
}

// ---------------------------------------------------------------------------
// Band backward, for slices whose image does not fit in shared memory: grid
// (G * nband, B), cluster (G, 1, 1).  CTA (band, g) of slice b owns the image
// rows [r0, r1) = [band*hb, band*hb + hb) and splats angles [g*apc, ...) of
// the samples whose footprint starts on a row i0 in [r0-1, r1-1] into a band
// image of rows r0-1 .. r1 (the two halo rows take the halves of footprints
// that belong to the neighbouring bands and are dropped).  Every footprint row
// is thus added by exactly the band that owns it, with plain shared-memory
// read-modify-writes: no global atomics.  Within an angle the samples are
// walked along lines -- sample columns when |cos| >= |sin|, else sample rows,
// so that a line crosses the band in at most (hb+1)*sqrt(2) + 6 samples --
// in six phases (line mod 3 x segment parity), as bwd_splat_angles does; x(h)
// and y(h) are computed by the forward's expressions, so each sample's
// weights, band and clamp class are the forward's.  Clamped samples go to
// band-local frame buffers (the column part indexed by local row), folded in
// at the end.  The cluster reduces the band over DSMEM and applies
// bwd_epilogue (mode 0: back-projection, mode 1: MLEM update).
// ---------------------------------------------------------------------------
template <int RC>
__device__ __forceinline__ void band_segment(const float* __restrict__ at, const float* q,
                                             float* sacc, float* srow, float* scol, int img,
                                             int pitch, int R, const Geo& g, int H, int W,
                                             int nrow, bool colmode, int L, int p0, int p1, int r0,
                                             Corners& cs) {
    // colmode: line = sample column w = L, position = h; else line = sample row h = L
    const float hfL = (float)L - g.cy;
    const float bxL = col_bx(g, L), byL = col_by(g, L);
    const int lmax = nrow - 2;           // local i0 in [0, nrow - 2]
    // attenuation address of position p: base + p * step
    const float* ap = colmode ? at + L : at + (int64_t)L * W;
    const int64_t step = colmode ? W : 1;
    const int n = p1 - p0;
    for (int j = 0; j < n; j += kSegU) {
        // the attenuation values of the next kSegU positions, loaded before
        // any is used (the loads of positions outside the band are wasted)
        float av[kSegU];
#pragma unroll
        for (int k = 0; k < kSegU; ++k) av[k] = __ldg(ap + (int64_t)(p0 + min(j + k, n - 1)) * step);
#pragma unroll
        for (int k = 0; k < kSegU; ++k) {
            if (j + k >= n) break;
            const int p = p0 + j + k;
            const int w = colmode ? L : p;
            float x, y;
            if (colmode) {
                const float hf = (float)p - g.cy;
                x = fmaf(g.c, hf, bxL);
                y = fmaf(g.s, hf, byL);
            } else {
                x = fmaf(g.c, hfL, col_bx(g, p));
                y = fmaf(g.s, hfL, col_by(g, p));
            }
            const float xc = fminf(fmaxf(x, 0.f), g.rmax), yc = fminf(fmaxf(y, 0.f), g.cmax);
            float fx, fy;
            const int i0 = ffloor(xc, fx), j0 = ffloor(yc, fy);
            const int li = i0 - r0 + 1;
            if ((unsigned)li > (unsigned)lmax) continue;
            if (x == xc && y == yc) {
                for (int r = 0; r < (RC > 0 ? RC : R); ++r) {
                    const float v = av[k] * q[r * W + w];
                    const float ra = v * fx, rb = v - ra;
                    const float a1 = ra * fy, b1 = rb * fy;
                    float* pp = sacc + r * img + li * pitch + j0;
                    const float s0 = pp[0], s1 = pp[1], s2 = pp[pitch], s3 = pp[pitch + 1];
                    pp[0] = s0 + (rb - b1);
                    pp[1] = s1 + b1;
                    pp[pitch] = s2 + (ra - a1);
                    pp[pitch + 1] = s3 + a1;
                }
            } else {
                Foot f;
                f.i0 = li;
                f.j0 = j0;
                f.fx = fx;
                f.fy = fy;
                f.kind = (x < 0.f ? 1 : 0) | (x > g.rmax ? 2 : 0) | (y < 0.f ? 4 : 0) |
                         (y > g.cmax ? 8 : 0);
                for (int r = 0; r < (RC > 0 ? RC : R); ++r)
                    frame_add<false>(f, av[k] * q[r * W + w], srow, scol, nrow, W, cs, r);
            }
        }
    }
}

// Adds the band's frame buffers into its image: the row part (slot 0: image
// row 0, slot 1: rows ih, ih+1 split by (1 - fxh, fxh)) where those rows lie
// in the band image, the column part (slot 0: column 0, slot 1: columns jh,
// jh+1) on every local row.
__device__ void band_fold(float* sacc, const float* sframe, int ncopy, int img, int pitch, int R,
                          int H, int W, int nrow, int r0) {
    __syncthreads();
    const Geo g0 = make_geo(0.f, H, W);
    const int copy = 2 * R * (nrow + W);
    const int l_lo = 0 - r0 + 1, l_hi = g0.ih - r0 + 1;
    for (int t = threadIdx.x; t < R * W; t += blockDim.x) {
        const int r = t / W, j = t - r * W;
        float lo = 0.f, hi = 0.f;
        for (int c = 0; c < ncopy; ++c) {
            lo += sframe[c * copy + 2 * r * W + j];
            hi += sframe[c * copy + 2 * r * W + W + j];
        }
        float* im = sacc + r * img + j;
        if (l_lo >= 0 && l_lo < nrow) im[l_lo * pitch] += lo;
        if (l_hi >= 0 && l_hi < nrow) im[l_hi * pitch] += hi * (1.f - g0.fxh);
        if (l_hi + 1 >= 0 && l_hi + 1 < nrow) im[(l_hi + 1) * pitch] += hi * g0.fxh;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < R * nrow; t += blockDim.x) {
        const int r = t / nrow, l = t - r * nrow;
        float lo = 0.f, hi = 0.f;
        for (int c = 0; c < ncopy; ++c) {
            lo += sframe[c * copy + 2 * R * W + 2 * r * nrow + l];
            hi += sframe[c * copy + 2 * R * W + 2 * r * nrow + nrow + l];
        }
        float* im = sacc + r * img + l * pitch;
        im[0] += lo;
        im[g0.jh] += hi * (1.f - g0.fyh);
        im[g0.jh + 1] += hi * g0.fyh;
    }
    __syncthreads();
}

template <int RC>
__global__ void __launch_bounds__(kT2, 3)
proj_bwd_band_kernel(const float* __restrict__ atten, const float* __restrict__ ratio,
                     const float* __restrict__ em, const float* __restrict__ theta,
                     float* __restrict__ out, const float* __restrict__ Cin,
                     const float* __restrict__ sens, int A, int B, int Rrt, int H, int W, int apc,
                     int hb, int seg, int ncopy, float clamp_min, int mode, float beta,
                     float delta) {
    extern __shared__ __align__(16) float smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int R = RC > 0 ? RC : Rrt;
    const int G = (int)cluster.num_blocks(), rank = (int)cluster.block_rank();
    const int band = blockIdx.x / G, b = blockIdx.y;
    const int r0 = band * hb, r1 = min(H, r0 + hb);
    const int nrow = r1 - r0 + 2;
    const int a0 = rank * apc, a1 = min(A, a0 + apc);
    const int pitch = slice_pitch(W);
    const int img = nrow * pitch;
    float* sacc = smem;                                          // [R][nrow][pitch]
    float* sframe = sacc + R * img;                              // ncopy x [R][2][W + nrow]
    float* sq = sframe + frame_floats(R, nrow, W, ncopy);        // [2][R][W]
    float* srow = sframe + ((threadIdx.x >> 5) % ncopy) * 2 * R * (nrow + W);
    float* scol = srow + 2 * R * W;
    __shared__ int s_ctr[2][6];             // per-phase item counters by angle parity
    if (threadIdx.x < 12) s_ctr[threadIdx.x / 6][threadIdx.x % 6] = 0;
    const int lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < R * img; i += blockDim.x) sacc[i] = 0.f;
    for (int i = threadIdx.x; i < frame_floats(R, nrow, W, ncopy); i += blockDim.x) sframe[i] = 0.f;
    if (a0 < a1) stage_q(sq + (a0 & 1) * R * W, ratio, em, a0, b, B, R, W);
    __syncthreads();
    Corners cs;
    cs.zero();
    // the band's x window: i0 in [r0-1, r1-1], i.e. the clamped x in [r0-1, r1);
    // x < 0 clamps to row 0 (i0 = 0) and x > rmax to i0 = ih = H-2
    const float xlo = r0 <= 1 ? -INFINITY : (float)(r0 - 1);
    const float xhi = r1 >= H - 1 ? INFINITY : (float)r1;
    for (int a = a0; a < a1; ++a) {
        const Geo g = make_geo(theta[a], H, W);
        const float* at = atten + ((int64_t)a * B + b) * H * W;
        const float* q = sq + (a & 1) * R * W;
        const bool colmode = fabsf(g.c) >= fabsf(g.s);
        const int nlines = colmode ? W : H, len = colmode ? H : W;
        // dx / d(position) along a line, and x at position 0 of line L:
        //   colmode x = c (h - cy) + bx(w);  else x = c (h - cy) - s (w - cx) + cy
        const float slope = colmode ? g.c : -g.s;
        const float islope = 1.f / slope;
        // the window [plo, phi) of line L: positions whose x lies in the
        // band's x window, two positions of margin on each side
        auto window = [&](int L, float& plo, float& phi) {
            const float x0 = colmode ? fmaf(g.c, -g.cy, col_bx(g, L))
                                     : fmaf(g.c, (float)L - g.cy, col_bx(g, 0));
            const float t1 = (xlo - x0) * islope, t2 = (xhi - x0) * islope;
            plo = fmaxf(floorf(fminf(t1, t2)) - 2.f, 0.f);
            phi = fminf(ceilf(fmaxf(t1, t2)) + 3.f, (float)len);
        };
        int nsegs = (len + seg - 1) / seg;
        if (xlo > -INFINITY && xhi < INFINITY) {
            // a window inside the line is at most (xhi - xlo) / |slope| + 7 long
            const int span = (int)((xhi - xlo) * fabsf(islope)) + 9;
            nsegs = min(nsegs, (span + seg - 1) / seg);
        }
        // (180 angles x 64 slices of 256^2: 9.43 ms with 6-sample segments
        // fetched dynamically, 9.87 / 9.98 ms with 4 / 8; 12.5 ms with
        // 16-sample segments assigned statically, 14.1 ms with longer ones
        // fitting one round of the block -- the line windows differ in length
        // and a static phase waits for the longest; 9.4 ms for the
        // global-atomic kernel this replaced.)
        if (threadIdx.x < 6) s_ctr[(a + 1) & 1][threadIdx.x] = 0;
        for (int ph = 0; ph < 6; ++ph) {
            const int pw = ph >> 1, ps = ph & 1;
            const int nl = (nlines - pw + 2) / 3, nsp = (nsegs - ps + 1) / 2;
            const int items = nl * nsp;
            // the phase's items touch disjoint pixels, so any warp may take
            // any of them: the warps take 32 at a time from the phase's
            // counter, and a warp whose lines have short windows in the band
            // takes more (blockDim.x is a multiple of 32)
            for (;;) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&s_ctr[a & 1][ph], 32);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base >= items) break;
                const int it = base + lane;
                if (it >= items) continue;
                const int k = it / nl, cl = it - k * nl;
                const int L = pw + 3 * cl;
                float plo, phi;
                window(L, plo, phi);
                if (!(plo < phi)) continue;
                const int p0 = (int)plo + (ps + 2 * k) * seg;
                const int p1 = min((int)phi, p0 + seg);
                if (p0 >= p1) continue;
                band_segment<RC>(at, q, sacc, srow, scol, img, pitch, R, g, H, W, nrow, colmode,
                                 L, p0, p1, r0, cs);
            }
            if (ph == 5 && a + 1 < a1) stage_q(sq + ((a + 1) & 1) * R * W, ratio, em, a + 1, b, B, R, W);
            __syncthreads();
        }
    }
    band_fold(sacc, sframe, ncopy, img, pitch, R, H, W, nrow, r0);
    cluster.sync();
    // reduce the band's own rows (local 1 .. nrow-2) over the cluster
    const int64_t n = (int64_t)R * (r1 - r0) * W;
    const int64_t share = (n + G - 1) / G;
    const int64_t i0 = rank * share, i1 = min(n, i0 + share);
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const int r = (int)(i / ((int64_t)(r1 - r0) * W));
        const int rem = (int)(i - (int64_t)r * (r1 - r0) * W);
        const int l = rem / W, w = rem - l * W;
        const int off = r * img + (l + 1) * pitch + w;
        float s = 0.f;
        for (int qq = 0; qq < G; ++qq) s += cluster.map_shared_rank(sacc, qq)[off];
        bwd_epilogue(mode, out, Cin, sens, clamp_min, beta, delta, r, b, B, H, W, r0 + l, w, s);
    }
    cluster.sync();
}

// ---------------------------------------------------------------------------
// Persistent MLEM over several problems (a problem: one element's -- or one
// volume's -- C, atten, em, theta, I; all with the same R; every problem of
// one launch with the same slice width W, which WC > 0 fixes at compile
// time).  Work item = (problem, slice); the clusters of G CTAs take items from
// a device counter (largest work per item first, as the host orders the
// problems) until none is left.  Per item, CTA g of the cluster takes the angles [g*apc, ...):
//   mode 0 (iteration): the forward of its angles with the slice of Cin in
//     shared memory, the ratio I / max(Pf, 1e-6) written to the problem's
//     ratio buffer; then the backward of the same angles (the image region is
//     reused as the accumulator), the cluster reduction and the update into
//     Cout (bwd_epilogue mode 1);
//   mode 1 (sensitivity): the backward of ratio = 1, max(P^T 1, 1e-6) into sens.
// One launch per slice width thus covers an MLEM iteration of every problem
// of that width, so that small problems fill the GPU beside large ones and no
// launch leaves a tail per problem; the shared memory of a launch is sized for
// its own width, so small slices keep three CTAs per SM.
// ---------------------------------------------------------------------------
constexpr int kMaxProbs = 64;

struct MlemProb {
    const float* atten;
    const float* em;
    const float* theta;
    const float* I;
    float* sens;
    const float* Cin;
    float* Cout;
    float* ratio;
    int A, B, H, W;
    int seg, parts;    // backward segment length, forward partial sums per column
};

struct MlemQueue {
    MlemProb p[kMaxProbs];
    int start[kMaxProbs + 1];   // item offsets: problem i owns items [start[i], start[i+1])
    int n_prob;
};

template <int RC, int WC>
__global__ void __launch_bounds__(kT2, 3)
mlem_queue_kernel(const MlemQueue* __restrict__ queue, int* __restrict__ counter, int Rrt,
                  int img_region, int frame_region, int ncopy, int mode, float beta, float delta) {
    extern __shared__ __align__(16) float smem[];
    __shared__ int s_item;
    cg::cluster_group cluster = cg::this_cluster();
    const int R = RC > 0 ? RC : Rrt;
    const int G = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    // regions sized by the host for the largest problem
    float* simg = smem;                                     // C (forward) / accumulator
    float* sframe = simg + img_region;                      // frames; partial sums (forward)
    float* sq = sframe + frame_region;                      // [2][R][W]
    const int n_items = queue->start[queue->n_prob];
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        cluster.sync();
        const int item = *cluster.map_shared_rank(&s_item, 0);
        cluster.sync();   // every CTA has read the item before rank 0 takes the next
        if (item >= n_items) break;
        int pi = 0;
        while (queue->start[pi + 1] <= item) ++pi;
        const MlemProb P = queue->p[pi];
        const int b = item - queue->start[pi];
        const int H = P.H, W = WC > 0 ? WC : P.W, seg = P.seg, parts = P.parts;
        const int pitch = slice_pitch(W);
        const int img = H * pitch;
        const int apc = (P.A + G - 1) / G;
        const int a0 = rank * apc, a1 = min(P.A, a0 + apc);
        if (mode == 0) {
            stage_slice(simg, P.Cin, R, P.B, b, H, W, pitch);
            __syncthreads();
            for (int a = a0; a < a1; ++a) {
                const Geo g = make_geo(P.theta[a], H, W);
                float* sp = sframe + (a & 1) * parts * W;
                fwd_angle2<RC, WC>(P.atten + ((int64_t)a * P.B + b) * H * W, simg, img, pitch,
                               P.em + (int64_t)a * R, R, g, H, W, parts, sp);
                __syncthreads();
                fwd_finish(sp, parts, W, RC == 1 ? __ldg(P.em + (int64_t)a * R) : 1.f, P.I,
                           P.ratio, (int64_t)a * P.B + b);
            }
            __syncthreads();   // the image and partials are reused below
        }
        bwd_splat_angles<RC, WC>(P.atten, mode == 0 ? P.ratio : nullptr, P.em, P.theta, simg, sframe,
                             sq, ncopy, a0, a1, b, P.B, R, H, W, seg);
        cluster.sync();
        cluster_reduce(cluster, simg, R, H, W, pitch, [&](int r, int h, int w, float s) {
            if (mode == 0)
                bwd_epilogue(1, P.Cout, P.Cin, P.sens, 0.f, beta, delta, r, b, P.B, H, W, h, w, s);
            else
                bwd_epilogue(0, P.sens, nullptr, nullptr, 1e-6f, 0.f, 0.f, r, b, P.B, H, W, h, w, s);
        });
        cluster.sync();   // remote images read before the next item overwrites them
    }
}

// Copies the problem table (passed by value: no host copy, capture-safe).
__global__ void mlem_queue_init_kernel(MlemQueue q, MlemQueue* __restrict__ dst) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = q;
}

__global__ void huber_kernel(const float* __restrict__ C, float* __restrict__ grad, int64_t n,
                             int H, int W, float delta) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t img = i / ((int64_t)H * W);
    int rem = (int)(i - img * H * W);
    int r = rem / W, c = rem - r * W;
    const float* p = C + img * H * W;
    float cp = p[rem], g = 0.f;
    if (r > 0) { float d = cp - p[rem - W]; g += fabsf(d) <= delta ? d : copysignf(delta, d); }
    if (r + 1 < H) { float d = cp - p[rem + W]; g += fabsf(d) <= delta ? d : copysignf(delta, d); }
    if (c > 0) { float d = cp - p[rem - 1]; g += fabsf(d) <= delta ? d : copysignf(delta, d); }
    if (c + 1 < W) { float d = cp - p[rem + 1]; g += fabsf(d) <= delta ? d : copysignf(delta, d); }
    grad[i] = g;
}

// ---------------------------------------------------------------------------
// Host-side planning
// ---------------------------------------------------------------------------
struct Plan {
    int G;      // CTAs per slice (cluster size) or angle groups
    int apc;    // angles per CTA
    size_t smem;
};

int check_proj_sizes(int64_t A, int64_t B, int64_t R, int64_t H, int64_t W) {
    FLC_REQUIRE(A >= 1 && B >= 1 && R >= 1 && H >= 2 && W >= 2,
                "projector sizes must satisfy A,B,R >= 1 and H,W >= 2 (got A=%lld B=%lld R=%lld H=%lld W=%lld)",
                (long long)A, (long long)B, (long long)R, (long long)H, (long long)W);
    FLC_REQUIRE(R <= kMaxR, "at most %d references per element are supported (R=%lld)", kMaxR,
                (long long)R);
    FLC_REQUIRE(H <= 4096 && W <= 4096 && A <= (1 << 24) && B <= 65535,
                "projector sizes out of range (A=%lld B=%lld H=%lld W=%lld)", (long long)A,
                (long long)B, (long long)H, (long long)W);
    return FLC_OK;
}

// Clusters of G CTAs of fn (kThreads threads, smem bytes each) that can be
// resident at once on the current device; 0 if G is not launchable.  Cached.
int active_clusters(const void* fn, int G, size_t smem, int threads = kThreads) {
    struct Entry {
        const void* fn;
        int dev, G;
        size_t smem;
        int n;
    };
    static std::mutex mu;
    static std::vector<Entry> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(mu);
        for (const Entry& e : cache)
            if (e.fn == fn && e.dev == dev && e.G == G && e.smem == smem) return e.n;
    }
    int n = 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
            cudaSuccess &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(G);
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = G;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess) n = 0;
    }
    (void)cudaGetLastError();  // a refused size is an answer, not a pending error
    std::lock_guard<std::mutex> lk(mu);
    cache.push_back({fn, dev, G, smem, n});
    return n;
}

// Cluster size G (CTAs per slice, each taking ceil(A/G) angles) minimising
// waves * (angles per CTA + 2): the B clusters run in ceil(B / resident)
// waves, and each CTA pays about two angles' worth of staging and reduction.
// The "proj.cluster" knob forces G.
Plan plan_cluster(const void* fn, int64_t A, int64_t B, size_t smem_per_cta,
                  int threads = kThreads) {
    Plan p;
    p.smem = smem_per_cta;
    int gmax = kMaxCluster < A ? kMaxCluster : (int)A;
    int best_g = 1;
    if (int64_t t = tune(kTuneProjCluster)) {
        best_g = (int)(t < gmax ? t : gmax);
    } else {
        int64_t best = -1;
        for (int G = 1; G <= gmax; ++G) {
            const int n = active_clusters(fn, G, smem_per_cta, threads);
            if (n < 1) continue;
            const int64_t cost = ceil_div(B, n) * (ceil_div(A, G) + 2);
            if (best < 0 || cost < best) {
                best = cost;
                best_g = G;
            }
        }
    }
    p.apc = (int)ceil_div(A, best_g);
    p.G = (int)ceil_div(A, p.apc);
    return p;
}

int launch_cluster(const void* fn, dim3 grid, int G, size_t smem, cudaStream_t st, void** args,
                   int threads = kThreads) {
    FLC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FLC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FLC_TRY_CUDA(cudaLaunchKernelExC(&cfg, fn, args));
    count_launches(1);
    return FLC_OK;
}

size_t tile_floats(int64_t H, int64_t W) { return (size_t)((H * W + 3) & ~3LL); }

size_t fwd_smem(int64_t R, int64_t H, int64_t W, bool stage_tile, bool stage_c) {
    int parts = col_parts((int)W, (int)H);
    return sizeof(float) * ((stage_tile ? tile_floats(H, W) : 0) +
                            (stage_c ? R * H * slice_pitch((int)W) : 0) + parts * W + kMaxR);
}

size_t bwd_smem(int64_t R, int64_t H, int64_t W, bool stage_tile, int ncopy) {
    return sizeof(float) * ((stage_tile ? tile_floats(H, W) : 0) + R * H * slice_pitch((int)W) +
                            frame_floats((int)R, (int)H, (int)W, ncopy) + W + kMaxR);
}

size_t mlem_smem(int64_t R, int64_t H, int64_t W, int ncopy) {
    int parts = col_parts((int)W, (int)H);
    return sizeof(float) * (tile_floats(H, W) + 2 * R * H * slice_pitch((int)W) +
                            frame_floats((int)R, (int)H, (int)W, ncopy) + parts * W + W + kMaxR);
}

// Segment length of the column-segment backward: the shortest (>= 2) for
// which one round of a segment phase's items fits the CTA's threads.
int seg_length(int64_t H, int64_t W) {
    const int64_t nw = (W + 2) / 3;
    int seg = 2;
    while (seg < H && nw * (((H + seg - 1) / seg + 1) / 2) > kThreads) ++seg;
    return seg;
}

// Backward form for the knob value 0 (automatic): the column segments (4)
// when one round of a segment phase's items fills 85-100% of the CTA's
// threads with segments of at most 8 samples -- measured faster there
// (fused MLEM iteration, 120 angles: 96^2 1.03 vs 1.14 ms, 112^2 2.30 vs
// 2.61, 128^2 2.80 vs 3.06) -- else the nine-phase splat (2), which wins
// when the segment phases leave threads idle or the segments grow long
// (192^2, 12 samples: 5.98 vs 5.75 ms).
int pick_bwd_mode(int64_t H, int64_t W) {
    int mode = (int)tune(kTuneProjBwd);
    if (mode != 0) return mode;
    const int seg = seg_length(H, W);
    const int64_t items = (W + 2) / 3 * (((H + seg - 1) / seg + 1) / 2);
    return (seg <= 8 && items <= kThreads && items * 100 >= 85 * kThreads) ? 4 : 2;
}

// The most frame copies (kMaxFrameCopies, halving down to 1) for which
// smem_of(ncopy) still fits in a CTA's shared memory.
template <class F>
int frame_copies(F smem_of) {
    const size_t cap = (size_t)max_smem_optin();
    int n = kMaxFrameCopies;
    while (n > 1 && smem_of(n) > cap) n /= 2;
    return n;
}

// ---- lean kernels: sizes and launches ------------------------------------
// Partial sums per column of the lean forward: about one item per thread.
int fwd2_parts(int64_t H, int64_t W) {
    int64_t p = kT2 / W;
    if (p < 1) p = 1;
    if (p > H) p = H;
    return (int)p;
}

size_t fwd2_smem(int64_t R, int64_t H, int64_t W) {
    return sizeof(float) * (R * H * slice_pitch((int)W) + 2 * fwd2_parts(H, W) * W);
}

size_t bwd2_smem(int64_t R, int64_t H, int64_t W, int ncopy) {
    return sizeof(float) * (R * H * slice_pitch((int)W) + frame_floats((int)R, (int)H, (int)W, ncopy) +
                            2 * R * W);
}

// Segment length of the lean backward: the shortest (>= 2) for which one
// round of a phase's items fits its kT2 threads.
int seg2_length(int64_t H, int64_t W) {
    const int64_t nw = (W + 2) / 3;
    int seg = 2;
    while (seg < H && nw * (((H + seg - 1) / seg + 1) / 2) > kT2) ++seg;
    return seg;
}

// Threads of the lean backward: its largest phase's items rounded up to whole
// warps (at most kT2), so that no warp of the CTA only waits at the phase
// barriers.
int bwd2_threads(int64_t H, int64_t W) {
    const int64_t seg = seg2_length(H, W);
    const int64_t items = ((W + 2) / 3) * ((((H + seg - 1) / seg) + 1) / 2);
    const int64_t t = (items + 31) / 32 * 32;
    return (int)(t < 64 ? 64 : (t > kT2 ? kT2 : t));
}

// Shared-memory budget per CTA for `per_sm` resident CTAs (1 KB of each CTA's
// shared memory is reserved by the runtime), capped by the opt-in limit.
size_t smem_budget(int per_sm) {
    size_t b = (size_t)smem_per_sm() / (size_t)per_sm;
    b = b > 1024 ? b - 1024 : 0;
    return b < (size_t)max_smem_optin() ? b : (size_t)max_smem_optin();
}

// Frame copies of the lean backward: as many (up to kMaxFrameCopies) as keep
// the CTAs per SM that the bare image allows.
int bwd2_copies(int64_t R, int64_t H, int64_t W) {
    int per_sm = 3;
    while (per_sm > 1 && bwd2_smem(R, H, W, 1) > smem_budget(per_sm)) --per_sm;
    int n = kMaxFrameCopies;
    while (n > 1 && bwd2_smem(R, H, W, n) > smem_budget(per_sm)) n /= 2;
    return n;
}

bool use_lean() { return tune(kTuneProjLegacy) == 0; }

// The lean kernels instantiated for the common slice widths (their row
// strides and pitch become immediates) and for any width at run time.
template <int RC>
const void* fwd2_for_width(int64_t W) {
    switch (W) {
        case 64: return (const void*)proj_fwd2_kernel<RC, 64>;
        case 96: return (const void*)proj_fwd2_kernel<RC, 96>;
        case 128: return (const void*)proj_fwd2_kernel<RC, 128>;
        case 160: return (const void*)proj_fwd2_kernel<RC, 160>;
        case 192: return (const void*)proj_fwd2_kernel<RC, 192>;
        default: return (const void*)proj_fwd2_kernel<RC, 0>;
    }
}

template <int RC>
const void* bwd2_for_width(int64_t W) {
    switch (W) {
        case 64: return (const void*)proj_bwd2_kernel<RC, 64>;
        case 96: return (const void*)proj_bwd2_kernel<RC, 96>;
        case 128: return (const void*)proj_bwd2_kernel<RC, 128>;
        case 160: return (const void*)proj_bwd2_kernel<RC, 160>;
        case 192: return (const void*)proj_bwd2_kernel<RC, 192>;
        default: return (const void*)proj_bwd2_kernel<RC, 0>;
    }
}

const void* fwd2_kernel_for(int64_t R, int64_t W) {
    return R == 1 ? fwd2_for_width<1>(W) : fwd2_for_width<0>(W);
}

const void* bwd2_kernel_for(int64_t R, int64_t W) {
    return R == 1 ? bwd2_for_width<1>(W) : bwd2_for_width<0>(W);
}
bool force_band() { return use_lean() && tune(kTuneProjBand) != 0; }

}  // namespace

// Lean forward (+ ratio when I != nullptr); FLC_ERR_UNSUPPORTED (nothing
// launched) when the slice does not fit in shared memory.
int fwd2_launch(const float* atten, const float* C, const float* em, const float* theta,
                float* out, const float* I, int64_t A, int64_t B, int64_t R, int64_t H, int64_t W,
                cudaStream_t st) {
    const size_t smem = fwd2_smem(R, H, W);
    if (smem > (size_t)max_smem_optin()) return FLC_ERR_UNSUPPORTED;
    const void* fn = fwd2_kernel_for(R, W);
    FLC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kT2, smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    (void)cudaGetLastError();
    // angle groups minimising waves x (angles per CTA + 1 for staging the slice)
    const int64_t slots = (int64_t)sm_count() * per_sm;
    int64_t best = -1, groups = 1;
    for (int64_t gcount = 1; gcount <= A && gcount <= 64; ++gcount) {
        const int64_t apc = ceil_div(A, gcount);
        const int64_t cost = ceil_div(B * ceil_div(A, apc), slots) * (apc + 1);
        if (best < 0 || cost < best) {
            best = cost;
            groups = gcount;
        }
    }
    int apc = (int)ceil_div(A, groups);
    if (int64_t t = tune(kTuneProjApc)) apc = (int)(t < A ? t : A);
    groups = ceil_div(A, apc);
    const int parts = fwd2_parts(H, W);
    int iA = (int)A, iB = (int)B, iR = (int)R, iH = (int)H, iW = (int)W;
    void* args[] = {(void*)&atten, (void*)&C, (void*)&em, (void*)&theta, (void*)&out, (void*)&I,
                    &iA, &iB, &iR, &iH, &iW, &apc, (void*)&parts};
    FLC_TRY_CUDA(cudaLaunchKernel(fn, dim3((unsigned)groups, (unsigned)B), dim3(kT2), args, smem, st));
    count_launches(1);
    return FLC_OK;
}

// Lean backward with its epilogue (mode 0: out = P^T ratio, clamped below by
// clamp_min when > 0; mode 1: the MLEM update of Cin into out).
// FLC_ERR_UNSUPPORTED (nothing launched) when the image does not fit.
int bwd2_launch(const float* atten, const float* ratio, const float* em, const float* theta,
                float* out, const float* Cin, const float* sens, int64_t A, int64_t B, int64_t R,
                int64_t H, int64_t W, float clamp_min, int mode, float beta, float delta,
                cudaStream_t st) {
    if (bwd2_smem(R, H, W, 1) > (size_t)max_smem_optin()) return FLC_ERR_UNSUPPORTED;
    const int ncopy = bwd2_copies(R, H, W);
    const size_t smem = bwd2_smem(R, H, W, ncopy);
    const void* fn = bwd2_kernel_for(R, W);
    const int threads = bwd2_threads(H, W);
    Plan p = plan_cluster(fn, A, B, smem, threads);
    int iA = (int)A, iB = (int)B, iR = (int)R, iH = (int)H, iW = (int)W, apc = p.apc;
    int seg = seg2_length(H, W);
    void* args[] = {(void*)&atten, (void*)&ratio, (void*)&em, (void*)&theta, (void*)&out,
                    (void*)&Cin, (void*)&sens, &iA, &iB, &iR, &iH, &iW, &apc, &seg,
                    (void*)&ncopy, &clamp_min, &mode, &beta, &delta};
    return launch_cluster(fn, dim3(p.G, (unsigned)B), p.G, smem, st, args, threads);
}

// Band backward (slices too large for the lean kernel): the band height is
// the largest that lets three CTAs share an SM (bands of at least 48 rows),
// else two, else one; the bands are evened out, and the angles are split over
// a cluster when the bands x slices do not fill the GPU.  FLC_ERR_UNSUPPORTED when even
// a 1-row band does not fit.
size_t band_smem(int64_t R, int64_t hb, int64_t W, int ncopy) {
    const int64_t nrow = hb + 2;
    return sizeof(float) * (R * nrow * slice_pitch((int)W) + frame_floats((int)R, (int)nrow, (int)W, ncopy) +
                            2 * R * W);
}

// Segment length of the band walk (the warps fetch items dynamically).
constexpr int kSegBand = 6;

int band_height(int64_t R, int64_t H, int64_t W, int* ncopy_out) {
    const size_t cap = (size_t)max_smem_optin();
    if (band_smem(R, 1, W, 1) > cap) return 0;
    // three CTAs per SM where bands of >= 48 rows (or the whole slice) fit,
    // else two where bands of >= 8 rows fit, else one
    const int64_t want3 = H < 48 ? H : 48;
    int per_sm = band_smem(R, want3, W, 1) <= smem_budget(3) ? 3
                 : band_smem(R, 8, W, 1) <= smem_budget(2) ? 2 : 1;
    const size_t budget = smem_budget(per_sm);
    int64_t hb = 1;
    while (hb < H && band_smem(R, hb + 1, W, 1) <= budget) ++hb;
    const int64_t nband = ceil_div(H, hb);
    hb = ceil_div(H, nband);                     // even bands
    int ncopy = kMaxFrameCopies;
    while (ncopy > 1 && band_smem(R, hb, W, ncopy) > budget) ncopy /= 2;
    *ncopy_out = ncopy;
    return (int)hb;
}

int band_launch(const float* atten, const float* ratio, const float* em, const float* theta,
                float* out, const float* Cin, const float* sens, int64_t A, int64_t B, int64_t R,
                int64_t H, int64_t W, float clamp_min, int mode, float beta, float delta,
                cudaStream_t st) {
    int ncopy = 1;
    const int hb = band_height(R, H, W, &ncopy);
    if (hb < 1) {
        set_error("backward projection: a slice row of W=%lld with R=%lld references does not fit "
                  "in shared memory", (long long)W, (long long)R);
        return FLC_ERR_UNSUPPORTED;
    }
    const int nband = (int)ceil_div(H, hb);
    const size_t smem = band_smem(R, hb, W, ncopy);
    const void* fn = R == 1 ? (const void*)proj_bwd_band_kernel<1> : (const void*)proj_bwd_band_kernel<0>;
    Plan p = plan_cluster(fn, A, (int64_t)nband * B, smem, kT2);
    int iA = (int)A, iB = (int)B, iR = (int)R, iH = (int)H, iW = (int)W, apc = p.apc, ihb = hb;
    int seg = kSegBand;
    void* args[] = {(void*)&atten, (void*)&ratio, (void*)&em, (void*)&theta, (void*)&out,
                    (void*)&Cin, (void*)&sens, &iA, &iB, &iR, &iH, &iW, &apc, &ihb, &seg,
                    (void*)&ncopy, &clamp_min, &mode, &beta, &delta};
    return launch_cluster(fn, dim3((unsigned)(p.G * nband), (unsigned)B), p.G, smem, st, args, kT2);
}

// Launches the backward projector (also used for the MLEM sensitivity).
int bwd_emission_launch(const float* atten, const float* ratio, const float* em,
                        const float* theta, float* out, int64_t A, int64_t B, int64_t R,
                        int64_t H, int64_t W, float clamp_min, cudaStream_t st) {
    if (use_lean()) {
        const int r = force_band() ? FLC_ERR_UNSUPPORTED
                                   : bwd2_launch(atten, ratio, em, theta, out, nullptr, nullptr, A,
                                                 B, R, H, W, clamp_min, 0, 0.f, 0.f, st);
        if (r != FLC_ERR_UNSUPPORTED) return r;
        return band_launch(atten, ratio, em, theta, out, nullptr, nullptr, A, B, R, H, W, clamp_min,
                           0, 0.f, 0.f, st);
    }
    const size_t cap = (size_t)max_smem_optin();
    int stage_tile = bwd_smem(R, H, W, true, 1) <= cap;
    if (!stage_tile && bwd_smem(R, H, W, false, 1) > cap) {
        // the slice image does not fit on chip: row bands
        return band_launch(atten, ratio, em, theta, out, nullptr, nullptr, A, B, R, H, W, clamp_min,
                           0, 0.f, 0.f, st);
    }
    int ncopy = frame_copies([&](int n) { return bwd_smem(R, H, W, stage_tile, n); });
    size_t smem = bwd_smem(R, H, W, stage_tile, ncopy);
    const void* fn = R == 1 ? (const void*)proj_bwd_kernel<1> : (const void*)proj_bwd_kernel<0>;
    Plan p = plan_cluster(fn, A, B, smem);
    int iA = (int)A, iB = (int)B, iR = (int)R, iH = (int)H, iW = (int)W, apc = p.apc;
    int bwd_mode = pick_bwd_mode(H, W), seg = seg_length(H, W);
    void* args[] = {(void*)&atten, (void*)&ratio, (void*)&em, (void*)&theta, (void*)&out,
                    &iA, &iB, &iR, &iH, &iW, &apc, &clamp_min, &stage_tile, &bwd_mode, &ncopy,
                    &seg};
    return launch_cluster(fn, dim3(p.G, (unsigned)B), p.G, smem, st, args);
}

int fwd_emission_launch(const float* atten, const float* C, const float* em, const float* theta,
                        float* Pf, const float* I, int64_t A, int64_t B, int64_t R, int64_t H,
                        int64_t W, cudaStream_t st) {
    if (use_lean()) {
        const int r = fwd2_launch(atten, C, em, theta, Pf, I, A, B, R, H, W, st);
        if (r != FLC_ERR_UNSUPPORTED) return r;
    }
    const size_t cap = (size_t)max_smem_optin();
    int stage_tile = 1, stage_c = 1;
    if (fwd_smem(R, H, W, true, true) > cap) stage_tile = 0;
    if (!stage_tile && fwd_smem(R, H, W, false, true) > cap) stage_c = 0;
    size_t smem = fwd_smem(R, H, W, stage_tile, stage_c);
    int per_sm = (int)(max_smem_optin() / (smem + 1024));
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 4) per_sm = 4;
    int64_t want = 3LL * sm_count() * per_sm;
    int64_t groups = ceil_div(want, B);
    if (groups > A) groups = A;
    if (groups < 1) groups = 1;
    int apc = (int)ceil_div(A, groups);
    if (int64_t t = tune(kTuneProjApc)) apc = (int)(t < A ? t : A);
    groups = ceil_div(A, apc);
    FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)proj_fwd_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    proj_fwd_kernel<<<dim3((unsigned)groups, (unsigned)B), kThreads, smem, st>>>(
        atten, C, em, theta, Pf, I, (int)A, (int)B, (int)R, (int)H, (int)W, apc, stage_tile,
        stage_c);
    return check_launch("proj_fwd_kernel");
}

int mlem_iter_launch(const float* atten, const float* em, const float* theta, const float* I,
                     const float* sens, const float* Cin, float* Cout, int64_t A, int64_t B,
                     int64_t R, int64_t H, int64_t W, float beta, float delta, cudaStream_t st,
                     bool* fused, float* ratio_ws) {
    if (use_lean() && !force_band() && fwd2_smem(R, H, W) <= (size_t)max_smem_optin() &&
        bwd2_smem(R, H, W, 1) <= (size_t)max_smem_optin()) {
        // forward + ratio, then backward + update: two launches
        *fused = true;
        FLC_TRY(fwd2_launch(atten, Cin, em, theta, ratio_ws, I, A, B, R, H, W, st));
        return bwd2_launch(atten, ratio_ws, em, theta, Cout, Cin, sens, A, B, R, H, W, 0.f, 1,
                           beta, delta, st);
    }
    if (use_lean() && (force_band() || bwd2_smem(R, H, W, 1) > (size_t)max_smem_optin())) {
        // large slices: forward + ratio, then the band backward + update
        *fused = true;
        FLC_TRY(fwd_emission_launch(atten, Cin, em, theta, ratio_ws, I, A, B, R, H, W, st));
        return band_launch(atten, ratio_ws, em, theta, Cout, Cin, sens, A, B, R, H, W, 0.f, 1, beta,
                           delta, st);
    }
    *fused = mlem_smem(R, H, W, 1) <= (size_t)max_smem_optin();
    if (!*fused) return FLC_OK;
    int ncopy = frame_copies([&](int n) { return mlem_smem(R, H, W, n); });
    const size_t smem = mlem_smem(R, H, W, ncopy);
    const void* fn = R == 1 ? (const void*)mlem_iter_kernel<1> : (const void*)mlem_iter_kernel<0>;
    Plan p = plan_cluster(fn, A, B, smem);
    int iA = (int)A, iB = (int)B, iR = (int)R, iH = (int)H, iW = (int)W, apc = p.apc;
    int bwd_mode = pick_bwd_mode(H, W), seg = seg_length(H, W);
    void* args[] = {(void*)&atten, (void*)&em, (void*)&theta, (void*)&I, (void*)&sens,
                    (void*)&Cin, (void*)&Cout, &iA, &iB, &iR, &iH, &iW, &apc, &beta, &delta,
                    &bwd_mode, &ncopy, &seg};
    return launch_cluster(fn, dim3(p.G, (unsigned)B), p.G, smem, st, args);
}

// Computes (and caches) the launch plan of the fused iteration, so that a
// later stream capture makes no occupancy queries.
void mlem_iter_prepare(int64_t A, int64_t B, int64_t R, int64_t H, int64_t W) {
    if (use_lean() && !force_band() && bwd2_smem(R, H, W, 1) <= (size_t)max_smem_optin()) {
        const size_t smem = bwd2_smem(R, H, W, bwd2_copies(R, H, W));
        const void* fn = bwd2_kernel_for(R, W);
        (void)plan_cluster(fn, A, B, smem, bwd2_threads(H, W));
        return;
    }
    if (use_lean()) {
        int ncopy = 1;
        const int hb = band_height(R, H, W, &ncopy);
        if (hb < 1) return;
        const void* fn = R == 1 ? (const void*)proj_bwd_band_kernel<1> : (const void*)proj_bwd_band_kernel<0>;
        (void)plan_cluster(fn, A, ceil_div(H, hb) * B, band_smem(R, hb, W, ncopy), kT2);
        return;
    }
    if (mlem_smem(R, H, W, 1) > (size_t)max_smem_optin()) return;
    const size_t smem = mlem_smem(R, H, W, frame_copies([&](int n) { return mlem_smem(R, H, W, n); }));
    const void* fn = R == 1 ? (const void*)mlem_iter_kernel<1> : (const void*)mlem_iter_kernel<0>;
    (void)plan_cluster(fn, A, B, smem);
}

int huber_launch(const float* C, float* grad, int64_t RB, int64_t H, int64_t W, float delta,
                 cudaStream_t st) {
    int64_t n = RB * H * W;
    huber_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(C, grad, n, (int)H, (int)W, delta);
    return check_launch("huber_kernel");
}

}  // namespace flc

// ===========================================================================
// C ABI
// ===========================================================================
using namespace flc;

extern "C" int flc_fwd_emission(const float* atten, const float* C, const float* em,
                                const float* theta, float* Pf, int64_t A, int64_t B, int64_t R,
                                int64_t H, int64_t W, void* stream) {
    clear_error();
    FLC_REQUIRE(atten && C && em && theta && Pf, "flc_fwd_emission: null pointer argument");
    FLC_TRY(check_proj_sizes(A, B, R, H, W));
    return fwd_emission_launch(atten, C, em, theta, Pf, nullptr, A, B, R, H, W, as_stream(stream));
}

extern "C" int flc_bwd_emission(const float* atten, const float* ratio, const float* em,
                                const float* theta, float* out, int64_t A, int64_t B, int64_t R,
                                int64_t H, int64_t W, void* stream) {
    clear_error();
    FLC_REQUIRE(atten && ratio && em && theta && out, "flc_bwd_emission: null pointer argument");
    FLC_TRY(check_proj_sizes(A, B, R, H, W));
    return bwd_emission_launch(atten, ratio, em, theta, out, A, B, R, H, W, 0.f, as_stream(stream));
}

// ---------------------------------------------------------------------------
// flc_mlem_multi: MLEM of P problems of the same R, H, W with the persistent
// queue kernel -- one launch per iteration for all of them.
// ---------------------------------------------------------------------------
namespace flc {
namespace {

size_t al256(size_t n) { return (n + 255) & ~(size_t)255; }

size_t multi_frame_floats(int64_t R, int64_t H, int64_t W, int ncopy) {
    const size_t f = (size_t)frame_floats((int)R, (int)H, (int)W, ncopy);
    const size_t pt = (size_t)2 * fwd2_parts(H, W) * W;   // forward partials share the region
    return f > pt ? f : pt;
}

// Shared-memory regions of the queue kernel for the largest of P problems
// (floats): image, frames / forward partials, q; the total in bytes.
struct MultiSmem {
    size_t img, frame, q, bytes;
};

MultiSmem multi_smem(int64_t P, int64_t R, const int64_t* H, const int64_t* W, int ncopy) {
    MultiSmem m = {0, 0, 0, 0};
    for (int64_t i = 0; i < P; ++i) {
        const size_t img = (size_t)R * H[i] * slice_pitch((int)W[i]);
        const size_t fr = multi_frame_floats(R, H[i], W[i], ncopy);
        const size_t q = 2 * (size_t)R * W[i];
        m.img = img > m.img ? img : m.img;
        m.frame = fr > m.frame ? fr : m.frame;
        m.q = q > m.q ? q : m.q;
    }
    m.img = (m.img + 3) & ~(size_t)3;       // keep the regions 16-byte aligned
    m.frame = (m.frame + 3) & ~(size_t)3;
    m.bytes = sizeof(float) * (m.img + m.frame + m.q);
    return m;
}

// Groups of the problems by slice width, in order of first appearance:
// gid[i] = group of problem i; returns the number of groups.
int width_groups(int64_t P, const int64_t* W, int* gid, int64_t* gw) {
    int ng = 0;
    for (int64_t i = 0; i < P; ++i) {
        int g = 0;
        while (g < ng && gw[g] != W[i]) ++g;
        if (g == ng) gw[ng++] = W[i];
        gid[i] = g;
    }
    return ng;
}

// Workspace: per width group two problem tables and a counter (256 bytes),
// then per problem the sensitivity, the second C buffer and the ratio.
size_t multi_layout(int64_t P, const int64_t* A, const int64_t* B, int64_t R, const int64_t* H,
                    const int64_t* W, size_t* prob_off) {
    int gid[kMaxProbs];
    int64_t gw[kMaxProbs];
    const int ng = width_groups(P, W, gid, gw);
    size_t off = (size_t)ng * (2 * al256(sizeof(MlemQueue)) + 256);
    for (int64_t i = 0; i < P; ++i) {
        if (prob_off) prob_off[i] = off;
        const size_t nC = al256(sizeof(float) * (size_t)(R * B[i] * H[i] * W[i]));
        off += 2 * nC + al256(sizeof(float) * (size_t)(A[i] * B[i] * W[i]));
    }
    return off;
}

int mlem_multi_impl(int64_t P, float* const* C, const float* const* atten, const float* const* em,
                    const float* const* theta, const float* const* I, const int64_t* A,
                    const int64_t* B, int64_t R, const int64_t* H, const int64_t* W, int64_t n_iter,
                    double beta, double delta, void* workspace, size_t workspace_bytes,
                    void* stream);

// The queue kernel for R references and slice width W (compile-time widths
// 64, 96, 128, 160, 192; any other width at run time).
template <int RC>
const void* queue_kernel_for_r(int64_t W) {
    switch (W) {
        case 64: return (const void*)mlem_queue_kernel<RC, 64>;
        case 96: return (const void*)mlem_queue_kernel<RC, 96>;
        case 128: return (const void*)mlem_queue_kernel<RC, 128>;
        case 160: return (const void*)mlem_queue_kernel<RC, 160>;
        case 192: return (const void*)mlem_queue_kernel<RC, 192>;
        default: return (const void*)mlem_queue_kernel<RC, 0>;
    }
}

const void* queue_kernel_for(int64_t R, int64_t W) {
    return R == 1 ? queue_kernel_for_r<1>(W) : queue_kernel_for_r<0>(W);
}

}  // namespace
}  // namespace flc

extern "C" size_t flc_mlem_multi_sizes_workspace_bytes(int64_t P, const int64_t* A,
                                                       const int64_t* B, int64_t R,
                                                       const int64_t* H, const int64_t* W) {
    if (P < 1 || P > kMaxProbs || !A || !B || !H || !W || R < 1) return 0;
    for (int64_t i = 0; i < P; ++i)
        if (A[i] < 1 || B[i] < 1 || H[i] < 1 || W[i] < 1) return 0;
    return multi_layout(P, A, B, R, H, W, nullptr);
}

extern "C" size_t flc_mlem_multi_workspace_bytes(int64_t P, const int64_t* A, const int64_t* B,
                                                 int64_t R, int64_t H, int64_t W) {
    if (P < 1 || P > kMaxProbs) return 0;
    int64_t hs[kMaxProbs], wsz[kMaxProbs];
    for (int64_t i = 0; i < P; ++i) hs[i] = H, wsz[i] = W;
    return flc_mlem_multi_sizes_workspace_bytes(P, A, B, R, hs, wsz);
}

extern "C" int flc_mlem_multi(int64_t P, float* const* C, const float* const* atten,
                              const float* const* em, const float* const* theta,
                              const float* const* I, const int64_t* A, const int64_t* B, int64_t R,
                              int64_t H, int64_t W, int64_t n_iter, double beta, double delta,
                              void* workspace, size_t workspace_bytes, void* stream) {
    clear_error();
    FLC_REQUIRE(P >= 1 && P <= kMaxProbs, "flc_mlem_multi: 1 <= P <= %d problems", kMaxProbs);
    int64_t hs[kMaxProbs], wsz[kMaxProbs];
    for (int64_t i = 0; i < P; ++i) hs[i] = H, wsz[i] = W;
    return mlem_multi_impl(P, C, atten, em, theta, I, A, B, R, hs, wsz, n_iter, beta, delta,
                           workspace, workspace_bytes, stream);
}

extern "C" int flc_mlem_multi_sizes(int64_t P, float* const* C, const float* const* atten,
                                    const float* const* em, const float* const* theta,
                                    const float* const* I, const int64_t* A, const int64_t* B,
                                    int64_t R, const int64_t* H, const int64_t* W, int64_t n_iter,
                                    double beta, double delta, void* workspace,
                                    size_t workspace_bytes, void* stream) {
    clear_error();
    FLC_REQUIRE(P >= 1 && P <= kMaxProbs, "flc_mlem_multi_sizes: 1 <= P <= %d problems", kMaxProbs);
    FLC_REQUIRE(H && W, "flc_mlem_multi_sizes: null pointer argument");
    return mlem_multi_impl(P, C, atten, em, theta, I, A, B, R, H, W, n_iter, beta, delta,
                           workspace, workspace_bytes, stream);
}

namespace flc {
namespace {

int mlem_multi_impl(int64_t P, float* const* C, const float* const* atten, const float* const* em,
                    const float* const* theta, const float* const* I, const int64_t* A,
                    const int64_t* B, int64_t R, const int64_t* H, const int64_t* W, int64_t n_iter,
                    double beta, double delta, void* workspace, size_t workspace_bytes,
                    void* stream) {
    FLC_REQUIRE(C && atten && em && theta && I && A && B && workspace,
                "flc_mlem_multi: null pointer argument");
    int64_t items = 0;
    for (int64_t i = 0; i < P; ++i) {
        FLC_REQUIRE(C[i] && atten[i] && em[i] && theta[i] && I[i],
                    "flc_mlem_multi: null pointer for problem %lld", (long long)i);
        FLC_TRY(check_proj_sizes(A[i], B[i], R, H[i], W[i]));
        items += B[i];
    }
    FLC_REQUIRE(n_iter >= 0 && items < (1LL << 30), "flc_mlem_multi: invalid sizes");
    if (((uintptr_t)workspace & 255) != 0) {
        set_error("flc_mlem_multi: workspace must be 256-byte aligned");
        return FLC_ERR_ALIGNMENT;
    }
    size_t prob_off[kMaxProbs];
    const size_t need = multi_layout(P, A, B, R, H, W, prob_off);
    if (workspace_bytes < need) {
        set_error("flc_mlem_multi: workspace of %zu bytes is smaller than the %zu required",
                  workspace_bytes, need);
        return FLC_ERR_WORKSPACE;
    }
    if (multi_smem(P, R, H, W, 1).bytes > (size_t)max_smem_optin()) {
        set_error("flc_mlem_multi: the largest slice does not fit in shared memory");
        return FLC_ERR_UNSUPPORTED;
    }
    cudaStream_t st = as_stream(stream);
    char* ws = (char*)workspace;
    int gid[kMaxProbs];
    int64_t gw[kMaxProbs];
    const int ng = width_groups(P, W, gid, gw);
    const size_t tbl = al256(sizeof(MlemQueue));
    struct GroupLaunch {
        const void* fn;
        MlemQueue *q_even, *q_odd;
        int* counter;
        int G, nclu, ncopy, img_region, frame_region;
        size_t smem;
    };
    GroupLaunch gl[kMaxProbs];
    for (int gi = 0; gi < ng; ++gi) {
        // this width's problems, in decreasing work per item (angles x slice
        // area): the long items are taken first
        int64_t n = 0, gA[kMaxProbs], gB[kMaxProbs], gH[kMaxProbs], gW[kMaxProbs];
        int order[kMaxProbs];
        for (int64_t i = 0; i < P; ++i)
            if (gid[i] == gi) order[n++] = (int)i;
        auto cost = [&](int i) { return A[i] * H[i] * W[i]; };
        for (int i = 1; i < n; ++i)
            for (int j = i; j > 0 && cost(order[j]) > cost(order[j - 1]); --j) std::swap(order[j], order[j - 1]);
        char* gbase = ws + (size_t)gi * (2 * tbl + 256);
        GroupLaunch& L = gl[gi];
        L.q_even = (MlemQueue*)gbase;
        L.q_odd = (MlemQueue*)(gbase + tbl);
        L.counter = (int*)(gbase + 2 * tbl);
        MlemQueue te = {}, to = {};
        te.n_prob = to.n_prob = (int)n;
        int64_t amax = 1, items = 0;
        for (int k = 0; k < n; ++k) {
            const int i = order[k];
            char* base = ws + prob_off[i];
            const size_t nC = al256(sizeof(float) * (size_t)(R * B[i] * H[i] * W[i]));
            float* sens = (float*)base;
            float* alt = (float*)(base + nC);
            float* ratio = (float*)(base + 2 * nC);
            const int hh = (int)H[i], ww = (int)W[i];
            const int sg = seg2_length(hh, ww), pt = fwd2_parts(hh, ww);
            te.p[k] = MlemProb{atten[i], em[i], theta[i], I[i], sens, C[i], alt, ratio,
                               (int)A[i], (int)B[i], hh, ww, sg, pt};
            to.p[k] = MlemProb{atten[i], em[i], theta[i], I[i], sens, alt, C[i], ratio,
                               (int)A[i], (int)B[i], hh, ww, sg, pt};
            te.start[k + 1] = to.start[k + 1] = te.start[k] + (int)B[i];
            amax = A[i] > amax ? A[i] : amax;
            items += B[i];
            gA[k] = A[i], gB[k] = B[i], gH[k] = H[i], gW[k] = W[i];
        }
        mlem_queue_init_kernel<<<1, 32, 0, st>>>(te, L.q_even);
        FLC_TRY(check_launch("mlem_queue_init_kernel"));
        mlem_queue_init_kernel<<<1, 32, 0, st>>>(to, L.q_odd);
        FLC_TRY(check_launch("mlem_queue_init_kernel"));
        // launch shape: frame copies that keep the CTAs per SM, cluster size by
        // (item work / clusters + the longest item), persistent grid
        int per_sm = 3;
        while (per_sm > 1 && multi_smem(n, R, gH, gW, 1).bytes > smem_budget(per_sm)) --per_sm;
        int ncopy = kMaxFrameCopies;
        while (ncopy > 1 && multi_smem(n, R, gH, gW, ncopy).bytes > smem_budget(per_sm)) ncopy /= 2;
        const MultiSmem ms = multi_smem(n, R, gH, gW, ncopy);
        const void* fn = queue_kernel_for(R, gw[gi]);
        int bestG = 1, nclu = 1;
        double best = -1;
        const int gmax = (int)(amax < kMaxCluster ? amax : kMaxCluster);
        if (int64_t t = tune(kTuneProjCluster)) {
            bestG = (int)(t < gmax ? t : gmax);
            nclu = active_clusters(fn, bestG, ms.bytes, kT2);
        } else {
            for (int G = 1; G <= gmax; ++G) {
                const int nc = active_clusters(fn, G, ms.bytes, kT2);
                if (nc < 1) continue;
                double total = 0, longest = 0;
                for (int64_t k = 0; k < n; ++k) {
                    const double item = (double)(ceil_div(gA[k], G) + 2) * (double)(gH[k] * gW[k]);
                    total += item * (double)gB[k];
                    longest = item > longest ? item : longest;
                }
                const double c = total / nc + longest;
                if (best < 0 || c < best) {
                    best = c;
                    bestG = G;
                    nclu = nc;
                }
            }
        }
        if (nclu < 1) {
            set_error("flc_mlem_multi: the queue kernel cannot be made resident");
            return FLC_ERR_UNSUPPORTED;
        }
        if (nclu > items) nclu = (int)items;
        L.fn = fn;
        L.G = bestG;
        L.nclu = nclu;
        L.ncopy = ncopy;
        L.img_region = (int)ms.img;
        L.frame_region = (int)ms.frame;
        L.smem = ms.bytes;
    }
    int iR = (int)R;
    float fb = (float)beta, fd = (float)delta;
    auto launch = [&](const GroupLaunch& L, bool odd, int mode) -> int {
        FLC_TRY_CUDA(cudaMemsetAsync(L.counter, 0, sizeof(int), st));
        const MlemQueue* q = odd ? L.q_odd : L.q_even;
        int img_region = L.img_region, frame_region = L.frame_region, ncopy = L.ncopy;
        void* args[] = {(void*)&q, (void*)&L.counter, &iR, &img_region, &frame_region, &ncopy,
                        &mode, &fb, &fd};
        return launch_cluster(L.fn, dim3((unsigned)(L.nclu * L.G)), L.G, L.smem, st, args, kT2);
    };
    for (int gi = 0; gi < ng; ++gi) FLC_TRY(launch(gl[gi], false, 1));   // sensitivities
    for (int64_t it = 0; it < n_iter; ++it)
        for (int gi = 0; gi < ng; ++gi) FLC_TRY(launch(gl[gi], (it & 1) != 0, 0));
    if (n_iter & 1) {
        for (int64_t i = 0; i < P; ++i) {
            const size_t n = sizeof(float) * (size_t)(R * B[i] * H[i] * W[i]);
            FLC_TRY_CUDA(cudaMemcpyAsync(C[i], ws + prob_off[i] + al256(n), n,
                                         cudaMemcpyDeviceToDevice, st));
        }
    }
    return FLC_OK;
}

}  // namespace
}  // namespace flc

extern "C" int flc_huber_grad(const float* C, float* grad, int64_t RB, int64_t H, int64_t W,
                              float delta, void* stream) {
    clear_error();
    FLC_REQUIRE(C && grad, "flc_huber_grad: null pointer argument");
    FLC_REQUIRE(RB >= 1 && H >= 1 && W >= 1, "flc_huber_grad: sizes must be positive");
    return huber_launch(C, grad, RB, H, W, delta, as_stream(stream));
}
