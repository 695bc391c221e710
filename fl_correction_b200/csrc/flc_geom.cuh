// Device geometry shared by the forward kernels and their adjoints, so that
// every adjoint samples exactly the points its forward sampled.
#pragma once

#include "flc_common.cuh"

namespace flc {

// Row pitch (floats) of a slice image staged in shared memory: >= W and
// == 9 (mod 32) (of the odd residues measured, 1, 3 and 9, the fastest for the
// column-segment splats).
__host__ __device__ inline int slice_pitch(int W) {
    int p = W;
    while ((p & 31) != 9) ++p;
    return p;
}

// ---------------------------------------------------------------------------
// Projector geometry (atten_cuda_kernel.cu:91-142, :271-337): the sample for
// detector column w at beam step h of angle th is
//   row x = c*(h-cy) - s*(w-cx) + cy,  col y = s*(h-cy) + c*(w-cx) + cx,
// c = cos(-th), s = sin(-th), cx = (W-1)/2, cy = (H-1)/2, clamped to
// [0, H-1.001] x [0, W-1.001], then bilinear on the four neighbours.
// ---------------------------------------------------------------------------
struct Geo {
    float c, s, cx, cy, rmax, cmax;
    int ih, jh;       // floor of rmax / cmax (H-2, W-2)
    float fxh, fyh;   // rmax - ih, cmax - jh: weights of the far clamp
};

__device__ __forceinline__ Geo make_geo(float th, int H, int W) {
    Geo g;
    g.c = cosf(-th);
    g.s = sinf(-th);
    g.cx = (W - 1) * 0.5f;
    g.cy = (H - 1) * 0.5f;
    g.rmax = H - 1.001f;
    g.cmax = W - 1.001f;
    g.ih = (int)floorf(g.rmax);
    g.jh = (int)floorf(g.cmax);
    g.fxh = g.rmax - (float)g.ih;
    g.fyh = g.cmax - (float)g.jh;
    return g;
}

// floor(x) and x - floor(x) for 0 <= x < 2^22: adding 1.5*2^23 with round-down
// leaves floor(x) in the low mantissa bits (exact), all on the FP32/INT pipes.
__device__ __forceinline__ int ffloor(float x, float& frac) {
    const float k = 12582912.0f;  // 1.5 * 2^23, bit pattern 0x4B400000
    float t = __fadd_rd(x, k);
    frac = x - (t - k);
    return __float_as_int(t) - 0x4B400000;
}

struct Smp {
    int i0, j0;
    float fx, fy;
    float x, y;   // unclamped
};

// Per-column offsets: x = c*(h-cy) + bx(w), y = s*(h-cy) + by(w).
__device__ __forceinline__ float col_bx(const Geo& g, int w) { return fmaf(-g.s, (float)w - g.cx, g.cy); }
__device__ __forceinline__ float col_by(const Geo& g, int w) { return fmaf(g.c, (float)w - g.cx, g.cx); }

__device__ __forceinline__ Smp sample_xy(const Geo& g, float x, float y) {
    Smp s;
    s.x = x;
    s.y = y;
    float xc = fminf(fmaxf(x, 0.f), g.rmax);
    float yc = fminf(fmaxf(y, 0.f), g.cmax);
    s.i0 = ffloor(xc, s.fx);
    s.j0 = ffloor(yc, s.fy);
    return s;
}

__device__ __forceinline__ Smp sample(const Geo& g, int h, int w) {
    const float hf = (float)h - g.cy;
    return sample_xy(g, fmaf(g.c, hf, col_bx(g, w)), fmaf(g.s, hf, col_by(g, w)));
}

// Bilinear value of img (row stride `pitch`) at a clamped sample.
__device__ __forceinline__ float bilerp(const float* img, int pitch, const Smp& s) {
    const float* p = img + s.i0 * pitch + s.j0;
    float t = fmaf(s.fy, p[1] - p[0], p[0]);
    float b = fmaf(s.fy, p[pitch + 1] - p[pitch], p[pitch]);
    return fmaf(s.fx, b - t, t);
}

// ---------------------------------------------------------------------------
// grid_sample rotation (FL/torch_image_util.py:13-114): out(h,w) samples the
// input at ix = c*(w-cx) - s*(h-cy)*(W/H) + cx, iy = s*(w-cx)*(H/W) + c*(h-cy) + cy
// (affine_grid [[c,-s,0],[s,c,0]], align_corners=False), bilinear, zero padding.
// ---------------------------------------------------------------------------
struct RotGeom {
    float c, s, cx, cy, sxw, syh;  // sxw = W/H, syh = H/W
};

__host__ __device__ inline RotGeom rot_geom(float c, float s, int H, int W) {
    RotGeom g;
    g.c = c;
    g.s = s;
    g.cx = (W - 1) * 0.5f;
    g.cy = (H - 1) * 0.5f;
    g.sxw = (float)W / (float)H;
    g.syh = (float)H / (float)W;
    return g;
}

// The four taps of a rotation sample: corner (x0, y0) and weights; a tap
// outside the image contributes zero.
struct RotTap {
    int x0, y0;
    float tx, ty;
    bool inside;   // the sample point lies in [0, W-1] x [0, H-1]
};

__device__ __forceinline__ RotTap rot_tap(const RotGeom& g, int h, int w) {
    float dw = (float)w - g.cx, dh = (float)h - g.cy;
    float ix = g.c * dw - g.s * dh * g.sxw + g.cx;
    float iy = g.s * dw * g.syh + g.c * dh + g.cy;
    float fx = floorf(ix), fy = floorf(iy);
    RotTap t;
    t.x0 = (int)fx;
    t.y0 = (int)fy;
    t.tx = ix - fx;
    t.ty = iy - fy;
    t.inside = ix >= 0.f && ix <= 2.f * g.cx && iy >= 0.f && iy <= 2.f * g.cy;
    return t;
}

// The row coordinate iy of rot_tap's sample point.
__device__ __forceinline__ float rot_tap_y(const RotGeom& g, int h, int w) {
    const float dw = (float)w - g.cx, dh = (float)h - g.cy;
    return g.s * dw * g.syh + g.c * dh + g.cy;
}

__device__ __forceinline__ float rot_sample_tap(const float* __restrict__ img, int H, int W,
                                                const RotTap& t) {
    const int x0 = t.x0, y0 = t.y0;
    bool xin0 = x0 >= 0 && x0 < W, xin1 = x0 + 1 >= 0 && x0 + 1 < W;
    bool yin0 = y0 >= 0 && y0 < H, yin1 = y0 + 1 >= 0 && y0 + 1 < H;
    float v00 = (yin0 && xin0) ? __ldg(img + y0 * W + x0) : 0.f;
    float v01 = (yin0 && xin1) ? __ldg(img + y0 * W + x0 + 1) : 0.f;
    float v10 = (yin1 && xin0) ? __ldg(img + (y0 + 1) * W + x0) : 0.f;
    float v11 = (yin1 && xin1) ? __ldg(img + (y0 + 1) * W + x0 + 1) : 0.f;
    float top = fmaf(t.tx, v01 - v00, v00);
    float bot = fmaf(t.tx, v11 - v10, v10);
    return fmaf(t.ty, bot - top, top);
}

__device__ __forceinline__ float rot_sample(const float* __restrict__ img, int H, int W,
                                            const RotGeom& g, int h, int w) {
    return rot_sample_tap(img, H, W, rot_tap(g, h, w));
}

// scipy.ndimage.rotate(order=1, reshape=False, mode='constant') -- the
// reference's rot3D (FL/image_util.py:165-203): the same sample point and
// bilinear weights as rot_sample inside [0, W-1] x [0, H-1], zero outside
// (no interpolation against the padding within one pixel of the border).
__device__ __forceinline__ float rot_sample_scipy(const float* __restrict__ img, int H, int W,
                                                  const RotGeom& g, int h, int w) {
    const RotTap t = rot_tap(g, h, w);
    return t.inside ? rot_sample_tap(img, H, W, t) : 0.f;
}

}  // namespace flc
