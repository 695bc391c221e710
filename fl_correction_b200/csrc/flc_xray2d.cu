// Incident X-ray attenuation of one slice from reference-spectrum volumes
// (FL/torch_functions.py:181-215 torch_2D_xray_atten_with_ref and :247-330
// torch_2D_xray_atten_with_ref_vectorize).
//
// Both reference functions scale the n_ref reference volumes C (n_ref, H, W)
// by 1 / (max over pixels of sum_j C_j + C_other + eps), rotate them to each
// angle, assemble mu = (sum_j cs_ref[a][j] * frac_j) * rho * pix with the
// UNROTATED per-pixel map rho, and take the product of max(1 - mu, floor)
// along the rows below each pixel.  They differ in details that change the
// numbers, and each variant keeps its own:
//
//   variant 0 (torch_2D_xray_atten_with_ref): eps 1e-9, rotation with
//     align_corners=False (torch_rotate_image_nd), floor 1e-6, exclusive
//     product  out[h] = prod_{h' > h} f[h'],  out[H-1] = 1;
//   variant 1 (_vectorize): eps 1e-8, rotation with align_corners=True,
//     mu clipped at 0 (relu), floor 1e-8, and the product of its
//     flip / cumprod / shift (:320-327): out[h] = prod_{h' >= h} f[h'] for
//     h < H-1 -- row h itself included -- and out[H-1] = 1.
//
// Layout: one thread per (angle, column); it walks its column from the
// bottom row up with the running product in a register, sampling every
// reference volume bilinearly at the rotated point (the volumes of one slice
// stay in L2).  A single-CTA kernel first reduces the normaliser.

#include "flc_common.cuh"
#include "flc_geom.cuh"

namespace flc {
namespace {

constexpr int kColThreads = 128;
constexpr int kNormThreads = 1024;

// den = max_p (sum_j C[j][p] + C_other[p]) + eps, in the reference's order
// (sum over j first, then C_other).
__global__ void __launch_bounds__(kNormThreads)
    ref2d_norm_kernel(const float* __restrict__ C, const float* __restrict__ C_other, int n_ref,
                      int64_t HW, float eps, float* __restrict__ den) {
    __shared__ float red[kNormThreads / 32];
    float m = -INFINITY;
    for (int64_t p = threadIdx.x; p < HW; p += blockDim.x) {
        float s = 0.f;
        for (int j = 0; j < n_ref; ++j) s += __ldg(C + j * HW + p);
        m = fmaxf(m, s + __ldg(C_other + p));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : -INFINITY;
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) *den = m + eps;
    }
}

struct Ref2dArgs {
    const float* C;        // (n_ref, H, W)
    const float* rho;      // (H, W)
    const float* cs;       // (A, n_ref)
    const float* theta;    // (A,) radians
    const float* den;      // normaliser (device scalar)
    float* out;            // (A, H, W)
    int n_ref, H, W, variant;
    float pix;
};

__global__ void __launch_bounds__(kColThreads) ref2d_atten_kernel(Ref2dArgs p) {
    const int w = blockIdx.x * kColThreads + threadIdx.x;
    const int a = blockIdx.y;
    if (w >= p.W) return;
    const int H = p.H, W = p.W;
    const int64_t HW = (int64_t)H * W;
    // the FP32 rotation matrix: variant 0 rounds the FP64 cos / sin of the
    // FP32 angle (math.cos of a tensor element), variant 1 takes the FP32
    // functions of the tensor (torch.cos)
    const float th = p.theta[a];
    const float c = p.variant == 1 ? cosf(th) : (float)cos((double)th);
    const float sn = p.variant == 1 ? sinf(th) : (float)sin((double)th);
    RotGeom g = rot_geom(c, sn, H, W);
    if (p.variant == 1) {
        // affine_grid / grid_sample with align_corners=True: the normalised
        // coordinates span pixel centres, so the aspect factors are (W-1)/(H-1)
        g.sxw = (float)(W - 1) / (float)(H - 1);
        g.syh = (float)(H - 1) / (float)(W - 1);
    }
    const float den = *p.den;
    const float floor_f = p.variant == 1 ? 1e-8f : 1e-6f;
    const float* cs = p.cs + (int64_t)a * p.n_ref;
    float* out = p.out + (int64_t)a * HW + w;
    float prod = 1.f;
    out[(int64_t)(H - 1) * W] = 1.f;
    for (int h = H - 1; h >= 0; --h) {
        const RotTap t = rot_tap(g, h, w);
        const float rp = __ldg(p.rho + (int64_t)h * W + w);
        float mu = 0.f;
        if (p.variant == 1) {
            for (int j = 0; j < p.n_ref; ++j)
                mu += (rot_sample_tap(p.C + j * HW, H, W, t) / den) * __ldg(cs + j);
            mu = fmaxf(mu * rp * p.pix, 0.f);
        } else {
            for (int j = 0; j < p.n_ref; ++j)
                mu += __ldg(cs + j) * (rot_sample_tap(p.C + j * HW, H, W, t) / den) * rp * p.pix;
        }
        const float f = fmaxf(1.f - mu, floor_f);
        if (p.variant == 1) {
            prod *= f;
            if (h < H - 1) out[(int64_t)h * W] = prod;
        } else {
            if (h < H - 1) out[(int64_t)h * W] = prod;
            prod *= f;
        }
    }
}

}  // namespace
}  // namespace flc

using namespace flc;

extern "C" size_t flc_xray_atten_ref2d_workspace_bytes(void) { return 256; }

extern "C" int flc_xray_atten_ref2d(const float* C, const float* C_other, const float* theta,
                                    const float* cs_ref, const float* rho, float pix, float* out,
                                    int64_t n_ref, int64_t A, int64_t H, int64_t W, int variant,
                                    void* workspace, size_t workspace_bytes, void* stream) {
    clear_error();
    FLC_REQUIRE(C && C_other && theta && cs_ref && rho && out && workspace,
                "flc_xray_atten_ref2d: null pointer argument");
    FLC_REQUIRE(n_ref >= 1 && A >= 1 && H >= 2 && W >= 2 && H * W <= ((int64_t)1 << 30) &&
                    A <= 65535,
                "flc_xray_atten_ref2d: bad sizes n_ref=%lld A=%lld H=%lld W=%lld",
                (long long)n_ref, (long long)A, (long long)H, (long long)W);
    FLC_REQUIRE(variant == 0 || variant == 1, "flc_xray_atten_ref2d: variant must be 0 or 1");
    if (workspace_bytes < flc_xray_atten_ref2d_workspace_bytes()) {
        set_error("flc_xray_atten_ref2d: workspace of %zu bytes is smaller than the %zu required",
                  workspace_bytes, flc_xray_atten_ref2d_workspace_bytes());
        return FLC_ERR_WORKSPACE;
    }
    cudaStream_t st = as_stream(stream);
    float* den = (float*)workspace;
    ref2d_norm_kernel<<<1, kNormThreads, 0, st>>>(C, C_other, (int)n_ref, H * W,
                                                  variant == 1 ? 1e-8f : 1e-9f, den);
    FLC_TRY(check_launch("ref2d_norm_kernel"));
    Ref2dArgs p{C, rho, cs_ref, theta, den, out, (int)n_ref, (int)H, (int)W, variant, pix};
    dim3 grid((unsigned)ceil_div(W, kColThreads), (unsigned)A);
    ref2d_atten_kernel<<<grid, kColThreads, 0, st>>>(p);
    return check_launch("ref2d_atten_kernel");
}
