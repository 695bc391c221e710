// cal_frac on the device (FL/core.py:159-205): the fractions that feed the
// attenuation from a set of concentration volumes.
//
//   img_sum = sum_i img[i] + 1e-12, times the threshold mask
//   tmp_i   = img[i] / img_sum with NaN, inf and negatives set to 0 (rm_abnormal)
//   scale_range (r0, r1): where tmp_i has more than 100 positive values,
//             tmp_i is clamped to [s_i[int(l*r0)], s_i[int(l*r1) - 1]], s_i the
//             sorted positive values of tmp_i and l their count
//   enable_scale: ratio = img_sum / p, p = the int(l*scale_limit)-th smallest
//             positive img_sum; else ratio = 1
//   frac_i  = tmp_i * mask * ratio
// The reference's threshold mask is scikit-image's multi-Otsu with hole
// filling and dilation (FL/image_util.py:337-371); when the threshold fails,
// as it does without scikit-image, cal_frac uses mask = 1 (FL/core.py:177-179).
// This entry point takes the mask from the caller (NULL: 1).
//
// The order statistics are exact: a radix select over the IEEE bit patterns
// of the positive values (which sort like unsigned integers), eight bits per
// pass from the most significant, every selection problem of the call in the
// same four histogram passes.  Arithmetic is FP32, as numpy does it on FP32
// volumes (the sum accumulates in channel order).

#include <algorithm>

#include "flc_common.cuh"

namespace flc {
namespace {

constexpr int kMaxFracCh = 8;
constexpr int kMaxSel = 1 + 2 * kMaxFracCh;

// One order-statistic problem: the k-th smallest positive value of src.
struct SelProb {
    const float* src;
    int64_t n;
    int rule;            // 0: k = int(l * a); 1: k = int(l * a) - 1 (l = positive count)
    double a;
    uint32_t prefix;     // bits fixed by the passes so far
    int64_t k;           // rank among the values that match the prefix
    int64_t count;       // positive values (set by the first pass)
    float value;
    int valid;           // 0 when there are no positive values (or the rank is out of range)
};

__global__ void frac_sum_kernel(const float* __restrict__ img, const float* __restrict__ mask,
                                float* __restrict__ sum, int n_ch, int64_t N) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N;
         v += (int64_t)gridDim.x * blockDim.x) {
        float s = __ldg(img + v);
        for (int i = 1; i < n_ch; ++i) s += __ldg(img + (int64_t)i * N + v);
        s += 1e-12f;
        if (mask) s *= __ldg(mask + v);
        sum[v] = s;
    }
}

__device__ __forceinline__ float rm_abnormal(float x) {
    return (isnan(x) || isinf(x) || x < 0.f) ? 0.f : x;
}

__global__ void frac_tmp_kernel(const float* __restrict__ img, const float* __restrict__ sum,
                                float* __restrict__ tmp, int n_ch, int64_t N) {
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N;
         v += (int64_t)gridDim.x * blockDim.x) {
        const float s = __ldg(sum + v);
        for (int i = 0; i < n_ch; ++i)
            tmp[(int64_t)i * N + v] = rm_abnormal(__ldg(img + (int64_t)i * N + v) / s);
    }
}

// Pass `pass` (0: bits 31..24, ... 3: bits 7..0): per problem, the histogram of
// the pass's digit over the positive values whose higher digits equal the
// prefix.  grid.y = problem.
__global__ void sel_hist_kernel(const SelProb* __restrict__ probs,
                                unsigned int* __restrict__ hist, int pass) {
    __shared__ unsigned int h[256];
    const SelProb p = probs[blockIdx.y];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int shift = 24 - 8 * pass;
    const uint32_t want = p.prefix;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < p.n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const float x = __ldg(p.src + v);
        if (!(x > 0.f)) continue;
        const uint32_t b = __float_as_uint(x);
        if (pass > 0 && (b >> (shift + 8)) != want) continue;
        atomicAdd(&h[(b >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[blockIdx.y * 256 + i], h[i]);
}

// One thread per problem: after the first pass, the positive count and the
// rank; then the bucket that holds the rank becomes the next prefix digit.
// Clears the histogram for the next pass.
__global__ void sel_step_kernel(SelProb* __restrict__ probs, unsigned int* __restrict__ hist,
                                int n_prob, int pass) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_prob) return;
    SelProb& p = probs[q];
    unsigned int* h = hist + q * 256;
    if (pass == 0) {
        int64_t l = 0;
        for (int i = 0; i < 256; ++i) l += h[i];
        p.count = l;
        int64_t k = (int64_t)((double)l * p.a) - (p.rule == 1 ? 1 : 0);
        p.valid = (l > 0 && k >= 0 && k < l) ? 1 : 0;
        p.k = p.valid ? k : 0;
        p.prefix = 0;
    }
    if (p.valid) {
        int64_t c = 0;
        int b = 0;
        for (; b < 255; ++b) {
            if (c + (int64_t)h[b] > p.k) break;
            c += h[b];
        }
        p.k -= c;
        p.prefix = (p.prefix << 8) | (uint32_t)b;
        if (pass == 3) p.value = __uint_as_float(p.prefix);
    }
    for (int i = 0; i < 256; ++i) h[i] = 0;
}

__global__ void frac_final_kernel(const float* __restrict__ tmp, const float* __restrict__ sum,
                                  const float* __restrict__ mask, const SelProb* __restrict__ probs,
                                  float* __restrict__ frac, int n_ch, int64_t N, int use_range,
                                  int enable_scale) {
    __shared__ float lo[kMaxFracCh], hi[kMaxFracCh], pmax;
    __shared__ int clamp_on[kMaxFracCh], scale_on;
    if (threadIdx.x == 0) {
        const SelProb& s0 = probs[0];
        scale_on = enable_scale && s0.valid;
        pmax = s0.value;
        for (int i = 0; i < n_ch; ++i) {
            const SelProb& a = probs[1 + 2 * i];
            const SelProb& b = probs[2 + 2 * i];
            clamp_on[i] = use_range && a.count > 100 && a.valid && b.valid;
            lo[i] = a.value;
            hi[i] = b.value;
        }
    }
    __syncthreads();
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N;
         v += (int64_t)gridDim.x * blockDim.x) {
        const float m = mask ? __ldg(mask + v) : 1.f;
        const float r = scale_on ? __ldg(sum + v) / pmax : 1.f;
        for (int i = 0; i < n_ch; ++i) {
            float t = __ldg(tmp + (int64_t)i * N + v);
            if (clamp_on[i]) {
                if (t >= hi[i]) t = hi[i];
                if (t <= lo[i]) t = lo[i];
            }
            frac[(int64_t)i * N + v] = t * m * r;
        }
    }
}

// The problem table, passed by value so that a call issues no host copy
// (and can be captured in a CUDA graph); also clears the histograms.
struct SelInit {
    SelProb p[kMaxSel];
    int n;
};

__global__ void sel_init_kernel(SelInit init, SelProb* __restrict__ probs,
                                unsigned int* __restrict__ hist) {
    for (int i = threadIdx.x; i < init.n; i += blockDim.x) probs[i] = init.p[i];
    for (int i = threadIdx.x; i < 256 * init.n; i += blockDim.x) hist[i] = 0;
}

size_t align256f(size_t n) { return (n + 255) & ~(size_t)255; }

size_t frac_ws_bytes(int64_t n_ch, int64_t N) {
    return align256f(sizeof(float) * (size_t)N) + align256f(sizeof(float) * (size_t)(n_ch * N)) +
           align256f(sizeof(SelProb) * kMaxSel) + align256f(sizeof(unsigned int) * 256 * kMaxSel);
}

}  // namespace
}  // namespace flc

using namespace flc;

extern "C" size_t flc_cal_frac_workspace_bytes(int64_t n_ch, int64_t N) {
    if (n_ch < 1 || n_ch > kMaxFracCh || N < 1) return 0;
    return frac_ws_bytes(n_ch, N);
}

extern "C" int flc_cal_frac(const float* img, const float* mask, float* frac, float* img_sum,
                            int64_t n_ch, int64_t N, int use_range, double r0, double r1,
                            int enable_scale, double scale_limit, void* workspace,
                            size_t workspace_bytes, void* stream) {
    clear_error();
    FLC_REQUIRE(img && frac && workspace, "flc_cal_frac: null pointer argument");
    FLC_REQUIRE(n_ch >= 1 && n_ch <= kMaxFracCh && N >= 1,
                "flc_cal_frac: 1 <= n_ch <= %d and N >= 1", kMaxFracCh);
    FLC_REQUIRE(!use_range || (r0 >= 0.0 && r1 <= 1.0 && r0 < r1),
                "flc_cal_frac: scale_range needs 0 <= r0 < r1 <= 1");
    FLC_REQUIRE(!enable_scale || (scale_limit >= 0.0 && scale_limit < 1.0),
                "flc_cal_frac: scale_limit must lie in [0, 1)");
    if (((uintptr_t)workspace & 255) != 0) {
        set_error("flc_cal_frac: workspace must be 256-byte aligned");
        return FLC_ERR_ALIGNMENT;
    }
    if (workspace_bytes < frac_ws_bytes(n_ch, N)) {
        set_error("flc_cal_frac: workspace of %zu bytes is smaller than the %zu required",
                  workspace_bytes, frac_ws_bytes(n_ch, N));
        return FLC_ERR_WORKSPACE;
    }
    cudaStream_t st = as_stream(stream);
    char* w = (char*)workspace;
    float* sum = (float*)w;
    w += align256f(sizeof(float) * (size_t)N);
    float* tmp = (float*)w;
    w += align256f(sizeof(float) * (size_t)(n_ch * N));
    SelProb* probs = (SelProb*)w;
    w += align256f(sizeof(SelProb) * kMaxSel);
    unsigned int* hist = (unsigned int*)w;
    const int threads = 256;
    const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(N, threads), 4L * sm_count());
    frac_sum_kernel<<<blocks, threads, 0, st>>>(img, mask, sum, (int)n_ch, N);
    FLC_TRY(check_launch("frac_sum_kernel"));
    frac_tmp_kernel<<<blocks, threads, 0, st>>>(img, sum, tmp, (int)n_ch, N);
    FLC_TRY(check_launch("frac_tmp_kernel"));
    // problems: 0 the scale percentile of the masked sum; 1 + 2i / 2 + 2i the
    // range ends of channel i
    SelInit init = {};
    const int n_prob = 1 + 2 * (int)n_ch;
    init.n = n_prob;
    init.p[0] = SelProb{sum, N, 0, enable_scale ? scale_limit : 0.0, 0, 0, 0, 0.f, 0};
    for (int i = 0; i < n_ch; ++i) {
        init.p[1 + 2 * i] = SelProb{tmp + i * N, N, 0, use_range ? r0 : 0.0, 0, 0, 0, 0.f, 0};
        init.p[2 + 2 * i] = SelProb{tmp + i * N, N, 1, use_range ? r1 : 1.0, 0, 0, 0, 0.f, 0};
    }
    sel_init_kernel<<<1, 256, 0, st>>>(init, probs, hist);
    FLC_TRY(check_launch("sel_init_kernel"));
    const unsigned hb = (unsigned)std::min<int64_t>(ceil_div(N, threads), 2L * sm_count());
    for (int pass = 0; pass < 4; ++pass) {
        sel_hist_kernel<<<dim3(hb, (unsigned)n_prob), threads, 0, st>>>(probs, hist, pass);
        FLC_TRY(check_launch("sel_hist_kernel"));
        sel_step_kernel<<<1, 32, 0, st>>>(probs, hist, n_prob, pass);
        FLC_TRY(check_launch("sel_step_kernel"));
    }
    frac_final_kernel<<<blocks, threads, 0, st>>>(tmp, sum, mask, probs, frac, (int)n_ch, N,
                                                  use_range, enable_scale);
    FLC_TRY(check_launch("frac_final_kernel"));
    if (img_sum)
        FLC_TRY_CUDA(cudaMemcpyAsync(img_sum, sum, sizeof(float) * N, cudaMemcpyDeviceToDevice, st));
    return FLC_OK;
}
