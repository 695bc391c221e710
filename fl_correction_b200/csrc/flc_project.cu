// Attenuated emission projector (forward / exact-transpose backward), the
// Huber term and the device-resident MLEM iteration, for sm_100a.
//
// Reference semantics: FL/cuda_lib/atten_cuda_kernel.cu:91-446,495-616 and
// FL/cuda_lib/atten_cuda.cpp:82-345.  The reference scatters with one global
// atomicAdd per sample (forward) and four per sample per reference
// (backward).  Here:
//  * one CTA owns one slice b and a group of angles; the slice of C is staged
//    once in shared memory (row pitch chosen to spread banks) and every
//    bilinear tap is a shared-memory load;
//  * the forward sums each detector column along the beam in registers and
//    combines a fixed number of partial sums in a fixed order (no atomics,
//    deterministic);
//  * the backward splats into a shared-memory accumulator of the whole slice;
//    the CTAs of one slice form a thread-block cluster and reduce their
//    accumulators through distributed shared memory in rank order, so no
//    partial buffer touches HBM;
//  * one MLEM iteration (forward, ratio, backward, Huber, update, clamp) is a
//    single cluster launch: atten streams from HBM once per iteration in the
//    forward pass and is re-read from L2 in the backward pass.

#include <cooperative_groups.h>

#include "flc_common.cuh"

namespace cg = cooperative_groups;

namespace flc {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxCluster = 8;
constexpr int kMaxR = 8;

// Row pitch (floats) of a staged slice: >= W and == 3 (mod 32), which keeps
// the warp's 32 rotated taps spread over banks for every angle class.
__host__ __device__ inline int slice_pitch(int W) {
    int p = W;
    while ((p & 31) != 3) ++p;
    return p;
}

// Partial sums per detector column: enough (w, part) items to fill the CTA.
__host__ __device__ inline int col_parts(int W, int H) {
    int p = (2 * kThreads + W - 1) / W;
    if (p > 8) p = 8;
    if (p > H) p = H;
    return p < 1 ? 1 : p;
}

__device__ __forceinline__ float bilerp(const float* img, int pitch, const Tap& t) {
    const float* p = img + t.i0 * pitch + t.j0;
    float v00 = p[0], v01 = p[1], v10 = p[pitch], v11 = p[pitch + 1];
    float top = fmaf(t.fc, v01 - v00, v00);
    float bot = fmaf(t.fc, v11 - v10, v10);
    return fmaf(t.fr, bot - top, top);
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

// Forward projection of one (angle, slice) into spart[parts][W]:
// spart[p][w] = sum over beam steps h of part p of atten * sum_r em_r * bilerp(C_r).
__device__ void forward_angle(const float* __restrict__ atten_ab, const float* sC,
                              int img_stride, int pitch, const float* em_a, int R,
                              const ProjGeom& g, int H, int W, int parts, float* spart) {
    int hper = (H + parts - 1) / parts;
    for (int item = threadIdx.x; item < parts * W; item += blockDim.x) {
        int part = item / W, w = item - part * W;
        int h0 = part * hper, h1 = min(H, h0 + hper);
        float wf = (float)w, acc = 0.f;
#pragma unroll 4
        for (int h = h0; h < h1; ++h) {
            float a = __ldg(atten_ab + (int64_t)h * W + w);
            Tap t = proj_tap(g, (float)h, wf);
            float val = 0.f;
            for (int r = 0; r < R; ++r) val = fmaf(em_a[r], bilerp(sC + r * img_stride, pitch, t), val);
            acc = fmaf(a, val, acc);
        }
        spart[part * W + w] = acc;
    }
}

// Backward (splat) of one (angle, slice) into the smem accumulator sacc[R][H][pitch]:
// sacc_r += em_r * atten * ratio[w] * bilinear weights, the transpose of forward_angle.
__device__ void backward_angle(const float* __restrict__ atten_ab, const float* sratio,
                               float* sacc, int img_stride, int pitch, const float* em_a, int R,
                               const ProjGeom& g, int H, int W, int parts) {
    int hper = (H + parts - 1) / parts;
    for (int item = threadIdx.x; item < parts * W; item += blockDim.x) {
        int part = item / W, w = item - part * W;
        int h0 = part * hper, h1 = min(H, h0 + hper);
        float wf = (float)w, rq = sratio[w];
#pragma unroll 2
        for (int h = h0; h < h1; ++h) {
            float av = __ldg(atten_ab + (int64_t)h * W + w) * rq;
            Tap t = proj_tap(g, (float)h, wf);
            float w00 = (1.f - t.fc) * (1.f - t.fr), w01 = t.fc * (1.f - t.fr);
            float w10 = (1.f - t.fc) * t.fr, w11 = t.fc * t.fr;
            for (int r = 0; r < R; ++r) {
                float v = em_a[r] * av;
                float* p = sacc + r * img_stride + t.i0 * pitch + t.j0;
                atomicAdd(p, v * w00);
                atomicAdd(p + 1, v * w01);
                atomicAdd(p + pitch, v * w10);
                atomicAdd(p + pitch + 1, v * w11);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Forward projection: grid (angle groups, B); optional MLEM ratio epilogue.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
proj_fwd_kernel(const float* __restrict__ atten, const float* __restrict__ C,
                const float* __restrict__ em, const float* __restrict__ theta,
                float* __restrict__ Pf, const float* __restrict__ I, int A, int B, int R,
                int H, int W, int apc, int staged) {
    extern __shared__ float smem[];
    const int b = blockIdx.y;
    const int a0 = blockIdx.x * apc, a1 = min(A, a0 + apc);
    const int pitch = staged ? slice_pitch(W) : W;
    const int parts = col_parts(W, H);
    const int img_stride = staged ? H * pitch : B * H * W;
    float* sC = smem;
    float* spart = smem + (staged ? R * H * pitch : 0);
    float* sem = spart + parts * W;
    const float* Cb = staged ? sC : C + (int64_t)b * H * W;
    if (staged) stage_slice(sC, C, R, B, b, H, W, pitch);
    for (int a = a0; a < a1; ++a) {
        if (threadIdx.x < R) sem[threadIdx.x] = em[a * R + threadIdx.x];
        __syncthreads();
        ProjGeom g = proj_geom(theta[a], H, W);
        const float* atten_ab = atten + ((int64_t)a * B + b) * H * W;
        forward_angle(atten_ab, Cb, img_stride, pitch, sem, R, g, H, W, parts, spart);
        __syncthreads();
        for (int w = threadIdx.x; w < W; w += blockDim.x) {
            float s = 0.f;
            for (int p = 0; p < parts; ++p) s += spart[p * W + w];
            int64_t o = ((int64_t)a * B + b) * W + w;
            if (I) s = I[o] / fmaxf(s, 1e-6f);
            Pf[o] = s;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Backward projection: grid (G, B), cluster (G, 1, 1).  CTA g of slice b
// splats angles [g*apc, (g+1)*apc) into its smem accumulator; the cluster
// then reduces the G accumulators in rank order, each CTA finishing a 1/G
// share of the slice.  ratio == nullptr means ratio = 1 (sensitivity).
// clamp_min > 0 applies max(out, clamp_min) (the reference's sens clamp).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
proj_bwd_kernel(const float* __restrict__ atten, const float* __restrict__ ratio,
                const float* __restrict__ em, const float* __restrict__ theta,
                float* __restrict__ out, int A, int B, int R, int H, int W, int apc,
                float clamp_min) {
    extern __shared__ float smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int G = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int b = blockIdx.y;
    const int a0 = blockIdx.x * apc, a1 = min(A, a0 + apc);
    const int pitch = slice_pitch(W);
    const int parts = col_parts(W, H);
    const int img_stride = H * pitch;
    float* sacc = smem;
    float* sratio = smem + R * img_stride;
    float* sem = sratio + W;
    for (int i = threadIdx.x; i < R * img_stride; i += blockDim.x) sacc[i] = 0.f;
    for (int a = a0; a < a1; ++a) {
        __syncthreads();
        if (threadIdx.x < R) sem[threadIdx.x] = em[a * R + threadIdx.x];
        for (int w = threadIdx.x; w < W; w += blockDim.x)
            sratio[w] = ratio ? ratio[((int64_t)a * B + b) * W + w] : 1.f;
        __syncthreads();
        ProjGeom g = proj_geom(theta[a], H, W);
        backward_angle(atten + ((int64_t)a * B + b) * H * W, sratio, sacc, img_stride, pitch,
                       sem, R, g, H, W, parts);
    }
    cluster.sync();
    const int64_t n = (int64_t)R * H * W;
    const int64_t share = (n + G - 1) / G;
    const int64_t i0 = rank * share, i1 = min(n, i0 + share);
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        int r = (int)(i / (H * W));
        int rem = (int)(i - (int64_t)r * H * W);
        int h = rem / W, w = rem - h * W;
        int off = r * img_stride + h * pitch + w;
        float s = 0.f;
        for (int q = 0; q < G; ++q) s += cluster.map_shared_rank(sacc, q)[off];
        if (clamp_min > 0.f) s = fmaxf(s, clamp_min);
        out[(((int64_t)r * B + b) * H + h) * W + w] = s;
    }
    cluster.sync();
}

// ---------------------------------------------------------------------------
// One fused MLEM iteration (grid (G, B), cluster (G,1,1)):
//   Pf = max(P C, 1e-6); ratio = I / Pf; back = P^T ratio;
//   C' = C*back / (sens + beta*huber(C))  (or C*back/sens), C' = max(C', 0)
// as atten_cuda.cpp:321-342.  Reads C from Cin, writes Cout (ping-pong:
// the Huber term needs the old neighbours).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
mlem_iter_kernel(const float* __restrict__ atten, const float* __restrict__ em,
                 const float* __restrict__ theta, const float* __restrict__ I,
                 const float* __restrict__ sens, const float* __restrict__ Cin,
                 float* __restrict__ Cout, int A, int B, int R, int H, int W, int apc,
                 float beta, float delta) {
    extern __shared__ float smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int G = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int b = blockIdx.y;
    const int a0 = blockIdx.x * apc, a1 = min(A, a0 + apc);
    const int pitch = slice_pitch(W);
    const int parts = col_parts(W, H);
    const int img_stride = H * pitch;
    float* sC = smem;
    float* sacc = sC + R * img_stride;
    float* spart = sacc + R * img_stride;
    float* sratio = spart + parts * W;
    float* sem = sratio + W;
    stage_slice(sC, Cin, R, B, b, H, W, pitch);
    for (int i = threadIdx.x; i < R * img_stride; i += blockDim.x) sacc[i] = 0.f;
    for (int a = a0; a < a1; ++a) {
        __syncthreads();
        if (threadIdx.x < R) sem[threadIdx.x] = em[a * R + threadIdx.x];
        __syncthreads();
        ProjGeom g = proj_geom(theta[a], H, W);
        const float* atten_ab = atten + ((int64_t)a * B + b) * H * W;
        forward_angle(atten_ab, sC, img_stride, pitch, sem, R, g, H, W, parts, spart);
        __syncthreads();
        for (int w = threadIdx.x; w < W; w += blockDim.x) {
            float s = 0.f;
            for (int p = 0; p < parts; ++p) s += spart[p * W + w];
            sratio[w] = I[((int64_t)a * B + b) * W + w] / fmaxf(s, 1e-6f);
        }
        __syncthreads();
        backward_angle(atten_ab, sratio, sacc, img_stride, pitch, sem, R, g, H, W, parts);
    }
    cluster.sync();
    const int64_t n = (int64_t)R * H * W;
    const int64_t share = (n + G - 1) / G;
    const int64_t i0 = rank * share, i1 = min(n, i0 + share);
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        int r = (int)(i / (H * W));
        int rem = (int)(i - (int64_t)r * H * W);
        int h = rem / W, w = rem - h * W;
        int off = r * img_stride + h * pitch + w;
        float back = 0.f;
        for (int q = 0; q < G; ++q) back += cluster.map_shared_rank(sacc, q)[off];
        const float* img = sC + r * img_stride;
        float cp = img[h * pitch + w];
        int64_t gi = (((int64_t)r * B + b) * H + h) * W + w;
        float den = sens[gi];
        if (beta > 0.f) {
            float hg = 0.f;
            const int dr[4] = {-1, 1, 0, 0};
            const int dc[4] = {0, 0, -1, 1};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                int rr = h + dr[k], cc = w + dc[k];
                if (rr < 0 || rr >= H || cc < 0 || cc >= W) continue;
                float d = cp - img[rr * pitch + cc];
                hg += fabsf(d) <= delta ? d : copysignf(delta, d);
            }
            den = __fadd_rn(den, __fmul_rn(beta, hg));
        }
        float c = __fmul_rn(cp, back) / den;
        Cout[gi] = fmaxf(c, 0.f);
    }
    cluster.sync();
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
    const int dr[4] = {-1, 1, 0, 0};
    const int dc[4] = {0, 0, -1, 1};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        int rr = r + dr[k], cc = c + dc[k];
        if (rr < 0 || rr >= H || cc < 0 || cc >= W) continue;
        float d = cp - p[rr * W + cc];
        g += fabsf(d) <= delta ? d : copysignf(delta, d);
    }
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

// Splits A angles into G groups so that G*B CTAs cover the SMs a few times.
Plan plan_cluster(int64_t A, int64_t B, size_t smem_per_cta) {
    Plan p;
    int sms = sm_count();
    int per_sm = (int)(max_smem_optin() / (smem_per_cta + 1024));
    if (per_sm < 1) per_sm = 1;
    int64_t want = 2LL * sms * per_sm;
    int G = (int)ceil_div(want, B);
    if (G > kMaxCluster) G = kMaxCluster;
    if (G > A) G = (int)A;
    if (G < 1) G = 1;
    p.G = G;
    p.apc = (int)ceil_div(A, G);
    p.G = (int)ceil_div(A, p.apc);
    p.smem = smem_per_cta;
    return p;
}

int launch_cluster(const void* fn, dim3 grid, int G, size_t smem, cudaStream_t st, void** args) {
    FLC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    FLC_TRY_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(kThreads);
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

size_t bwd_smem(int64_t R, int64_t H, int64_t W) {
    return sizeof(float) * (R * H * slice_pitch((int)W) + W + kMaxR);
}

size_t mlem_smem(int64_t R, int64_t H, int64_t W) {
    int parts = col_parts((int)W, (int)H);
    return sizeof(float) * (2 * R * H * slice_pitch((int)W) + parts * W + W + kMaxR);
}

}  // namespace

// Launches the backward projector (also used for the MLEM sensitivity).
int bwd_emission_launch(const float* atten, const float* ratio, const float* em,
                        const float* theta, float* out, int64_t A, int64_t B, int64_t R,
                        int64_t H, int64_t W, float clamp_min, cudaStream_t st) {
    size_t smem = bwd_smem(R, H, W);
    if (smem > (size_t)max_smem_optin()) {
        set_error("backward projector: slice %lldx%lld x R=%lld needs %zu B of shared memory (max %d)",
                  (long long)H, (long long)W, (long long)R, smem, max_smem_optin());
        return FLC_ERR_UNSUPPORTED;
    }
    Plan p = plan_cluster(A, B, smem);
    int iA = (int)A, iB = (int)B, iR = (int)R, iH = (int)H, iW = (int)W, apc = p.apc;
    void* args[] = {(void*)&atten, (void*)&ratio, (void*)&em, (void*)&theta, (void*)&out,
                    &iA, &iB, &iR, &iH, &iW, &apc, &clamp_min};
    return launch_cluster((const void*)proj_bwd_kernel, dim3(p.G, (unsigned)B), p.G, smem, st, args);
}

int fwd_emission_launch(const float* atten, const float* C, const float* em, const float* theta,
                        float* Pf, const float* I, int64_t A, int64_t B, int64_t R, int64_t H,
                        int64_t W, cudaStream_t st) {
    int parts = col_parts((int)W, (int)H);
    size_t staged_bytes = sizeof(float) * (R * H * slice_pitch((int)W) + parts * W + kMaxR);
    int staged = staged_bytes <= (size_t)max_smem_optin() ? 1 : 0;
    size_t smem = staged ? staged_bytes : sizeof(float) * (parts * W + kMaxR);
    int per_sm = (int)(max_smem_optin() / (smem + 1024));
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 8) per_sm = 8;
    int64_t want = 3LL * sm_count() * per_sm;
    int64_t groups = ceil_div(want, B);
    if (groups > A) groups = A;
    if (groups < 1) groups = 1;
    int apc = (int)ceil_div(A, groups);
    groups = ceil_div(A, apc);
    FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)proj_fwd_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    proj_fwd_kernel<<<dim3((unsigned)groups, (unsigned)B), kThreads, smem, st>>>(
        atten, C, em, theta, Pf, I, (int)A, (int)B, (int)R, (int)H, (int)W, apc, staged);
    return check_launch("proj_fwd_kernel");
}

int mlem_iter_launch(const float* atten, const float* em, const float* theta, const float* I,
                     const float* sens, const float* Cin, float* Cout, int64_t A, int64_t B,
                     int64_t R, int64_t H, int64_t W, float beta, float delta, cudaStream_t st,
                     bool* fused) {
    size_t smem = mlem_smem(R, H, W);
    *fused = smem <= (size_t)max_smem_optin();
    if (!*fused) return FLC_OK;
    Plan p = plan_cluster(A, B, smem);
    int iA = (int)A, iB = (int)B, iR = (int)R, iH = (int)H, iW = (int)W, apc = p.apc;
    void* args[] = {(void*)&atten, (void*)&em, (void*)&theta, (void*)&I, (void*)&sens,
                    (void*)&Cin, (void*)&Cout, &iA, &iB, &iR, &iH, &iW, &apc, &beta, &delta};
    return launch_cluster((const void*)mlem_iter_kernel, dim3(p.G, (unsigned)B), p.G, smem, st, args);
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

extern "C" int flc_huber_grad(const float* C, float* grad, int64_t RB, int64_t H, int64_t W,
                              float delta, void* stream) {
    clear_error();
    FLC_REQUIRE(C && grad, "flc_huber_grad: null pointer argument");
    FLC_REQUIRE(RB >= 1 && H >= 1 && W >= 1, "flc_huber_grad: sizes must be positive");
    return huber_launch(C, grad, RB, H, W, delta, as_stream(stream));
}
