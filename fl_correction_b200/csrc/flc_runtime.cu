// Error reporting, device queries and the device-resident MLEM driver.
//
// MLEM follows FL/cuda_lib/atten_cuda.cpp:283-345 (mlem_cuda_batch) step by
// step, but nothing is allocated per iteration: the caller hands in one
// workspace, the sensitivity is computed once, and each iteration is either
// one fused cluster launch (when a slice of C plus its accumulator fit in
// shared memory) or three launches (forward+ratio, backward, update).  With
// use_graph the two-iteration ping-pong body is captured once into a CUDA
// graph and replayed.

#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>

#include "flc_common.cuh"

namespace flc {

namespace {
std::atomic<uint64_t> g_launches{0};
thread_local char g_err[1024] = {0};
int g_sms[64] = {0};
int g_smem[64] = {0};
int g_smem_sm[64] = {0};
std::mutex g_mu;
}  // namespace

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

void clear_error() { g_err[0] = 0; }

void count_launches(int64_t n) { g_launches.fetch_add((uint64_t)n); }
uint64_t launches() { return g_launches.load(); }

int cuda_fail(cudaError_t e, const char* what) {
    set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return FLC_ERR_CUDA;
}

static void query_device(int dev) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= 64 || g_sms[dev]) return;
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    g_sms[dev] = v > 0 ? v : 1;
    v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    g_smem[dev] = v > 0 ? v : 48 * 1024;
    v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    g_smem_sm[dev] = v > 0 ? v : g_smem[dev];
}

namespace {
std::atomic<int64_t> g_tune[kTuneCount];
const char* const kTuneNames[kTuneCount] = {"proj.cluster", "proj.apc", "cone.variant",
                                            "atten.chunk", "proj.bwd", "cone.test_wait_limit",
                                            "cone.test_skip_load", "proj.legacy", "proj.band",
                                            "xrf.band"};
}  // namespace

int64_t tune(int key) { return (key >= 0 && key < kTuneCount) ? g_tune[key].load() : 0; }

int tune_index(const char* name) {
    for (int i = 0; i < kTuneCount; ++i)
        if (name && strcmp(name, kTuneNames[i]) == 0) return i;
    return -1;
}

int sm_count() {
    int dev = 0;
    cudaGetDevice(&dev);
    query_device(dev);
    return (dev >= 0 && dev < 64) ? g_sms[dev] : 148;
}

int smem_per_sm() {
    int dev = 0;
    cudaGetDevice(&dev);
    query_device(dev);
    return (dev >= 0 && dev < 64) ? g_smem_sm[dev] : 228 * 1024;
}

int max_smem_optin() {
    int dev = 0;
    cudaGetDevice(&dev);
    query_device(dev);
    return (dev >= 0 && dev < 64) ? g_smem[dev] : 227 * 1024;
}

// Launchers defined in flc_project.cu.
int bwd_emission_launch(const float* atten, const float* ratio, const float* em,
                        const float* theta, float* out, int64_t A, int64_t B, int64_t R,
                        int64_t H, int64_t W, float clamp_min, cudaStream_t st);
int fwd_emission_launch(const float* atten, const float* C, const float* em, const float* theta,
                        float* Pf, const float* I, int64_t A, int64_t B, int64_t R, int64_t H,
                        int64_t W, cudaStream_t st);
int mlem_iter_launch(const float* atten, const float* em, const float* theta, const float* I,
                     const float* sens, const float* Cin, float* Cout, int64_t A, int64_t B,
                     int64_t R, int64_t H, int64_t W, float beta, float delta, cudaStream_t st,
                     bool* fused, float* ratio_ws);
void mlem_iter_prepare(int64_t A, int64_t B, int64_t R, int64_t H, int64_t W);

namespace {

// Unfused update: C' = max(C*back/(sens + beta*huber(C)), 0).
__global__ void mlem_update_kernel(const float* __restrict__ back, const float* __restrict__ sens,
                                   const float* __restrict__ Cin, float* __restrict__ Cout,
                                   int64_t n, int H, int W, float beta, float delta) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float cp = Cin[i];
    float den = sens[i];
    if (beta > 0.f) {
        int64_t img = i / ((int64_t)H * W);
        int rem = (int)(i - img * H * W);
        int r = rem / W, c = rem - r * W;
        const float* p = Cin + img * H * W;
        const int dr[4] = {-1, 1, 0, 0};
        const int dc[4] = {0, 0, -1, 1};
        float g = 0.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int rr = r + dr[k], cc = c + dc[k];
            if (rr < 0 || rr >= H || cc < 0 || cc >= W) continue;
            float d = cp - p[rr * W + cc];
            g += fabsf(d) <= delta ? d : copysignf(delta, d);
        }
        den = __fadd_rn(den, __fmul_rn(beta, g));
    }
    Cout[i] = fmaxf(__fmul_rn(cp, back[i]) / den, 0.f);
}

struct MlemBufs {
    float* sens;
    float* alt;    // ping-pong partner of C
    float* ratio;  // (A,B,W)      unfused path only
    float* back;   // (R,B,H,W)    unfused path only
};

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

size_t mlem_layout(int64_t A, int64_t B, int64_t R, int64_t H, int64_t W, char* base,
                   MlemBufs* m) {
    size_t nC = align256(sizeof(float) * R * B * H * W);
    size_t nP = align256(sizeof(float) * A * B * W);
    if (m) {
        m->sens = (float*)(base);
        m->alt = (float*)(base + nC);
        m->ratio = (float*)(base + 2 * nC);
        m->back = (float*)(base + 2 * nC + nP);
    }
    return 3 * nC + nP;
}

int mlem_step(const float* atten, const float* em, const float* theta, const float* I,
              const MlemBufs& m, const float* Cin, float* Cout, int64_t A, int64_t B, int64_t R,
              int64_t H, int64_t W, float beta, float delta, cudaStream_t st) {
    bool fused = false;
    FLC_TRY(mlem_iter_launch(atten, em, theta, I, m.sens, Cin, Cout, A, B, R, H, W, beta, delta,
                             st, &fused, m.ratio));
    if (fused) return FLC_OK;
    FLC_TRY(fwd_emission_launch(atten, Cin, em, theta, m.ratio, I, A, B, R, H, W, st));
    FLC_TRY(bwd_emission_launch(atten, m.ratio, em, theta, m.back, A, B, R, H, W, 0.f, st));
    int64_t n = R * B * H * W;
    mlem_update_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(m.back, m.sens, Cin, Cout, n,
                                                                   (int)H, (int)W, beta, delta);
    return check_launch("mlem_update_kernel");
}

}  // namespace
}  // namespace flc

using namespace flc;

extern "C" const char* flc_status_string(int s) {
    switch (s) {
        case FLC_OK: return "FLC_OK";
        case FLC_ERR_INVALID_ARG: return "FLC_ERR_INVALID_ARG";
        case FLC_ERR_UNSUPPORTED: return "FLC_ERR_UNSUPPORTED";
        case FLC_ERR_ALIGNMENT: return "FLC_ERR_ALIGNMENT";
        case FLC_ERR_WORKSPACE: return "FLC_ERR_WORKSPACE";
        case FLC_ERR_CUDA: return "FLC_ERR_CUDA";
        case FLC_ERR_TIMEOUT: return "FLC_ERR_TIMEOUT";
        case FLC_ERR_OOM: return "FLC_ERR_OOM";
        default: return "FLC_ERR_UNKNOWN";
    }
}

extern "C" const char* flc_last_error(void) { return g_err; }

extern "C" const char* flc_version(void) { return "flc-b200 0.1.0 (sm_100a)"; }

extern "C" uint64_t flc_launch_count(void) { return launches(); }

extern "C" size_t flc_mlem_workspace_bytes(int64_t A, int64_t B, int64_t R, int64_t H, int64_t W) {
    if (A < 1 || B < 1 || R < 1 || H < 1 || W < 1) return 0;
    return mlem_layout(A, B, R, H, W, nullptr, nullptr);
}

extern "C" int flc_mlem(float* C, const float* atten, const float* em, const float* theta,
                        const float* I, int64_t n_iter, double beta, double delta, int64_t A,
                        int64_t B, int64_t R, int64_t H, int64_t W, void* workspace,
                        size_t workspace_bytes, int use_graph, void* stream) {
    clear_error();
    FLC_REQUIRE(C && atten && em && theta && I, "flc_mlem: null pointer argument");
    FLC_REQUIRE(A >= 1 && B >= 1 && R >= 1 && H >= 2 && W >= 2 && n_iter >= 0,
                "flc_mlem: invalid sizes");
    FLC_REQUIRE(workspace != nullptr, "flc_mlem: workspace is required");
    if (((uintptr_t)workspace & 255) != 0) {
        set_error("flc_mlem: workspace must be 256-byte aligned");
        return FLC_ERR_ALIGNMENT;
    }
    size_t need = mlem_layout(A, B, R, H, W, nullptr, nullptr);
    if (workspace_bytes < need) {
        set_error("flc_mlem: workspace of %zu bytes is smaller than the %zu required",
                  workspace_bytes, need);
        return FLC_ERR_WORKSPACE;
    }
    cudaStream_t st = as_stream(stream);
    MlemBufs m;
    mlem_layout(A, B, R, H, W, (char*)workspace, &m);
    // sens = max(P^T 1, 1e-6)   (atten_cuda.cpp:308-314)
    FLC_TRY(bwd_emission_launch(atten, nullptr, em, theta, m.sens, A, B, R, H, W, 1e-6f, st));
    if (n_iter == 0) return FLC_OK;
    const float fb = (float)beta, fd = (float)delta;
    const int64_t nC = R * B * H * W;
    if (!use_graph || n_iter < 4) {
        const float* cur = C;
        float* nxt = m.alt;
        for (int64_t it = 0; it < n_iter; ++it) {
            FLC_TRY(mlem_step(atten, em, theta, I, m, cur, nxt, A, B, R, H, W, fb, fd, st));
            float* done = nxt;
            nxt = (float*)cur;
            cur = done;
        }
        if (cur != C)
            FLC_TRY_CUDA(cudaMemcpyAsync(C, cur, sizeof(float) * nC, cudaMemcpyDeviceToDevice, st));
        return check_launch("flc_mlem");
    }
    // Capture C -> alt -> C once; replay n_iter/2 times; odd tail runs eagerly.
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int status = FLC_OK;
    mlem_iter_prepare(A, B, R, H, W);
    FLC_TRY_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    do {
        const uint64_t before = launches();
        if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            status = cuda_fail(cudaGetLastError(), "cudaStreamBeginCapture");
            break;
        }
        int s1 = mlem_step(atten, em, theta, I, m, C, m.alt, A, B, R, H, W, fb, fd, cap);
        int s2 = s1 == FLC_OK ? mlem_step(atten, em, theta, I, m, m.alt, C, A, B, R, H, W, fb, fd, cap)
                              : s1;
        cudaError_t e = cudaStreamEndCapture(cap, &graph);
        // captured launches run only when the graph is replayed
        const int64_t body = (int64_t)(launches() - before);
        count_launches(-body);
        if (s2 != FLC_OK) { status = s2; break; }
        if (e != cudaSuccess) { status = cuda_fail(e, "cudaStreamEndCapture"); break; }
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) { status = cuda_fail(e, "cudaGraphInstantiate"); break; }
        for (int64_t it = 0; it + 1 < n_iter; it += 2) {
            e = cudaGraphLaunch(exec, st);
            if (e != cudaSuccess) { status = cuda_fail(e, "cudaGraphLaunch"); break; }
            count_launches(body);
        }
        if (status != FLC_OK) break;
        if (n_iter & 1) {
            status = mlem_step(atten, em, theta, I, m, C, m.alt, A, B, R, H, W, fb, fd, st);
            if (status != FLC_OK) break;
            e = cudaMemcpyAsync(C, m.alt, sizeof(float) * nC, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) { status = cuda_fail(e, "cudaMemcpyAsync"); break; }
        }
    } while (0);
    // An executable graph destroyed while in flight is released on completion.
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cap);
    return status;
}

extern "C" int flc_tune_set(const char* name, int64_t value) {
    clear_error();
    int k = tune_index(name);
    if (k < 0) {
        set_error("flc_tune_set: unknown knob '%s'", name ? name : "(null)");
        return FLC_ERR_INVALID_ARG;
    }
    if (value < 0) {
        set_error("flc_tune_set: value must be >= 0 (0 = automatic)");
        return FLC_ERR_INVALID_ARG;
    }
    g_tune[k].store(value);
    return FLC_OK;
}

extern "C" int64_t flc_tune_get(const char* name) {
    int k = tune_index(name);
    return k < 0 ? -1 : g_tune[k].load();
}
