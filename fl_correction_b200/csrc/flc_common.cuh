// Shared helpers for the sm_100a kernels of the XRF self-absorption path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/flc.h"

namespace flc {

// Records a printf-style message as the calling thread's last error.
void set_error(const char* fmt, ...);
void clear_error();

// Maps a CUDA error to FLC_ERR_CUDA with a message naming `what`.
int cuda_fail(cudaError_t e, const char* what);

// Kernel-launch counter behind flc_launch_count().
void count_launches(int64_t n);
uint64_t launches();

// Checks the launch just issued (configuration errors are synchronous) and
// counts it.
inline int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, what);
    count_launches(1);
    return FLC_OK;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Launch-shape knobs (set by the autotuner through flc_tune_set; 0 = auto).
enum TuneKey {
    kTuneProjCluster = 0,   // CTAs per slice cluster for the backward / MLEM kernels
    kTuneProjApc = 1,       // angles per CTA for the projector kernels
    kTuneConeVariant = 2,   // 1: TMA 16x8 tile, 2: TMA 8x4 tile, 3: plain kernel
    kTuneAttenChunk = 3,    // angles per attenuation-pipeline pass
    kTuneProjBwd = 4,       // backward splat: 1 shared atomics, 0/2 nine disjoint phases
    kTuneCount = 5
};
int64_t tune(int key);

// Number of SMs of the current device (cached per device).
int sm_count();
// Opt-in shared memory per block of the current device (cached per device).
int max_smem_optin();

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Bit of the cone `mode` argument that selects the plain separable kernel
// over the TMA-pipelined one (for parity tests of both).
constexpr int kConePlain = 0x100;

// Device-side status left by bounded waits that gave up (flc_cone.cu).
int cone_device_status(int reset);

}  // namespace flc

#define FLC_REQUIRE(cond, ...)                      \
    do {                                            \
        if (!(cond)) {                              \
            flc::set_error(__VA_ARGS__);            \
            return FLC_ERR_INVALID_ARG;             \
        }                                           \
    } while (0)

#define FLC_TRY_CUDA(call)                                   \
    do {                                                     \
        cudaError_t e__ = (call);                            \
        if (e__ != cudaSuccess) return flc::cuda_fail(e__, #call); \
    } while (0)

#define FLC_TRY(call)                  \
    do {                               \
        int s__ = (call);              \
        if (s__ != FLC_OK) return s__; \
    } while (0)

// -------------------------------------------------------------------------
// Projector geometry of the reference (atten_cuda_kernel.cu:91-142,
// :271-337): the sample for detector column w at beam step h of angle th is
//   row = c*(h-cy) - s*(w-cx) + cy,   col = s*(h-cy) + c*(w-cx) + cx
// with c = cos(-th), s = sin(-th), cx = (W-1)/2, cy = (H-1)/2, clamped to
// [0, H-1.001] x [0, W-1.001], then bilinear on the four neighbours.
// -------------------------------------------------------------------------
struct ProjGeom {
    float c, s, cx, cy, rmax, cmax;
};

__device__ __forceinline__ ProjGeom proj_geom(float th, int H, int W) {
    ProjGeom g;
    g.c = cosf(-th);
    g.s = sinf(-th);
    g.cx = (W - 1) * 0.5f;
    g.cy = (H - 1) * 0.5f;
    g.rmax = H - 1.001f;
    g.cmax = W - 1.001f;
    return g;
}

// One clamped bilinear sample: top-left corner (i0, j0) and fractions.
struct Tap {
    int i0, j0;
    float fr, fc;
};

__device__ __forceinline__ Tap proj_tap(const ProjGeom& g, float hf, float wf) {
    float r = g.c * (hf - g.cy) - g.s * (wf - g.cx) + g.cy;
    float q = g.s * (hf - g.cy) + g.c * (wf - g.cx) + g.cx;
    r = fminf(fmaxf(r, 0.f), g.rmax);
    q = fminf(fmaxf(q, 0.f), g.cmax);
    Tap t;
    float r0 = floorf(r), q0 = floorf(q);
    t.i0 = (int)r0;
    t.j0 = (int)q0;
    t.fr = r - r0;
    t.fc = q - q0;
    return t;
}
