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
    kTuneConeVariant = 2,   // 1: TMA 16x8 tile, 2: TMA 8x4 tile, 3: plain kernel, 4: spectral
    kTuneAttenChunk = 3,    // angles per attenuation-pipeline pass
    kTuneProjBwd = 4,       // backward: 0 automatic, 1 shared-atomic splat, 2 nine-phase
                            // splat, 3 gather, 4 column segments
    // test hooks of the bounded waits (0 = off): the polls a TMA-cone wait
    // makes before it gives up, and a plane step (1-based) whose TMA load is
    // not issued, so that its wait runs out and the kernel reports
    // FLC_ERR_TIMEOUT without faulting
    kTuneConeWaitLimit = 5,
    kTuneConeSkipLoad = 6,
    kTuneProjLegacy = 7,    // 1: the earlier projector / fused-MLEM kernels instead of
                            // the two lean kernels (for comparison)
    kTuneProjBand = 8,      // 1: the band backward at every slice size (it runs by
                            // itself only where the lean kernel's image does not fit)
    kTuneXrfBand = 9,       // rows per band of the XRF rotation adjoint (by itself it
                            // bands only slices that do not fit in shared memory)
    kTuneCount = 10
};
int64_t tune(int key);

// Number of SMs of the current device (cached per device).
int sm_count();
// Opt-in shared memory per block of the current device (cached per device).
int max_smem_optin();
// Shared memory per SM of the current device (cached per device).
int smem_per_sm();

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
