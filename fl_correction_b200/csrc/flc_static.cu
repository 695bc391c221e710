// MLEM with its scratch in a fixed device array instead of a caller workspace.
//
// flc_mlem needs flc_mlem_workspace_bytes(...) of device scratch from its
// caller.  Some callers cannot provide it: a host bound to the C ABI through
// an FFI that hands over only the data buffers and owns no device allocator,
// or a process whose device memory is reserved up front by another
// framework's pool.  flc_mlem_static serves them: the scratch is the
// file-scope array below, so the call allocates nothing.
//
// Limits and rules:
//  * the scratch holds kStaticScratchBytes (32 MiB); problems whose MLEM
//    workspace is larger are refused with FLC_ERR_UNSUPPORTED;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current) -- make
//    that first call before any stream capture.  Under lazy module loading
//    (the CUDA default) that lookup is also when the driver loads this module
//    and commits the 32 MiB on the device (CUDA_MODULE_LOADING=EAGER commits
//    it when the library loads): a process that hands its device memory to
//    another framework's pool should make the first call at start-up, before
//    the pool reserves the memory;
//  * the looked-up address is kept per device ordinal and belongs to the
//    device's primary context: only the runtime's primary context is
//    supported, and cudaDeviceReset must not be called between calls;
//  * every call uses the same array, so calls that overlap in time (other
//    streams, other host threads) race on it;
//  * the eager iteration path runs (no CUDA graph, no stream creation).
//    Nothing in the MLEM scratch is read before it is written within a call,
//    so nothing needs clearing between calls.

#include <mutex>

#include "flc_common.cuh"

namespace flc {
namespace {

constexpr size_t kStaticScratchBytes = 32u << 20;

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mu;
void* g_static_ptr[64] = {nullptr};

// Device address of g_static_scratch on the current device (looked up once).
int static_scratch(void** out) {
    int dev = 0;
    FLC_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("flc_mlem_static: device ordinal %d out of range", dev);
        return FLC_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_ptr[dev]) {
        void* p = nullptr;
        FLC_TRY_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
        g_static_ptr[dev] = p;
    }
    *out = g_static_ptr[dev];
    return FLC_OK;
}

}  // namespace
}  // namespace flc

using namespace flc;

extern "C" size_t flc_mlem_workspace_bytes(int64_t A, int64_t B, int64_t R, int64_t H, int64_t W);
extern "C" int flc_mlem(float* C, const float* atten, const float* em, const float* theta,
                        const float* I, int64_t n_iter, double beta, double delta, int64_t A,
                        int64_t B, int64_t R, int64_t H, int64_t W, void* workspace,
                        size_t workspace_bytes, int use_graph, void* stream);

extern "C" int flc_mlem_static(float* C, const float* atten, const float* em, const float* theta,
                               const float* I, int64_t n_iter, double beta, double delta,
                               int64_t A, int64_t B, int64_t R, int64_t H, int64_t W,
                               void* stream) {
    clear_error();
    const size_t need = flc_mlem_workspace_bytes(A, B, R, H, W);
    FLC_REQUIRE(need > 0, "flc_mlem_static: invalid sizes");
    if (need > kStaticScratchBytes) {
        set_error("flc_mlem_static: this problem needs %zu bytes of scratch, more than the %zu "
                  "of the static array; use flc_mlem with a caller workspace",
                  need, kStaticScratchBytes);
        return FLC_ERR_UNSUPPORTED;
    }
    void* ws = nullptr;
    FLC_TRY(static_scratch(&ws));
    return flc_mlem(C, atten, em, theta, I, n_iter, beta, delta, A, B, R, H, W, ws,
                    kStaticScratchBytes, 0, stream);
}
