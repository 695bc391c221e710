/*
 * flc.h -- C ABI of the B200 (sm_100a) XRF self-absorption hot path.
 *
 * This library replaces the native layer of FL_correction
 * (FL/cuda_lib/atten_cuda.cpp + FL/cuda_lib/atten_cuda_kernel.cu).  Every
 * entry point takes plain device pointers, 64-bit sizes and a CUDA stream
 * (cudaStream_t passed as void*, NULL = legacy default stream), allocates
 * nothing unless it says so, and returns an flc_status.  It never aborts;
 * flc_last_error() returns a message describing the last failure on the
 * calling host thread.
 *
 * Layouts are C-contiguous float32 unless stated:
 *   atten  (A, B, H, W)   attenuation per angle, slice, row, column
 *   C      (R, B, H, W)   concentration per reference, slice, row, column
 *   em     (A, R)         emission cross-section per angle and reference
 *   theta  (A)            angles in radians
 *   Pf     (A, B, W)      projection per angle, slice, detector column
 * The single-slice reference functions are the B == 1 case.
 */
#ifndef FLC_H
#define FLC_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FLC_API __attribute__((visibility("default")))
#else
#define FLC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FLC_OK = 0,
    FLC_ERR_INVALID_ARG = 1,  /* null pointer, non-positive or inconsistent size */
    FLC_ERR_UNSUPPORTED = 2,  /* valid request outside what this library supports */
    FLC_ERR_ALIGNMENT = 3,    /* pointer not aligned as the entry point requires */
    FLC_ERR_WORKSPACE = 4,    /* caller-provided workspace too small */
    FLC_ERR_CUDA = 5,         /* CUDA runtime / launch error */
    FLC_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up */
    FLC_ERR_OOM = 7           /* an entry point that allocates could not */
} flc_status;

/* Human-readable name of a status code. */
FLC_API const char* flc_status_string(int status);
/* Message for the last failure on this host thread ("" if none). */
FLC_API const char* flc_last_error(void);
/* Library version string. */
FLC_API const char* flc_version(void);
/* Status left on the device by kernels whose bounded waits gave up
 * (FLC_ERR_TIMEOUT) or FLC_OK; synchronizes the device.  reset != 0 clears it. */
FLC_API int flc_device_status(int reset);
/* Number of kernels this library has launched in this process (graph
 * replays count every kernel node they run).  For instrumentation. */
FLC_API uint64_t flc_launch_count(void);
/* Launch-shape knobs of this library (no counterpart in the reference; the
 * autotuner in fl_correction_b200/tune.py sets them).  Names:
 *   "proj.cluster"  CTAs per slice cluster, backward/MLEM kernels (1..8)
 *   "proj.apc"      angles per CTA, projector kernels
 *   "cone.variant"  1: TMA 16x8 tile, 2: TMA 8x4 tile, 3: plain kernel, 4: spectral,
 *                   5: spectral with the plane transforms split into row and column
 *                   passes (where scratch is given; automatic: spectral where it fits,
 *                   split where a padded plane does not fit one CTA twice)
 *   "atten.chunk"   angles per attenuation-pipeline pass
 *   "proj.bwd"      backward: 2 nine-phase splat, 1 shared-memory atomics,
 *                   3 gather per pixel, 4 splat by column segments; automatic:
 *                   4 where one round of its items fills the thread block, else 2
 *                   (these four are the earlier kernels, run with "proj.legacy")
 *   "proj.legacy"   1: the earlier projector and fused-MLEM kernels instead of the
 *                   lean forward / backward pair (for comparison)
 *   "proj.band"     1: the row-band backward (no global atomics; it runs by itself
 *                   where a slice image does not fit in shared memory) at every size
 *   "xrf.band"      rows per band of the XRF rotation adjoint (automatic: the whole
 *                   slice, or the fewest even bands that fit in shared memory)
 * Test hooks of the direct cone's bounded waits (for failure-path tests):
 *   "cone.test_wait_limit"  polls before a TMA-plane wait gives up (default 2^26)
 *   "cone.test_skip_load"   k > 0: the load of the k-th staged plane of every
 *                   CTA is not issued, so its wait runs out; the kernel waits
 *                   for its other loads, stops, and flc_device_status then
 *                   reports FLC_ERR_TIMEOUT (no fault, the context stays usable)
 * 0 restores the automatic choice.  flc_tune_get returns -1 for an unknown
 * name.  Process-wide; not synchronized with launches in flight. */
FLC_API int flc_tune_set(const char* name, int64_t value);
FLC_API int64_t flc_tune_get(const char* name);

/* ---------------------------------------------------------------------
 * Cone-mask (fluorescence) path sum, reference layout.
 * Replaces cal_atten_cuda / atten_kernel
 * (FL/cuda_lib/atten_cuda.cpp:12-28, atten_cuda_kernel.cu:10-86):
 *   out[k,z,x,y] = sum_{dz,dx,dy} mask[dz,dx,dy] * mu[k, z+dz-Mz/2, x+dx, y+dy-My/2]
 * with taps outside the volume skipped.  mu (K,Z,X,Y), mask (Mz,Mx,My).
 * When every depth plane mask[:,dx,:] is rank one (true of the masks that
 * FL.detector_mask builds) the separable forms run -- the spectral form where
 * the padded planes fit in shared memory (its scratch is allocated with
 * cudaMallocAsync and freed on the same stream), else the direct separable
 * kernel; otherwise a general gather over the non-zero taps.  `flags` is a
 * bit set of FLC_CONE_*.
 * --------------------------------------------------------------------- */
#define FLC_CONE_FORCE_GENERAL 1  /* skip the rank-one test, use the general kernel */
#define FLC_CONE_PLAIN_KERNEL 16  /* separable: plain kernel, not the TMA pipeline */
FLC_API int flc_cone_atten(const float* mu, const float* mask, float* out,
                   int64_t K, int64_t Z, int64_t X, int64_t Y,
                   int64_t Mz, int64_t Mx, int64_t My, int flags, void* stream);

/* Separable cone path sum with a caller-factored mask:
 *   mask[dz,dx,dy] == u[dx*Mz + dz] * v[dx*My + dy].
 * mode: 0 writes the sum, 1 writes exp(-sum); OR FLC_CONE_PLAIN_KERNEL to use
 * the plain separable kernel instead of the TMA-pipelined one.
 * No counterpart entry point in the reference (it is the fast path of
 * cal_atten_cuda, atten_cuda.cpp:12-28). */
FLC_API int flc_cone_atten_separable(const float* mu, const float* u, const float* v, float* out,
                             int64_t K, int64_t Z, int64_t X, int64_t Y,
                             int64_t Mz, int64_t Mx, int64_t My, int mode, void* stream);

/* flc_cone_atten_separable with caller scratch for the spectral form (the
 * form flc_cone_atten picks, without its per-call mask read-back,
 * factorisation and scratch allocation): `workspace` (256-byte aligned) of
 * flc_cone_atten_workspace_bytes(K, Z, X, Y, Mz, Mx, My) bytes; where that is
 * 0 (the padded planes do not fit) or workspace is NULL, the direct separable
 * kernel runs.  mode 0 writes the sum, 1 exp(-sum).  Same results as
 * flc_cone_atten to FP32 rounding.  Counterpart: cal_atten_cuda
 * (atten_cuda.cpp:12-28) with the mask factored once by the caller. */
FLC_API size_t flc_cone_atten_workspace_bytes(int64_t K, int64_t Z, int64_t X, int64_t Y,
                                              int64_t Mz, int64_t Mx, int64_t My);
FLC_API int flc_cone_atten_separable_ws(const float* mu, const float* u, const float* v,
                                        float* out, int64_t K, int64_t Z, int64_t X, int64_t Y,
                                        int64_t Mz, int64_t Mx, int64_t My, int mode,
                                        void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------
 * Attenuated emission projector.
 * forward: Pf[a,b,w] = sum_h atten[a,b,h,w] * sum_r em[a,r] * bilerp(C[r,b], row(a,h,w), col(a,h,w))
 *   Replaces forward_emission_batch / forward_emission
 *   (atten_cuda.cpp:142-182 / :82-108; kernels atten_cuda_kernel.cu:298-337 / :91-142).
 * backward: out[r,b] = exact transpose of the forward applied to ratio (A,B,W).
 *   Replaces backward_emission_batch / backward_emission
 *   (atten_cuda.cpp:188-214 / :113-135; kernels :390-446 / :177-231).
 * The sample point is the reference's: rotation about ((H-1)/2,(W-1)/2),
 * clamp to [0,H-1.001]x[0,W-1.001], bilinear.  Requires H, W >= 2.
 * --------------------------------------------------------------------- */
FLC_API int flc_fwd_emission(const float* atten, const float* C, const float* em, const float* theta,
                     float* Pf, int64_t A, int64_t B, int64_t R, int64_t H, int64_t W,
                     void* stream);
FLC_API int flc_bwd_emission(const float* atten, const float* ratio, const float* em,
                     const float* theta, float* out, int64_t A, int64_t B, int64_t R,
                     int64_t H, int64_t W, void* stream);

/* Huber gradient over the four in-plane neighbours of each pixel of
 * C (RB, H, W).  Replaces huber_grad[_batch]
 * (atten_cuda.cpp:218-238; atten_cuda_kernel.cu:495-616). */
FLC_API int flc_huber_grad(const float* C, float* grad, int64_t RB, int64_t H, int64_t W,
                   float delta, void* stream);

/* ---------------------------------------------------------------------
 * MLEM with optional Huber regularisation, device resident.
 * Replaces mlem_cuda_batch / mlem_cuda (atten_cuda.cpp:283-345 / :244-281).
 * C (R,B,H,W) holds C_init on entry and the result on return (the caller
 * copies C_init first, as the reference's clone does).  I is (A,B,W).
 * The caller provides `workspace` of at least flc_mlem_workspace_bytes(...)
 * bytes (256-byte aligned).  With use_graph != 0 the iteration is captured
 * once into a CUDA graph and replayed n_iter times.
 * --------------------------------------------------------------------- */
FLC_API size_t flc_mlem_workspace_bytes(int64_t A, int64_t B, int64_t R, int64_t H, int64_t W);
FLC_API int flc_mlem(float* C, const float* atten, const float* em, const float* theta,
             const float* I, int64_t n_iter, double beta, double delta,
             int64_t A, int64_t B, int64_t R, int64_t H, int64_t W,
             void* workspace, size_t workspace_bytes, int use_graph, void* stream);
/* flc_mlem without a caller workspace: the scratch is a static 32 MiB device
 * array inside the library, so the call allocates nothing.  For callers that
 * cannot allocate device memory (an FFI host that passes only the data
 * buffers, a process whose device memory another framework has reserved).
 * No counterpart in the reference.  Problems whose flc_mlem_workspace_bytes
 * exceeds 32 MiB return FLC_ERR_UNSUPPORTED.  The first call on a device
 * looks up the array's address (make it before any stream capture); with
 * lazy module loading, the CUDA default, that first call is also when the
 * driver commits the 32 MiB, so make it at start-up, before another pool
 * reserves the device's memory.  The address is kept per device for the
 * primary context: do not call cudaDeviceReset between calls.  Calls that
 * overlap in time share the array and race.  Runs the eager iteration path
 * (use_graph = 0). */
FLC_API int flc_mlem_static(float* C, const float* atten, const float* em, const float* theta,
                    const float* I, int64_t n_iter, double beta, double delta,
                    int64_t A, int64_t B, int64_t R, int64_t H, int64_t W, void* stream);

/* MLEM of P independent problems at once (P <= 64; for instance the elements
 * of one volume, or several volumes): problem i has C[i] (R, B[i], H, W),
 * atten[i] (A[i], B[i], H, W), em[i] (A[i], R), theta[i] (A[i]) and I[i]
 * (A[i], B[i], W), all device pointers held in host arrays of length P; R,
 * H, W are shared (flc_mlem_multi_sizes: H[i], W[i] per problem).  Each C[i]
 * is updated in place by n_iter iterations of flc_mlem.  One persistent
 * launch per iteration and slice width covers every problem of that width:
 * clusters of CTAs take (problem, slice) items from a device counter, the
 * largest work per item (angles x slice area) first, and for each item run
 * the forward of their angles, the backward of the same angles and the
 * update; the shared memory of a launch is sized for its width (every width
 * must fit the lean kernels).  Workspace:
 * flc_mlem_multi[_sizes]_workspace_bytes (256-byte aligned).  Issues no host
 * copies (the problem table travels as a kernel argument).  No counterpart
 * in the reference, which runs mlem_cuda_batch once per element and volume
 * (FL/torch_recon.py:50-99, FL/example/demo.py:177-232). */
FLC_API size_t flc_mlem_multi_workspace_bytes(int64_t P, const int64_t* A, const int64_t* B,
                                              int64_t R, int64_t H, int64_t W);
FLC_API int flc_mlem_multi(int64_t P, float* const* C, const float* const* atten,
                           const float* const* em, const float* const* theta,
                           const float* const* I, const int64_t* A, const int64_t* B, int64_t R,
                           int64_t H, int64_t W, int64_t n_iter, double beta, double delta,
                           void* workspace, size_t workspace_bytes, void* stream);
FLC_API size_t flc_mlem_multi_sizes_workspace_bytes(int64_t P, const int64_t* A,
                                                    const int64_t* B, int64_t R,
                                                    const int64_t* H, const int64_t* W);
FLC_API int flc_mlem_multi_sizes(int64_t P, float* const* C, const float* const* atten,
                                 const float* const* em, const float* const* theta,
                                 const float* const* I, const int64_t* A, const int64_t* B,
                                 int64_t R, const int64_t* H, const int64_t* W, int64_t n_iter,
                                 double beta, double delta, void* workspace,
                                 size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------
 * Per-angle attenuation maps (rotation + mu assembly + incident scan +
 * fluorescence cone + product), the path of FL.core.cal_xrf_atten_at_angles,
 * cal_xray_atten_at_angles and cal_total_atten_at_angles
 * (FL/core.py:19-101, FL/torch_functions.py:8-176,
 * FL/torch_image_util.py:13-155) without the TIFF round trips.
 *
 *   frac    (n_ch, S, H, W)   unrotated fractions (H == W)
 *   theta   (A)               rotation angles, radians
 *   coef_x  (A, n_ch)         cs[comp_j-x] * rho_j * pix per angle
 *   coef_f  (A, L, n_ch)      cs[comp_j-elem_i] * rho_j * pix per angle
 *   u, v                      factored cone mask (see flc_cone_atten_separable)
 *   out     (L, A, S, H, W)   atten[i] = incident(i) * exp(-cone(mu_f[i]))
 * incident_mode 0: element i uses channel i only (FL/torch_functions.py:39-50,
 *   FL/core.py:80-81 -- the current package); 1: product over all channels
 *   (FL/legacy/FL_correction_core.py:1855-1860).  2: no incident term.
 * xrf_mode 0: fluorescence term on; 1: off (incident only).
 * workspace: flc_atten_workspace_bytes(...) bytes; `chunk` angles are
 * processed per pass (0 = choose).  A workspace larger by
 * flc_cone_fft_workspace_bytes(chunk * L, S, H, W, Mz, Mx, My) bytes (the
 * chunk as chosen, pick it explicitly to size this) lets the cone run in its
 * spectral form (2-D FFTs of the depth planes, a per-frequency correlation
 * along the depth, inverse FFTs); without it the direct separable kernels run.
 * --------------------------------------------------------------------- */
FLC_API size_t flc_atten_workspace_bytes(int64_t n_ch, int64_t S, int64_t H, int64_t W, int64_t A,
                                 int64_t L, int64_t chunk);
FLC_API int flc_atten_maps(const float* frac, const float* theta, const float* coef_x,
                   const float* coef_f, const float* u, const float* v, float* out,
                   int64_t n_ch, int64_t S, int64_t H, int64_t W, int64_t A, int64_t L,
                   int64_t Mz, int64_t Mx, int64_t My, int incident_mode, int xrf_mode,
                   int64_t chunk, void* workspace, size_t workspace_bytes, void* stream);

/* flc_atten_maps with a reference-spectrum incident cross section (the
 * XANES case of FL/torch_functions.py:22-37, FL/cross_section_util.py:44-66):
 * frac holds n_ch compound fractions followed by n_ref raw reference volumes
 * (n_ch + n_ref channels); coef_x (A, n_ch) and coef_f (A, L, n_ch) cover the
 * compounds only.  All channels rotate about the same centre with the same
 * sample points; the reference volumes take the reference's scipy boundary
 * rule (see flc_rotate_ex, mode 1), the fractions grid_sample's.  The
 * incident coefficient of compound ref_ch is, per voxel, sum_i coef_ref[a][i] *
 * max(ref_i / (sum_k ref_k + 1e-12), 0), with coef_ref (A, n_ref) the spectrum
 * values cs[comp-x_ref{i+1}] * rho * pix per angle.  n_ref = 0 is
 * flc_atten_maps.  Workspace: flc_atten_workspace_bytes(n_ch + n_ref, ...). */
FLC_API int flc_atten_maps_ref(const float* frac, const float* theta, const float* coef_x,
                               const float* coef_f, const float* coef_ref, const float* u,
                               const float* v, float* out, int64_t n_ch, int64_t n_ref,
                               int64_t ref_ch, int64_t S, int64_t H, int64_t W, int64_t A,
                               int64_t L, int64_t Mz, int64_t Mx, int64_t My, int incident_mode,
                               int xrf_mode, int64_t chunk, void* workspace,
                               size_t workspace_bytes, void* stream);

/* The two stages of flc_atten_maps, for callers that schedule angle chunks
 * themselves.  flc_atten_stage writes the incident term of angles
 * [a0, a0+n_a) into out (L, A, S, H, W) and, if write_mu, the fluorescence mu
 * of those angles into mu_ref (n_a, L, S, W, H) -- the detector-depth-major
 * layout of the reference's rot90 frame (FL/torch_functions.py:142-143).
 * flc_cone_atten_apply multiplies exp(-cone(mu_ref)) into the same angles of
 * out.  No counterpart entry points in the reference (FL/core.py:19-101 runs
 * these steps per angle in Python). */
FLC_API int flc_atten_stage(const float* frac, const float* theta, const float* coef_x,
                            const float* coef_f, float* out, float* mu_ref, int64_t n_ch,
                            int64_t S, int64_t H, int64_t W, int64_t A, int64_t L, int64_t a0,
                            int64_t n_a, int incident_mode, int write_mu, void* stream);
/* flc_atten_stage with scratch (flc_atten_stage_workspace_bytes(n_ch, S, H,
 * W) bytes, 256-byte aligned) for a channel-interleaved copy of frac, made
 * on each call: the rotation then reads every channel's bilinear tap in one
 * 16-byte load.  Same results as flc_atten_stage. */
FLC_API size_t flc_atten_stage_workspace_bytes(int64_t n_ch, int64_t S, int64_t H, int64_t W);
FLC_API int flc_atten_stage_ws(const float* frac, const float* theta, const float* coef_x,
                               const float* coef_f, float* out, float* mu_ref, int64_t n_ch,
                               int64_t S, int64_t H, int64_t W, int64_t A, int64_t L, int64_t a0,
                               int64_t n_a, int incident_mode, int write_mu, void* workspace,
                               size_t workspace_bytes, void* stream);
FLC_API int flc_cone_atten_apply(const float* mu_ref, const float* u, const float* v,
                                 float* atten, int64_t n_a, int64_t L, int64_t S, int64_t H,
                                 int64_t W, int64_t A, int64_t a0, int64_t Mz, int64_t Mx,
                                 int64_t My, void* stream);
/* flc_cone_atten_apply with scratch for the spectral cone: `workspace`
 * (256-byte aligned) of flc_cone_fft_workspace_bytes(n_a * L, S, H, W, Mz,
 * Mx, My) bytes, or NULL for the direct kernels.  The query returns 0 for a
 * shape the spectral form does not take (its planes must fit in shared
 * memory); the "cone.variant" knob selects among the forms. */
FLC_API size_t flc_cone_fft_workspace_bytes(int64_t n_vol, int64_t S, int64_t H, int64_t W,
                                            int64_t Mz, int64_t Mx, int64_t My);
FLC_API int flc_cone_atten_apply_ws(const float* mu_ref, const float* u, const float* v,
                                    float* atten, int64_t n_a, int64_t L, int64_t S, int64_t H,
                                    int64_t W, int64_t A, int64_t a0, int64_t Mz, int64_t Mx,
                                    int64_t My, void* workspace, size_t workspace_bytes,
                                    void* stream);

/* ---------------------------------------------------------------------
 * Differentiable corrected projection with per-angle recomputation.
 *
 * flc_xrf_project: Pf (L, A, S, W) of the concentrations frac[0:L] through
 *   their own self-absorption: for each chunk of angles the attenuation
 *   (incident scan x exp(-cone)) is rebuilt from frac (n_ch, S, H, W, the
 *   first L channels are the element concentrations C_l) and used at once;
 *   nothing of size A x volume is kept.  em (L, A) is em_cs * rho * pix.
 * flc_xrf_project_adjoint: dC (L, S, H, W) = d<gPf, Pf>/dC, including the
 *   dependence of the attenuation on C (rotation, mu assembly, incident scan
 *   and cone are differentiated by hand).  uf, vf are u, v with the taps of
 *   every depth reversed (uf[d][k] = u[d][Mz-1-k]); Mz and My must be odd.
 * Both take flc_xrf_workspace_bytes(...) of scratch (256-byte aligned);
 * with flc_xrf_workspace_bytes_ex(..., Mz, Mx, My) bytes they also keep a
 * channel-interleaved copy of frac for the stage and run the spectral cone
 * where its planes fit (same results to FP32 rounding).
 * Counterpart: the reference differentiates only the projector in C
 * (FL/cuda_lib/autograd.py:5-77) with attenuation held fixed
 * (FL/example/demo.py:413-475); this is the full-mu extension of that path.
 * --------------------------------------------------------------------- */
FLC_API size_t flc_xrf_workspace_bytes(int64_t n_ch, int64_t S, int64_t H, int64_t W, int64_t A,
                                       int64_t L, int64_t chunk);
FLC_API size_t flc_xrf_workspace_bytes_ex(int64_t n_ch, int64_t S, int64_t H, int64_t W,
                                          int64_t A, int64_t L, int64_t chunk, int64_t Mz,
                                          int64_t Mx, int64_t My);
FLC_API int flc_xrf_project(const float* frac, const float* theta, const float* coef_x,
                            const float* coef_f, const float* u, const float* v, const float* em,
                            float* Pf, int64_t n_ch, int64_t S, int64_t H, int64_t W, int64_t A,
                            int64_t L, int64_t Mz, int64_t Mx, int64_t My, int incident_mode,
                            int64_t chunk, void* workspace, size_t workspace_bytes, void* stream);
FLC_API int flc_xrf_project_adjoint(const float* frac, const float* theta, const float* coef_x,
                                    const float* coef_f, const float* u, const float* v,
                                    const float* uf, const float* vf, const float* em,
                                    const float* gPf, float* dC, int64_t n_ch, int64_t S,
                                    int64_t H, int64_t W, int64_t A, int64_t L, int64_t Mz,
                                    int64_t Mx, int64_t My, int incident_mode, int64_t chunk,
                                    void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------
 * Detector cone mask on the device (FL/detector_mask.py:22-151,
 * generate_detector_mask with g_mask and g_radial_mask_approximate).
 * alfa0, theta0: full horizontal / vertical cone angles in degrees; leng0:
 * depth in voxels.  flc_detector_mask_shape gives the mask extents (Mz, Mx =
 * leng0, My) and the FP64 scratch the generator needs.  flc_detector_mask
 * writes the rank-one factors of every depth plane, u (Mx, Mz) and v (Mx, My)
 * as FP32 (mask[dz][d][dy] = u[d][dz] * v[d][dy], the input of
 * flc_cone_atten_separable and flc_atten_maps), and, when dense != NULL, the
 * FP64 mask (Mz, Mx, My) the reference returns.  No counterpart entry point
 * in the reference (it builds the mask on the host with numba).
 * --------------------------------------------------------------------- */
FLC_API int flc_detector_mask_shape(double alfa0, double theta0, int64_t leng0, int64_t* Mz,
                                    int64_t* Mx, int64_t* My, size_t* scratch_bytes);
FLC_API int flc_detector_mask(double alfa0, double theta0, int64_t leng0, float* u, float* v,
                              double* dense, void* scratch, size_t scratch_bytes, void* stream);

/* ---------------------------------------------------------------------
 * cal_frac on the device (FL/core.py:159-205): frac (n_ch, N) from
 * concentrations img (n_ch, N), N voxels per channel.
 *   img_sum = (sum_i img_i + 1e-12) * mask      (mask NULL: 1)
 *   tmp_i   = img_i / img_sum, NaN / inf / negative -> 0
 *   use_range: where tmp_i has more than 100 positive values it is clamped
 *     to its int(l*r0)-th and (int(l*r1)-1)-th smallest positive values
 *   enable_scale: frac_i = tmp_i * mask * img_sum / p, p the
 *     int(l*scale_limit)-th smallest positive img_sum; else tmp_i * mask
 * img_sum (optional, N) receives the masked sum.  The order statistics are
 * exact (radix select on the FP32 bit patterns).  The reference's mask is a
 * multi-Otsu threshold that falls back to 1 without scikit-image; the caller
 * passes a mask or NULL.  Workspace: flc_cal_frac_workspace_bytes.  n_ch <= 8.
 * No counterpart entry point in the reference (numpy on the host).
 * --------------------------------------------------------------------- */
FLC_API size_t flc_cal_frac_workspace_bytes(int64_t n_ch, int64_t N);
FLC_API int flc_cal_frac(const float* img, const float* mask, float* frac, float* img_sum,
                         int64_t n_ch, int64_t N, int use_range, double r0, double r1,
                         int enable_scale, double scale_limit, void* workspace,
                         size_t workspace_bytes, void* stream);

/* Incident X-ray attenuation of one slice from reference-spectrum volumes,
 * replacing torch_2D_xray_atten_with_ref (variant 0, FL/torch_functions.py:
 * 181-215) and torch_2D_xray_atten_with_ref_vectorize (variant 1, :247-330).
 * C (n_ref, H, W) reference volumes, C_other (H, W), theta (A,) radians,
 * cs_ref (A, n_ref), rho (H, W) (applied unrotated), pix; out (A, H, W), all
 * device FP32.  With frac = C / (max_p(sum_j C_j + C_other) + eps) rotated to
 * each angle and mu = (sum_j cs_ref[a][j] frac_j) rho pix, f = max(1 - mu, fl):
 *   variant 0: eps 1e-9, grid_sample rotation with align_corners=False,
 *              fl 1e-6, out[h] = prod_{h' > h} f[h'], out[H-1] = 1;
 *   variant 1: eps 1e-8, align_corners=True, mu clipped at 0, fl 1e-8,
 *              out[h] = prod_{h' >= h} f[h'] for h < H-1, out[H-1] = 1
 *              (the reference's shifted cumulative product includes row h).
 * H, W >= 2.  Workspace: flc_xray_atten_ref2d_workspace_bytes() bytes of
 * device memory (the normaliser). */
FLC_API size_t flc_xray_atten_ref2d_workspace_bytes(void);
FLC_API int flc_xray_atten_ref2d(const float* C, const float* C_other, const float* theta,
                                 const float* cs_ref, const float* rho, float pix, float* out,
                                 int64_t n_ref, int64_t A, int64_t H, int64_t W, int variant,
                                 void* workspace, size_t workspace_bytes, void* stream);

/* Rotation with torch grid_sample semantics (bilinear, zero padding,
 * align_corners=False, same-size output): out (N, H, W) from x (N, H, W).
 * cos_t/sin_t are the FP32 matrix entries.  Replaces torch_rotate_image_nd
 * (FL/torch_image_util.py:13-114, enable_crop=True). */
FLC_API int flc_rotate(const float* x, float* out, int64_t N, int64_t H, int64_t W,
               float cos_t, float sin_t, void* stream);

/* flc_rotate with a choice of boundary rule: mode 0 is flc_rotate
 * (grid_sample, zero padding: within one pixel of the border the sample
 * interpolates against the padding); mode 1 is scipy.ndimage.rotate with
 * order=1, reshape=False, mode='constant' -- the reference's rot3D
 * (FL/image_util.py:165-203), which rotates the reference-spectrum volumes
 * (FL/atten_util.py:79-88): the same sample points and weights, but zero for
 * every sample outside [0, W-1] x [0, H-1]. */
FLC_API int flc_rotate_ex(const float* x, float* out, int64_t N, int64_t H, int64_t W,
                          float cos_t, float sin_t, int mode, void* stream);

/* Incident attenuation: out[n,h,w] = prod_{h'>h} (1 - mu[n,h',w]), out[n,H-1,w] = 1.
 * Replaces the flip/cumprod/flip of torch_xray_atten_3D (FL/torch_functions.py:95-102). */
FLC_API int flc_incident_scan(const float* mu, float* out, int64_t N, int64_t H, int64_t W,
                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FLC_H */
