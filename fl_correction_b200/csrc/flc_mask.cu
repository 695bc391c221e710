// Detector cone mask generated on the device (FL/detector_mask.py:22-151).
//
// The reference builds, on the host with numba, two 1-D cone profiles
// M1 (horizontal angle alfa, cells x depth) and M2 (vertical angle theta)
// (g_mask, :110-151), the pyramid Mask = M1 (x) M2 per depth, normalises each
// depth plane by its sum (g_radial_mask_approximate, :179-186), multiplies
// once more by Mask, crops the centre and transposes to (slice, row=depth,
// col).  Per depth d the result is therefore
//     mask[dz][d][dy] = M2[dz][d]^2 * M1[dy][d]^2 / (sum M1[:, d] * sum M2[:, d]),
// an outer product.  Here one kernel evaluates both profiles cell by cell
// (FP64, the reference's arithmetic) and a second writes the rank-one factors
//     u[d][dz] = M2[dz][d]^2 / sum M2[:, d],   v[d][dy] = M1[dy][d]^2 / sum M1[:, d]
// (FP32, the form the separable cone kernels consume) and, when asked, the
// dense FP64 mask.  Depth planes whose sum is 0 (depth 0: the NaN of the
// reference's 0 / 0, set to 0 at :103) are zero.
//
// The scalars that decide the shape -- FP32 half angles, N1 = ceil(L tan),
// the cut -- follow the numpy steps of generate_detector_mask exactly: FP32
// arithmetic for the angle and the products L * tan(alfa), the FP32 tan of
// the FP32 angle for the sizes, and inside the profiles the FP32 rounding of
// the FP64 tan / cos (the numba kernel's values).

#include <math.h>

#include "flc_common.cuh"

namespace flc {
namespace {

struct MaskDims {
    int leng0, leng;       // cut depth, working depth (leng0 + 30)
    int n1, n2, n1_0, n2_0;
    int s0, s1;            // profile cells: 2 n1 - 1, 2 n2 - 1
    int My, Mz;            // cut extents: 2 n1_0 - 1, 2 n2_0 - 1
    double tan_a, cos_a, tan_t, cos_t;   // FP32 values held in FP64
};

float deg_half_rad(double deg) {
    // np.float32(alfa0) / 2 / 180 * np.pi in FP32 arithmetic
    float a = (float)deg;
    a = a / 2.0f;
    a = a / 180.0f;
    a = a * (float)M_PI;
    return a;
}

MaskDims mask_dims(double alfa0, double theta0, int64_t leng0) {
    MaskDims m;
    const float alfa = deg_half_rad(alfa0), theta = deg_half_rad(theta0);
    const float ta32 = tanf(alfa), tt32 = tanf(theta);
    m.leng0 = (int)leng0;
    m.leng = (int)leng0 + 30;
    m.n1_0 = (int)ceilf((float)leng0 * ta32);
    m.n2_0 = (int)ceilf((float)leng0 * tt32);
    m.n1 = (int)ceilf((float)m.leng * ta32);
    m.n2 = (int)ceilf((float)m.leng * tt32);
    m.s0 = 2 * m.n1 - 1;
    m.s1 = 2 * m.n2 - 1;
    m.My = 2 * m.n1_0 - 1;
    m.Mz = 2 * m.n2_0 - 1;
    m.tan_a = (double)(float)tan((double)alfa);
    m.cos_a = (double)(float)cos((double)alfa);
    m.tan_t = (double)(float)tan((double)theta);
    m.cos_t = (double)(float)cos((double)theta);
    return m;
}

// One cell (I, J) of g_mask (FL/detector_mask.py:110-151), 0-based indices.
__device__ double profile_cell(int I, int J, double t, double cos_a, int N) {
    const double i = I + 1, j = J + 1;
    if (I == N - 1) return J == 0 ? 0.0 : 1.0;   // the apex row (:64-67)
    const double o = fabs((double)N - i);
    const double jt = j * t, j1t = (j - 1) * t;
    if (o >= jt) return 0.0;
    if (o < j1t && o + 1 > jt) {
        const double d1 = j1t - floor(j1t), d2 = jt - floor(jt);
        return 0.5 * (d1 + d2) / cos_a;
    }
    if (o < jt && o + 1 > jt && o > j1t) {
        const double d1 = jt - floor(jt);
        return 0.5 * d1 * (d1 / t) / cos_a;
    }
    if (o + 1 < jt && o < j1t && o + 1 > j1t) {
        const double d1 = ceil(j1t) - j1t;
        return (1.0 - 0.5 * d1 * (d1 / t)) / cos_a;
    }
    return 1.0 / cos(atan(((double)N - i) / j));
}

// prof1 (s0 x leng) and prof2 (s1 x leng), one thread per cell.
__global__ void mask_profile_kernel(double* __restrict__ prof1, double* __restrict__ prof2,
                                    MaskDims m) {
    const int64_t n1 = (int64_t)m.s0 * m.leng, n2 = (int64_t)m.s1 * m.leng;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n1 + n2;
         k += (int64_t)gridDim.x * blockDim.x) {
        if (k < n1) {
            const int I = (int)(k / m.leng), J = (int)(k - (int64_t)I * m.leng);
            prof1[k] = profile_cell(I, J, m.tan_a, m.cos_a, m.n1);
        } else {
            const int64_t q = k - n1;
            const int I = (int)(q / m.leng), J = (int)(q - (int64_t)I * m.leng);
            prof2[q] = profile_cell(I, J, m.tan_t, m.cos_t, m.n2);
        }
    }
}

// One CTA per cut depth d: the profile sums over all cells (warp-shuffle
// reductions in a fixed order), then the factors and the dense planes.
__global__ void mask_factor_kernel(const double* __restrict__ prof1,
                                   const double* __restrict__ prof2, float* __restrict__ u,
                                   float* __restrict__ v, double* __restrict__ dense, MaskDims m) {
    __shared__ double part[2][32];
    const int d = blockIdx.x;
    double a = 0.0, b = 0.0;
    for (int I = threadIdx.x; I < m.s0; I += blockDim.x) a += prof1[(int64_t)I * m.leng + d];
    for (int I = threadIdx.x; I < m.s1; I += blockDim.x) b += prof2[(int64_t)I * m.leng + d];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) {
        part[0][wid] = a;
        part[1][wid] = b;
    }
    __syncthreads();
    double s1 = 0.0, s2 = 0.0;
    for (int k = 0; k < nw; ++k) {
        s1 += part[0][k];
        s2 += part[1][k];
    }
    const double den = s1 * s2;
    const int c0 = m.s0 / 2, c1 = m.s1 / 2, d0 = m.My / 2, d1 = m.Mz / 2;
    for (int k = threadIdx.x; k < m.My; k += blockDim.x) {
        const double p = prof1[(int64_t)(c0 - d0 + k) * m.leng + d];
        v[(int64_t)d * m.My + k] = s1 != 0.0 ? (float)(p * p / s1) : 0.f;
    }
    for (int k = threadIdx.x; k < m.Mz; k += blockDim.x) {
        const double p = prof2[(int64_t)(c1 - d1 + k) * m.leng + d];
        u[(int64_t)d * m.Mz + k] = s2 != 0.0 ? (float)(p * p / s2) : 0.f;
    }
    if (dense) {
        for (int k = threadIdx.x; k < m.Mz * m.My; k += blockDim.x) {
            const int dz = k / m.My, dy = k - dz * m.My;
            const double p1 = prof1[(int64_t)(c0 - d0 + dy) * m.leng + d];
            const double p2 = prof2[(int64_t)(c1 - d1 + dz) * m.leng + d];
            const double mk = p1 * p2;
            dense[((int64_t)dz * m.leng0 + d) * m.My + dy] = den != 0.0 ? (mk / den) * mk : 0.0;
        }
    }
}

int check_mask_args(double alfa0, double theta0, int64_t leng0, const char* who) {
    FLC_REQUIRE(alfa0 > 0.0 && alfa0 < 180.0 && theta0 > 0.0 && theta0 < 180.0,
                "%s: full angles must lie in (0, 180) degrees", who);
    FLC_REQUIRE(leng0 >= 1 && leng0 <= 4096, "%s: length must be in [1, 4096]", who);
    return FLC_OK;
}

}  // namespace
}  // namespace flc

using namespace flc;

extern "C" int flc_detector_mask_shape(double alfa0, double theta0, int64_t leng0, int64_t* Mz,
                                       int64_t* Mx, int64_t* My, size_t* scratch_bytes) {
    clear_error();
    FLC_TRY(check_mask_args(alfa0, theta0, leng0, "flc_detector_mask_shape"));
    const MaskDims m = mask_dims(alfa0, theta0, leng0);
    FLC_REQUIRE(m.n1_0 >= 1 && m.n2_0 >= 1, "flc_detector_mask_shape: degenerate cone");
    if (Mz) *Mz = m.Mz;
    if (Mx) *Mx = m.leng0;
    if (My) *My = m.My;
    if (scratch_bytes)
        *scratch_bytes = sizeof(double) * ((size_t)m.s0 + (size_t)m.s1) * (size_t)m.leng;
    return FLC_OK;
}

extern "C" int flc_detector_mask(double alfa0, double theta0, int64_t leng0, float* u, float* v,
                                 double* dense, void* scratch, size_t scratch_bytes,
                                 void* stream) {
    clear_error();
    FLC_TRY(check_mask_args(alfa0, theta0, leng0, "flc_detector_mask"));
    FLC_REQUIRE(u && v && scratch, "flc_detector_mask: null pointer argument");
    const MaskDims m = mask_dims(alfa0, theta0, leng0);
    FLC_REQUIRE(m.n1_0 >= 1 && m.n2_0 >= 1, "flc_detector_mask: degenerate cone");
    const size_t need = sizeof(double) * ((size_t)m.s0 + (size_t)m.s1) * (size_t)m.leng;
    if (scratch_bytes < need) {
        set_error("flc_detector_mask: scratch of %zu bytes is smaller than the %zu required",
                  scratch_bytes, need);
        return FLC_ERR_WORKSPACE;
    }
    if (((uintptr_t)scratch & 7) != 0) {
        set_error("flc_detector_mask: scratch must be 8-byte aligned");
        return FLC_ERR_ALIGNMENT;
    }
    cudaStream_t st = as_stream(stream);
    double* p1 = (double*)scratch;
    double* p2 = p1 + (size_t)m.s0 * m.leng;
    const int64_t cells = ((int64_t)m.s0 + m.s1) * m.leng;
    mask_profile_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(p1, p2, m);
    FLC_TRY(check_launch("mask_profile_kernel"));
    mask_factor_kernel<<<(unsigned)m.leng0, 256, 0, st>>>(p1, p2, u, v, dense, m);
    return check_launch("mask_factor_kernel");
}
