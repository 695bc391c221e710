// Separable cone path sum, TMA-pipelined (sm_100a).
//
// Computes, in the reference layout of atten_kernel (atten_cuda_kernel.cu:10-57),
//   res[v,z,x,y] = sum_{d} sum_{dz} u[d][dz] sum_{dy} v[d][dy] mu[v, z+dz-hz, x+d, y+dy-hy]
// for a mask whose every depth plane is an outer product u[d] (x) v[d]
// (FL/detector_mask.py builds exactly such masks).
//
// One CTA owns XB consecutive target planes x0.. and a TY-wide strip of y,
// for every z.  It streams the source planes p = x0 .. x0+XB-1+Mx-1 through
// shared memory: one thread issues a 3-D TMA tensor load of
// mu[v, 0:Z, p, y0-HYP : y0-HYP+boxW] (zero fill outside [0, Y)) into a
// double buffer and waits for it on an mbarrier (bounded wait).  For every
// target the plane feeds (d = p - x), the y filter runs row by row from the
// staged plane into a z-major scratch X, and the z filter accumulates column
// by column into registers.  Both filters keep sliding windows of the input
// in registers, rotated over blocks of four taps, and run several windows
// under one weight row: a y-filter thread owns two rows at a time and a
// z-filter thread 32 consecutive outputs, so a block of four taps costs one
// broadcast weight load and one 128-bit input load per 32 FMAs.
//
// Taps are zero-padded to blocks of four; the reference's zero-skip order of
// summation is not reproduced (FP32 sums in a different order; the result
// agrees with the FP64 oracle to ~1e-6 relative).

#include <cuda.h>
#include <cudaTypedefs.h>

#include "flc_common.cuh"

namespace flc {

// Set by a kernel whose bounded wait gave up; read by flc_device_status().
__device__ int g_cone_status = 0;

namespace {

constexpr int kWaitLimit = 1 << 26;  // default polls before a wait gives up (~ seconds)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Polls the mbarrier phase `parity` at most `limit` times; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit) {
    for (int i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

struct ConeGeom {
    int Z, X, Y, Mz, Mx, My;
    int hz, hy;
    int HYP, offy;   // y halo in the staged plane (multiple of 4), HYP - hy
    int HZP, offz;   // z halo in X (multiple of 4), HZP - hz
    int boxW;        // staged row width (floats)
    int PZ;          // X row pitch (floats)
    int WY, WZ;      // padded weight row lengths
    int zblocks;     // Z / 32 rounded up
    int ring;        // 0: every depth's filters preloaded; 1: a ring of 2 XB rows
    int wait_limit;  // polls of a bounded wait before it gives up
    int skip_step;   // test hook: the plane step whose load is not issued (-1: none)
};

// 4 taps x 8 outputs from a 12-value window (a,b,c) and 4 weights w.
__device__ __forceinline__ void fma_block(float (&acc)[8], const float4& a, const float4& b,
                                          const float4& c, const float4& w) {
    const float v[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        acc[t] = fmaf(w.x, v[t], acc[t]);
        acc[t] = fmaf(w.y, v[t + 1], acc[t]);
        acc[t] = fmaf(w.z, v[t + 2], acc[t]);
        acc[t] = fmaf(w.w, v[t + 3], acc[t]);
    }
}

// NR independent 1-D correlations sharing one weight row: acc[k][t] +=
// sum_m w[m] * in[k * rs + t + m].  Each block of four taps costs one
// broadcast weight load and NR input loads for NR x 32 FMAs (the windows
// slide by one float4 per block).  `rs` is a multiple of 4 floats.
template <int NR>
__device__ __forceinline__ void corr8_rows(float (&acc)[NR][8], const float* in, int rs,
                                           const float* w, int mlo, int mhi) {
    if (mlo >= mhi) return;
    float4 g0[NR], g1[NR], g2[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
        g0[k] = *reinterpret_cast<const float4*>(in + k * rs + mlo);
        g1[k] = *reinterpret_cast<const float4*>(in + k * rs + mlo + 4);
    }
    int m = mlo;
    while (true) {
        float4 wv = *reinterpret_cast<const float4*>(w + m);
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            g2[k] = *reinterpret_cast<const float4*>(in + k * rs + m + 8);
            fma_block(acc[k], g0[k], g1[k], g2[k], wv);
        }
        m += 4;
        if (m >= mhi) break;
        wv = *reinterpret_cast<const float4*>(w + m);
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            g0[k] = *reinterpret_cast<const float4*>(in + k * rs + m + 8);
            fma_block(acc[k], g1[k], g2[k], g0[k], wv);
        }
        m += 4;
        if (m >= mhi) break;
        wv = *reinterpret_cast<const float4*>(w + m);
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            g1[k] = *reinterpret_cast<const float4*>(in + k * rs + m + 8);
            fma_block(acc[k], g2[k], g0[k], g1[k], wv);
        }
        m += 4;
        if (m >= mhi) break;
    }
}

// Output modes (see flc.h): 0 res, 1 exp(-res) in the reference layout;
// 2 multiply exp(-res) into the beam-layout attenuation out[l][a][z][Y-1-y][x],
// volume v = a_local * L + l.
template <int TY, int XB, bool RING>
__global__ void __launch_bounds__(512)
cone_tma_kernel(const __grid_constant__ CUtensorMap tmap, const float* __restrict__ U,
                const float* __restrict__ V, float* __restrict__ out, ConeGeom g, int mode, int L,
                int a_base, int64_t out_a_stride, int64_t out_l_stride) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const int Z = g.Z, X = g.X, Y = g.Y;
    const int v = blockIdx.z;
    const int x0 = blockIdx.y * XB;
    const int y0 = blockIdx.x * TY;
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;

    // shared layout: S[2][Z][boxW] | X[XB][TY][PZ] | wy[nw][WY] | wz[nw][WZ] |
    //               meta[Mx][8] | bars[2]
    // nw = Mx: every depth's filters are preloaded.  nw = 2 XB (long masks,
    // whose filters do not fit): depth d sits in ring slot d % (2 XB); at
    // plane p the CTA's targets meet depths p-x0-XB+1 .. p-x0, and the depth
    // that enters at the next plane reuses the slot of one last used XB
    // planes ago.
    const int nw = RING ? 2 * XB : g.Mx;
    const int sbuf = (Z * g.boxW + 31) & ~31;  // 128-byte aligned TMA destinations
    float* S = reinterpret_cast<float*>(smem_raw);
    float* Xs = S + 2 * sbuf;
    float* wy = Xs + XB * TY * g.PZ;
    float* wz = wy + nw * g.WY;
    int* meta = reinterpret_cast<int*>(wz + nw * g.WZ);  // per depth: on, ylo, yhi, zlo, zhi
    uint64_t* bars = reinterpret_cast<uint64_t*>(meta + g.Mx * 8);
    __shared__ int s_fail;

    const int p_begin = x0;
    const int p_end = min(X, x0 + XB - 1 + g.Mx);
    const uint32_t plane_bytes = (uint32_t)(Z * g.boxW * sizeof(float));

    if (tid == 0) {
        s_fail = 0;
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < XB * TY * g.PZ; i += nthr) Xs[i] = 0.f;
    __syncthreads();
    if (tid == 0) {
        for (int q = 0; q < 2 && p_begin + q < p_end; ++q) {
            if (q == g.skip_step) continue;   // test hook: this wait will run out
            mbar_expect_tx(&bars[q], plane_bytes);
            tma_load_3d(S + q * sbuf, &tmap, y0 - g.HYP, p_begin + q, v * Z, &bars[q]);
        }
    }
    // Element e of depth d's filter row, zero-padded and shifted so that tap m
    // lines up with input column t + m (y, e < WY) / row z + m (z, e >= WY).
    auto wval = [&](int d, int e) -> float {
        if (e < g.WY) {
            const int dy = e - g.offy;
            return (dy >= 0 && dy < g.My) ? __ldg(V + (int64_t)d * g.My + dy) : 0.f;
        }
        const int dz = e - g.WY - g.offz;
        return (dz >= 0 && dz < g.Mz) ? __ldg(U + (int64_t)d * g.Mz + dz) : 0.f;
    };
    auto wput = [&](int d, int e, float x) {
        const int slot = RING ? d % (2 * XB) : d;
        if (e < g.WY) wy[slot * g.WY + e] = x;
        else wz[slot * g.WZ + e - g.WY] = x;
    };
    // depth 0's filters into the ring (the others stream in one per plane)
    for (int e = tid; e < g.WY + g.WZ; e += nthr) wput(0, e, wval(0, e));
    // each depth's tap support [lo, hi] in y and z: every element of every
    // depth's rows is loaded once, in parallel, and the non-zero ones fold
    // into shared min / max (integer atomics)
    for (int d = tid; d < g.Mx; d += nthr) {
        meta[d * 8 + 1] = 1 << 30;
        meta[d * 8 + 2] = -1;
        meta[d * 8 + 3] = 1 << 30;
        meta[d * 8 + 4] = -1;
    }
    __syncthreads();
    {
        const int row = g.WY + g.WZ;
        for (int e = tid; e < g.Mx * row; e += nthr) {
            const int d = e / row, k = e - d * row;
            const float wv = wval(d, k);
            if (!RING) wput(d, k, wv);
            if (wv == 0.f) continue;
            const int lo = k < g.WY ? 1 : 3, m = k < g.WY ? k : k - g.WY;
            atomicMin(&meta[d * 8 + lo], m);
            atomicMax(&meta[d * 8 + lo + 1], m);
        }
    }
    __syncthreads();
    for (int d = tid; d < g.Mx; d += nthr) {
        int* md = meta + d * 8;
        const int on = md[2] >= 0 && md[4] >= 0;
        md[0] = on;
        md[1] = on ? (md[1] & ~3) : 0;
        md[2] = on ? md[2] + 1 : 0;
        md[3] = on ? (md[3] & ~3) : 0;
        md[4] = on ? md[4] + 1 : 0;
    }

    // y-filter ownership: (yf_j, yf_half, yf_r0) with yf_r0 fastest; each
    // thread takes rows yf_r0 + zq * {0, 1, 2, 3}, zq = 8 * zblocks
    const int zq = 8 * g.zblocks;
    const int yf_r0 = tid % zq;
    const int yf_half = (tid / zq) % (TY / 8);
    const int yf_j = tid / (zq * (TY / 8));
    // z-filter ownership: (j, t, zb) with t fastest
    const int zt_t = tid % TY;
    const int zt_j = (tid / TY) % XB;
    const int zt_zb = tid / (TY * XB);
    const bool zt_on = zt_zb < g.zblocks;
    float acc[4][8];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[q][k] = 0.f;

    for (int p = p_begin; p < p_end; ++p) {
        const int step = p - p_begin;
        const int buf = step & 1;
        const uint32_t parity = (uint32_t)((step >> 1) & 1);
        if (tid == 0 && !mbar_wait(&bars[buf], parity, g.wait_limit)) s_fail = 1 + step;
        __syncthreads();
        if (s_fail) break;
        // the filters of the depth that enters at the next plane: loaded now,
        // stored after this plane's work (its ring slot is already free)
        const int dn = RING ? p + 1 - x0 : g.Mx;
        const float wn0 = (dn < g.Mx && tid < g.WY + g.WZ) ? wval(dn, tid) : 0.f;
        const float wn1 = (dn < g.Mx && tid + nthr < g.WY + g.WZ) ? wval(dn, tid + nthr) : 0.f;
        // ---- y filter: X[j][t][HZP + z] = sum_m wy[j][m] * S[z][t + m] ----
        // this thread: target yf_j, columns yf_half*8.., rows yf_r0 + zq*{0..3}
        {
            const float* Sb = S + buf * sbuf;
            const int d = p - (x0 + yf_j);
            if (d >= 0 && d < g.Mx && x0 + yf_j < X && meta[d * 8]) {
                const int mlo = meta[d * 8 + 1], mhi = meta[d * 8 + 2];
                const float* wr = wy + (RING ? d % (2 * XB) : d) * g.WY;
#pragma unroll
                for (int pr = 0; pr < 2; ++pr) {
                    // rows z0, z0 + zq (clamped to the staged plane; extra rows are not stored)
                    const int z0 = yf_r0 + 2 * pr * zq;
                    const int za = min(z0, Z - 1), zb2 = min(z0 + zq, Z - 1);
                    float a8[2][8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) a8[0][k] = a8[1][k] = 0.f;
                    corr8_rows<2>(a8, Sb + za * g.boxW + yf_half * 8, (zb2 - za) * g.boxW, wr,
                                  mlo, mhi);
                    float* xo = Xs + (yf_j * TY + yf_half * 8) * g.PZ + g.HZP;
                    if (z0 < Z) {
#pragma unroll
                        for (int k = 0; k < 8; ++k) xo[k * g.PZ + z0] = a8[0][k];
                    }
                    if (z0 + zq < Z) {
#pragma unroll
                        for (int k = 0; k < 8; ++k) xo[k * g.PZ + z0 + zq] = a8[1][k];
                    }
                }
            }
        }
        __syncthreads();
        // plane buffer `buf` is free: prefetch plane p + 2 into it
        if (tid == 0 && p + 2 < p_end && step + 2 != g.skip_step) {
            fence_proxy_async();
            mbar_expect_tx(&bars[buf], plane_bytes);
            tma_load_3d(S + buf * sbuf, &tmap, y0 - g.HYP, p + 2, v * Z, &bars[buf]);
        }
        // ---- z filter: acc[z] += sum_m wz[j][m] * X[j][t][z + m] ----
        const int dz_ = p - (x0 + zt_j);
        if (zt_on && dz_ >= 0 && dz_ < g.Mx && x0 + zt_j < X && meta[dz_ * 8]) {
            const float* xr = Xs + (zt_j * TY + zt_t) * g.PZ;
            const float* wr = wz + (RING ? dz_ % (2 * XB) : dz_) * g.WZ;
            const int mlo = meta[dz_ * 8 + 3], mhi = meta[dz_ * 8 + 4];
            corr8_rows<4>(acc, xr + zt_zb * 32, 8, wr, mlo, mhi);
        }
        if (dn < g.Mx) {
            if (tid < g.WY + g.WZ) wput(dn, tid, wn0);
            if (tid + nthr < g.WY + g.WZ) wput(dn, tid + nthr, wn1);
        }
        // the next iteration's first barrier orders this z filter before the
        // next y filter overwrites X
    }
    // Every load issued on the normal path was waited for.  After a timeout
    // the loads still pending are waited for (again with a bound) before exit.
    if (s_fail) {
        if (tid == 0) {
            atomicExch(&g_cone_status, FLC_ERR_TIMEOUT);
            // the load the wait gave up on (if it was issued and is only slow)
            // and the load of the following plane may still be in flight
            const int step = s_fail - 1;
            for (int q = step; q <= step + 1; ++q)
                if (p_begin + q < p_end && q != g.skip_step)
                    mbar_wait(&bars[q & 1], (uint32_t)((q >> 1) & 1), g.wait_limit);
        }
        __syncthreads();
        return;
    }
    // ---- epilogue ----
    const int y = y0 + zt_t;
    const int x = x0 + zt_j;
    if (mode >= 2) {
        // beam layout (2: multiply exp(-res) in, 3: store exp(-res)); transpose
        // through shared memory so that stores run along x
        float* T = S;  // [Z][TY][XB], spans the S and X buffers (contiguous)
        __syncthreads();
        if (zt_on) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    int z = zt_zb * 32 + q * 8 + k;
                    if (z < Z) T[(z * TY + zt_t) * XB + zt_j] = acc[q][k];
                }
        }
        __syncthreads();
        const int al = v / L, l = v - al * L;
        float* ob = out + l * out_l_stride + (int64_t)(a_base + al) * out_a_stride;
        for (int i = tid; i < Z * TY * XB; i += nthr) {
            int j = i % XB, rest = i / XB;
            int t = rest % TY, z = rest / TY;
            int yy = y0 + t, xx = x0 + j;
            if (yy >= Y || xx >= X) continue;
            float* o = ob + ((int64_t)z * Y + (Y - 1 - yy)) * X + xx;
            const float e = expf(-T[i]);
            if (mode == 2) *o *= e; else *o = e;
        }
        return;
    }
    if (!zt_on || y >= Y || x >= X) return;
    float* ov = out + (int64_t)v * Z * X * Y;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            int z = zt_zb * 32 + q * 8 + k;
            if (z >= Z) continue;
            float r = acc[q][k];
            ov[((int64_t)z * X + x) * Y + y] = mode == 1 ? expf(-r) : r;
        }
}

int pad_mod8_4(int n) {  // smallest >= n with n*4/16 odd, i.e. n == 4 (mod 8)
    while ((n & 7) != 4) ++n;
    return n;
}

template <int TY, int XB>
bool cone_tma_geom(int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My, ConeGeom* g,
                   size_t* smem, int* threads) {
    if (Y % 4 != 0 || Z > 256 || Z < 1) return false;
    g->Z = (int)Z; g->X = (int)X; g->Y = (int)Y;
    g->Mz = (int)Mz; g->Mx = (int)Mx; g->My = (int)My;
    g->hz = (int)Mz / 2; g->hy = (int)My / 2;
    g->HYP = (g->hy + 3) & ~3;
    g->offy = g->HYP - g->hy;
    g->HZP = (g->hz + 3) & ~3;
    g->offz = g->HZP - g->hz;
    int wy_core = (g->offy + g->My + 3) & ~3;
    int wz_core = (g->offz + g->Mz + 3) & ~3;
    g->WY = wy_core + 4;
    g->WZ = wz_core + 4;
    // y window reads up to (TY-8) + wy_core + 8 columns past the strip start
    g->boxW = pad_mod8_4(TY - 8 + wy_core + 8);
    if (g->boxW > 256) return false;
    // z window reads up to Z-8 (+ rounding to 32) + wz_core + 8 rows past HZP - offz
    int zspan = ((g->Z + 31) & ~31);
    g->PZ = pad_mod8_4(zspan + wz_core + 8 + g->HZP);
    g->zblocks = (g->Z + 31) / 32;
    *threads = TY * XB * g->zblocks;
    if (*threads > 512) return false;
    size_t sb = ((size_t)g->Z * g->boxW + 31) & ~(size_t)31;
    if (g->WY + g->WZ > 2 * *threads) return false;   // two filter elements per thread
    // preload every depth's filters when they fit, else stream them through a ring
    const size_t fixed = sizeof(float) * (2 * sb + (size_t)XB * TY * g->PZ) +
                         sizeof(int) * (size_t)g->Mx * 8 + 2 * sizeof(uint64_t) + 64;
    g->ring = fixed + sizeof(float) * (size_t)g->Mx * (g->WY + g->WZ) >
              (size_t)max_smem_optin();
    const int nw = g->ring ? 2 * XB : g->Mx;
    size_t s = sizeof(float) * (2 * sb + (size_t)XB * TY * g->PZ +
                                (size_t)nw * (g->WY + g->WZ)) +
               sizeof(int) * (size_t)g->Mx * 8 + 2 * sizeof(uint64_t) + 64;
    // the mode-2 epilogue reuses S for a [Z][TY][XB] tile
    // the mode-2 epilogue stages a [Z][TY][XB] tile over the S and X buffers
    if ((size_t)g->Z * TY * XB > 2 * sb + (size_t)XB * TY * g->PZ) return false;
    *smem = s;
    return s <= (size_t)max_smem_optin();
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

template <int TY, int XB>
int cone_tma_launch_t(const float* mu, const float* U, const float* Vw, float* out, int64_t Vn,
                      const ConeGeom& g, size_t smem, int threads, int mode, int L, int a_base,
                      int64_t out_a_stride, int64_t out_l_stride, cudaStream_t st) {
    auto enc = encode_fn();
    if (!enc) {
        set_error("cuTensorMapEncodeTiled is not available from the driver");
        return FLC_ERR_UNSUPPORTED;
    }
    CUtensorMap map;
    cuuint64_t dims[3] = {(cuuint64_t)g.Y, (cuuint64_t)g.X, (cuuint64_t)(Vn * g.Z)};
    cuuint64_t strides[2] = {(cuuint64_t)g.Y * 4, (cuuint64_t)g.X * g.Y * 4};
    cuuint32_t box[3] = {(cuuint32_t)g.boxW, 1, (cuuint32_t)g.Z};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)mu, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return FLC_ERR_UNSUPPORTED;
    }
    auto kern = g.ring ? cone_tma_kernel<TY, XB, true> : cone_tma_kernel<TY, XB, false>;
    FLC_TRY_CUDA(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    dim3 grid((unsigned)ceil_div(g.Y, TY), (unsigned)ceil_div(g.X, XB), (unsigned)Vn);
    kern<<<grid, threads, smem, st>>>(map, U, Vw, out, g, mode, L, a_base, out_a_stride, out_l_stride);
    return check_launch("cone_tma_kernel");
}

}  // namespace

// Returns FLC_ERR_UNSUPPORTED (without launching) when the shape does not
// fit the pipelined kernel; the caller then uses the plain separable kernel.
int cone_tma_launch(const float* mu, const float* U, const float* Vw, float* out, int64_t Vn,
                    int64_t Z, int64_t X, int64_t Y, int64_t Mz, int64_t Mx, int64_t My, int mode,
                    int L, int a_base, int64_t out_a_stride, int64_t out_l_stride, cudaStream_t st) {
    if (((uintptr_t)mu & 15) != 0 || Vn * Z > (int64_t)1 << 31 || Vn > 65535) return FLC_ERR_UNSUPPORTED;
    ConeGeom g;
    size_t smem;
    int threads;
    const int64_t wl = tune(kTuneConeWaitLimit), sk = tune(kTuneConeSkipLoad);
    g.wait_limit = (wl > 0 && wl < kWaitLimit) ? (int)wl : kWaitLimit;
    g.skip_step = (sk > 0 && sk < (1 << 30)) ? (int)sk - 1 : -1;
    int64_t variant = tune(kTuneConeVariant);  // 0 auto, 1 16x8, 2 8x4, 3 plain, 4 spectral
    if (variant == 4) variant = 0;              // the spectral form fell back to this kernel
    if (variant == 3) return FLC_ERR_UNSUPPORTED;
    if ((variant == 1 || (variant == 0 && Z <= 128)) &&
        cone_tma_geom<16, 8>(Z, X, Y, Mz, Mx, My, &g, &smem, &threads))
        return cone_tma_launch_t<16, 8>(mu, U, Vw, out, Vn, g, smem, threads, mode, L, a_base,
                                        out_a_stride, out_l_stride, st);
    if (cone_tma_geom<8, 4>(Z, X, Y, Mz, Mx, My, &g, &smem, &threads))
        return cone_tma_launch_t<8, 4>(mu, U, Vw, out, Vn, g, smem, threads, mode, L, a_base,
                                       out_a_stride, out_l_stride, st);
    return FLC_ERR_UNSUPPORTED;
}

int cone_device_status(int reset) {
    int v = 0;
    cudaMemcpyFromSymbol(&v, g_cone_status, sizeof(int));
    if (reset) {
        int z = 0;
        cudaMemcpyToSymbol(g_cone_status, &z, sizeof(int));
    }
    return v;
}

}  // namespace flc
