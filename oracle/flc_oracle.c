/*
 * CPU oracle for the FL_correction XRF self-absorption hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C with FP64
 * arithmetic, what the reference computes on the hot path, so that the CUDA
 * product can be checked against it.  Only tests/, __graft_entry__.smoke()
 * and the CPU-baseline legs of bench.py load it; the product never does.
 *
 * Every function names the reference file:line it restates.  Sample
 * coordinates use the reference's FP32 constants (cos/sin rounded to float,
 * the clamp bound `N - 1.001f`) and are then evaluated in FP64, so the oracle
 * differs from the FP32 reference only by FP32 rounding.
 *
 * Parallelism: OpenMP over independent outputs (slices / angles), used when
 * this file is timed as the CPU baseline.  Results do not depend on the
 * thread count: each output is owned by one thread and summed in a fixed
 * order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------
 * In-plane rotation with torch grid_sample semantics.
 * Restates FL/torch_image_util.py:13-114 (affine_grid + grid_sample,
 * bilinear, zeros padding, align_corners=False, output size == input size).
 * `cos_t`/`sin_t` are the entries of the FP32 theta matrix (:80-85).
 * Base grid (align_corners=False): xn = (2w+1)/W - 1, yn = (2h+1)/H - 1.
 * grid = [[c,-s],[s,c]] (xn,yn); unnormalise ix = ((gx+1)W-1)/2.
 * ---------------------------------------------------------------------- */
void orc_rotate(const double* in, double* out, i64 nimg, i64 H, i64 W,
                double cos_t, double sin_t) {
#pragma omp parallel for schedule(static)
    for (i64 n = 0; n < nimg; ++n) {
        const double* src = in + n * H * W;
        double* dst = out + n * H * W;
        for (i64 h = 0; h < H; ++h) {
            double yn = (2.0 * h + 1.0) / (double)H - 1.0;
            for (i64 w = 0; w < W; ++w) {
                double xn = (2.0 * w + 1.0) / (double)W - 1.0;
                double gx = cos_t * xn - sin_t * yn;
                double gy = sin_t * xn + cos_t * yn;
                double ix = ((gx + 1.0) * (double)W - 1.0) * 0.5;
                double iy = ((gy + 1.0) * (double)H - 1.0) * 0.5;
                double fx = floor(ix), fy = floor(iy);
                i64 x0 = (i64)fx, y0 = (i64)fy;
                double tx = ix - fx, ty = iy - fy;
                double acc = 0.0;
                for (int dy = 0; dy < 2; ++dy) {
                    i64 yy = y0 + dy;
                    if (yy < 0 || yy >= H) continue;
                    double wy = dy ? ty : 1.0 - ty;
                    for (int dx = 0; dx < 2; ++dx) {
                        i64 xx = x0 + dx;
                        if (xx < 0 || xx >= W) continue;
                        double wx = dx ? tx : 1.0 - tx;
                        acc += src[yy * W + xx] * wx * wy;
                    }
                }
                dst[h * W + w] = acc;
            }
        }
    }
}

/* Adjoint of orc_rotate (grid_sample's input gradient): scatter. */
void orc_rotate_adjoint(const double* gout, double* gin, i64 nimg, i64 H, i64 W,
                        double cos_t, double sin_t) {
#pragma omp parallel for schedule(static)
    for (i64 n = 0; n < nimg; ++n) {
        const double* g = gout + n * H * W;
        double* dst = gin + n * H * W;
        memset(dst, 0, sizeof(double) * H * W);
        for (i64 h = 0; h < H; ++h) {
            double yn = (2.0 * h + 1.0) / (double)H - 1.0;
            for (i64 w = 0; w < W; ++w) {
                double xn = (2.0 * w + 1.0) / (double)W - 1.0;
                double gx = cos_t * xn - sin_t * yn;
                double gy = sin_t * xn + cos_t * yn;
                double ix = ((gx + 1.0) * (double)W - 1.0) * 0.5;
                double iy = ((gy + 1.0) * (double)H - 1.0) * 0.5;
                double fx = floor(ix), fy = floor(iy);
                i64 x0 = (i64)fx, y0 = (i64)fy;
                double tx = ix - fx, ty = iy - fy;
                double v = g[h * W + w];
                for (int dy = 0; dy < 2; ++dy) {
                    i64 yy = y0 + dy;
                    if (yy < 0 || yy >= H) continue;
                    double wy = dy ? ty : 1.0 - ty;
                    for (int dx = 0; dx < 2; ++dx) {
                        i64 xx = x0 + dx;
                        if (xx < 0 || xx >= W) continue;
                        double wx = dx ? tx : 1.0 - tx;
                        dst[yy * W + xx] += v * wx * wy;
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------
 * Incident-beam attenuation: exclusive reverse product along H.
 * Restates FL/torch_functions.py:95-102:
 *   atten[h] = prod_{h' > h} (1 - mu[h']),  atten[H-1] = 1.
 * ---------------------------------------------------------------------- */
void orc_incident_scan(const double* mu, double* out, i64 nimg, i64 H, i64 W) {
#pragma omp parallel for schedule(static)
    for (i64 n = 0; n < nimg; ++n) {
        const double* m = mu + n * H * W;
        double* o = out + n * H * W;
        for (i64 w = 0; w < W; ++w) {
            double p = 1.0;
            for (i64 h = H - 1; h >= 0; --h) {
                o[h * W + w] = p;
                p *= 1.0 - m[h * W + w];
            }
        }
    }
}

/* ------------------------------------------------------------------------
 * Cone-mask correlation, reference layout.
 * Restates FL/cuda_lib/atten_cuda_kernel.cu:10-57 (atten_kernel):
 *   out[k,z,x,y] = sum_{dz,dx,dy} mu[k, z+dz-Mz/2, x+dx, y+dy-My/2] * mask[dz,dx,dy]
 * with out-of-range taps skipped; loop order dz, dx, dy as in the kernel.
 * ---------------------------------------------------------------------- */
void orc_cone_ref(const double* mu, const double* mask, double* out,
                  i64 K, i64 Z, i64 X, i64 Y, i64 Mz, i64 Mx, i64 My) {
    i64 hz = Mz / 2, hy = My / 2;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (i64 k = 0; k < K; ++k)
        for (i64 z = 0; z < Z; ++z)
            for (i64 x = 0; x < X; ++x)
                for (i64 y = 0; y < Y; ++y) {
                    double acc = 0.0;
                    for (i64 dz = 0; dz < Mz; ++dz) {
                        i64 zz = z + dz - hz;
                        if (zz < 0 || zz >= Z) continue;
                        for (i64 dx = 0; dx < Mx; ++dx) {
                            i64 xx = x + dx;
                            if (xx >= X) break;
                            const double* mrow = mask + (dz * Mx + dx) * My;
                            const double* src = mu + ((k * Z + zz) * X + xx) * Y;
                            for (i64 dy = 0; dy < My; ++dy) {
                                i64 yy = y + dy - hy;
                                if (yy < 0 || yy >= Y) continue;
                                double m = mrow[dy];
                                if (m != 0.0) acc += src[yy] * m;
                            }
                        }
                    }
                    out[((k * Z + z) * X + x) * Y + y] = acc;
                }
}

/* ------------------------------------------------------------------------
 * Cone-mask correlation in the unrotated (beam) frame.
 * FL/torch_functions.py:142-171 applies rot90(clock) -> atten_kernel ->
 * rot90(c-clock) (FL/torch_image_util.py:129-134).  Composing the index maps
 * gives, for mu[k,z,h,w] with the detector on the +w side:
 *   res[k,z,h,w] = sum mask[dz,dx,dy] * mu[k, z+dz-Mz/2, h-(dy-My/2), w+dx].
 * (Requires H == W, as rot90 of the reference does.)
 * ---------------------------------------------------------------------- */
void orc_cone_beam(const double* mu, const double* mask, double* out,
                   i64 K, i64 Z, i64 H, i64 W, i64 Mz, i64 Mx, i64 My) {
    i64 hz = Mz / 2, hy = My / 2;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (i64 k = 0; k < K; ++k)
        for (i64 z = 0; z < Z; ++z)
            for (i64 h = 0; h < H; ++h)
                for (i64 w = 0; w < W; ++w) {
                    double acc = 0.0;
                    for (i64 dz = 0; dz < Mz; ++dz) {
                        i64 zz = z + dz - hz;
                        if (zz < 0 || zz >= Z) continue;
                        for (i64 dx = 0; dx < Mx; ++dx) {
                            i64 ww = w + dx;
                            if (ww >= W) break;
                            const double* mrow = mask + (dz * Mx + dx) * My;
                            for (i64 dy = 0; dy < My; ++dy) {
                                i64 hh = h - (dy - hy);
                                if (hh < 0 || hh >= H) continue;
                                double m = mrow[dy];
                                if (m != 0.0) acc += mu[((k * Z + zz) * H + hh) * W + ww] * m;
                            }
                        }
                    }
                    out[((k * Z + z) * H + h) * W + w] = acc;
                }
}

/* orc_cone_beam restricted to output slices [z0, z1) of every volume
 * (out has the full (K,Z,H,W) shape; other slices are left untouched).
 * Used to time a bounded sample of the full computation. */
void orc_cone_beam_slab(const double* mu, const double* mask, double* out,
                        i64 K, i64 Z, i64 H, i64 W, i64 Mz, i64 Mx, i64 My, i64 z0, i64 z1) {
    i64 hz = Mz / 2, hy = My / 2;
#pragma omp parallel for collapse(3) schedule(dynamic, 1)
    for (i64 k = 0; k < K; ++k)
        for (i64 z = z0; z < z1; ++z)
            for (i64 h = 0; h < H; ++h)
                for (i64 w = 0; w < W; ++w) {
                    double acc = 0.0;
                    for (i64 dz = 0; dz < Mz; ++dz) {
                        i64 zz = z + dz - hz;
                        if (zz < 0 || zz >= Z) continue;
                        for (i64 dx = 0; dx < Mx; ++dx) {
                            i64 ww = w + dx;
                            if (ww >= W) break;
                            const double* mrow = mask + (dz * Mx + dx) * My;
                            for (i64 dy = 0; dy < My; ++dy) {
                                i64 hh = h - (dy - hy);
                                if (hh < 0 || hh >= H) continue;
                                double m = mrow[dy];
                                if (m != 0.0) acc += mu[((k * Z + zz) * H + hh) * W + ww] * m;
                            }
                        }
                    }
                    out[((k * Z + z) * H + h) * W + w] = acc;
                }
}

/* Adjoint of orc_cone_beam: g_mu[k,z',h',w'] = sum over outputs that read it. */
void orc_cone_beam_adjoint(const double* g, const double* mask, double* gmu,
                           i64 K, i64 Z, i64 H, i64 W, i64 Mz, i64 Mx, i64 My) {
    i64 hz = Mz / 2, hy = My / 2;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (i64 k = 0; k < K; ++k)
        for (i64 zz = 0; zz < Z; ++zz)
            for (i64 hh = 0; hh < H; ++hh)
                for (i64 ww = 0; ww < W; ++ww) {
                    double acc = 0.0;
                    for (i64 dz = 0; dz < Mz; ++dz) {
                        i64 z = zz - dz + hz;
                        if (z < 0 || z >= Z) continue;
                        for (i64 dx = 0; dx < Mx; ++dx) {
                            i64 w = ww - dx;
                            if (w < 0) break;
                            const double* mrow = mask + (dz * Mx + dx) * My;
                            for (i64 dy = 0; dy < My; ++dy) {
                                i64 h = hh + (dy - hy);
                                if (h < 0 || h >= H) continue;
                                double m = mrow[dy];
                                if (m != 0.0) acc += g[((k * Z + z) * H + h) * W + w] * m;
                            }
                        }
                    }
                    gmu[((k * Z + zz) * H + hh) * W + ww] = acc;
                }
}

/* ------------------------------------------------------------------------
 * Projector geometry, FL/cuda_lib/atten_cuda_kernel.cu:271-296,298-337:
 *   c = cosf(-th), s = sinf(-th), cx = (W-1)/2, cy = (H-1)/2
 *   row = c*(h-cy) - s*(w-cx) + cy,  col = s*(h-cy) + c*(w-cx) + cx
 *   clamp row to [0, H-1.001f], col to [0, W-1.001f]; floor; bilinear.
 * The backward kernels (:177-231, :390-446) use cos(th), sin(th) and the
 * algebraically identical expressions, so one geometry serves both.
 * ---------------------------------------------------------------------- */
typedef struct {
    i64 i0, j0;     /* top-left corner (row, col) */
    double dr, dc;  /* fractional offsets */
} orc_tap;

static inline orc_tap orc_sample(double c, double s, double cy, double cx,
                                 double rmax, double cmax, i64 h, i64 w) {
    double r = c * ((double)h - cy) - s * ((double)w - cx) + cy;
    double q = s * ((double)h - cy) + c * ((double)w - cx) + cx;
    r = fmin(fmax(r, 0.0), rmax);
    q = fmin(fmax(q, 0.0), cmax);
    orc_tap t;
    double fr = floor(r), fq = floor(q);
    t.i0 = (i64)fr; t.j0 = (i64)fq;
    t.dr = r - fr; t.dc = q - fq;
    return t;
}

static inline void orc_geom(float th, i64 H, i64 W, double* c, double* s,
                            double* cy, double* cx, double* rmax, double* cmax) {
    *c = (double)cosf(-th);
    *s = (double)sinf(-th);
    *cx = (double)((float)(W - 1) * 0.5f);
    *cy = (double)((float)(H - 1) * 0.5f);
    *rmax = (double)((float)H - 1.001f);
    *cmax = (double)((float)W - 1.001f);
}

/* Forward emission, batched slices: atten (A,B,H,W), C (R,B,H,W), em (A,R)
 * -> Pf (A,B,W).  Restates atten_cuda_kernel.cu:298-337 and :91-142 (B=1). */
void orc_fwd_emission(const double* atten, const double* C, const double* em,
                      const float* theta, double* Pf,
                      i64 A, i64 B, i64 R, i64 H, i64 W) {
#pragma omp parallel for collapse(2) schedule(static)
    for (i64 a = 0; a < A; ++a)
        for (i64 b = 0; b < B; ++b) {
            double c, s, cy, cx, rmax, cmax;
            orc_geom(theta[a], H, W, &c, &s, &cy, &cx, &rmax, &cmax);
            for (i64 w = 0; w < W; ++w) {
                double acc = 0.0;
                for (i64 h = 0; h < H; ++h) {
                    orc_tap t = orc_sample(c, s, cy, cx, rmax, cmax, h, w);
                    double val = 0.0;
                    for (i64 r = 0; r < R; ++r) {
                        const double* img = C + (r * B + b) * H * W;
                        double v00 = img[t.i0 * W + t.j0];
                        double v01 = img[t.i0 * W + t.j0 + 1];
                        double v10 = img[(t.i0 + 1) * W + t.j0];
                        double v11 = img[(t.i0 + 1) * W + t.j0 + 1];
                        double interp = (1 - t.dc) * (1 - t.dr) * v00 + t.dc * (1 - t.dr) * v01 +
                                        (1 - t.dc) * t.dr * v10 + t.dc * t.dr * v11;
                        val += em[a * R + r] * interp;
                    }
                    acc += atten[((a * B + b) * H + h) * W + w] * val;
                }
                Pf[(a * B + b) * W + w] = acc;
            }
        }
}

/* Backward emission (exact transpose of orc_fwd_emission): ratio (A,B,W)
 * -> out (R,B,H,W).  Restates atten_cuda_kernel.cu:390-446 and :177-231. */
void orc_bwd_emission(const double* atten, const double* ratio, const double* em,
                      const float* theta, double* out,
                      i64 A, i64 B, i64 R, i64 H, i64 W) {
    memset(out, 0, sizeof(double) * R * B * H * W);
#pragma omp parallel for schedule(static)
    for (i64 b = 0; b < B; ++b) {
        for (i64 a = 0; a < A; ++a) {
            double c, s, cy, cx, rmax, cmax;
            orc_geom(theta[a], H, W, &c, &s, &cy, &cx, &rmax, &cmax);
            for (i64 w = 0; w < W; ++w) {
                double rq = ratio[(a * B + b) * W + w];
                for (i64 h = 0; h < H; ++h) {
                    orc_tap t = orc_sample(c, s, cy, cx, rmax, cmax, h, w);
                    double av = atten[((a * B + b) * H + h) * W + w];
                    for (i64 r = 0; r < R; ++r) {
                        double wgt = em[a * R + r] * av * rq;
                        double* o = out + (r * B + b) * H * W;
                        o[t.i0 * W + t.j0] += wgt * (1 - t.dc) * (1 - t.dr);
                        o[t.i0 * W + t.j0 + 1] += wgt * t.dc * (1 - t.dr);
                        o[(t.i0 + 1) * W + t.j0] += wgt * (1 - t.dc) * t.dr;
                        o[(t.i0 + 1) * W + t.j0 + 1] += wgt * t.dc * t.dr;
                    }
                }
            }
        }
    }
}

/* Derivative of Pf w.r.t. atten: g_atten[a,b,h,w] = g_Pf[a,b,w] * sum_r em[a,r] * interp_r(h,w). */
void orc_fwd_emission_datten(const double* gPf, const double* C, const double* em,
                             const float* theta, double* gatten,
                             i64 A, i64 B, i64 R, i64 H, i64 W) {
#pragma omp parallel for collapse(2) schedule(static)
    for (i64 a = 0; a < A; ++a)
        for (i64 b = 0; b < B; ++b) {
            double c, s, cy, cx, rmax, cmax;
            orc_geom(theta[a], H, W, &c, &s, &cy, &cx, &rmax, &cmax);
            for (i64 w = 0; w < W; ++w) {
                double g = gPf[(a * B + b) * W + w];
                for (i64 h = 0; h < H; ++h) {
                    orc_tap t = orc_sample(c, s, cy, cx, rmax, cmax, h, w);
                    double val = 0.0;
                    for (i64 r = 0; r < R; ++r) {
                        const double* img = C + (r * B + b) * H * W;
                        double interp = (1 - t.dc) * (1 - t.dr) * img[t.i0 * W + t.j0] +
                                        t.dc * (1 - t.dr) * img[t.i0 * W + t.j0 + 1] +
                                        (1 - t.dc) * t.dr * img[(t.i0 + 1) * W + t.j0] +
                                        t.dc * t.dr * img[(t.i0 + 1) * W + t.j0 + 1];
                        val += em[a * R + r] * interp;
                    }
                    gatten[((a * B + b) * H + h) * W + w] = g * val;
                }
            }
        }
}

/* ------------------------------------------------------------------------
 * Huber gradient over the 4 in-plane neighbours.
 * Restates atten_cuda_kernel.cu:564-616 (huber_grad_batch_kernel).
 * ---------------------------------------------------------------------- */
void orc_huber_grad(const double* C, double* g, i64 RB, i64 H, i64 W, double delta) {
    static const int dr[4] = {-1, 1, 0, 0};
    static const int dc[4] = {0, 0, -1, 1};
#pragma omp parallel for schedule(static)
    for (i64 n = 0; n < RB; ++n)
        for (i64 r = 0; r < H; ++r)
            for (i64 c = 0; c < W; ++c) {
                const double* img = C + n * H * W;
                double cp = img[r * W + c], acc = 0.0;
                for (int k = 0; k < 4; ++k) {
                    i64 rr = r + dr[k], cc = c + dc[k];
                    if (rr < 0 || rr >= H || cc < 0 || cc >= W) continue;
                    double d = cp - img[rr * W + cc];
                    acc += fabs(d) <= delta ? d : (d > 0 ? delta : -delta);
                }
                g[n * H * W + r * W + c] = acc;
            }
}

/* ------------------------------------------------------------------------
 * MLEM with optional Huber term.  Restates FL/cuda_lib/atten_cuda.cpp:283-345
 * (mlem_cuda_batch; mlem_cuda :244-281 is the B=1 case):
 *   sens = max(P^T 1, 1e-6)
 *   repeat: Pf = max(P C, 1e-6); back = P^T (I / Pf);
 *           C = C*back / (sens + beta*huber(C))   (beta > 0)
 *           C = C*back / sens                      (beta == 0)
 *           C = max(C, 0)
 * `C` is updated in place (the caller passes a copy of C_init).
 * ---------------------------------------------------------------------- */
void orc_mlem(double* C, const double* atten, const double* em, const float* theta,
              const double* I, i64 n_iter, double beta, double delta,
              i64 A, i64 B, i64 R, i64 H, i64 W) {
    i64 nC = R * B * H * W, nP = A * B * W;
    double* sens = (double*)malloc(sizeof(double) * nC);
    double* back = (double*)malloc(sizeof(double) * nC);
    double* grad = (double*)malloc(sizeof(double) * nC);
    double* Pf = (double*)malloc(sizeof(double) * nP);
    for (i64 i = 0; i < nP; ++i) Pf[i] = 1.0;
    orc_bwd_emission(atten, Pf, em, theta, sens, A, B, R, H, W);
    for (i64 i = 0; i < nC; ++i) sens[i] = sens[i] < 1e-6 ? 1e-6 : sens[i];
    for (i64 it = 0; it < n_iter; ++it) {
        orc_fwd_emission(atten, C, em, theta, Pf, A, B, R, H, W);
        for (i64 i = 0; i < nP; ++i) Pf[i] = I[i] / (Pf[i] < 1e-6 ? 1e-6 : Pf[i]);
        orc_bwd_emission(atten, Pf, em, theta, back, A, B, R, H, W);
        if (beta > 0.0) {
            orc_huber_grad(C, grad, R * B, H, W, delta);
            for (i64 i = 0; i < nC; ++i) C[i] = C[i] * back[i] / (sens[i] + beta * grad[i]);
        } else {
            for (i64 i = 0; i < nC; ++i) C[i] = C[i] * back[i] / sens[i];
        }
        for (i64 i = 0; i < nC; ++i) C[i] = C[i] < 0.0 ? 0.0 : C[i];
    }
    free(sens); free(back); free(grad); free(Pf);
}
