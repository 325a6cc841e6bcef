/*
 * Gradients of the multi-view NCC cost, for plane and pose polishing after PatchMatch.
 *
 * Objective of reference pixel p: c(p) = sum over the sources s of view_cost(p, s), the
 * bilateral-weighted 1 - NCC over the window of frontend/src/app/vision/mvs/patchmatch.wgsl.ts
 * (prepare_window :90-110, view_cost :130-159), with exact bilinear samples of the stored
 * images.  Parameters:
 *   - a plane per reference pixel: z-depth d and two normal angles (a, b),
 *     n = (sin a cos b, sin b, -cos a cos b)     (a = b = 0 faces the camera);
 *   - an se(3) increment per view, delta = (v, w): the view's world -> camera map becomes
 *     X -> Exp(w) (R0 X + t0) + v, with (R0, t0) the handle's FP64 pose.
 * A source whose window leaves the image or passes behind the camera costs 2, a window without
 * texture 1, and every source costs 2 for a plane seen edge-on or from behind
 * (n . ray >= -1e-3) or with d <= 0; those constants carry no gradient.
 *
 * Chain rule, per window sample i of a (pixel, source) pair; q = H x_i with H = B + kt u^T,
 * u = K_r^-T n / (d n.ray), sample value s_i at (q.x / q.z, q.y / q.z):
 *   dc/ds_i = -(w_i / W) ((r_i - mr) / den - NCC (s_i - ms) / vs)
 *   dc/dq   = dc/ds_i / q.z (gx, gy, -(gx u + gy v))      (gx, gy: bilinear image gradient)
 *   dc/du  += (dc/dq . kt) x_i                            -> depth and angles of the pixel
 *   e_i = (u . x_i) K_s^T dc/dq       the gradient at the source-camera point
 *                                     Y_i = K_s^-1 q / (u . x_i)
 *   S1 += e_i,  S2 += Y_i x e_i       summed per (reference, source) pair over all pixels
 * k_finalize turns S1 and S2 into the gradients of both views' increments in FP64 with the
 * exact SO(3) left Jacobians; k_compose builds each pair's relative pose and homography base
 * from the FP64 base poses and the increments, in FP64 on the device.  The warped samples are
 * recomputed in the gradient pass instead of being stored.
 */
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/luvas3d.h"
#include "l3d_fmath.h"
#include "l3d_internal.h"

namespace {

/* ---- FP64 SO(3) helpers ---- */

/* Coefficients of I + A [w]x + B [w]x^2: the exponential (A = sin t / t, B = (1 - cos t) / t^2)
 * or the left Jacobian (A = (1 - cos t) / t^2, B = (t - sin t) / t^3), t = |w|; Taylor series
 * for tiny angles. */
__device__ void so3_coeffs(const double* w, bool jacobian, double* A, double* B) {
    const double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    if (th2 < 1e-8) {
        if (jacobian) {
            *A = 0.5 - th2 / 24.0;
            *B = 1.0 / 6.0 - th2 / 120.0;
        } else {
            *A = 1.0 - th2 / 6.0;
            *B = 0.5 - th2 / 24.0;
        }
        return;
    }
    const double th = sqrt(th2);
    const double s = sin(th), c = cos(th);
    if (jacobian) {
        *A = (1.0 - c) / th2;
        *B = (th - s) / (th2 * th);
    } else {
        *A = s / th;
        *B = (1.0 - c) / th2;
    }
}

__device__ void so3_matrix(const double* w, double A, double B, double* M) {
    const double K[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            const double kk = K[r * 3] * K[c] + K[r * 3 + 1] * K[3 + c] + K[r * 3 + 2] * K[6 + c];
            M[r * 3 + c] = (r == c ? 1.0 : 0.0) + A * K[r * 3 + c] + B * kk;
        }
}

__device__ void exp_so3(const double* w, double* R) {
    double A, B;
    so3_coeffs(w, false, &A, &B);
    so3_matrix(w, A, B, R);
}

/* left Jacobian: Exp(w + e) ~ Exp(Jl(w) e) Exp(w) */
__device__ void jl_so3(const double* w, double* J) {
    double A, B;
    so3_coeffs(w, true, &A, &B);
    so3_matrix(w, A, B, J);
}

__device__ void mat_mul(const double* A, const double* B, double* C) {
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            C[r * 3 + c] = A[r * 3] * B[c] + A[r * 3 + 1] * B[3 + c] + A[r * 3 + 2] * B[6 + c];
}
__device__ void mat_vec(const double* A, const double* x, double* y) {
    for (int r = 0; r < 3; r++) y[r] = A[r * 3] * x[0] + A[r * 3 + 1] * x[1] + A[r * 3 + 2] * x[2];
}
__device__ void mat_tvec(const double* A, const double* x, double* y) {
    for (int c = 0; c < 3; c++) y[c] = A[c] * x[0] + A[3 + c] * x[1] + A[6 + c] * x[2];
}
__device__ void transpose(const double* A, double* T) {
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) T[c * 3 + r] = A[r * 3 + c];
}
__device__ void cross(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ void load_delta(const float* deltas, int view, double* v, double* w) {
    for (int i = 0; i < 3; i++) {
        v[i] = deltas ? (double)deltas[6 * view + i] : 0.0;
        w[i] = deltas ? (double)deltas[6 * view + 3 + i] : 0.0;
    }
}

/* Current pose of a view: R = Exp(w) R0, t = Exp(w) t0 + v. */
__device__ void current_pose(const L3dGradView& b, const float* deltas, int view, double* R,
                             double* t) {
    double v[3], w[3], E[9], et[3];
    load_delta(deltas, view, v, w);
    exp_so3(w, E);
    mat_mul(E, b.R, R);
    mat_vec(E, b.t, et);
    for (int i = 0; i < 3; i++) t[i] = et[i] + v[i];
}

/* One thread per (reference, source) pair: relative pose (relativePose, geometry/camera.ts:73-77)
 * and homography base B = K_s R K_r^-1, kt = K_s t (DenseStereo.params, dense-stereo.ts:314-355)
 * in FP64, rounded to f32. */
__global__ void k_compose(const L3dGradView* __restrict__ views, const float* __restrict__ deltas,
                          const L3dGradJob job, L3dGradPair* __restrict__ pairs) {
    const int k = threadIdx.x;
    if (k >= job.n) return;
    const int s = job.src[k];
    const L3dGradView& vr = views[job.ref];
    const L3dGradView& vs = views[s];
    double Rr[9], tr[3], Rs[9], ts[3], RrT[9], R[9], rt[3];
    current_pose(vr, deltas, job.ref, Rr, tr);
    current_pose(vs, deltas, s, Rs, ts);
    /* X_s = Rs Rr^T (X_r - tr) + ts */
    transpose(Rr, RrT);
    mat_mul(Rs, RrT, R);
    mat_vec(R, tr, rt);
    const double t[3] = {ts[0] - rt[0], ts[1] - rt[1], ts[2] - rt[2]};
    const double* kr = vr.k;
    const double* kv = vs.k;
    double A[9];
    for (int c = 0; c < 3; c++) {
        A[c] = kv[0] * R[c] + kv[2] * R[6 + c];
        A[3 + c] = kv[1] * R[3 + c] + kv[3] * R[6 + c];
        A[6 + c] = R[6 + c];
    }
    L3dGradPair& o = pairs[k];
    for (int r = 0; r < 3; r++) {
        o.B[r * 3 + 0] = (float)(A[r * 3 + 0] / kr[0]);
        o.B[r * 3 + 1] = (float)(A[r * 3 + 1] / kr[1]);
        o.B[r * 3 + 2] =
            (float)(A[r * 3 + 2] - A[r * 3 + 0] * kr[2] / kr[0] - A[r * 3 + 1] * kr[3] / kr[1]);
    }
    o.kt[0] = (float)(kv[0] * t[0] + kv[2] * t[2]);
    o.kt[1] = (float)(kv[1] * t[1] + kv[3] * t[2]);
    o.kt[2] = (float)t[2];
    for (int i = 0; i < 4; i++) o.ks[i] = (float)kv[i];
    o.W = vs.W;
    o.H = vs.H;
    o.img_off = vs.img_off;
}

/* Texel loads of the handle's image storage (u8 texels are value / 255). */
template <int ST>
__device__ __forceinline__ float texel(const void* img, long long i) {
    if (ST == L3D_DTYPE_F32) return __ldg((const float*)img + i);
    if (ST == L3D_DTYPE_F16) return __half2float(__ldg((const __half*)img + i));
    if (ST == L3D_DTYPE_BF16) return __bfloat162float(__ldg((const __nv_bfloat16*)img + i));
    return (float)__ldg((const uint8_t*)img + i) / 255.0f;
}

/* Bilinear sample (clamp to edge) at texel coordinates (u, v) and its gradient. */
template <int ST>
__device__ __forceinline__ float bilinear_grad(const void* img, int W, int H, float u, float v,
                                               float* gu, float* gv) {
    const float x0f = floorf(u), y0f = floorf(v);
    const float fx = u - x0f, fy = v - y0f;
    const int x0 = min(max((int)x0f, 0), W - 1), y0 = min(max((int)y0f, 0), H - 1);
    const int x1 = min(x0 + 1, W - 1), y1 = min(y0 + 1, H - 1);
    const float a = texel<ST>(img, (long long)y0 * W + x0);
    const float b = texel<ST>(img, (long long)y0 * W + x1);
    const float c = texel<ST>(img, (long long)y1 * W + x0);
    const float e = texel<ST>(img, (long long)y1 * W + x1);
    const float top = fmaf(fx, b - a, a), bot = fmaf(fx, e - c, c);
    *gu = fmaf(fy, (e - c) - (b - a), b - a);
    *gv = bot - top;
    return fmaf(fy, bot - top, top);
}

constexpr int kTileX = 32, kTileY = 4;

/* One thread per reference pixel, blocks of 32 x 4 pixels.  Each (pixel, source) pair takes
 * one pass over the window for the statistics and, when gradients are wanted, a second pass
 * that recomputes the samples and pushes the gradient through them.  Per-pair sums S1, S2 are
 * reduced per block and added to pair_sums in FP64. */
template <int N, int DIL, int ST>
__global__ void __launch_bounds__(kTileX * kTileY) k_ncc_grad(
        const L3dGradDev d, const L3dGradPair* __restrict__ pairs, int n,
        const float* __restrict__ planes, const float* __restrict__ grad_cost,
        float* __restrict__ cost_out, float* __restrict__ grad_planes,
        double* __restrict__ pair_sums) {
    constexpr int S = N * N;
    constexpr int HALF = ((N - 1) * DIL) / 2;
    __shared__ float red[kTileY][6];
    const int W = d.W, H = d.H;
    const int x = blockIdx.x * kTileX + (int)(threadIdx.x % kTileX);
    const int y = blockIdx.y * kTileY + (int)(threadIdx.x / kTileX);
    const bool active = x < W && y < H;
    const long long idx = active ? (long long)y * W + x : 0;
    const bool want_grad = grad_planes != nullptr || pair_sums != nullptr;
    const float px = (float)x, py = (float)y;

    /* reference window: values and bilateral weights (prepare_window) */
    /* the reference window in shared memory (lane-major) when it fits: the gradient pass
     * indexes it in a loop that is not fully unrolled, which puts register arrays in local
     * memory; the 11 x 11 window stays in (local) per-thread arrays */
    constexpr bool kSharedWin = S <= 36;
    constexpr int LS = kSharedWin ? kTileX * kTileY : 1;
    __shared__ float rv_s[kSharedWin ? S : 1][kTileX * kTileY], rw_s[kSharedWin ? S : 1][kTileX * kTileY];
    float rv_l[kSharedWin ? 1 : S], rw_l[kSharedWin ? 1 : S];
    float* const rv = kSharedWin ? &rv_s[0][threadIdx.x] : rv_l;
    float* const rw = kSharedWin ? &rw_s[0][threadIdx.x] : rw_l;
    float rsum = 1.0f, rmean = 0.0f, rvar = 0.0f;
    if (active) {
        const float center = texel<ST>(d.images, d.ref_img_off + idx);
        float sw = 0.0f, sr = 0.0f, srr = 0.0f;
#pragma unroll
        for (int i = 0; i < S; i++) {
            const int ox = (i % N) * DIL - HALF, oy = (i / N) * DIL - HALF;
            const int xx = min(max(x + ox, 0), W - 1), yy = min(max(y + oy, 0), H - 1);
            const float v = texel<ST>(d.images, d.ref_img_off + (long long)yy * W + xx);
            const float dc = v - center;
            const float wgt = l3d_expf(-(dc * dc) / (2.0f * 0.06f * 0.06f) -
                                       (float)(ox * ox + oy * oy) / (2.0f * 5.0f * 5.0f));
            rv[i * LS] = v;
            rw[i * LS] = wgt;
            sw = sw + wgt;
            sr = fmaf(wgt, v, sr);
            srr = fmaf(wgt * v, v, srr);
        }
        rsum = sw;
        rmean = sr / sw;
        rvar = fmaxf(fmaf(-rmean, rmean, srr / sw), 0.0f);
    }

    /* plane -> u = K_r^-T n / (d n.ray) */
    float dd = 1.0f, al = 0.0f, be = 0.0f;
    if (active) {
        dd = planes[idx * 3];
        al = planes[idx * 3 + 1];
        be = planes[idx * 3 + 2];
    }
    float sa, ca, sb, cb;
    sincosf(al, &sa, &ca);
    sincosf(be, &sb, &cb);
    const float nx = sa * cb, ny = sb, nz = -ca * cb;
    const float m0 = nx * d.kinv[0], m1 = ny * d.kinv[1];
    const float m2 = fmaf(nx, d.kinv[2], fmaf(ny, d.kinv[3], nz));
    const float mu = fmaf(m0, px, fmaf(m1, py, m2));  /* n . ray */
    const float rho = dd * mu;
    const bool plane_ok = active && dd > 0.0f && mu < -1e-3f;
    const float ir = plane_ok ? 1.0f / rho : 0.0f;
    const float u0 = m0 * ir, u1 = m1 * ir, u2 = m2 * ir;
    const float gout = grad_cost ? (active ? grad_cost[idx] : 0.0f) : 1.0f;

    float total = 0.0f;
    float gu0 = 0.0f, gu1 = 0.0f, gu2 = 0.0f;
    for (int k = 0; k < n; k++) {
        const L3dGradPair& pr = pairs[k];
        float c = 2.0f;
        float S1x = 0.0f, S1y = 0.0f, S1z = 0.0f, S2x = 0.0f, S2y = 0.0f, S2z = 0.0f;
        if (plane_ok) {
            float h[9];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                h[r * 3 + 0] = fmaf(pr.kt[r], u0, pr.B[r * 3 + 0]);
                h[r * 3 + 1] = fmaf(pr.kt[r], u1, pr.B[r * 3 + 1]);
                h[r * 3 + 2] = fmaf(pr.kt[r], u2, pr.B[r * 3 + 2]);
            }
            const void* img = (const char*)d.images + pr.img_off * d.elem;
            const float wmax = (float)(pr.W - 1), hmax = (float)(pr.H - 1);
            bool ok = true;
            float ss = 0.0f, sss = 0.0f, srs = 0.0f;
#pragma unroll
            for (int i = 0; i < S; i++) {
                const float xi = px + (float)((i % N) * DIL - HALF);
                const float yi = py + (float)((i / N) * DIL - HALF);
                const float qz = fmaf(h[6], xi, fmaf(h[7], yi, h[8]));
                const float qx = fmaf(h[0], xi, fmaf(h[1], yi, h[2]));
                const float qy = fmaf(h[3], xi, fmaf(h[4], yi, h[5]));
                const float iz = 1.0f / qz;
                const float uu = qx * iz, vv = qy * iz;
                ok = ok && qz > 1e-6f && uu >= 0.0f && vv >= 0.0f && uu <= wmax && vv <= hmax;
                float gx, gy;
                const float val = ok ? bilinear_grad<ST>(img, pr.W, pr.H, uu, vv, &gx, &gy) : 0.0f;
                ss = fmaf(rw[i * LS], val, ss);
                const float wv = rw[i * LS] * val;
                sss = fmaf(wv, val, sss);
                srs = fmaf(wv, rv[i * LS], srs);
            }
            if (ok) {
                const float ms = ss / rsum;
                const float vs = fmaxf(fmaf(-ms, ms, sss / rsum), 0.0f);
                const float den = sqrtf(rvar * vs);
                if (den < 1e-5f) {
                    c = 1.0f;
                } else {
                    const float cov = fmaf(-rmean, ms, srs / rsum);
                    const float ncc = cov / den;
                    const float raw = 1.0f - ncc;
                    c = fminf(fmaxf(raw, 0.0f), 2.0f);
                    if (want_grad && raw > 0.0f && raw < 2.0f) {
                        const float inv_w = 1.0f / rsum, iden = 1.0f / den, ivs = 1.0f / vs;
                        const float ks0 = pr.ks[0], ks1 = pr.ks[1], ks2 = pr.ks[2], ks3 = pr.ks[3];
                        const float iks0 = 1.0f / ks0, iks1 = 1.0f / ks1;
                        const float kt0 = pr.kt[0], kt1 = pr.kt[1], kt2 = pr.kt[2];
#pragma unroll 4
                        for (int i = 0; i < S; i++) {
                            const float xi = px + (float)((i % N) * DIL - HALF);
                            const float yi = py + (float)((i / N) * DIL - HALF);
                            const float qz = fmaf(h[6], xi, fmaf(h[7], yi, h[8]));
                            const float qx = fmaf(h[0], xi, fmaf(h[1], yi, h[2]));
                            const float qy = fmaf(h[3], xi, fmaf(h[4], yi, h[5]));
                            const float iz = 1.0f / qz;
                            const float uu = qx * iz, vv = qy * iz;
                            float gx, gy;
                            const float val = bilinear_grad<ST>(img, pr.W, pr.H, uu, vv, &gx, &gy);
                            const float dcs = -gout * (rw[i * LS] * inv_w) *
                                              ((rv[i * LS] - rmean) * iden - ncc * (val - ms) * ivs);
                            const float g0 = dcs * iz * gx, g1 = dcs * iz * gy;
                            const float g2 = -(g0 * uu + g1 * vv);
                            /* plane */
                            const float a = fmaf(g0, kt0, fmaf(g1, kt1, g2 * kt2));
                            gu0 = fmaf(a, xi, gu0);
                            gu1 = fmaf(a, yi, gu1);
                            gu2 += a;
                            /* pose: e = lambda K_s^T g at Y = K_s^-1 q / lambda */
                            const float lam = fmaf(u0, xi, fmaf(u1, yi, u2));
                            const float e0 = lam * (ks0 * g0);
                            const float e1 = lam * (ks1 * g1);
                            const float e2 = lam * fmaf(ks2, g0, fmaf(ks3, g1, g2));
                            const float il = 1.0f / lam;
                            const float Y2 = qz * il;
                            const float Y0 = (fmaf(-ks2, qz, qx) * iks0) * il;
                            const float Y1 = (fmaf(-ks3, qz, qy) * iks1) * il;
                            S1x += e0;
                            S1y += e1;
                            S1z += e2;
                            S2x += Y1 * e2 - Y2 * e1;
                            S2y += Y2 * e0 - Y0 * e2;
                            S2z += Y0 * e1 - Y1 * e0;
                        }
                    }
                }
            }
        }
        total += c;
        if (pair_sums) {
            const float v6[6] = {S1x, S1y, S1z, S2x, S2y, S2z};
#pragma unroll
            for (int j = 0; j < 6; j++) {
                float v = v6[j];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][j] = v;
            }
            __syncthreads();
            if (threadIdx.x < 6) {
                double acc = 0.0;
#pragma unroll
                for (int wi = 0; wi < kTileY; wi++) acc += (double)red[wi][threadIdx.x];
                if (acc != 0.0) atomicAdd(pair_sums + k * 6 + threadIdx.x, acc);
            }
            __syncthreads();
        }
    }
    if (!active) return;
    if (cost_out) cost_out[idx] = total;
    if (grad_planes) {
        float g_d = 0.0f, g_a = 0.0f, g_b = 0.0f;
        if (plane_ok) {
            /* u = m / (d mu), mu = m . (px, py, 1):  du/dd = -u / d,
             * dL/dm = gu / (d mu) - (gu . m) (px, py, 1) / (d mu^2) */
            const float gdotu = fmaf(gu0, u0, fmaf(gu1, u1, gu2 * u2));
            g_d = -gdotu / dd;
            const float gm = fmaf(gu0, m0, fmaf(gu1, m1, gu2 * m2));
            const float f = 1.0f / rho, f2 = gm / (rho * mu);
            const float dm0 = fmaf(gu0, f, -f2 * px), dm1 = fmaf(gu1, f, -f2 * py);
            const float dm2 = gu2 * f - f2;
            /* m = K^-T n  ->  dL/dn = K^-1 dL/dm */
            const float dn0 = fmaf(dm2, d.kinv[2], dm0 * d.kinv[0]);
            const float dn1 = fmaf(dm2, d.kinv[3], dm1 * d.kinv[1]);
            const float dn2 = dm2;
            /* n = (sa cb, sb, -ca cb) */
            g_a = fmaf(dn0, ca * cb, dn2 * (sa * cb));
            g_b = fmaf(dn0, -sa * sb, fmaf(dn1, cb, dn2 * (ca * sb)));
        }
        grad_planes[idx * 3] = g_d;
        grad_planes[idx * 3 + 1] = g_a;
        grad_planes[idx * 3 + 2] = g_b;
    }
}

/* One thread per pair: S1, S2 -> gradients of the source's and the reference's increments
 * (FP64), added into grad (6 per view).
 *   source:    g_v += S1,  g_w += Jl(w_s)^T (S2 - v_s x S1)
 *   reference: with E = Exp(w_s), Rm = R0_s R0_r^T, tm = t0_s - Rm t0_r,
 *              g_v -= (E Rm Exp(w_r)^T)^T S1,
 *              g_w -= Jl(-w_r)^T Rm^T (E^T (S2 - v_s x S1) - tm x E^T S1) */
__global__ void k_finalize(const L3dGradView* __restrict__ views, const float* __restrict__ deltas,
                           const L3dGradJob job, const double* __restrict__ pair_sums,
                           double* __restrict__ grad) {
    const int k = threadIdx.x;
    if (k >= job.n) return;
    const int s = job.src[k];
    const int ref = job.ref;
    const double* S1 = pair_sums + 6 * k;
    const double* S2 = S1 + 3;
    double vs_[3], ws[3], vr_[3], wr[3];
    load_delta(deltas, s, vs_, ws);
    load_delta(deltas, ref, vr_, wr);
    double vx[3], A[3], J[9], JA[3];
    cross(vs_, S1, vx);
    for (int i = 0; i < 3; i++) A[i] = S2[i] - vx[i];
    jl_so3(ws, J);
    mat_tvec(J, A, JA);
    for (int i = 0; i < 3; i++) {
        atomicAdd(grad + 6 * s + i, S1[i]);
        atomicAdd(grad + 6 * s + 3 + i, JA[i]);
    }
    const L3dGradView& vr = views[ref];
    const L3dGradView& vsv = views[s];
    double RrT[9], Rm[9], rt[3];
    transpose(vr.R, RrT);
    mat_mul(vsv.R, RrT, Rm);
    mat_vec(Rm, vr.t, rt);
    const double tm[3] = {vsv.t[0] - rt[0], vsv.t[1] - rt[1], vsv.t[2] - rt[2]};
    double E[9], Er[9], ErT[9], ERm[9], Rrs[9];
    exp_so3(ws, E);
    exp_so3(wr, Er);
    transpose(Er, ErT);
    mat_mul(E, Rm, ERm);
    mat_mul(ERm, ErT, Rrs);
    double gv[3], EtA[3], EtS1[3], tx[3], inner[3], RmT_in[3];
    mat_tvec(Rrs, S1, gv);
    mat_tvec(E, A, EtA);
    mat_tvec(E, S1, EtS1);
    cross(tm, EtS1, tx);
    for (int i = 0; i < 3; i++) inner[i] = EtA[i] - tx[i];
    mat_tvec(Rm, inner, RmT_in);
    const double mwr[3] = {-wr[0], -wr[1], -wr[2]};
    double Jr[9], gw[3];
    jl_so3(mwr, Jr);
    mat_tvec(Jr, RmT_in, gw);
    for (int i = 0; i < 3; i++) {
        atomicAdd(grad + 6 * ref + i, -gv[i]);
        atomicAdd(grad + 6 * ref + 3 + i, -gw[i]);
    }
}

template <int N, int DIL>
cudaError_t launch_window(const L3dGradDev& d, dim3 grid, const L3dGradPair* pairs, int n,
                          const float* planes, const float* grad_cost, float* cost,
                          float* grad_planes, double* sums, cudaStream_t stream) {
    const int threads = kTileX * kTileY;
    switch (d.storage) {
        case L3D_DTYPE_F32:
            k_ncc_grad<N, DIL, L3D_DTYPE_F32><<<grid, threads, 0, stream>>>(d, pairs, n, planes, grad_cost, cost, grad_planes, sums);
            break;
        case L3D_DTYPE_F16:
            k_ncc_grad<N, DIL, L3D_DTYPE_F16><<<grid, threads, 0, stream>>>(d, pairs, n, planes, grad_cost, cost, grad_planes, sums);
            break;
        case L3D_DTYPE_BF16:
            k_ncc_grad<N, DIL, L3D_DTYPE_BF16><<<grid, threads, 0, stream>>>(d, pairs, n, planes, grad_cost, cost, grad_planes, sums);
            break;
        default:
            k_ncc_grad<N, DIL, L3D_DTYPE_U8><<<grid, threads, 0, stream>>>(d, pairs, n, planes, grad_cost, cost, grad_planes, sums);
            break;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t l3d_launch_ncc_grad(const L3dGradDev& d, const L3dGradView* views_dev,
                                const float* deltas, const L3dGradJob& job, L3dGradPair* pairs_dev,
                                double* pair_sums, const float* planes, const float* grad_cost,
                                float* cost, float* grad_planes, double* grad_deltas,
                                cudaStream_t stream) {
    if (job.n <= 0 || job.n > L3D_MAX_SOURCES) return cudaErrorInvalidValue;
    k_compose<<<1, 32, 0, stream>>>(views_dev, deltas, job, pairs_dev);
    if (grad_deltas) {
        cudaError_t e = cudaMemsetAsync(pair_sums, 0, (size_t)job.n * 6 * sizeof(double), stream);
        if (e != cudaSuccess) return e;
    }
    const dim3 grid((d.W + kTileX - 1) / kTileX, (d.H + kTileY - 1) / kTileY);
    double* sums = grad_deltas ? pair_sums : nullptr;
    cudaError_t e;
    if (d.window == 11)
        e = launch_window<11, 1>(d, grid, pairs_dev, job.n, planes, grad_cost, cost, grad_planes, sums, stream);
    else
        e = launch_window<6, 2>(d, grid, pairs_dev, job.n, planes, grad_cost, cost, grad_planes, sums, stream);
    if (e != cudaSuccess) return e;
    if (grad_deltas) k_finalize<<<1, 32, 0, stream>>>(views_dev, deltas, job, pair_sums, grad_deltas);
    return cudaGetLastError();
}
