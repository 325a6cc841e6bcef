/*
 * PatchMatch multi-view stereo, plain FP32 form (one reference view per launch).
 *
 * Kernels of frontend/src/app/vision/mvs/patchmatch.wgsl.ts rebuilt for sm_100a: init (255-289),
 * init_coarse (296-333), propagate (349-423, one launch per colour), pack (425-433) and
 * consistency (436-469), plus a per-pixel plane-cost probe.  One thread owns one pixel; its
 * reference window (values and bilateral weights) lives in registers for the whole launch and
 * source images are read through the read-only data path (L1/L2), since each pixel's warped
 * footprint follows its own plane.
 *
 * Arithmetic: this form is the bit-exact twin of the FP32 CPU restatement.  The operation
 * order is fixed (explicit fmaf, IEEE division and sqrt, l3d_fmath.h transcendentals) and the
 * file is compiled with --fmad=false so that no other multiply-add is fused:
 *   dot(a, b) = fma(a.z, b.z, fma(a.y, b.y, a.x * b.x)); normalize(v) = v * (1 / sqrt(v.v));
 *   homography H = B_s + kt_s u^T with u = (K_r^-T n) / rho; bilinear samples at texel
 *   coordinates q.xy / q.z with exact weights and clamp-to-edge; window sums in sample order.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "l3d_fmath.h"
#include "l3d_internal.h"

namespace {

__device__ __forceinline__ float dot3f(float3 a, float3 b) {
    return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x));
}
__device__ __forceinline__ float3 normalize3f(float3 v) {
    float il = 1.0f / sqrtf(dot3f(v, v));
    return make_float3(v.x * il, v.y * il, v.z * il);
}
__device__ __forceinline__ float maxw(float a, float b) { return a > b ? a : b; }  /* WGSL max */
__device__ __forceinline__ float minw(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float clampw(float v, float lo, float hi) { return minw(maxw(v, lo), hi); }

/* depth-packing.wgsl.ts:3-19 */
__device__ __forceinline__ float unpack_depth(uint32_t packed) {
    return l3d_f16_to_f32(packed & 0xffffu);
}
__device__ __forceinline__ float3 unpack_normal(uint32_t packed) {
    float ex = ((float)((packed >> 16) & 63u) / 63.0f) * 2.0f - 1.0f;
    float ey = ((float)((packed >> 22) & 63u) / 63.0f) * 2.0f - 1.0f;
    float3 n = make_float3(ex, ey, (1.0f - fabsf(ex)) - fabsf(ey));
    if (n.z < 0.0f) {
        float sx = n.x >= 0.0f ? 1.0f : -1.0f;
        float sy = n.y >= 0.0f ? 1.0f : -1.0f;
        float nx = (1.0f - fabsf(n.y)) * sx;
        float ny = (1.0f - fabsf(n.x)) * sy;
        n.x = nx;
        n.y = ny;
    }
    return normalize3f(n);
}

/* depth-packing.wgsl.ts:21-33 */
__device__ __forceinline__ uint32_t pack_sample(float depth, float3 n, float cost) {
    if (!(depth > 0.0f) || !(cost < 1.0f)) return 0u;
    float s = (fabsf(n.x) + fabsf(n.y)) + fabsf(n.z);
    float ex = n.x / s, ey = n.y / s;
    if (n.z < 0.0f) {
        float sx = ex >= 0.0f ? 1.0f : -1.0f;
        float sy = ey >= 0.0f ? 1.0f : -1.0f;
        float nx = (1.0f - fabsf(ey)) * sx;
        float ny = (1.0f - fabsf(ex)) * sy;
        ex = nx;
        ey = ny;
    }
    float cx = clampw(fmaf(ex, 0.5f, 0.5f), 0.0f, 1.0f);
    float cy = clampw(fmaf(ey, 0.5f, 0.5f), 0.0f, 1.0f);
    uint32_t qx = (uint32_t)fmaf(cx, 63.0f, 0.5f);
    uint32_t qy = (uint32_t)fmaf(cy, 63.0f, 0.5f);
    uint32_t c = min(15u, (uint32_t)(cost * 15.0f));
    uint32_t h = l3d_f32_to_f16(depth);
    return (h & 0xffffu) | (qx << 16) | (qy << 22) | (c << 28);
}

template <int N, int DIL>
struct Win {
    static constexpr int S = N * N;
    static constexpr int HALF = ((N - 1) * DIL) / 2;
    static_assert(((N - 1) * DIL) % 2 == 0, "window must be centred");
    __device__ static constexpr int ox(int i) { return (i % N) * DIL - HALF; }
    __device__ static constexpr int oy(int i) { return (i / N) * DIL - HALF; }
};

/* Private state of one invocation (the var<private> block of patchmatch.wgsl.ts:49-54). */
template <int N, int DIL>
struct Pix {
    float rv[N * N], rw[N * N];
    float rsum, rmean, rvar;
    uint32_t rng;
    float px, py;
    float3 ray;
};

template <int N, int DIL>
struct Stereo {
    using W_ = Win<N, DIL>;
    const L3dParams& p;
    const L3dStereoDev& d;

    __device__ Stereo(const L3dParams& params, const L3dStereoDev& dev) : p(params), d(dev) {}

    __device__ float3 ray_of(float x, float y) const {
        return make_float3((x - p.k[2]) / p.k[0], (y - p.k[3]) / p.k[1], 1.0f);
    }

    __device__ float random(Pix<N, DIL>& s) const { return l3d_random(&s.rng); }

    __device__ float ref_pixel(int x, int y) const {
        x = min(max(x, 0), p.W - 1);
        y = min(max(y, 0), p.H - 1);
        return __ldg(d.images + p.ref_off + (long long)y * p.W + x);
    }

    /* prepare_window (patchmatch.wgsl.ts:90-110) */
    __device__ void prepare_window(Pix<N, DIL>& s, int x, int y) const {
        const float c1 = 2.0f * 0.06f * 0.06f;
        const float c2 = 2.0f * 5.0f * 5.0f;
        float center = ref_pixel(x, y);
        float sw = 0.0f, sr = 0.0f, srr = 0.0f;
#pragma unroll
        for (int i = 0; i < W_::S; i++) {
            const int ox = W_::ox(i), oy = W_::oy(i);
            float v = ref_pixel(x + ox, y + oy);
            float dc = v - center;
            float w = l3d_expf(-(dc * dc) / c1 - (float)(ox * ox + oy * oy) / c2);
            s.rv[i] = v;
            s.rw[i] = w;
            sw = sw + w;
            sr = fmaf(w, v, sr);
            srr = fmaf(w * v, v, srr);
        }
        s.rsum = sw;
        s.rmean = sr / sw;
        s.rvar = maxw(fmaf(-s.rmean, s.rmean, srr / sw), 0.0f);
    }

    __device__ float bilinear(const L3dSrc& src, float u, float v) const {
        float x0 = floorf(u), y0 = floorf(v);
        float fx = u - x0, fy = v - y0;
        int ix0 = (int)x0, iy0 = (int)y0;
        int ix1 = min(ix0 + 1, src.W - 1), iy1 = min(iy0 + 1, src.H - 1);
        const float* img = d.images + src.img_off;
        float a = __ldg(img + (long long)iy0 * src.W + ix0);
        float b = __ldg(img + (long long)iy0 * src.W + ix1);
        float c = __ldg(img + (long long)iy1 * src.W + ix0);
        float e = __ldg(img + (long long)iy1 * src.W + ix1);
        float top = fmaf(fx, b - a, a);
        float bot = fmaf(fx, e - c, c);
        return fmaf(fy, bot - top, top);
    }

    /* view_cost (patchmatch.wgsl.ts:130-159) */
    __device__ float view_cost(const Pix<N, DIL>& s, const L3dSrc& src, const float* u) const {
        float h[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) h[r * 3 + c] = fmaf(src.kt[r], u[c], src.B[r * 3 + c]);
        const float wmax = (float)(src.W - 1), hmax = (float)(src.H - 1);
        float ss = 0.0f, sss = 0.0f, srs = 0.0f;
#pragma unroll
        for (int i = 0; i < W_::S; i++) {
            float x = s.px + (float)W_::ox(i);
            float y = s.py + (float)W_::oy(i);
            float qz = fmaf(h[6], x, fmaf(h[7], y, h[8]));
            if (!(qz > 1e-6f)) return 2.0f;
            float qx = fmaf(h[0], x, fmaf(h[1], y, h[2]));
            float qy = fmaf(h[3], x, fmaf(h[4], y, h[5]));
            float iz = 1.0f / qz;
            float uu = qx * iz, vv = qy * iz;
            if (!(uu >= 0.0f && vv >= 0.0f && uu <= wmax && vv <= hmax)) return 2.0f;
            float val = bilinear(src, uu, vv);
            float w = s.rw[i];
            ss = fmaf(w, val, ss);
            float wv = w * val;
            sss = fmaf(wv, val, sss);
            srs = fmaf(wv, s.rv[i], srs);
        }
        float mean = ss / s.rsum;
        float var_s = maxw(fmaf(-mean, mean, sss / s.rsum), 0.0f);
        float den = sqrtf(s.rvar * var_s);
        if (den < 1e-5f) return 1.0f;
        float cov = fmaf(-s.rmean, mean, srs / s.rsum);
        return clampw(1.0f - cov / den, 0.0f, 2.0f);
    }

    /* reproject (patchmatch.wgsl.ts:166-190); returns false when invalid. */
    __device__ bool reproject(const L3dSrc& v, float px, float py, float3 x, float* dist,
                              float* z) const {
        const float* R = v.R;
        float3 xs = make_float3(fmaf(R[2], x.z, fmaf(R[1], x.y, fmaf(R[0], x.x, v.t[0]))),
                                fmaf(R[5], x.z, fmaf(R[4], x.y, fmaf(R[3], x.x, v.t[1]))),
                                fmaf(R[8], x.z, fmaf(R[7], x.y, fmaf(R[6], x.x, v.t[2]))));
        if (!(xs.z > 1e-6f)) return false;
        float iz = 1.0f / xs.z;
        float rx = rintf(fmaf(v.k[0] * xs.x, iz, v.k[2]));
        float ry = rintf(fmaf(v.k[1] * xs.y, iz, v.k[3]));
        if (!(rx >= 0.0f && ry >= 0.0f && rx < (float)v.W && ry < (float)v.H)) return false;
        int ix = (int)rx, iy = (int)ry;
        uint32_t packed = __ldg(d.depths + v.dep_off + (long long)iy * v.W + ix);
        float ds = unpack_depth(packed);
        if (!(ds > 0.0f) || (packed >> 28) > L3D_FILTER_COST) return false;
        float3 bs = make_float3(((rx - v.k[2]) / v.k[0]) * ds, ((ry - v.k[3]) / v.k[1]) * ds, ds);
        float3 e = make_float3(bs.x - v.t[0], bs.y - v.t[1], bs.z - v.t[2]);
        float3 back = make_float3(fmaf(R[6], e.z, fmaf(R[3], e.y, R[0] * e.x)),
                                  fmaf(R[7], e.z, fmaf(R[4], e.y, R[1] * e.x)),
                                  fmaf(R[8], e.z, fmaf(R[5], e.y, R[2] * e.x)));
        if (!(back.z > 1e-6f)) return false;
        float bz = 1.0f / back.z;
        float qx = fmaf(p.k[0] * back.x, bz, p.k[2]);
        float qy = fmaf(p.k[1] * back.y, bz, p.k[3]);
        float dx = qx - px, dy = qy - py;
        *dist = sqrtf(fmaf(dx, dx, dy * dy));
        *z = back.z;
        return true;
    }

    /* hypothesis_cost (patchmatch.wgsl.ts:192-233) */
    __device__ float hypothesis_cost(const Pix<N, DIL>& s, float3 n, float dd,
                                     float* view_costs = nullptr) const {
        float inv = 1.0f / dd;
        if (!(dd > 0.0f) || inv > p.range[0] || inv < p.range[1]) return 2.0f;
        if (dot3f(n, s.ray) >= -1e-3f) return 2.0f;
        float3 x = make_float3(s.ray.x * dd, s.ray.y * dd, s.ray.z * dd);
        float rho = dot3f(n, x);
        const int count = p.n;
        if (count == 0) return 2.0f;
        float ir = 1.0f / rho;
        float u[3];
        u[0] = (n.x * p.kinv[0]) * ir;
        u[1] = (n.y * p.kinv[1]) * ir;
        u[2] = fmaf(n.x, p.kinv[2], fmaf(n.y, p.kinv[3], n.z)) * ir;
        const bool geometric = (p.flags & 1u) != 0u;
        float costs[L3D_MAX_SOURCES];
        for (int k = 0; k < count; k++) {
            float c = view_cost(s, p.src[k], u);
            if (geometric) {
                float dist, z;
                bool ok = reproject(p.src[k], s.px, s.py, x, &dist, &z);
                float e = ok ? minw(dist, 3.0f) : 3.0f;
                c = fmaf(p.range[3], e, c);
            }
            costs[k] = c;
            if (view_costs) view_costs[k] = c;
        }
        const int kk = max(1, min(3, count - 1));
        float total = 0.0f;
        for (int pick = 0; pick < kk; pick++) {
            int best = pick;
            for (int j = pick + 1; j < count; j++)
                if (costs[j] < costs[best]) best = j;
            float tmp = costs[pick];
            costs[pick] = costs[best];
            costs[best] = tmp;
            total = total + costs[pick];
        }
        return total / (float)kk;
    }

    /* random_normal, random_depth (patchmatch.wgsl.ts:235-249) */
    __device__ float3 random_normal(Pix<N, DIL>& s) const {
        float z = fmaf(random(s), 2.0f, -1.0f);
        float a = random(s) * 6.2831853f;
        float r = sqrtf(maxw(0.0f, fmaf(-z, z, 1.0f)));
        float sn, cs;
        l3d_sincosf(a, &sn, &cs);
        float3 n = make_float3(r * cs, r * sn, z);
        float3 view = normalize3f(s.ray);
        if (dot3f(n, view) > 0.0f) n = make_float3(-n.x, -n.y, -n.z);
        return normalize3f(make_float3(fmaf(view.x, -0.5f, n.x), fmaf(view.y, -0.5f, n.y),
                                       fmaf(view.z, -0.5f, n.z)));
    }
    __device__ float random_depth(Pix<N, DIL>& s) const {
        float t = random(s);
        float m = fmaf(p.range[0], t, p.range[1] * (1.0f - t));
        return 1.0f / m;
    }

    __device__ void begin(Pix<N, DIL>& s, int x, int y) const {
        s.px = (float)x;
        s.py = (float)y;
        /* seed (patchmatch.wgsl.ts:251-253) */
        s.rng = l3d_pcg((uint32_t)(y * p.W + x) ^ l3d_pcg(p.seed + p.iter * 7919u + p.phase * 104729u));
        prepare_window(s, x, y);
        s.ray = ray_of(s.px, s.py);
    }
};

__device__ __forceinline__ void near_offset(int i, int* ox, int* oy) {
    int m = (i + 1) / 2;
    *ox = (i & 1) ? -m : m;
    *oy = -(m + 1);
}
__device__ __forceinline__ void orient(int ox, int oy, int dir, int* rx, int* ry) {
    switch (dir) {
        case 1: *rx = ox; *ry = -oy; break;
        case 2: *rx = oy; *ry = ox; break;
        case 3: *rx = -oy; *ry = ox; break;
        default: *rx = ox; *ry = oy; break;
    }
}

template <int N, int DIL>
__global__ void __launch_bounds__(128) k_init(const L3dParams p, const L3dStereoDev d) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.W || y >= p.H) return;
    Stereo<N, DIL> st(p, d);
    Pix<N, DIL> s;
    st.begin(s, x, y);
    const long long index = (long long)y * p.W + x;
    float3 n = st.random_normal(s);
    float dd = st.random_depth(s);
    if (p.flags & 1u) {
        uint32_t packed = d.depths[p.ref_dep_off + index];
        if (unpack_depth(packed) > 0.0f) {
            dd = unpack_depth(packed);
            n = unpack_normal(packed);
        }
    }
    float c = st.hypothesis_cost(s, n, dd);
    if (!(p.flags & 1u) && d.prior && d.prior[index] > 0.0f) {
        float3 v = normalize3f(s.ray);
        float3 pn = make_float3(-v.x, -v.y, -v.z);
        float pd = d.prior[index];
        float pc = st.hypothesis_cost(s, pn, pd);
        if (pc < c) {
            c = pc;
            n = pn;
            dd = pd;
        }
    }
    d.hyp[index] = make_float4(n.x, n.y, n.z, dd);
    d.cost[index] = c;
}

template <int N, int DIL>
__global__ void __launch_bounds__(128) k_init_coarse(const L3dParams p, const L3dStereoDev d) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.W || y >= p.H) return;
    Stereo<N, DIL> st(p, d);
    Pix<N, DIL> s;
    st.begin(s, x, y);
    const long long index = (long long)y * p.W + x;
    float3 bn = st.random_normal(s);
    float bd = st.random_depth(s);
    float best_cost = st.hypothesis_cost(s, bn, bd);
    float qx = ((s.px + 0.5f) * (float)p.cW) / (float)p.W - 0.5f;
    float qy = ((s.py + 0.5f) * (float)p.cH) / (float)p.H - 0.5f;
    int bx = (int)floorf(qx), by = (int)floorf(qy);
    for (int corner = 0; corner < 4; corner++) {
        int cx = min(max(bx + (corner & 1), 0), p.cW - 1);
        int cy = min(max(by + (corner >> 1), 0), p.cH - 1);
        float4 h = d.coarse[(long long)cy * p.cW + cx];
        if (!(h.w > 0.0f)) continue;
        float3 hn = make_float3(h.x, h.y, h.z);
        float3 point = make_float3(((float)cx - p.ck[2]) / p.ck[0] * h.w,
                                   ((float)cy - p.ck[3]) / p.ck[1] * h.w, h.w);
        float den = dot3f(hn, s.ray);
        if (fabsf(den) < 1e-6f) continue;
        float dd = dot3f(hn, point) / den;
        float c = st.hypothesis_cost(s, hn, dd);
        if (c < best_cost) {
            best_cost = c;
            bn = hn;
            bd = dd;
        }
    }
    d.hyp[index] = make_float4(bn.x, bn.y, bn.z, bd);
    d.cost[index] = best_cost;
}

/* propagate (patchmatch.wgsl.ts:349-423); threads cover the pixels of one colour. */
template <int N, int DIL>
__global__ void __launch_bounds__(128) k_propagate(const L3dParams p, const L3dStereoDev d) {
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = (blockIdx.x * blockDim.x + threadIdx.x) * 2 + (int)((y + p.phase) & 1u);
    if (x >= p.W || y >= p.H) return;
    Stereo<N, DIL> st(p, d);
    Pix<N, DIL> s;
    st.begin(s, x, y);
    const long long index = (long long)y * p.W + x;
    float4 b = d.hyp[index];
    float3 bn = make_float3(b.x, b.y, b.z);
    float bd = b.w;
    float best_cost = d.cost[index];
    for (int region = 0; region < 8; region++) {
        const int count = region < 4 ? 7 : 11;
        long long chosen = -1;
        float chosen_cost = 1e9f;
        for (int i = 0; i < count; i++) {
            int ox = 0, oy = -3 - 2 * i;
            if (region < 4) near_offset(i, &ox, &oy);
            int rx, ry;
            orient(ox, oy, region & 3, &rx, &ry);
            int qx = x + rx, qy = y + ry;
            if (qx < 0 || qy < 0 || qx >= p.W || qy >= p.H) continue;
            long long qi = (long long)qy * p.W + qx;
            float c = d.cost[qi];
            if (c < chosen_cost) {
                chosen_cost = c;
                chosen = qi;
            }
        }
        if (chosen < 0) continue;
        float4 h = d.hyp[chosen];
        float3 hn = make_float3(h.x, h.y, h.z);
        float3 rq = st.ray_of((float)(chosen % p.W), (float)(chosen / p.W));
        float den = dot3f(hn, s.ray);
        if (fabsf(den) < 1e-6f) continue;
        float dd = dot3f(hn, make_float3(rq.x * h.w, rq.y * h.w, rq.z * h.w)) / den;
        float c = st.hypothesis_cost(s, hn, dd);
        if (c < best_cost) {
            best_cost = c;
            bn = hn;
            bd = dd;
        }
    }
    const float step = p.range[2];
    float3 view = normalize3f(s.ray);
    float3 n_random = st.random_normal(s);
    float d_random = st.random_depth(s);
    float e = (fmaf(st.random(s), 2.0f, -1.0f) * 0.15f) * step;
    float d_perturbed = 1.0f / ((1.0f / bd) * (1.0f + e));
    float r1 = st.random(s), r2 = st.random(s), r3 = st.random(s);
    float3 np = make_float3(bn.x + (fmaf(r1, 2.0f, -1.0f) * 0.6f) * step,
                            bn.y + (fmaf(r2, 2.0f, -1.0f) * 0.6f) * step,
                            bn.z + (fmaf(r3, 2.0f, -1.0f) * 0.6f) * step);
    float3 n_perturbed = normalize3f(np);
    if (dot3f(n_perturbed, view) >= 0.0f) n_perturbed = bn;
    const float3 cur_n = bn;
    const float cur_d = bd;
    for (int c = 0; c < 6; c++) {
        /* candidates (n_random, d_random), (n_perturbed, d_perturbed), (current, d_random),
         * (n_random, current), (current, d_perturbed), (n_perturbed, current) */
        float3 nn = (c == 0 || c == 3) ? n_random : ((c == 1 || c == 5) ? n_perturbed : cur_n);
        float dv = (c == 0 || c == 2) ? d_random : ((c == 1 || c == 4) ? d_perturbed : cur_d);
        float cand = st.hypothesis_cost(s, nn, dv);
        if (cand < best_cost) {
            best_cost = cand;
            bn = nn;
            bd = dv;
        }
    }
    d.hyp[index] = make_float4(bn.x, bn.y, bn.z, bd);
    d.cost[index] = best_cost;
}

__global__ void k_pack(const L3dParams p, const L3dStereoDev d) {
    const long long total = (long long)p.W * p.H;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    float4 h = d.hyp[i];
    d.depths[p.ref_dep_off + i] = pack_sample(h.w, make_float3(h.x, h.y, h.z), d.cost[i]);
}

/* consistency (patchmatch.wgsl.ts:436-469) */
__global__ void __launch_bounds__(128) k_consistency(const L3dParams p, const L3dStereoDev d) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.W || y >= p.H) return;
    const long long index = (long long)y * p.W + x;
    Stereo<6, 2> st(p, d);
    uint32_t packed = d.depths[p.ref_dep_off + index];
    float dd = unpack_depth(packed);
    if (!(dd > 0.0f) || (packed >> 28) > L3D_FILTER_COST) {
        d.filtered[index] = 0u;
        return;
    }
    float px = (float)x, py = (float)y;
    float3 r = st.ray_of(px, py);
    float3 X = make_float3(r.x * dd, r.y * dd, r.z * dd);
    uint32_t agree = 0;
    float sum = dd;
    for (int k = 0; k < p.n; k++) {
        float dist, z;
        bool ok = st.reproject(p.src[k], px, py, X, &dist, &z);
        if (ok && dist < 1.0f && fabsf(z - dd) < 0.01f * dd) {
            agree++;
            sum = sum + z;
        }
    }
    uint32_t needed = min((uint32_t)p.n, max(1u, p.needed));
    if (agree < needed) {
        d.filtered[index] = 0u;
        return;
    }
    float mean = sum / (float)(agree + 1u);
    d.filtered[index] = (packed & 0xffff0000u) | (l3d_f32_to_f16(mean) & 0xffffu);
}

template <int N, int DIL>
__global__ void __launch_bounds__(128) k_plane_cost(const L3dParams p, const L3dStereoDev d,
                                                    const float4* planes, float* cost,
                                                    float* view_costs) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.W || y >= p.H) return;
    Stereo<N, DIL> st(p, d);
    Pix<N, DIL> s;
    st.begin(s, x, y);
    const long long index = (long long)y * p.W + x;
    float4 pl = planes[index];
    float vc[L3D_MAX_SOURCES];
    for (int k = 0; k < L3D_MAX_SOURCES; k++) vc[k] = 0.0f;
    cost[index] = st.hypothesis_cost(s, make_float3(pl.x, pl.y, pl.z), pl.w, vc);
    if (view_costs)
        for (int k = 0; k < L3D_MAX_SOURCES; k++) view_costs[index * L3D_MAX_SOURCES + k] = vc[k];
}

template <int N, int DIL>
cudaError_t launch_win(int kernel, const L3dParams& p, const L3dStereoDev& d, cudaStream_t stream) {
    dim3 block(32, 4);
    switch (kernel) {
        case L3D_K_INIT: {
            dim3 grid((p.W + 31) / 32, (p.H + 3) / 4);
            k_init<N, DIL><<<grid, block, 0, stream>>>(p, d);
            break;
        }
        case L3D_K_INIT_COARSE: {
            dim3 grid((p.W + 31) / 32, (p.H + 3) / 4);
            k_init_coarse<N, DIL><<<grid, block, 0, stream>>>(p, d);
            break;
        }
        case L3D_K_PROPAGATE: {
            int half = (p.W + 1) / 2;
            dim3 grid((half + 31) / 32, (p.H + 3) / 4);
            k_propagate<N, DIL><<<grid, block, 0, stream>>>(p, d);
            break;
        }
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t l3d_launch_plain(int kernel, const L3dParams& p, const L3dStereoDev& d, int win,
                             int dil, cudaStream_t stream) {
    if (kernel == L3D_K_PACK) {
        long long total = (long long)p.W * p.H;
        k_pack<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(p, d);
        return cudaGetLastError();
    }
    if (kernel == L3D_K_CONSISTENCY) {
        dim3 block(32, 4), grid((p.W + 31) / 32, (p.H + 3) / 4);
        k_consistency<<<grid, block, 0, stream>>>(p, d);
        return cudaGetLastError();
    }
    if (win == 6 && dil == 2) return launch_win<6, 2>(kernel, p, d, stream);
    if (win == 11 && dil == 1) return launch_win<11, 1>(kernel, p, d, stream);
    return cudaErrorInvalidValue;
}

cudaError_t l3d_launch_plane_cost(const L3dParams& p, const L3dStereoDev& d, const float4* planes,
                                  float* cost, float* view_costs, int win, int dil,
                                  cudaStream_t stream) {
    dim3 block(32, 4), grid((p.W + 31) / 32, (p.H + 3) / 4);
    if (win == 6 && dil == 2)
        k_plane_cost<6, 2><<<grid, block, 0, stream>>>(p, d, planes, cost, view_costs);
    else if (win == 11 && dil == 1)
        k_plane_cost<11, 1><<<grid, block, 0, stream>>>(p, d, planes, cost, view_costs);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

/* ---- image upload conversion ---- */

namespace {
__global__ void k_convert(const uint8_t* src, int dtype, long long stride, int W, int H, void* dst,
                          int storage) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W || y >= H) return;
    const uint8_t* row = src + (long long)y * stride;
    float v;
    switch (dtype) {
        case 0: v = (float)row[x] / 255.0f; break;                              /* r8unorm */
        case 1: v = ((const float*)row)[x]; break;
        case 2: v = l3d_f16_to_f32(((const uint16_t*)row)[x]); break;
        default: v = l3d_u2f((uint32_t)((const uint16_t*)row)[x] << 16); break; /* bf16 */
    }
    long long o = (long long)y * W + x;
    if (storage == 0) {
        /* r8unorm: round to the nearest of 256 levels */
        ((uint8_t*)dst)[o] = (uint8_t)rintf(fminf(fmaxf(v, 0.0f), 1.0f) * 255.0f);
    } else if (storage == 1) {
        ((float*)dst)[o] = v;
    } else if (storage == 2) {
        ((uint16_t*)dst)[o] = (uint16_t)l3d_f32_to_f16(v);
    } else {
        /* bf16, round to nearest even */
        uint32_t u = l3d_f2u(v);
        uint32_t r = ((u >> 16) & 1u) + 0x7fffu;
        ((uint16_t*)dst)[o] = (uint16_t)((u + r) >> 16);
    }
}
}  // namespace

cudaError_t l3d_launch_convert(const void* src, int dtype, int64_t row_stride, int W, int H,
                               void* dst, int storage, cudaStream_t stream) {
    dim3 block(128), grid((W + 127) / 128, H);
    k_convert<<<grid, block, 0, stream>>>((const uint8_t*)src, dtype, row_stride, W, H, dst, storage);
    return cudaGetLastError();
}
