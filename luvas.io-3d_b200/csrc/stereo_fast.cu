/*
 * PatchMatch multi-view stereo, batched forms: every reference view of a batch in one launch
 * per kernel (init, each red/black colour, pack).
 *
 * Same algorithm, RNG stream and candidate schedule as frontend/src/app/vision/mvs/
 * patchmatch.wgsl.ts (init 255-289, propagate 349-423, pack 425-433).  Two evaluators of the
 * multi-view NCC share the kernels:
 *
 * Fast (L3D_FORM_FAST, mixed precision):
 *   - source images are FP16 (or FP32, U8) CUDA arrays read through the texture unit with
 *     hardware bilinear filtering at q.xy / q.z (the same filtered fetch the WGSL's
 *     textureSampleLevel does); BF16 storage is sampled from linear memory with FP32 weights;
 *   - the warped window is convex (q.z is affine and each image bound is a linear inequality in
 *     the reference pixel once multiplied by q.z > 0), so its four corner samples decide whether
 *     any of the 36 samples leaves the image: one test replaces 36 per-sample bounds checks and
 *     the sample loop runs branch-free with incremental homogeneous coordinates;
 *   - the NCC sums are accumulated in FP32 on values shifted by the reference window's centre
 *     pixel (the shifted-data form of the weighted variance, which removes the cancellation of
 *     E[x^2] - E[x]^2), with the reference terms w and w (r - c) precomputed per pixel;
 *     optionally compensated: FP32 row partials added with Neumaier compensation;
 *   - the k-best view mean keeps the three smallest costs in registers (same sum order as the
 *     reference's partial selection sort).
 *
 * Exact (L3D_FORM_EXACT): the plain form's arithmetic, operation for operation (per-sample
 * homogeneous coordinates, IEEE reciprocal, exact bilinear weights, raw-value sums, l3d_fmath.h
 * transcendentals), so a batched solve equals the plain per-view solve and the FP32 oracle bit
 * for bit.  Samples come from FP32 CUDA arrays through texture gathers: the four texels of a
 * bilinear footprint are fetched by one tld4 at the footprint's centre (integer coordinates
 * chosen in software, so the hardware's coordinate rounding cannot move the footprint) and
 * weighted in FP32 exactly as the oracle does.  With compensation on, every window sum is a
 * Neumaier sum (the oracle's compensated mode restates the same operations).
 *
 * Blocks are tiles of 16 x 8 pixels of one colour of one view; a block loads its view's
 * parameters (homography bases composed in FP64 on the host) into shared memory.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include <cuda_fp16.h>

#include "l3d_fmath.h"
#include "l3d_internal.h"

namespace {

constexpr int TX = 16;   /* colour columns per tile */
constexpr int TY = 8;    /* rows per tile */
constexpr int S = 36;    /* 6 x 6 window, offsets -5, -3, ..., 5 */
#ifndef L3D_EXACT_MIN_BLOCKS
#define L3D_EXACT_MIN_BLOCKS 5 /* resident blocks per SM of the exact propagate kernel (5: 81 M px-iters/s on the scan, 4: 72 M) */
#endif
/* Resident blocks per SM of the fast propagate kernel with the window in shared memory, with
 * gathers (4: 168.9 M px-iters/s on the scan with FP32 texels, 5: 166.8 M) and with filtered
 * samples (5: 249.7 M with FP16 texels, 4: 248.0 M). */
#ifndef L3D_SHWIN_GATHER_MIN_BLOCKS
#define L3D_SHWIN_GATHER_MIN_BLOCKS 4
#endif
#ifndef L3D_SHWIN_MIN_BLOCKS
#define L3D_SHWIN_MIN_BLOCKS 5
#endif

__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float dot3f(float3 a, float3 b) {
    return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x));
}
__device__ __forceinline__ float3 normalize_fast(float3 v) {
    float il = rsqrtf(dot3f(v, v));
    return make_float3(v.x * il, v.y * il, v.z * il);
}
/* normalize with an IEEE square root and reciprocal (the plain form's and oracle's order) */
__device__ __forceinline__ float3 normalize_ieee(float3 v) {
    float il = 1.0f / sqrtf(dot3f(v, v));
    return make_float3(v.x * il, v.y * il, v.z * il);
}
__device__ __forceinline__ float maxw(float a, float b) { return a > b ? a : b; }  /* WGSL max */
__device__ __forceinline__ float minw(float a, float b) { return a < b ? a : b; }

/* A running FP32 sum, plain (COMP = false: s += x, s = fma(a, b, s)) or Neumaier-compensated
 * (COMP = true): every addend, products rounded to FP32 first, goes through
 *   t = s + x;  c += |s| >= |x| ? (s - t) + x : (x - t) + s;  s = t,
 * and the sum is s + c.  The error of the compensated sum is bounded by about 2 ulp of the sum
 * of magnitudes independently of the number of terms (Neumaier 1974); the plain sum's bound
 * grows with the 36 terms of a window. */
template <bool COMP>
struct Acc {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add(float x) {
        if (COMP) {
            const float t = s + x;
            const bool big = fabsf(s) >= fabsf(x);
            const float hi = big ? s : x, lo = big ? x : s;
            c = c + ((hi - t) + lo);
            s = t;
        } else {
            s = s + x;
        }
    }
    /* s + a * b: one fused multiply-add, or the rounded product added with compensation */
    __device__ __forceinline__ void fma_add(float a, float b) {
        if (COMP) add(a * b);
        else s = fmaf(a, b, s);
    }
    __device__ __forceinline__ float value() const { return COMP ? s + c : s; }
};

/* The three source-window sums of the fast evaluator (sum w s', sum w s'^2, sum w r' s' over
 * shifted values).  Plain (COMP = false): sequential FP32 sums in sample order.  Compensated:
 * each 6-sample window row is summed in FP32 (a row partial), and the row partials are added
 * with Neumaier compensation; the rounding error is then bounded by about 7 ulp of the sum of
 * magnitudes instead of 35 for the sequential sum, at 7 extra operations per row and sum
 * instead of per sample (the fast propagate kernel is bound by the texture pipe, not by issue,
 * so the row-level compensation costs it next to nothing; per-sample compensation did). */
template <bool COMP>
struct WinSums {
    Acc<COMP> ss, sss, srs;
    float rs = 0.0f, rss = 0.0f, rrs = 0.0f;
    __device__ __forceinline__ void term(float t, float sv, float rwr) {
        if (COMP) {
            rs = rs + t;
            rss = fmaf(t, sv, rss);
            rrs = fmaf(rwr, sv, rrs);
        } else {
            ss.s = ss.s + t;
            sss.s = fmaf(t, sv, sss.s);
            srs.s = fmaf(rwr, sv, srs.s);
        }
    }
    __device__ __forceinline__ void end_row() {
        if (COMP) {
            ss.add(rs);
            sss.add(rss);
            srs.add(rrs);
            rs = rss = rrs = 0.0f;
        }
    }
};

__device__ __forceinline__ float unpack_depth(uint32_t packed) {
    return l3d_f16_to_f32(packed & 0xffffu);
}
/* unpack_normal of depth-packing.wgsl.ts:3-19 in the plain form's operation order */
__device__ __forceinline__ float3 unpack_normal_ieee(uint32_t packed) {
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
    return normalize_ieee(n);
}
__device__ __forceinline__ float3 unpack_normal(uint32_t packed) {
    float ex = (float)((packed >> 16) & 63u) * (2.0f / 63.0f) - 1.0f;
    float ey = (float)((packed >> 22) & 63u) * (2.0f / 63.0f) - 1.0f;
    float3 n = make_float3(ex, ey, (1.0f - fabsf(ex)) - fabsf(ey));
    if (n.z < 0.0f) {
        float nx = (1.0f - fabsf(n.y)) * (n.x >= 0.0f ? 1.0f : -1.0f);
        float ny = (1.0f - fabsf(n.x)) * (n.y >= 0.0f ? 1.0f : -1.0f);
        n.x = nx;
        n.y = ny;
    }
    return normalize_fast(n);
}
__device__ __forceinline__ uint32_t pack_sample(float depth, float3 n, float cost) {
    if (!(depth > 0.0f) || !(cost < 1.0f)) return 0u;
    float s = (fabsf(n.x) + fabsf(n.y)) + fabsf(n.z);
    float ex = n.x / s, ey = n.y / s;
    if (n.z < 0.0f) {
        float nx = (1.0f - fabsf(ey)) * (ex >= 0.0f ? 1.0f : -1.0f);
        float ny = (1.0f - fabsf(ex)) * (ey >= 0.0f ? 1.0f : -1.0f);
        ex = nx;
        ey = ny;
    }
    float cx = fminf(fmaxf(fmaf(ex, 0.5f, 0.5f), 0.0f), 1.0f);
    float cy = fminf(fmaxf(fmaf(ey, 0.5f, 0.5f), 0.0f), 1.0f);
    uint32_t qx = (uint32_t)fmaf(cx, 63.0f, 0.5f);
    uint32_t qy = (uint32_t)fmaf(cy, 63.0f, 0.5f);
    uint32_t c = min(15u, (uint32_t)(cost * 15.0f));
    return (l3d_f32_to_f16(depth) & 0xffffu) | (qx << 16) | (qy << 22) | (c << 28);
}

/* The four texels of the bilinear footprint whose top-left texel is (x0, y0), from a texture
 * gather (tld4) at the footprint's centre: in unnormalised coordinates the centre of texel i is
 * i + 0.5, so coordinate x0 + 1 lies exactly between texels x0 and x0 + 1 and the footprint
 * cannot shift with the texture unit's coordinate rounding.  Clamp addressing repeats the last
 * row and column like the oracle's min(i + 1, size - 1).  The gather returns the footprint as
 * (x0, y0+1), (x0+1, y0+1), (x0+1, y0), (x0, y0) in x, y, z, w. */
__device__ __forceinline__ float bilinear_gather(unsigned long long tex, float u, float v) {
    const float x0 = floorf(u), y0 = floorf(v);
    const float fx = u - x0, fy = v - y0;
    const float4 g = tex2Dgather<float4>((cudaTextureObject_t)tex, x0 + 1.0f, y0 + 1.0f, 0);
    const float a = g.w, b = g.z, c = g.x, e = g.y;
    const float top = fmaf(fx, b - a, a);
    const float bot = fmaf(fx, e - c, c);
    return fmaf(fy, bot - top, top);
}

/* Image access: texture path (F16/F32 CUDA arrays, hardware bilinear) or BF16 linear memory. */
template <bool TEX>
struct Img {
    /* value at filtering coordinate (u, v) = texel coordinate + 0.5 */
    static __device__ __forceinline__ float sample(unsigned long long tex, const uint16_t* img,
                                                   int W, int H, float u, float v) {
        if (TEX) {
            return tex2D<float>((cudaTextureObject_t)tex, u, v);
        } else {
            float x = u - 0.5f, y = v - 0.5f;
            float x0 = floorf(x), y0 = floorf(y);
            float fx = x - x0, fy = y - y0;
            int ix0 = min(max((int)x0, 0), W - 1), iy0 = min(max((int)y0, 0), H - 1);
            int ix1 = min(ix0 + 1, W - 1), iy1 = min(iy0 + 1, H - 1);
            const uint16_t* r0 = img + (long long)iy0 * W;
            const uint16_t* r1 = img + (long long)iy1 * W;
            float a = __uint_as_float((uint32_t)__ldg(r0 + ix0) << 16);
            float b = __uint_as_float((uint32_t)__ldg(r0 + ix1) << 16);
            float c = __uint_as_float((uint32_t)__ldg(r1 + ix0) << 16);
            float e = __uint_as_float((uint32_t)__ldg(r1 + ix1) << 16);
            float top = fmaf(fx, b - a, a);
            float bot = fmaf(fx, e - c, c);
            return fmaf(fy, bot - top, top);
        }
    }
    static __device__ __forceinline__ float texel(unsigned long long tex, const uint16_t* img,
                                                  int W, int H, int x, int y) {
        if (TEX) {
            return tex2D<float>((cudaTextureObject_t)tex, (float)x + 0.5f, (float)y + 0.5f);
        } else {
            x = min(max(x, 0), W - 1);
            y = min(max(y, 0), H - 1);
            return __uint_as_float((uint32_t)__ldg(img + (long long)y * W + x) << 16);
        }
    }
};

/* Software bilinear sample from the pair image (each texel stores itself and its right
 * neighbour as half2), at filtering coordinate (u, v): two 32-bit loads on the LSU path, FP32
 * weights.  Used for the window rows the texture unit does not take. */
__device__ __forceinline__ float pair_sample(const uint32_t* __restrict__ pairs, int W, int H,
                                             float u, float v) {
    float x = u - 0.5f, y = v - 0.5f;
    int x0 = __float2int_rd(x), y0 = __float2int_rd(y);
    float fx = x - (float)x0, fy = y - (float)y0;
    x0 = min(max(x0, 0), W - 1);
    y0 = min(max(y0, 0), H - 1);
    int y1 = min(y0 + 1, H - 1);
    uint32_t t = __ldg(pairs + (long long)y0 * W + x0);
    uint32_t b = __ldg(pairs + (long long)y1 * W + x0);
    float2 tf = __half22float2(*reinterpret_cast<const __half2*>(&t));
    float2 bf = __half22float2(*reinterpret_cast<const __half2*>(&b));
    float top = fmaf(fx, tf.y - tf.x, tf.x);
    float bot = fmaf(fx, bf.y - bf.x, bf.x);
    return fmaf(fy, bot - top, top);
}

/* reproject (patchmatch.wgsl.ts:166-190): the reference point x seen from source sv, rounded to
 * a source pixel, back-projected with that pixel's packed depth; false when any step fails.
 * Operation order of the plain form. */
__device__ __forceinline__ bool reproject(const L3dFastView& v, const L3dFastDev& d,
                                          const L3dFastSrc& sv, float px, float py, float3 x,
                                          float* dist, float* z) {
    const float* R = sv.R;
    float3 xs = make_float3(fmaf(R[2], x.z, fmaf(R[1], x.y, fmaf(R[0], x.x, sv.t[0]))),
                            fmaf(R[5], x.z, fmaf(R[4], x.y, fmaf(R[3], x.x, sv.t[1]))),
                            fmaf(R[8], x.z, fmaf(R[7], x.y, fmaf(R[6], x.x, sv.t[2]))));
    if (!(xs.z > 1e-6f)) return false;
    float iz = 1.0f / xs.z;
    float rx = rintf(fmaf(sv.k[0] * xs.x, iz, sv.k[2]));
    float ry = rintf(fmaf(sv.k[1] * xs.y, iz, sv.k[3]));
    if (!(rx >= 0.0f && ry >= 0.0f && rx < (float)sv.W && ry < (float)sv.H)) return false;
    uint32_t packed = __ldg(d.depths + sv.dep_off + (long long)(int)ry * sv.W + (int)rx);
    float ds = unpack_depth(packed);
    if (!(ds > 0.0f) || (packed >> 28) > L3D_FILTER_COST) return false;
    float3 e = make_float3(((rx - sv.k[2]) / sv.k[0]) * ds - sv.t[0],
                           ((ry - sv.k[3]) / sv.k[1]) * ds - sv.t[1], ds - sv.t[2]);
    float3 back = make_float3(fmaf(R[6], e.z, fmaf(R[3], e.y, R[0] * e.x)),
                              fmaf(R[7], e.z, fmaf(R[4], e.y, R[1] * e.x)),
                              fmaf(R[8], e.z, fmaf(R[5], e.y, R[2] * e.x)));
    if (!(back.z > 1e-6f)) return false;
    float bz = 1.0f / back.z;
    float dx = fmaf(v.k[0] * back.x, bz, v.k[2]) - px;
    float dy = fmaf(v.k[1] * back.y, bz, v.k[3]) - py;
    *dist = sqrtf(fmaf(dx, dx, dy * dy));
    *z = back.z;
    return true;
}

/* hypothesis_cost (patchmatch.wgsl.ts:192-233) over evaluator E's view_cost: range and
 * orientation tests, u = (K_r^-T n) / rho, per-source cost (+ geometric term), mean of the
 * k = max(1, min(3, S - 1)) smallest.  The three smallest are kept in registers, ascending; the
 * reference's partial selection sort adds the same values in the same order. */
template <class E>
__device__ __forceinline__ float hyp_cost(const E& e, const L3dFastView& v, const L3dFastDev& d,
                                          const typename E::Pix& s, float3 n, float dd) {
    if (!(dd > 0.0f)) return 2.0f;
    float inv = 1.0f / dd;
    if (inv > v.range[0] || inv < v.range[1]) return 2.0f;
    if (dot3f(n, s.ray) >= -1e-3f) return 2.0f;
    const int count = v.n;
    if (count == 0) return 2.0f;
    float3 x = make_float3(s.ray.x * dd, s.ray.y * dd, dd);
    float ir = 1.0f / dot3f(n, x);
    float u[3];
    u[0] = (n.x * v.kinv[0]) * ir;
    u[1] = (n.y * v.kinv[1]) * ir;
    u[2] = fmaf(n.x, v.kinv[2], fmaf(n.y, v.kinv[3], n.z)) * ir;
    const bool geometric = (v.flags & 1u) != 0u;
    float b0 = 3.0e38f, b1 = 3.0e38f, b2 = 3.0e38f;
    for (int k = 0; k < count; k++) {
        float c = e.view_cost(s, v.src[k], u);
        if (geometric) {
            float dist, z;
            bool ok = reproject(v, d, v.src[k], s.px, s.py, x, &dist, &z);
            c = fmaf(v.range[3], ok ? minw(dist, 3.0f) : 3.0f, c);
        }
        if (c < b2) {
            if (c < b1) {
                b2 = b1;
                if (c < b0) {
                    b1 = b0;
                    b0 = c;
                } else {
                    b1 = c;
                }
            } else {
                b2 = c;
            }
        }
    }
    const int kk = max(1, min(3, count - 1));
    float total = b0;
    if (kk > 1) total = total + b1;
    if (kk > 2) total = total + b2;
    return total / (float)kk;
}

/* This thread's window column in shared memory: element i (sample i's pair of window values)
 * at [i * XBLOCK]; consecutive threads read consecutive float2, so a warp's access is
 * conflict-free.  The exact evaluator keeps (w, r) there, the fast evaluator with a shared
 * window (w, w (r - c)). */
constexpr int XBLOCK = 128;
__device__ __forceinline__ float2* exact_window() {
    __shared__ float2 win[S * XBLOCK];
    return win + threadIdx.x;
}

/* Per-pixel state: the reference window as w and w (r - c), c = centre pixel. */
struct FPix {
    float rw[S], rwr[S];
    float center, inv_sum, mean_r, var_r;
    uint32_t rng;
    float px, py;
    float3 ray;
};

/* The same without the window, which lives in shared memory (exact_window). */
struct FPixS {
    float center, inv_sum, mean_r, var_r;
    uint32_t rng;
    float px, py;
    float3 ray;
};

/* TEX: texture-unit sampling of F16/F32 arrays (false: BF16 linear memory).  TEXROWS: window
 * rows (of 6) sampled by the texture unit; the other rows use pair_sample (TEX only).  COMP:
 * compensated window sums.  GATHER: the texture rows are texture gathers weighted with exact
 * FP32 bilinear weights instead of hardware-filtered fetches (8-bit weights).  SHWIN: the
 * reference window lives in shared memory instead of 72 registers, so that more warps are
 * resident to cover the texture latency; the arithmetic, and so every result, is unchanged. */
template <bool TEX, int TEXROWS = 6, bool COMP = false, bool GATHER = false, bool SHWIN = false>
struct Fast {
    using Pix = typename std::conditional<SHWIN, FPixS, FPix>::type;
    /* resident blocks per SM the propagate kernel targets */
    static constexpr int kMinBlocks =
        SHWIN ? (GATHER ? L3D_SHWIN_GATHER_MIN_BLOCKS : L3D_SHWIN_MIN_BLOCKS) : 3;
    const L3dFastView& v;
    const L3dFastDev& d;
    __device__ Fast(const L3dFastView& view, const L3dFastDev& dev) : v(view), d(dev) {}

    static __device__ __forceinline__ float3 normalize(float3 a) { return normalize_fast(a); }
    static __device__ __forceinline__ float3 unpack_n(uint32_t packed) { return unpack_normal(packed); }

    __device__ const uint16_t* img(long long off) const {
        return (const uint16_t*)d.images + off;
    }

    __device__ float3 ray_of(float x, float y) const {
        return make_float3((x - v.k[2]) / v.k[0], (y - v.k[3]) / v.k[1], 1.0f);
    }

    __device__ float random(Pix& s) const { return l3d_random(&s.rng); }

    /* prepare_window (patchmatch.wgsl.ts:90-110), shifted by the centre pixel */
    __device__ void prepare(Pix& s, int x, int y) const {
        const uint16_t* ri = img(v.ref_img_off);
        const float center = Img<TEX>::texel(v.ref_tex, ri, v.W, v.H, x, y);
        const float ic1 = 1.0f / (2.0f * 0.06f * 0.06f);
        Acc<COMP> sw, sr, srr;
#pragma unroll
        for (int i = 0; i < S; i++) {
            const int ox = (i % 6) * 2 - 5, oy = (i / 6) * 2 - 5;
            const float spatial = (float)(ox * ox + oy * oy) / (2.0f * 5.0f * 5.0f);
            float val = Img<TEX>::texel(v.ref_tex, ri, v.W, v.H, x + ox, y + oy);
            float dc = val - center;
            float w = __expf(-(dc * dc) * ic1 - spatial);
            if constexpr (SHWIN) {
                exact_window()[i * XBLOCK] = make_float2(w, w * dc);
            } else {
                s.rw[i] = w;
                s.rwr[i] = w * dc;
            }
            sw.add(w);
            sr.fma_add(w, dc);
            srr.fma_add(w * dc, dc);
        }
        s.center = center;
        s.inv_sum = 1.0f / sw.value();
        s.mean_r = sr.value() * s.inv_sum;
        s.var_r = fmaxf(fmaf(-s.mean_r, s.mean_r, srr.value() * s.inv_sum), 0.0f);
    }

    /* one sample's terms of the window sums: w s', s' and (w r') s' (s' = s - c, r' = r - c) */
    static __device__ __forceinline__ void window_term(WinSums<COMP>& ws, const Pix& s, int i, float sv) {
        if constexpr (SHWIN) {
            const float2 w = exact_window()[i * XBLOCK];
            ws.term(w.x * sv, sv, w.y);
        } else {
            ws.term(s.rw[i] * sv, sv, s.rwr[i]);
        }
    }

    /* view_cost (patchmatch.wgsl.ts:130-159) with H = Bt + ktt u^T. */
    __device__ float view_cost(const Pix& s, const L3dFastSrc& src, const float* u) const {
        float h[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) h[r * 3 + c] = fmaf(src.ktt[r], u[c], src.Bt[r * 3 + c]);
        const float x0 = s.px - 5.0f, y0 = s.py - 5.0f;
        /* q at the window's top-left sample and its steps along x and y (2 pixels) */
        const float qx0 = fmaf(h[0], x0, fmaf(h[1], y0, h[2]));
        const float qy0 = fmaf(h[3], x0, fmaf(h[4], y0, h[5]));
        const float qz0 = fmaf(h[6], x0, fmaf(h[7], y0, h[8]));
        const float dxx = 2.0f * h[0], dxy = 2.0f * h[3], dxz = 2.0f * h[6];
        const float dyx = 2.0f * h[1], dyy = 2.0f * h[4], dyz = 2.0f * h[7];
        /* the four corner samples decide validity for the whole (convex) window */
        const float umax = (float)src.W - 0.5f, vmax = (float)src.H - 0.5f;
        bool ok = true;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float fx = (c & 1) ? 5.0f : 0.0f, fy = (c & 2) ? 5.0f : 0.0f;
            float qz = fmaf(dyz, fy, fmaf(dxz, fx, qz0));
            float qx = fmaf(dyx, fy, fmaf(dxx, fx, qx0));
            float qy = fmaf(dyy, fy, fmaf(dxy, fx, qy0));
            ok = ok && qz > 1e-6f && qx >= 0.5f * qz && qy >= 0.5f * qz && qx <= umax * qz &&
                 qy <= vmax * qz;
        }
        if (!ok) return 2.0f;
        const uint16_t* si = img(src.img_off);
        WinSums<COMP> ws;
        /* rows [0, TEXROWS) through the texture unit, rows [TEXROWS, 6) through pair_sample: two
         * loops with constant bounds, so each unrolls into straight-line code with all its
         * fetches in flight together */
        constexpr int RT = TEX ? TEXROWS : 6;
        float rx = qx0, ry = qy0, rz = qz0;
#pragma unroll
        for (int r = 0; r < RT; r++) {
            float qx = rx, qy = ry, qz = rz;
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const int i = r * 6 + c;
                float iz = rcp_fast(qz);
                float val = GATHER ? bilinear_gather(src.tex, fmaf(qx, iz, -0.5f), fmaf(qy, iz, -0.5f))
                                   : Img<TEX>::sample(src.tex, si, src.W, src.H, qx * iz, qy * iz);
                float sv = val - s.center;  /* s' = s - c; r' = r - c lives in rwr / rw */
                window_term(ws, s, i, sv);
                qx += dxx;
                qy += dxy;
                qz += dxz;
            }
            ws.end_row();
            rx += dyx;
            ry += dyy;
            rz += dyz;
        }
        if constexpr (TEX && TEXROWS < 6) {
            const uint32_t* sp = d.pairs + src.img_off;
#pragma unroll
            for (int r = TEXROWS; r < 6; r++) {
                float qx = rx, qy = ry, qz = rz;
#pragma unroll
                for (int c = 0; c < 6; c++) {
                    const int i = r * 6 + c;
                    float iz = rcp_fast(qz);
                    float val = pair_sample(sp, src.W, src.H, qx * iz, qy * iz);
                    float sv = val - s.center;
                    window_term(ws, s, i, sv);
                    qx += dxx;
                    qy += dxy;
                    qz += dxz;
                }
                ws.end_row();
                rx += dyx;
                ry += dyy;
                rz += dyz;
            }
        }
        float mean = ws.ss.value() * s.inv_sum;
        float var_s = fmaxf(fmaf(-mean, mean, ws.sss.value() * s.inv_sum), 0.0f);
        float prod = s.var_r * var_s;
        if (prod < 1e-10f) return 1.0f;  /* sqrt(prod) < 1e-5 */
        float cov = fmaf(-s.mean_r, mean, ws.srs.value() * s.inv_sum);
        return fminf(fmaxf(1.0f - cov * rsqrtf(prod), 0.0f), 2.0f);
    }

    /* hypothesis_cost (patchmatch.wgsl.ts:192-233) */
    __device__ float hypothesis_cost(const Pix& s, float3 n, float dd) const {
        return hyp_cost(*this, v, d, s, n, dd);
    }

    /* random_normal, random_depth (patchmatch.wgsl.ts:235-249) */
    __device__ float3 random_normal(Pix& s) const {
        float z = fmaf(random(s), 2.0f, -1.0f);
        float a = random(s) * 6.2831853f;
        float r = sqrtf(fmaxf(0.0f, fmaf(-z, z, 1.0f)));
        float sn, cs;
        __sincosf(a, &sn, &cs);
        float3 n = make_float3(r * cs, r * sn, z);
        float3 view = normalize_fast(s.ray);
        if (dot3f(n, view) > 0.0f) n = make_float3(-n.x, -n.y, -n.z);
        return normalize_fast(make_float3(fmaf(view.x, -0.5f, n.x), fmaf(view.y, -0.5f, n.y),
                                          fmaf(view.z, -0.5f, n.z)));
    }
    __device__ float random_depth(Pix& s) const {
        float t = random(s);
        return 1.0f / fmaf(v.range[0], t, v.range[1] * (1.0f - t));
    }

    __device__ void begin(Pix& s, int x, int y, int iteration, int phase) const {
        s.px = (float)x;
        s.py = (float)y;
        uint32_t seed = (uint32_t)(v.ref + 1) * 0x9e3779b1u + (uint32_t)iteration * 97u +
                        (uint32_t)phase * 13u + (v.flags & 1u) * 7u;
        s.rng = l3d_pcg((uint32_t)(y * v.W + x) ^
                        l3d_pcg(seed + (uint32_t)iteration * 7919u + (uint32_t)phase * 104729u));
        prepare(s, x, y);
        s.ray = ray_of(s.px, s.py);
    }
};

/* Per-pixel state of the exact evaluator: the private block of patchmatch.wgsl.ts:49-54.  The
 * window's bilateral weights and values (w, v) live in shared memory, one column of S float2 per
 * thread (exact_window), so that the registers they would take go to more resident warps and
 * more gathers in flight; the weighted sum, mean and variance stay in registers. */
struct XPix {
    float rsum, rmean, rvar;
    uint32_t rng;
    float px, py;
    float3 ray;
};

/* The plain form's arithmetic in the batched kernels (see the file header).  COMP: Neumaier-
 * compensated window sums (the oracle's compensated mode). */
template <bool COMP>
struct Exact {
    using Pix = XPix;
    static constexpr int kMinBlocks = L3D_EXACT_MIN_BLOCKS;
    const L3dFastView& v;
    const L3dFastDev& d;
    __device__ Exact(const L3dFastView& view, const L3dFastDev& dev) : v(view), d(dev) {}

    static __device__ __forceinline__ float3 normalize(float3 a) { return normalize_ieee(a); }
    static __device__ __forceinline__ float3 unpack_n(uint32_t packed) { return unpack_normal_ieee(packed); }

    __device__ float3 ray_of(float x, float y) const {
        return make_float3((x - v.k[2]) / v.k[0], (y - v.k[3]) / v.k[1], 1.0f);
    }

    __device__ float random(XPix& s) const { return l3d_random(&s.rng); }

    __device__ float ref_pixel(int x, int y) const {
        x = min(max(x, 0), v.W - 1);
        y = min(max(y, 0), v.H - 1);
        return __ldg((const float*)d.images + v.ref_img_off + (long long)y * v.W + x);
    }

    /* prepare_window (patchmatch.wgsl.ts:90-110) */
    __device__ void prepare(XPix& s, int x, int y) const {
        const float c1 = 2.0f * 0.06f * 0.06f;
        const float c2 = 2.0f * 5.0f * 5.0f;
        const float center = ref_pixel(x, y);
        Acc<COMP> sw, sr, srr;
#pragma unroll
        for (int i = 0; i < S; i++) {
            const int ox = (i % 6) * 2 - 5, oy = (i / 6) * 2 - 5;
            float val = ref_pixel(x + ox, y + oy);
            float dc = val - center;
            float w = l3d_expf(-(dc * dc) / c1 - (float)(ox * ox + oy * oy) / c2);
            exact_window()[i * XBLOCK] = make_float2(w, val);
            sw.add(w);
            sr.fma_add(w, val);
            srr.fma_add(w * val, val);
        }
        s.rsum = sw.value();
        s.rmean = sr.value() / s.rsum;
        s.rvar = maxw(fmaf(-s.rmean, s.rmean, srr.value() / s.rsum), 0.0f);
    }

    /* view_cost (patchmatch.wgsl.ts:130-159) with H = B + kt u^T (Bt/ktt hold the unshifted
     * base in this form).  Every sample is computed as the oracle computes it; a sample with
     * q.z <= 1e-6 or outside [0, W-1] x [0, H-1] makes the cost 2.  The four corner samples are
     * tested first (with the same arithmetic), so most windows that leave the image stop there;
     * the per-sample test in the loop keeps the result exact for windows that graze an edge. */
    __device__ float view_cost(const XPix& s, const L3dFastSrc& src, const float* u) const {
        float h[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) h[r * 3 + c] = fmaf(src.ktt[r], u[c], src.Bt[r * 3 + c]);
        const float wmax = (float)(src.W - 1), hmax = (float)(src.H - 1);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float x = s.px + ((c & 1) ? 5.0f : -5.0f);
            const float y = s.py + ((c & 2) ? 5.0f : -5.0f);
            const float qz = fmaf(h[6], x, fmaf(h[7], y, h[8]));
            const float qx = fmaf(h[0], x, fmaf(h[1], y, h[2]));
            const float qy = fmaf(h[3], x, fmaf(h[4], y, h[5]));
            const float iz = 1.0f / qz;
            const float uu = qx * iz, vv = qy * iz;
            if (!(qz > 1e-6f) || !(uu >= 0.0f && vv >= 0.0f && uu <= wmax && vv <= hmax)) return 2.0f;
        }
        Acc<COMP> ss, sss, srs;
        const float2* win = exact_window();
        bool ok = true;
#pragma unroll
        for (int r = 0; r < 6; r++) {
            const float y = s.py + (float)(r * 2 - 5);
            const float hz = fmaf(h[7], y, h[8]);
            const float hx = fmaf(h[1], y, h[2]);
            const float hy = fmaf(h[4], y, h[5]);
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const int i = r * 6 + c;
                const float x = s.px + (float)(c * 2 - 5);
                const float qz = fmaf(h[6], x, hz);
                const float qx = fmaf(h[0], x, hx);
                const float qy = fmaf(h[3], x, hy);
                const float iz = 1.0f / qz;
                const float uu = qx * iz, vv = qy * iz;
                ok = ok && qz > 1e-6f && uu >= 0.0f && vv >= 0.0f && uu <= wmax && vv <= hmax;
                const float val = bilinear_gather(src.tex, uu, vv);
                const float2 rwv = win[i * XBLOCK];
                const float w = rwv.x;
                ss.fma_add(w, val);
                const float wv = w * val;
                sss.fma_add(wv, val);
                srs.fma_add(wv, rwv.y);
            }
        }
        if (!ok) return 2.0f;
        const float mean = ss.value() / s.rsum;
        const float var_s = maxw(fmaf(-mean, mean, sss.value() / s.rsum), 0.0f);
        const float den = sqrtf(s.rvar * var_s);
        if (den < 1e-5f) return 1.0f;
        const float cov = fmaf(-s.rmean, mean, srs.value() / s.rsum);
        return minw(maxw(1.0f - cov / den, 0.0f), 2.0f);
    }

    /* hypothesis_cost (patchmatch.wgsl.ts:192-233) */
    __device__ float hypothesis_cost(const XPix& s, float3 n, float dd) const {
        return hyp_cost(*this, v, d, s, n, dd);
    }

    /* random_normal, random_depth (patchmatch.wgsl.ts:235-249) */
    __device__ float3 random_normal(XPix& s) const {
        float z = fmaf(random(s), 2.0f, -1.0f);
        float a = random(s) * 6.2831853f;
        float r = sqrtf(maxw(0.0f, fmaf(-z, z, 1.0f)));
        float sn, cs;
        l3d_sincosf(a, &sn, &cs);
        float3 n = make_float3(r * cs, r * sn, z);
        float3 view = normalize_ieee(s.ray);
        if (dot3f(n, view) > 0.0f) n = make_float3(-n.x, -n.y, -n.z);
        return normalize_ieee(make_float3(fmaf(view.x, -0.5f, n.x), fmaf(view.y, -0.5f, n.y),
                                          fmaf(view.z, -0.5f, n.z)));
    }
    __device__ float random_depth(XPix& s) const {
        float t = random(s);
        return 1.0f / fmaf(v.range[0], t, v.range[1] * (1.0f - t));
    }

    __device__ void begin(XPix& s, int x, int y, int iteration, int phase) const {
        s.px = (float)x;
        s.py = (float)y;
        uint32_t seed = (uint32_t)(v.ref + 1) * 0x9e3779b1u + (uint32_t)iteration * 97u +
                        (uint32_t)phase * 13u + (v.flags & 1u) * 7u;
        s.rng = l3d_pcg((uint32_t)(y * v.W + x) ^
                        l3d_pcg(seed + (uint32_t)iteration * 7919u + (uint32_t)phase * 104729u));
        prepare(s, x, y);
        s.ray = ray_of(s.px, s.py);
    }
};

/* Block -> (view, tile) and the view's parameters in shared memory. */
__device__ __forceinline__ int find_view(const L3dFastDev& d, int tile) {
    int lo = 0, hi = d.n_views - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(d.tile_start + mid) <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

/* The view table has an 8-byte aligned stride (static_assert below), so it is copied in 8-byte
 * words. */
static_assert(sizeof(L3dFastView) % 8 == 0, "view table stride must be a multiple of 8 bytes");
static_assert(alignof(L3dFastView) >= 8, "view table must be 8-byte aligned");
__device__ __forceinline__ void load_view(L3dFastView& dst, const L3dFastView* src) {
    const unsigned long long* s = (const unsigned long long*)src;
    unsigned long long* o = (unsigned long long*)&dst;
    for (int i = threadIdx.x; i < (int)(sizeof(L3dFastView) / 8); i += blockDim.x) o[i] = __ldg(s + i);
    __syncthreads();
}

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

template <class E>
__global__ void __launch_bounds__(128) k_fast_init(const L3dFastDev d) {
    __shared__ __align__(16) L3dFastView sv;
    load_view(sv, d.views + find_view(d, blockIdx.x));
    const int local = blockIdx.x - sv.tile_start;
    const int y = (local / sv.tiles_x) * TY + threadIdx.x / TX;
    /* init covers every pixel: a tile spans 32 image columns, two pixels per thread */
    E f(sv, d);
    for (int half = 0; half < 2; half++) {
        const int xx = (local % sv.tiles_x) * (2 * TX) + (threadIdx.x % TX) * 2 + half;
        if (xx >= sv.W || y >= sv.H) continue;
        typename E::Pix s;
        f.begin(s, xx, y, 0, 0);
        const long long index = (long long)y * sv.W + xx;
        float3 n = f.random_normal(s);
        float dd = f.random_depth(s);
        if (sv.has_coarse && d.coarse) {
            /* init_coarse (patchmatch.wgsl.ts:296-333): the random plane against the planes of
             * the four nearest coarse pixels, re-intersected with this pixel's ray */
            float c = f.hypothesis_cost(s, n, dd);
            const float qx = ((s.px + 0.5f) * (float)sv.cW) / (float)sv.W - 0.5f;
            const float qy = ((s.py + 0.5f) * (float)sv.cH) / (float)sv.H - 0.5f;
            const int bx = (int)floorf(qx), by = (int)floorf(qy);
            for (int corner = 0; corner < 4; corner++) {
                const int cx = min(max(bx + (corner & 1), 0), sv.cW - 1);
                const int cy = min(max(by + (corner >> 1), 0), sv.cH - 1);
                const float4 h = d.coarse[sv.coarse_off + (long long)cy * sv.cW + cx];
                if (!(h.w > 0.0f)) continue;
                const float3 hn = make_float3(h.x, h.y, h.z);
                const float3 point = make_float3(((float)cx - sv.ck[2]) / sv.ck[0] * h.w,
                                                 ((float)cy - sv.ck[3]) / sv.ck[1] * h.w, h.w);
                const float den = dot3f(hn, s.ray);
                if (fabsf(den) < 1e-6f) continue;
                const float hd = dot3f(hn, point) / den;
                const float hc = f.hypothesis_cost(s, hn, hd);
                if (hc < c) {
                    c = hc;
                    n = hn;
                    dd = hd;
                }
            }
            d.hyp[sv.pix_off + index] = make_float4(n.x, n.y, n.z, dd);
            d.cost[sv.pix_off + index] = c;
            continue;
        }
        if (sv.flags & 1u) {
            uint32_t packed = d.depths[sv.ref_dep_off + index];
            if (unpack_depth(packed) > 0.0f) {
                dd = unpack_depth(packed);
                n = E::unpack_n(packed);
            }
        }
        float c = f.hypothesis_cost(s, n, dd);
        if (!(sv.flags & 1u) && sv.has_prior) {
            float pd = d.prior[sv.pix_off + index];
            if (pd > 0.0f) {
                float3 vv = E::normalize(s.ray);
                float3 pn = make_float3(-vv.x, -vv.y, -vv.z);
                float pc = f.hypothesis_cost(s, pn, pd);
                if (pc < c) {
                    c = pc;
                    n = pn;
                    dd = pd;
                }
            }
        }
        d.hyp[sv.pix_off + index] = make_float4(n.x, n.y, n.z, dd);
        d.cost[sv.pix_off + index] = c;
    }
}

/* QUAD: the four lanes of each hardware quad take a 2 x 2 block of this colour's pixels (tighter
 * texture footprints per quad request); otherwise four consecutive pixels of one row. */
template <class E, bool QUAD>
__global__ void __launch_bounds__(128, E::kMinBlocks) k_fast_propagate(const L3dFastDev d, int iteration,
                                                        int phase, float step) {
    __shared__ __align__(16) L3dFastView sv;
    load_view(sv, d.views + find_view(d, blockIdx.x));
    if (iteration >= sv.iterations) return;
    const int local = blockIdx.x - sv.tile_start;
    int tx, ty;
    if (QUAD) {
        const int q = threadIdx.x >> 2, j = threadIdx.x & 3;
        tx = (q % (TX / 2)) * 2 + (j & 1);
        ty = (q / (TX / 2)) * 2 + (j >> 1);
    } else {
        tx = threadIdx.x % TX;
        ty = threadIdx.x / TX;
    }
    const int y = (local / sv.tiles_x) * TY + ty;
    const int x = ((local % sv.tiles_x) * TX + tx) * 2 + ((y + phase) & 1);
    if (x >= sv.W || y >= sv.H) return;
    E f(sv, d);
    typename E::Pix s;
    f.begin(s, x, y, iteration, phase);
    const int W = sv.W, H = sv.H;
    const long long base = sv.pix_off;
    const long long index = (long long)y * W + x;
    float4 b = d.hyp[base + index];
    float3 bn = make_float3(b.x, b.y, b.z);
    float bd = b.w;
    float best_cost = d.cost[base + index];
    for (int region = 0; region < 8; region++) {
        const int count = region < 4 ? 7 : 11;
        int chosen = -1;
        float chosen_cost = 1e9f;
        for (int i = 0; i < count; i++) {
            int ox = 0, oy = -3 - 2 * i;
            if (region < 4) near_offset(i, &ox, &oy);
            int rx, ry;
            orient(ox, oy, region & 3, &rx, &ry);
            int qx = x + rx, qy = y + ry;
            if (qx < 0 || qy < 0 || qx >= W || qy >= H) continue;
            int qi = qy * W + qx;
            float c = d.cost[base + qi];
            if (c < chosen_cost) {
                chosen_cost = c;
                chosen = qi;
            }
        }
        if (chosen < 0) continue;
        float4 h = d.hyp[base + chosen];
        float3 hn = make_float3(h.x, h.y, h.z);
        float3 rq = f.ray_of((float)(chosen % W), (float)(chosen / W));
        float den = dot3f(hn, s.ray);
        if (fabsf(den) < 1e-6f) continue;
        float dd = dot3f(hn, make_float3(rq.x * h.w, rq.y * h.w, h.w)) / den;
        float c = f.hypothesis_cost(s, hn, dd);
        if (c < best_cost) {
            best_cost = c;
            bn = hn;
            bd = dd;
        }
    }
    float3 view = E::normalize(s.ray);
    float3 n_random = f.random_normal(s);
    float d_random = f.random_depth(s);
    float e = (fmaf(f.random(s), 2.0f, -1.0f) * 0.15f) * step;
    float d_perturbed = 1.0f / ((1.0f / bd) * (1.0f + e));
    float r1 = f.random(s), r2 = f.random(s), r3 = f.random(s);
    float3 n_perturbed = E::normalize(make_float3(bn.x + (fmaf(r1, 2.0f, -1.0f) * 0.6f) * step,
                                                    bn.y + (fmaf(r2, 2.0f, -1.0f) * 0.6f) * step,
                                                    bn.z + (fmaf(r3, 2.0f, -1.0f) * 0.6f) * step));
    if (dot3f(n_perturbed, view) >= 0.0f) n_perturbed = bn;
    const float3 cur_n = bn;
    const float cur_d = bd;
    for (int c = 0; c < 6; c++) {
        float3 nn = (c == 0 || c == 3) ? n_random : ((c == 1 || c == 5) ? n_perturbed : cur_n);
        float dv = (c == 0 || c == 2) ? d_random : ((c == 1 || c == 4) ? d_perturbed : cur_d);
        float cand = f.hypothesis_cost(s, nn, dv);
        if (cand < best_cost) {
            best_cost = cand;
            bn = nn;
            bd = dv;
        }
    }
    d.hyp[base + index] = make_float4(bn.x, bn.y, bn.z, bd);
    d.cost[base + index] = best_cost;
}

__global__ void k_fast_pack(const L3dFastDev d) {
    const L3dFastView* v = d.views + blockIdx.y;
    if (!__ldg(&v->pack)) return;
    const int W = __ldg(&v->W), H = __ldg(&v->H);
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)W * H) return;
    const long long base = __ldg(&v->pix_off);
    float4 h = d.hyp[base + i];
    d.depths[__ldg(&v->ref_dep_off) + i] = pack_sample(h.w, make_float3(h.x, h.y, h.z), d.cost[base + i]);
}

template <class E>
__global__ void __launch_bounds__(128) k_fast_plane_cost(const L3dFastDev d, const float4* planes,
                                                         float* cost) {
    __shared__ __align__(16) L3dFastView sv;
    load_view(sv, d.views + find_view(d, blockIdx.x));
    const int local = blockIdx.x - sv.tile_start;
    const int y = (local / sv.tiles_x) * TY + threadIdx.x / TX;
    E f(sv, d);
    for (int half = 0; half < 2; half++) {
        const int x = (local % sv.tiles_x) * (2 * TX) + (threadIdx.x % TX) * 2 + half;
        if (x >= sv.W || y >= sv.H) continue;
        typename E::Pix s;
        f.begin(s, x, y, 0, 0);
        const long long index = (long long)y * sv.W + x;
        float4 p = planes[sv.pix_off + index];
        cost[sv.pix_off + index] = f.hypothesis_cost(s, make_float3(p.x, p.y, p.z), p.w);
    }
}

}  // namespace

namespace {

template <class E, bool QUAD>
cudaError_t launch_eval(int kernel, const L3dFastDev& d, int iteration, int phase, cudaStream_t st) {
    if (kernel == L3D_K_INIT) {
        k_fast_init<E><<<d.total_tiles, 128, 0, st>>>(d);
    } else {
        float step = ldexpf(1.0f, -iteration);
        k_fast_propagate<E, QUAD><<<d.total_tiles, 128, 0, st>>>(d, iteration, phase, step);
    }
    return cudaGetLastError();
}

__global__ void k_make_pairs(const void* img, int storage, int W, int H, uint32_t* pairs) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    const long long row = (long long)y * W;
    const int x1 = min(x + 1, W - 1);
    float a, b;
    if (storage == 0) {
        a = (float)((const uint8_t*)img)[row + x] / 255.0f;
        b = (float)((const uint8_t*)img)[row + x1] / 255.0f;
    } else if (storage == 1) {
        a = ((const float*)img)[row + x];
        b = ((const float*)img)[row + x1];
    } else if (storage == 2) {
        a = l3d_f16_to_f32(((const uint16_t*)img)[row + x]);
        b = l3d_f16_to_f32(((const uint16_t*)img)[row + x1]);
    } else {
        a = __uint_as_float((uint32_t)((const uint16_t*)img)[row + x] << 16);
        b = __uint_as_float((uint32_t)((const uint16_t*)img)[row + x1] << 16);
    }
    pairs[row + x] = l3d_f32_to_f16(a) | (l3d_f32_to_f16(b) << 16);
}

}  // namespace

cudaError_t l3d_launch_make_pairs(const void* img, int storage, int W, int H, uint32_t* pairs,
                                  cudaStream_t stream) {
    dim3 grid((W + 127) / 128, H);
    k_make_pairs<<<grid, 128, 0, stream>>>(img, storage, W, H, pairs);
    return cudaGetLastError();
}

/* variant = texture rows (6, 4, 3, 2; the exact evaluator, compensated sums, gathers and the
 * shared window take 6 only) + 8 x quad mapping + 16 x texture gathers with exact weights (fast
 * evaluator, F16/F32/U8) + 32 x the reference window in shared memory (fast evaluator). */
cudaError_t l3d_launch_fast(int kernel, const L3dFastDev& d, int iteration, int phase, int variant,
                            cudaStream_t stream) {
    if (d.total_tiles <= 0) return cudaSuccess;
    if (kernel != L3D_K_INIT && kernel != L3D_K_PROPAGATE) return cudaErrorInvalidValue;
    const int rows = variant & 7;
    const bool quad = (variant & 8) != 0;
    if (d.exact) {
        if (rows != 6) return cudaErrorInvalidValue;
        if (d.comp) return quad ? launch_eval<Exact<true>, true>(kernel, d, iteration, phase, stream)
                                : launch_eval<Exact<true>, false>(kernel, d, iteration, phase, stream);
        return quad ? launch_eval<Exact<false>, true>(kernel, d, iteration, phase, stream)
                    : launch_eval<Exact<false>, false>(kernel, d, iteration, phase, stream);
    }
    if (d.storage == 3) { /* BF16 is sampled from linear memory */
        if (d.comp) return launch_eval<Fast<false, 6, true>, false>(kernel, d, iteration, phase, stream);
        return launch_eval<Fast<false, 6, false>, false>(kernel, d, iteration, phase, stream);
    }
    if (variant & 32) { /* the reference window in shared memory (six texture rows) */
        if (rows != 6) return cudaErrorInvalidValue;
        switch ((d.comp ? 1 : 0) + ((variant & 16) ? 2 : 0) + (quad ? 4 : 0)) {
            case 0: return launch_eval<Fast<true, 6, false, false, true>, false>(kernel, d, iteration, phase, stream);
            case 1: return launch_eval<Fast<true, 6, true, false, true>, false>(kernel, d, iteration, phase, stream);
            case 2: return launch_eval<Fast<true, 6, false, true, true>, false>(kernel, d, iteration, phase, stream);
            case 3: return launch_eval<Fast<true, 6, true, true, true>, false>(kernel, d, iteration, phase, stream);
            case 4: return launch_eval<Fast<true, 6, false, false, true>, true>(kernel, d, iteration, phase, stream);
            case 5: return launch_eval<Fast<true, 6, true, false, true>, true>(kernel, d, iteration, phase, stream);
            case 6: return launch_eval<Fast<true, 6, false, true, true>, true>(kernel, d, iteration, phase, stream);
            default: return launch_eval<Fast<true, 6, true, true, true>, true>(kernel, d, iteration, phase, stream);
        }
    }
    if (variant & 16) { /* texture gathers with exact weights */
        if (rows != 6) return cudaErrorInvalidValue;
        if (d.comp) return quad ? launch_eval<Fast<true, 6, true, true>, true>(kernel, d, iteration, phase, stream)
                                : launch_eval<Fast<true, 6, true, true>, false>(kernel, d, iteration, phase, stream);
        return quad ? launch_eval<Fast<true, 6, false, true>, true>(kernel, d, iteration, phase, stream)
                    : launch_eval<Fast<true, 6, false, true>, false>(kernel, d, iteration, phase, stream);
    }
    if (d.comp) {
        if (rows != 6) return cudaErrorInvalidValue;
        return quad ? launch_eval<Fast<true, 6, true>, true>(kernel, d, iteration, phase, stream)
                    : launch_eval<Fast<true, 6, true>, false>(kernel, d, iteration, phase, stream);
    }
    if (!d.pairs && rows < 6) return cudaErrorInvalidValue;
    switch (rows + (quad ? 8 : 0)) {
        case 6: return launch_eval<Fast<true, 6>, false>(kernel, d, iteration, phase, stream);
        case 4: return launch_eval<Fast<true, 4>, false>(kernel, d, iteration, phase, stream);
        case 3: return launch_eval<Fast<true, 3>, false>(kernel, d, iteration, phase, stream);
        case 2: return launch_eval<Fast<true, 2>, false>(kernel, d, iteration, phase, stream);
        case 14: return launch_eval<Fast<true, 6>, true>(kernel, d, iteration, phase, stream);
        case 12: return launch_eval<Fast<true, 4>, true>(kernel, d, iteration, phase, stream);
        case 11: return launch_eval<Fast<true, 3>, true>(kernel, d, iteration, phase, stream);
        case 10: return launch_eval<Fast<true, 2>, true>(kernel, d, iteration, phase, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t l3d_launch_fast_pack(const L3dFastDev& d, long long max_pixels, cudaStream_t stream) {
    if (d.n_views <= 0 || max_pixels <= 0) return cudaSuccess;
    dim3 grid((unsigned)((max_pixels + 255) / 256), (unsigned)d.n_views);
    k_fast_pack<<<grid, 256, 0, stream>>>(d);
    return cudaGetLastError();
}

cudaError_t l3d_launch_fast_plane_cost(const L3dFastDev& d, const float4* planes, float* cost,
                                       int variant, cudaStream_t stream) {
    if (d.total_tiles <= 0) return cudaSuccess;
    const int rows = variant & 7;
    const unsigned n = (unsigned)d.total_tiles;
    if (d.exact) {
        if (d.comp) k_fast_plane_cost<Exact<true>><<<n, 128, 0, stream>>>(d, planes, cost);
        else k_fast_plane_cost<Exact<false>><<<n, 128, 0, stream>>>(d, planes, cost);
    } else if (d.storage == 3) {
        if (d.comp) k_fast_plane_cost<Fast<false, 6, true>><<<n, 128, 0, stream>>>(d, planes, cost);
        else k_fast_plane_cost<Fast<false, 6>><<<n, 128, 0, stream>>>(d, planes, cost);
    } else if (variant & 16) {
        if (d.comp) k_fast_plane_cost<Fast<true, 6, true, true>><<<n, 128, 0, stream>>>(d, planes, cost);
        else k_fast_plane_cost<Fast<true, 6, false, true>><<<n, 128, 0, stream>>>(d, planes, cost);
    } else if (d.comp) {
        k_fast_plane_cost<Fast<true, 6, true>><<<n, 128, 0, stream>>>(d, planes, cost);
    } else if (rows == 6 || !d.pairs) {
        k_fast_plane_cost<Fast<true, 6>><<<n, 128, 0, stream>>>(d, planes, cost);
    } else if (rows == 4) {
        k_fast_plane_cost<Fast<true, 4>><<<n, 128, 0, stream>>>(d, planes, cost);
    } else if (rows == 3) {
        k_fast_plane_cost<Fast<true, 3>><<<n, 128, 0, stream>>>(d, planes, cost);
    } else {
        k_fast_plane_cost<Fast<true, 2>><<<n, 128, 0, stream>>>(d, planes, cost);
    }
    return cudaGetLastError();
}
