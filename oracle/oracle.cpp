/*
 * CPU oracle of the dense-reconstruction path: a C++ restatement of the reference's WGSL.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Parity unpinned: the reference has no CPU
 * implementation and no golden vectors for these stages; the known-answer tests under tests/
 * pin this restatement instead.
 *
 * Two instantiations:
 *   float  - the FP32 parity oracle.  Every operation is an IEEE f32 operation in a fixed order,
 *            fused multiply-adds are explicit (built with -ffp-contract=off), transcendentals
 *            come from l3d_fmath.h.  The product's plain FP32 kernels follow the same arithmetic
 *            and must agree bit for bit.
 *   double - the FP64 accuracy oracle: the same algorithm, same RNG stream and same f32
 *            constants, in double with libm exp/sin/cos.
 *
 * Sources restated (paths inside the reference project):
 *   frontend/src/app/vision/mvs/patchmatch.wgsl.ts:38-469      kernels and helpers
 *   frontend/src/app/vision/mvs/depth-packing.wgsl.ts:3-33     packed depth format
 *   frontend/src/app/vision/mvs/dense-stereo.ts:185-239,314-355 schedule, uniforms, seeds
 *   frontend/src/app/vision/geometry/camera.ts:28-36,73-77      scaleIntrinsics, relativePose
 *   frontend/src/app/vision/fusion/tsdf-volume.ts:103-154,220-268 TSDF integrate and culling
 *
 * Arithmetic contract (where WGSL leaves the order free, this file fixes it and the CUDA
 * kernels follow it):
 *   dot(a, b)          = fma(a.z, b.z, fma(a.y, b.y, a.x * b.x))
 *   R x + t            = fma(R_i2, x.z, fma(R_i1, x.y, fma(R_i0, x.x, t_i)))
 *   normalize(v)       = v * (1 / sqrt(dot(v, v)))
 *   mix(a, b, t)       = fma(b, t, a * (1 - t))
 *   projection         = fma(f * x, 1 / z, c)            (one reciprocal per point)
 *   homography         = B_s + kt_s u^T, B_s = K_s R_s K_r^-1 and kt_s = K_s t_s composed in
 *                        FP64 on the host, u = (K_r^-T n) / rho per candidate
 *   bilinear sample    = at texel coordinates (u, v) = q.xy / q.z (the centre-aligned texture
 *                        coordinate of textureSampleLevel), exact weights, clamp-to-edge:
 *                        top = fma(fx, b - a, a), bot = fma(fx, d - c, c), fma(fy, bot-top, top)
 *   window sums        = sequential in sample order, sr = fma(w, v, sr), srr = fma(w v, v, srr);
 *                        with args.compensated, Neumaier sums of the rounded products instead
 *   range checks       = written NaN-safe (a NaN coordinate is out of range)
 */
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../luvas.io-3d_b200/csrc/l3d_fmath.h"

namespace {

constexpr int MAX_SOURCES = 8;     /* dense-stereo.ts:44 */
constexpr int MAX_WINDOW = 121;    /* 11 x 11 samples */
constexpr uint32_t FILTER_COST = 7u;

template <typename T> struct Mth;
template <> struct Mth<float> {
    static float fma(float a, float b, float c) { return fmaf(a, b, c); }
    static float exp(float x) { return l3d_expf(x); }
    static void sincos(float a, float* s, float* c) { l3d_sincosf(a, s, c); }
    static float sqrt(float x) { return sqrtf(x); }
    static float rint(float x) { return rintf(x); }
    static float floor(float x) { return floorf(x); }
    static float abs(float x) { return fabsf(x); }
};
template <> struct Mth<double> {
    static double fma(double a, double b, double c) { return std::fma(a, b, c); }
    static double exp(double x) { return std::exp(x); }
    static void sincos(double a, double* s, double* c) { *s = std::sin(a); *c = std::cos(a); }
    static double sqrt(double x) { return std::sqrt(x); }
    static double rint(double x) { return std::rint(x); }
    static double floor(double x) { return std::floor(x); }
    static double abs(double x) { return std::fabs(x); }
};

template <typename T> struct V3 { T x, y, z; };

/* A window sum: plain (s = s + x, s = fma(a, b, s): the reference's running sums) or, with
 * comp, Neumaier's compensated summation (Neumaier 1974) of the addends, products rounded first:
 *   t = s + x;  c = c + (|s| >= |x| ? (s - t) + x : (x - t) + s);  s = t;  sum = s + c. */
template <typename T> struct Sum {
    bool comp;
    T s = 0, c = 0;
    explicit Sum(bool compensated) : comp(compensated) {}
    void add(T x) {
        if (comp) {
            T t = s + x;
            bool big = Mth<T>::abs(s) >= Mth<T>::abs(x);
            T hi = big ? s : x, lo = big ? x : s;
            c = c + ((hi - t) + lo);
            s = t;
        } else {
            s = s + x;
        }
    }
    void fma_add(T a, T b) {
        if (comp) add(a * b);
        else s = Mth<T>::fma(a, b, s);
    }
    T value() const { return comp ? s + c : s; }
};

template <typename T> inline T dot3(V3<T> a, V3<T> b) {
    return Mth<T>::fma(a.z, b.z, Mth<T>::fma(a.y, b.y, a.x * b.x));
}
template <typename T> inline V3<T> normalize3(V3<T> v) {
    T il = T(1) / Mth<T>::sqrt(dot3(v, v));
    return {v.x * il, v.y * il, v.z * il};
}
template <typename T> inline T maxT(T a, T b) { return a > b ? a : b; }  /* WGSL max */
template <typename T> inline T minT(T a, T b) { return a < b ? a : b; }
template <typename T> inline T clampT(T v, T lo, T hi) { return minT(maxT(v, lo), hi); }

/* One source view of a dispatch (View struct of patchmatch.wgsl.ts:4-10, plus the homography
 * base composed on the host). */
template <typename T> struct Src {
    T k[4];
    T R[9];
    T t[3];
    T B[9];
    T kt[3];
    int layer;
    int W, H;                   /* source image size */
    size_t off;                 /* offset of the source's image and depth map */
};

/* Params of patchmatch.wgsl.ts:12-26 as built by DenseStereo.params (dense-stereo.ts:314-355). */
template <typename T> struct Params {
    T k[4];
    T kinv[4];                  /* 1/fx, 1/fy, -cx/fx, -cy/fy in T */
    int W, H, ref, n;
    T range[4];                 /* 1/minD, 1/maxD, step, geometric weight */
    uint32_t iter, phase, seed, flags, needed;
    T ck[4];
    int cW, cH;
    int win_n, win_dil;
    int comp;                   /* compensated window sums */
    size_t ref_off;             /* offset of the reference image and depth map */
    Src<T> src[MAX_SOURCES];
};

/* Size and offset of view i in the concatenated image / depth-map arrays. */
inline void view_size(const orc_stereo_args* a, int i, int* W, int* H, size_t* off) {
    size_t o = 0;
    for (int j = 0; j < i; j++)
        o += a->sizes ? (size_t)a->sizes[2 * j] * a->sizes[2 * j + 1] : (size_t)a->width * a->height;
    *W = a->sizes ? a->sizes[2 * i] : a->width;
    *H = a->sizes ? a->sizes[2 * i + 1] : a->height;
    *off = o;
}

/* relativePose (camera.ts:73-77) in FP64 with the reference's summation order. */
void relative_pose(const double* a, const double* b, double* R, double* t) {
    const double* Ra = a + 4;
    const double* Rb = b + 4;
    double At[9] = {Ra[0], Ra[3], Ra[6], Ra[1], Ra[4], Ra[7], Ra[2], Ra[5], Ra[8]};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            R[r * 3 + c] = Rb[r * 3] * At[c] + Rb[r * 3 + 1] * At[3 + c] + Rb[r * 3 + 2] * At[6 + c];
    const double* ta = a + 13;
    const double* tb = b + 13;
    for (int r = 0; r < 3; r++) {
        double rt = R[r * 3] * ta[0] + R[r * 3 + 1] * ta[1] + R[r * 3 + 2] * ta[2];
        t[r] = tb[r] - rt;
    }
}

uint32_t seed_of(int ref, int iteration, int phase, int flags) {
    /* Math.imul(ref + 1, 0x9e3779b1) + iteration * 97 + phase * 13 + flags * 7, >>> 0 */
    uint32_t s = (uint32_t)(ref + 1) * 0x9e3779b1u;
    return s + (uint32_t)iteration * 97u + (uint32_t)phase * 13u + (uint32_t)flags * 7u;
}

template <typename T>
Params<T> build_params(const orc_stereo_args* a, int iteration, int phase, double step, int flags,
                       int needed, double min_depth, double max_depth) {
    Params<T> p;
    std::memset(&p, 0, sizeof(p));
    const double* ref = a->views + (size_t)a->ref * ORC_VIEW_DOUBLES;
    for (int i = 0; i < 4; i++) p.k[i] = (T)ref[i];
    p.kinv[0] = T(1) / p.k[0];
    p.kinv[1] = T(1) / p.k[1];
    p.kinv[2] = (-p.k[2]) / p.k[0];
    p.kinv[3] = (-p.k[3]) / p.k[1];
    view_size(a, a->ref, &p.W, &p.H, &p.ref_off);
    p.ref = a->ref;
    p.n = std::min(a->n_sources, MAX_SOURCES);
    p.range[0] = (T)(1.0 / min_depth);
    p.range[1] = (T)(1.0 / max_depth);
    p.range[2] = (T)step;
    p.range[3] = (T)0.2;
    p.iter = (uint32_t)iteration;
    p.phase = (uint32_t)phase;
    p.seed = seed_of(a->ref, iteration, phase, flags);
    p.flags = (uint32_t)flags;
    p.needed = (uint32_t)needed;
    if (a->coarse_w > 0 && a->coarse_h > 0) {
        /* scaleIntrinsics (camera.ts:28-36) */
        double sx = (double)a->coarse_w / p.W, sy = (double)a->coarse_h / p.H;
        p.ck[0] = (T)(ref[0] * sx);
        p.ck[1] = (T)(ref[1] * sy);
        p.ck[2] = (T)((ref[2] + 0.5) * sx - 0.5);
        p.ck[3] = (T)((ref[3] + 0.5) * sy - 0.5);
        p.cW = a->coarse_w;
        p.cH = a->coarse_h;
    }
    p.win_n = a->win_n > 0 ? a->win_n : 6;
    p.win_dil = a->win_dil > 0 ? a->win_dil : 2;
    p.comp = a->compensated ? 1 : 0;
    const double kr[4] = {ref[0], ref[1], ref[2], ref[3]};
    for (int s = 0; s < p.n; s++) {
        const double* v = a->views + (size_t)a->sources[s] * ORC_VIEW_DOUBLES;
        double R[9], t[3];
        relative_pose(ref, v, R, t);
        Src<T>& o = p.src[s];
        for (int i = 0; i < 4; i++) o.k[i] = (T)v[i];
        for (int i = 0; i < 9; i++) o.R[i] = (T)R[i];
        for (int i = 0; i < 3; i++) o.t[i] = (T)t[i];
        /* B = K_s R K_r^-1 and kt = K_s t in FP64 */
        double A[9];
        for (int c = 0; c < 3; c++) {
            A[0 * 3 + c] = v[0] * R[0 * 3 + c] + v[2] * R[2 * 3 + c];
            A[1 * 3 + c] = v[1] * R[1 * 3 + c] + v[3] * R[2 * 3 + c];
            A[2 * 3 + c] = R[2 * 3 + c];
        }
        for (int r = 0; r < 3; r++) {
            o.B[r * 3 + 0] = (T)(A[r * 3 + 0] / kr[0]);
            o.B[r * 3 + 1] = (T)(A[r * 3 + 1] / kr[1]);
            o.B[r * 3 + 2] =
                (T)(A[r * 3 + 2] - A[r * 3 + 0] * kr[2] / kr[0] - A[r * 3 + 1] * kr[3] / kr[1]);
        }
        o.kt[0] = (T)(v[0] * t[0] + v[2] * t[2]);
        o.kt[1] = (T)(v[1] * t[1] + v[3] * t[2]);
        o.kt[2] = (T)t[2];
        o.layer = a->sources[s];
        view_size(a, o.layer, &o.W, &o.H, &o.off);
    }
    return p;
}

/* unpack helpers (depth-packing.wgsl.ts:3-19) */
template <typename T> inline T unpack_depth(uint32_t packed) {
    return (T)l3d_f16_to_f32(packed & 0xffffu);
}
template <typename T> inline V3<T> unpack_normal(uint32_t packed) {
    T ex = ((T)((packed >> 16) & 63u) / T(63)) * T(2) - T(1);
    T ey = ((T)((packed >> 22) & 63u) / T(63)) * T(2) - T(1);
    V3<T> n = {ex, ey, (T(1) - Mth<T>::abs(ex)) - Mth<T>::abs(ey)};
    if (n.z < T(0)) {
        T sx = n.x >= T(0) ? T(1) : T(-1);
        T sy = n.y >= T(0) ? T(1) : T(-1);
        T nx = (T(1) - Mth<T>::abs(n.y)) * sx;
        T ny = (T(1) - Mth<T>::abs(n.x)) * sy;
        n.x = nx;
        n.y = ny;
    }
    return normalize3(n);
}
inline uint32_t unpack_cost(uint32_t packed) { return packed >> 28; }

/* pack_sample (depth-packing.wgsl.ts:21-33). */
template <typename T> uint32_t pack_sample(T depth, V3<T> n, T cost) {
    if (!(depth > T(0)) || !(cost < T(1))) return 0u;
    T s = (Mth<T>::abs(n.x) + Mth<T>::abs(n.y)) + Mth<T>::abs(n.z);
    T ex = n.x / s, ey = n.y / s;
    if (n.z < T(0)) {
        T sx = ex >= T(0) ? T(1) : T(-1);
        T sy = ey >= T(0) ? T(1) : T(-1);
        T nx = (T(1) - Mth<T>::abs(ey)) * sx;
        T ny = (T(1) - Mth<T>::abs(ex)) * sy;
        ex = nx;
        ey = ny;
    }
    T cx = clampT(Mth<T>::fma(ex, T(0.5), T(0.5)), T(0), T(1));
    T cy = clampT(Mth<T>::fma(ey, T(0.5), T(0.5)), T(0), T(1));
    uint32_t qx = (uint32_t)Mth<T>::fma(cx, T(63), T(0.5));
    uint32_t qy = (uint32_t)Mth<T>::fma(cy, T(63), T(0.5));
    uint32_t c = std::min(15u, (uint32_t)(cost * T(15)));
    uint32_t h = l3d_f32_to_f16((float)depth);
    return (h & 0xffffu) | (qx << 16) | (qy << 22) | (c << 28);
}

/* One dispatch over one image: the state a WGSL invocation keeps in private variables. */
template <typename T> struct Kernel {
    const Params<T>& p;
    const float* images;
    const uint32_t* depths;
    const float* prior;
    const T* coarse;
    int S;                      /* samples per window */
    int off[MAX_WINDOW][2];
    T ds[MAX_WINDOW];

    Kernel(const Params<T>& params, const float* img, const uint32_t* dep, const float* pri,
           const T* crs)
        : p(params), images(img), depths(dep), prior(pri), coarse(crs) {
        int n = p.win_n, dil = p.win_dil, half = ((n - 1) * dil) / 2;
        S = n * n;
        for (int i = 0; i < S; i++) {
            /* offset_of (patchmatch.wgsl.ts:76-78): 6 x 6 samples at -5, -3, ..., 5 */
            off[i][0] = (i % n) * dil - half;
            off[i][1] = (i / n) * dil - half;
            ds[i] = (T)(off[i][0] * off[i][0] + off[i][1] * off[i][1]);
        }
    }

    T image(size_t off, int W, int x, int y) const {
        return (T)images[off + (size_t)y * W + x];
    }

    V3<T> ray_of(T x, T y) const {
        return {(x - p.k[2]) / p.k[0], (y - p.k[3]) / p.k[1], T(1)};
    }

    /* Per-invocation state. */
    struct Pix {
        T rv[MAX_WINDOW], rw[MAX_WINDOW];
        T rsum, rmean, rvar;
        uint32_t rng;
        T px, py;
        V3<T> ray;
    };

    T random(Pix& s) const { return (T)l3d_random(&s.rng); }

    void seed(Pix& s, uint32_t index) const {
        s.rng = l3d_pcg(index ^ l3d_pcg(p.seed + p.iter * 7919u + p.phase * 104729u));
    }

    T ref_pixel(int x, int y) const {
        x = std::min(std::max(x, 0), p.W - 1);
        y = std::min(std::max(y, 0), p.H - 1);
        return image(p.ref_off, p.W, x, y);
    }

    /* prepare_window (patchmatch.wgsl.ts:90-110) */
    void prepare_window(Pix& s, int x, int y) const {
        const T c1 = T(2.0f) * T(0.06f) * T(0.06f);
        const T c2 = T(2.0f) * T(5.0f) * T(5.0f);
        T center = ref_pixel(x, y);
        Sum<T> sw(p.comp), sr(p.comp), srr(p.comp);
        for (int i = 0; i < S; i++) {
            T v = ref_pixel(x + off[i][0], y + off[i][1]);
            T dc = v - center;
            T w = Mth<T>::exp(-(dc * dc) / c1 - ds[i] / c2);
            s.rv[i] = v;
            s.rw[i] = w;
            sw.add(w);
            sr.fma_add(w, v);
            srr.fma_add(w * v, v);
        }
        s.rsum = sw.value();
        s.rmean = sr.value() / s.rsum;
        s.rvar = maxT(Mth<T>::fma(-s.rmean, s.rmean, srr.value() / s.rsum), T(0));
    }

    T bilinear(const Src<T>& src, T u, T v) const {
        T x0 = Mth<T>::floor(u), y0 = Mth<T>::floor(v);
        T fx = u - x0, fy = v - y0;
        int ix0 = (int)x0, iy0 = (int)y0;
        int ix1 = std::min(ix0 + 1, src.W - 1), iy1 = std::min(iy0 + 1, src.H - 1);
        T a = image(src.off, src.W, ix0, iy0), b = image(src.off, src.W, ix1, iy0);
        T c = image(src.off, src.W, ix0, iy1), d = image(src.off, src.W, ix1, iy1);
        T top = Mth<T>::fma(fx, b - a, a);
        T bot = Mth<T>::fma(fx, d - c, c);
        return Mth<T>::fma(fy, bot - top, top);
    }

    /* view_cost (patchmatch.wgsl.ts:130-159) with H = B_s + kt_s u^T. */
    T view_cost(const Pix& s, const Src<T>& src, const T u[3]) const {
        T h[9];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) h[r * 3 + c] = Mth<T>::fma(src.kt[r], u[c], src.B[r * 3 + c]);
        const T wmax = (T)(src.W - 1), hmax = (T)(src.H - 1);
        Sum<T> ss(p.comp), sss(p.comp), srs(p.comp);
        for (int i = 0; i < S; i++) {
            T x = s.px + (T)off[i][0];
            T y = s.py + (T)off[i][1];
            T qz = Mth<T>::fma(h[6], x, Mth<T>::fma(h[7], y, h[8]));
            if (!(qz > T(1e-6f))) return T(2);
            T qx = Mth<T>::fma(h[0], x, Mth<T>::fma(h[1], y, h[2]));
            T qy = Mth<T>::fma(h[3], x, Mth<T>::fma(h[4], y, h[5]));
            T iz = T(1) / qz;
            T uu = qx * iz, vv = qy * iz;
            if (!(uu >= T(0) && vv >= T(0) && uu <= wmax && vv <= hmax)) return T(2);
            T val = bilinear(src, uu, vv);
            T w = s.rw[i];
            ss.fma_add(w, val);
            T wv = w * val;
            sss.fma_add(wv, val);
            srs.fma_add(wv, s.rv[i]);
        }
        T mean = ss.value() / s.rsum;
        T var_s = maxT(Mth<T>::fma(-mean, mean, sss.value() / s.rsum), T(0));
        T den = Mth<T>::sqrt(s.rvar * var_s);
        if (den < T(1e-5f)) return T(1);
        T cov = Mth<T>::fma(-s.rmean, mean, srs.value() / s.rsum);
        return clampT(T(1) - cov / den, T(0), T(2));
    }

    struct Reproj { T dist, z; bool ok; };

    /* reproject (patchmatch.wgsl.ts:166-190) */
    Reproj reproject(const Src<T>& v, T px, T py, V3<T> x) const {
        Reproj bad = {T(-1), T(-1), false};
        const T* R = v.R;
        V3<T> xs = {
            Mth<T>::fma(R[2], x.z, Mth<T>::fma(R[1], x.y, Mth<T>::fma(R[0], x.x, v.t[0]))),
            Mth<T>::fma(R[5], x.z, Mth<T>::fma(R[4], x.y, Mth<T>::fma(R[3], x.x, v.t[1]))),
            Mth<T>::fma(R[8], x.z, Mth<T>::fma(R[7], x.y, Mth<T>::fma(R[6], x.x, v.t[2])))};
        if (!(xs.z > T(1e-6f))) return bad;
        T iz = T(1) / xs.z;
        T rx = Mth<T>::rint(Mth<T>::fma(v.k[0] * xs.x, iz, v.k[2]));
        T ry = Mth<T>::rint(Mth<T>::fma(v.k[1] * xs.y, iz, v.k[3]));
        if (!(rx >= T(0) && ry >= T(0) && rx < (T)v.W && ry < (T)v.H)) return bad;
        int ix = (int)rx, iy = (int)ry;
        uint32_t packed = depths[v.off + (size_t)iy * v.W + ix];
        T ds_ = unpack_depth<T>(packed);
        if (!(ds_ > T(0)) || unpack_cost(packed) > FILTER_COST) return bad;
        V3<T> bs = {((rx - v.k[2]) / v.k[0]) * ds_, ((ry - v.k[3]) / v.k[1]) * ds_, ds_};
        V3<T> d = {bs.x - v.t[0], bs.y - v.t[1], bs.z - v.t[2]};
        V3<T> back = {
            Mth<T>::fma(R[6], d.z, Mth<T>::fma(R[3], d.y, R[0] * d.x)),
            Mth<T>::fma(R[7], d.z, Mth<T>::fma(R[4], d.y, R[1] * d.x)),
            Mth<T>::fma(R[8], d.z, Mth<T>::fma(R[5], d.y, R[2] * d.x))};
        if (!(back.z > T(1e-6f))) return bad;
        T bz = T(1) / back.z;
        T qx = Mth<T>::fma(p.k[0] * back.x, bz, p.k[2]);
        T qy = Mth<T>::fma(p.k[1] * back.y, bz, p.k[3]);
        T dx = qx - px, dy = qy - py;
        return {Mth<T>::sqrt(Mth<T>::fma(dx, dx, dy * dy)), back.z, true};
    }

    /* hypothesis_cost (patchmatch.wgsl.ts:192-233). view_costs, when given, receives the
     * per-source costs (before the best-k selection). */
    T hypothesis_cost(const Pix& s, V3<T> n, T d, T* view_costs = nullptr) const {
        T inv = T(1) / d;
        if (!(d > T(0)) || inv > p.range[0] || inv < p.range[1]) return T(2);
        if (dot3(n, s.ray) >= T(-1e-3f)) return T(2);
        V3<T> x = {s.ray.x * d, s.ray.y * d, s.ray.z * d};
        T rho = dot3(n, x);
        int count = p.n;
        if (count == 0) return T(2);
        T u[3];
        T ir = T(1) / rho;
        u[0] = (n.x * p.kinv[0]) * ir;
        u[1] = (n.y * p.kinv[1]) * ir;
        u[2] = Mth<T>::fma(n.x, p.kinv[2], Mth<T>::fma(n.y, p.kinv[3], n.z)) * ir;
        bool geometric = (p.flags & 1u) != 0u;
        T costs[MAX_SOURCES];
        for (int k = 0; k < count; k++) {
            T c = view_cost(s, p.src[k], u);
            if (geometric) {
                Reproj r = reproject(p.src[k], s.px, s.py, x);
                T e = r.ok ? minT(r.dist, T(3)) : T(3);
                c = Mth<T>::fma(p.range[3], e, c);
            }
            costs[k] = c;
            if (view_costs) view_costs[k] = c;
        }
        int k = std::max(1, std::min(3, count - 1));
        T total = 0;
        for (int pick = 0; pick < k; pick++) {
            int best = pick;
            for (int j = pick + 1; j < count; j++)
                if (costs[j] < costs[best]) best = j;
            T tmp = costs[pick];
            costs[pick] = costs[best];
            costs[best] = tmp;
            total = total + costs[pick];
        }
        return total / (T)k;
    }

    /* random_normal, random_depth (patchmatch.wgsl.ts:235-249) */
    V3<T> random_normal(Pix& s) const {
        T z = Mth<T>::fma(random(s), T(2), T(-1));
        T a = random(s) * T(6.2831853f);
        T r = Mth<T>::sqrt(maxT(T(0), Mth<T>::fma(-z, z, T(1))));
        T sn, cs;
        Mth<T>::sincos(a, &sn, &cs);
        V3<T> n = {r * cs, r * sn, z};
        V3<T> view = normalize3(s.ray);
        if (dot3(n, view) > T(0)) n = {-n.x, -n.y, -n.z};
        return normalize3(V3<T>{Mth<T>::fma(view.x, T(-0.5f), n.x),
                                Mth<T>::fma(view.y, T(-0.5f), n.y),
                                Mth<T>::fma(view.z, T(-0.5f), n.z)});
    }
    T random_depth(Pix& s) const {
        T t = random(s);
        T m = Mth<T>::fma(p.range[0], t, p.range[1] * (T(1) - t));
        return T(1) / m;
    }

    void begin(Pix& s, int x, int y) const {
        s.px = (T)x;
        s.py = (T)y;
        seed(s, (uint32_t)(y * p.W + x));
        prepare_window(s, x, y);
        s.ray = ray_of(s.px, s.py);
    }

    /* init (patchmatch.wgsl.ts:255-289) */
    void init(int x, int y, T* hyp, T* cost) const {
        Pix s;
        begin(s, x, y);
        size_t index = (size_t)y * p.W + x;
        V3<T> n = random_normal(s);
        T d = random_depth(s);
        if (p.flags & 1u) {
            uint32_t packed = depths[p.ref_off + index];
            if (unpack_depth<T>(packed) > T(0)) {
                d = unpack_depth<T>(packed);
                n = unpack_normal<T>(packed);
            }
        }
        T c = hypothesis_cost(s, n, d);
        if (!(p.flags & 1u) && prior && (T)prior[index] > T(0)) {
            V3<T> v = normalize3(s.ray);
            V3<T> pn = {-v.x, -v.y, -v.z};
            T pd = (T)prior[index];
            T pc = hypothesis_cost(s, pn, pd);
            if (pc < c) {
                c = pc;
                n = pn;
                d = pd;
            }
        }
        hyp[index * 4 + 0] = n.x;
        hyp[index * 4 + 1] = n.y;
        hyp[index * 4 + 2] = n.z;
        hyp[index * 4 + 3] = d;
        cost[index] = c;
    }

    /* init_coarse (patchmatch.wgsl.ts:296-333) */
    void init_coarse(int x, int y, T* hyp, T* cost) const {
        Pix s;
        begin(s, x, y);
        size_t index = (size_t)y * p.W + x;
        V3<T> bn = random_normal(s);
        T bd = random_depth(s);
        T best_cost = hypothesis_cost(s, bn, bd);
        T qx = ((s.px + T(0.5f)) * (T)p.cW) / (T)p.W - T(0.5f);
        T qy = ((s.py + T(0.5f)) * (T)p.cH) / (T)p.H - T(0.5f);
        int bx = (int)Mth<T>::floor(qx), by = (int)Mth<T>::floor(qy);
        for (int corner = 0; corner < 4; corner++) {
            int cx = std::min(std::max(bx + (corner & 1), 0), p.cW - 1);
            int cy = std::min(std::max(by + (corner >> 1), 0), p.cH - 1);
            const T* h = coarse + ((size_t)cy * p.cW + cx) * 4;
            if (!(h[3] > T(0))) continue;
            V3<T> hn = {h[0], h[1], h[2]};
            V3<T> point = {((T)cx - p.ck[2]) / p.ck[0] * h[3], ((T)cy - p.ck[3]) / p.ck[1] * h[3],
                           h[3]};
            T den = dot3(hn, s.ray);
            if (Mth<T>::abs(den) < T(1e-6f)) continue;
            T d = dot3(hn, point) / den;
            T c = hypothesis_cost(s, hn, d);
            if (c < best_cost) {
                best_cost = c;
                bn = hn;
                bd = d;
            }
        }
        hyp[index * 4 + 0] = bn.x;
        hyp[index * 4 + 1] = bn.y;
        hyp[index * 4 + 2] = bn.z;
        hyp[index * 4 + 3] = bd;
        cost[index] = best_cost;
    }

    static void near_offset(int i, int* ox, int* oy) {
        int m = (i + 1) / 2;
        *ox = (i & 1) ? -m : m;
        *oy = -(m + 1);
    }
    static void orient(int ox, int oy, int dir, int* rx, int* ry) {
        switch (dir) {
            case 1: *rx = ox; *ry = -oy; break;
            case 2: *rx = oy; *ry = ox; break;
            case 3: *rx = -oy; *ry = ox; break;
            default: *rx = ox; *ry = oy; break;
        }
    }

    /* propagate (patchmatch.wgsl.ts:349-423): hyp/cost are read for the other colour and
     * written for this pixel only. */
    void propagate(int x, int y, T* hyp, T* cost) const {
        Pix s;
        begin(s, x, y);
        size_t index = (size_t)y * p.W + x;
        V3<T> bn = {hyp[index * 4], hyp[index * 4 + 1], hyp[index * 4 + 2]};
        T bd = hyp[index * 4 + 3];
        T best_cost = cost[index];
        for (int region = 0; region < 8; region++) {
            int count = region < 4 ? 7 : 11;
            long chosen = -1;
            T chosen_cost = T(1e9f);
            for (int i = 0; i < count; i++) {
                int ox = 0, oy = -3 - 2 * i;
                if (region < 4) near_offset(i, &ox, &oy);
                int rx, ry;
                orient(ox, oy, region % 4, &rx, &ry);
                int qx = x + rx, qy = y + ry;
                if (qx < 0 || qy < 0 || qx >= p.W || qy >= p.H) continue;
                size_t qi = (size_t)qy * p.W + qx;
                if (cost[qi] < chosen_cost) {
                    chosen_cost = cost[qi];
                    chosen = (long)qi;
                }
            }
            if (chosen < 0) continue;
            const T* h = hyp + (size_t)chosen * 4;
            V3<T> hn = {h[0], h[1], h[2]};
            V3<T> rq = ray_of((T)(chosen % p.W), (T)(chosen / p.W));
            T den = dot3(hn, s.ray);
            if (Mth<T>::abs(den) < T(1e-6f)) continue;
            T d = dot3(hn, V3<T>{rq.x * h[3], rq.y * h[3], rq.z * h[3]}) / den;
            T c = hypothesis_cost(s, hn, d);
            if (c < best_cost) {
                best_cost = c;
                bn = hn;
                bd = d;
            }
        }
        T step = p.range[2];
        V3<T> view = normalize3(s.ray);
        V3<T> n_random = random_normal(s);
        T d_random = random_depth(s);
        T e = ((Mth<T>::fma(random(s), T(2), T(-1)) * T(0.15f)) * step);
        T d_perturbed = T(1) / ((T(1) / bd) * (T(1) + e));
        T r1 = random(s), r2 = random(s), r3 = random(s);
        V3<T> np = {bn.x + (Mth<T>::fma(r1, T(2), T(-1)) * T(0.6f)) * step,
                    bn.y + (Mth<T>::fma(r2, T(2), T(-1)) * T(0.6f)) * step,
                    bn.z + (Mth<T>::fma(r3, T(2), T(-1)) * T(0.6f)) * step};
        V3<T> n_perturbed = normalize3(np);
        if (dot3(n_perturbed, view) >= T(0)) n_perturbed = bn;
        V3<T> cur_n = bn;
        T cur_d = bd;
        V3<T> normals[6] = {n_random, n_perturbed, cur_n, n_random, cur_n, n_perturbed};
        T dtry[6] = {d_random, d_perturbed, d_random, cur_d, d_perturbed, cur_d};
        for (int c = 0; c < 6; c++) {
            T cand = hypothesis_cost(s, normals[c], dtry[c]);
            if (cand < best_cost) {
                best_cost = cand;
                bn = normals[c];
                bd = dtry[c];
            }
        }
        hyp[index * 4 + 0] = bn.x;
        hyp[index * 4 + 1] = bn.y;
        hyp[index * 4 + 2] = bn.z;
        hyp[index * 4 + 3] = bd;
        cost[index] = best_cost;
    }

    /* consistency (patchmatch.wgsl.ts:436-469) */
    uint32_t consistency(int x, int y) const {
        size_t index = (size_t)y * p.W + x;
        uint32_t packed = depths[p.ref_off + index];
        T d = unpack_depth<T>(packed);
        if (!(d > T(0)) || unpack_cost(packed) > FILTER_COST) return 0u;
        T px = (T)x, py = (T)y;
        V3<T> r = ray_of(px, py);
        V3<T> X = {r.x * d, r.y * d, r.z * d};
        uint32_t agree = 0;
        T sum = d;
        for (int k = 0; k < p.n; k++) {
            Reproj q = reproject(p.src[k], px, py, X);
            if (q.ok && q.dist < T(1) && Mth<T>::abs(q.z - d) < T(0.01f) * d) {
                agree++;
                sum = sum + q.z;
            }
        }
        uint32_t needed = std::min((uint32_t)p.n, std::max(1u, p.needed));
        if (agree < needed) return 0u;
        T mean = sum / (T)(agree + 1u);
        return (packed & 0xffff0000u) | (l3d_f32_to_f16((float)mean) & 0xffffu);
    }
};

template <typename T>
void run_kernel(const orc_stereo_args* a, const Params<T>& p, int kernel, T* hyp, T* cost,
                uint32_t* depths, uint32_t* filtered) {
    Kernel<T> K(p, a->images, depths, a->prior, (const T*)a->coarse_hyp);
    const int W = p.W, H = p.H;
#ifdef _OPENMP
    int threads = a->threads > 0 ? a->threads : omp_get_max_threads();
#endif
    if (kernel == ORC_PACK) {
        size_t total = (size_t)W * H;
        uint32_t* out = depths + p.ref_off;
        for (size_t i = 0; i < total; i++) {
            V3<T> n = {hyp[i * 4], hyp[i * 4 + 1], hyp[i * 4 + 2]};
            out[i] = pack_sample<T>(hyp[i * 4 + 3], n, cost[i]);
        }
        return;
    }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (int y = 0; y < H; y++) {
        if (kernel == ORC_PROPAGATE) {
            for (int x = (int)((y + p.phase) & 1u); x < W; x += 2) K.propagate(x, y, hyp, cost);
        } else {
            for (int x = 0; x < W; x++) {
                if (kernel == ORC_INIT) K.init(x, y, hyp, cost);
                else if (kernel == ORC_INIT_COARSE) K.init_coarse(x, y, hyp, cost);
                else if (kernel == ORC_CONSISTENCY) filtered[(size_t)y * W + x] = K.consistency(x, y);
            }
        }
    }
}

bool valid_args(const orc_stereo_args* a) {
    if (!a || a->n_views <= 0 || !a->views || !a->images) return false;
    if (!a->sizes && (a->width <= 0 || a->height <= 0)) return false;
    if (a->sizes)
        for (int i = 0; i < a->n_views; i++)
            if (a->sizes[2 * i] <= 0 || a->sizes[2 * i + 1] <= 0) return false;
    if (a->ref < 0 || a->ref >= a->n_views || a->n_sources < 0) return false;
    for (int s = 0; s < std::min(a->n_sources, MAX_SOURCES); s++)
        if (a->sources[s] < 0 || a->sources[s] >= a->n_views) return false;
    int n = a->win_n > 0 ? a->win_n : 6, dil = a->win_dil > 0 ? a->win_dil : 2;
    if (n * n > MAX_WINDOW || ((n - 1) * dil) % 2) return false;
    return true;
}

template <typename T>
int kernel_impl(const orc_stereo_args* a, int kernel, int iteration, int phase, T* hyp, T* cost,
                uint32_t* depths, uint32_t* filtered) {
    if (!valid_args(a)) return 1;
    int flags = a->geometric ? 1 : 0;
    double step = std::pow(0.5, iteration);
    Params<T> p;
    if (kernel == ORC_CONSISTENCY) {
        /* DenseStereo.filter (dense-stereo.ts:250-263): range 0.01-100 m, no flags */
        p = build_params<T>(a, 0, 0, 0.0, 0, a->needed, 0.01, 100.0);
    } else if (kernel == ORC_PACK) {
        p = build_params<T>(a, 0, 0, 0.0, flags, 0, a->min_depth, a->max_depth);
    } else {
        p = build_params<T>(a, iteration, phase, step, flags, 0, a->min_depth, a->max_depth);
    }
    run_kernel<T>(a, p, kernel, hyp, cost, depths, filtered);
    return 0;
}

template <typename T>
int solve_impl(const orc_stereo_args* a, T* hyp, T* cost, uint32_t* depths) {
    if (!valid_args(a)) return 1;
    if (a->n_sources == 0) return 0;   /* dense-stereo.ts:187 */
    int start = (a->from_coarse && a->coarse_hyp) ? ORC_INIT_COARSE : ORC_INIT;
    kernel_impl<T>(a, start, 0, 0, hyp, cost, depths, nullptr);
    for (int it = 0; it < a->iterations; it++)
        for (int phase = 0; phase < 2; phase++)
            kernel_impl<T>(a, ORC_PROPAGATE, it, phase, hyp, cost, depths, nullptr);
    if (a->pack) kernel_impl<T>(a, ORC_PACK, 0, 0, hyp, cost, depths, nullptr);
    return 0;
}

template <typename T>
int plane_cost_impl(const orc_stereo_args* a, const T* planes, T* cost, T* view_costs) {
    if (!valid_args(a)) return 1;
    int flags = a->geometric ? 1 : 0;
    Params<T> p = build_params<T>(a, 0, 0, 1.0, flags, 0, a->min_depth, a->max_depth);
    Kernel<T> K(p, a->images, nullptr, a->prior, nullptr);
    const int W = p.W, H = p.H;
#ifdef _OPENMP
    int threads = a->threads > 0 ? a->threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (int y = 0; y < H; y++) {
        typename Kernel<T>::Pix s;
        for (int x = 0; x < W; x++) {
            size_t i = (size_t)y * W + x;
            K.begin(s, x, y);
            V3<T> n = {planes[i * 4], planes[i * 4 + 1], planes[i * 4 + 2]};
            T vc[MAX_SOURCES] = {0};
            cost[i] = K.hypothesis_cost(s, n, planes[i * 4 + 3], vc);
            if (view_costs)
                for (int k = 0; k < MAX_SOURCES; k++) view_costs[i * MAX_SOURCES + k] = vc[k];
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- TSDF -------------------- */

/* visibleBricks (tsdf-volume.ts:220-234) in FP64 with the reference's operation order. */
bool brick_visible(const orc_tsdf_desc* d, const orc_tsdf_view* v, int bx, int by, int bz) {
    double side = d->voxel * 8.0;
    double c[3] = {d->origin[0] + (bx + 0.5) * side, d->origin[1] + (by + 0.5) * side,
                   d->origin[2] + (bz + 0.5) * side};
    double radius = d->voxel * 8.0 * 0.87 + d->truncation;
    const double* R = v->R;
    double p0 = R[0] * c[0] + R[1] * c[1] + R[2] * c[2] + v->t[0];
    double p1 = R[3] * c[0] + R[4] * c[1] + R[5] * c[2] + v->t[1];
    double p2 = R[6] * c[0] + R[7] * c[1] + R[8] * c[2] + v->t[2];
    double u = (v->k[0] * p0) / p2 + v->k[2];
    double w = (v->k[1] * p1) / p2 + v->k[3];
    double z = p2;
    if (z < 0.02 - radius || z > v->max_depth + radius) return false;
    double margin = (v->k[0] * radius) / std::max(0.02, z);
    if (u < -margin || w < -margin || u > d->width + margin || w > d->height + margin) return false;
    return true;
}

inline void brick_count(const orc_tsdf_desc* d, int* nb) {
    nb[0] = (d->dims[0] + 7) / 8;
    nb[1] = (d->dims[1] + 7) / 8;
    nb[2] = (d->dims[2] + 7) / 8;
}

/* Per-voxel body of integrate (tsdf-volume.ts:111-153). */
template <typename T, bool Q8>
inline void integrate_voxel(const orc_tsdf_desc* dsc, const T* tf, const T* kk, int W, int H,
                            const uint32_t* depth, const float* prior, int gx, int gy, int gz,
                            size_t idx, T* tsdf, void* weight) {
    const T* origin = tf;          /* [0..2] origin, [3] voxel, [4] mu, [5] prior weight,
                                      [6] max weight, [7] confidence, [8..16] R, [17..19] t */
    const T vox = tf[3], mu = tf[4];
    const T* R = tf + 8;
    const T* t = tf + 17;
    T wx = Mth<T>::fma((T)gx + T(0.5f), vox, origin[0]);
    T wy = Mth<T>::fma((T)gy + T(0.5f), vox, origin[1]);
    T wz = Mth<T>::fma((T)gz + T(0.5f), vox, origin[2]);
    V3<T> cam = {Mth<T>::fma(R[2], wz, Mth<T>::fma(R[1], wy, Mth<T>::fma(R[0], wx, t[0]))),
                 Mth<T>::fma(R[5], wz, Mth<T>::fma(R[4], wy, Mth<T>::fma(R[3], wx, t[1]))),
                 Mth<T>::fma(R[8], wz, Mth<T>::fma(R[7], wy, Mth<T>::fma(R[6], wx, t[2])))};
    if (!(cam.z > T(0.01f))) return;
    T iz = T(1) / cam.z;
    T rx = Mth<T>::rint(Mth<T>::fma(kk[0] * cam.x, iz, kk[2]));
    T ry = Mth<T>::rint(Mth<T>::fma(kk[1] * cam.y, iz, kk[3]));
    if (!(rx >= T(0) && ry >= T(0) && rx < (T)W && ry < (T)H)) return;
    size_t i = (size_t)(int)ry * W + (size_t)(int)rx;
    uint32_t packed = depth[i];
    T d = unpack_depth<T>(packed);
    T w = 0;
    if (d > T(0)) {
        V3<T> n = unpack_normal<T>(packed);
        V3<T> cn = normalize3(cam);
        w = maxT(T(0.2f), Mth<T>::abs(dot3(n, cn)));
        T conf = tf[7];
        if (conf > T(0)) {
            T c = (T)unpack_cost(packed) / T(8);
            T r = clampT(conf / d, T(0.5f), T(2));
            w = w * ((maxT(T(0.15f), (T(1) - c) * (T(1) - c)) * r) * r);
        }
    } else {
        d = prior ? (T)prior[i] : T(0);
        w = tf[5];
    }
    if (!(d > T(0))) return;
    T sdf = d - cam.z;
    if (sdf < -mu) return;
    T obs = minT(T(1), sdf / mu);
    if (Q8) {
        uint16_t* wq = (uint16_t*)weight;
        uint32_t wi = (uint32_t)Mth<T>::rint(w * T(256));
        if (wi == 0u) return;
        uint32_t w0i = wq[idx];
        T w0 = (T)w0i * T(0.00390625f);
        T wf = (T)wi * T(0.00390625f);
        tsdf[idx] = Mth<T>::fma(tsdf[idx], w0, obs * wf) / (w0 + wf);
        uint32_t maxq = (uint32_t)Mth<T>::rint(tf[6] * T(256));
        wq[idx] = (uint16_t)std::min(w0i + wi, maxq);
    } else {
        T* wt = (T*)weight;
        T w0 = wt[idx];
        tsdf[idx] = Mth<T>::fma(tsdf[idx], w0, obs * w) / (w0 + w);
        wt[idx] = minT(w0 + w, tf[6]);
    }
}

template <typename T>
int tsdf_impl(const orc_tsdf_desc* d, const orc_tsdf_view* v, const uint32_t* depth, T* tsdf,
              void* weight, int threads) {
    if (!d || !v || !depth || !tsdf || !weight || d->width <= 0 || d->height <= 0) return 1;
    if (d->weight_q8 && sizeof(T) != sizeof(float)) return 1;
    /* Uniform block of TsdfVolume.integrate (tsdf-volume.ts:244-253), rounded to T. */
    T tf[20];
    for (int i = 0; i < 3; i++) tf[i] = (T)d->origin[i];
    tf[3] = (T)d->voxel;
    tf[4] = (T)d->truncation;
    tf[5] = (T)d->prior_weight;
    tf[6] = (T)d->max_weight;
    tf[7] = (T)v->confidence;
    for (int i = 0; i < 9; i++) tf[8 + i] = (T)v->R[i];
    for (int i = 0; i < 3; i++) tf[17 + i] = (T)v->t[i];
    T kk[4] = {(T)v->k[0], (T)v->k[1], (T)v->k[2], (T)v->k[3]};
    const int W = d->width, H = d->height;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#endif
    if (d->dense) {
        int nb[3];
        brick_count(d, nb);
        long bricks = (long)nb[0] * nb[1] * nb[2];
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
        for (long b = 0; b < bricks; b++) {
            int bx = (int)(b % nb[0]), by = (int)((b / nb[0]) % nb[1]), bz = (int)(b / ((long)nb[0] * nb[1]));
            if (!brick_visible(d, v, bx, by, bz)) continue;
            for (int l = 0; l < 512; l++) {
                int gx = bx * 8 + (l & 7), gy = by * 8 + ((l >> 3) & 7), gz = bz * 8 + (l >> 6);
                if (gx >= d->dims[0] || gy >= d->dims[1] || gz >= d->dims[2]) continue;
                size_t idx = ((size_t)gz * d->dims[1] + gy) * d->dims[0] + gx;
                if (d->weight_q8)
                    integrate_voxel<T, true>(d, tf, kk, W, H, depth, v->prior, gx, gy, gz, idx, tsdf, weight);
                else
                    integrate_voxel<T, false>(d, tf, kk, W, H, depth, v->prior, gx, gy, gz, idx, tsdf, weight);
            }
        }
    } else {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
        for (long b = 0; b < d->count; b++) {
            const int32_t* c = d->coords + b * 4;
            if (!brick_visible(d, v, c[0], c[1], c[2])) continue;
            for (int l = 0; l < 512; l++) {
                int gx = c[0] * 8 + (l & 7), gy = c[1] * 8 + ((l >> 3) & 7), gz = c[2] * 8 + (l >> 6);
                size_t idx = (size_t)b * 512 + l;
                if (d->weight_q8)
                    integrate_voxel<T, true>(d, tf, kk, W, H, depth, v->prior, gx, gy, gz, idx, tsdf, weight);
                else
                    integrate_voxel<T, false>(d, tf, kk, W, H, depth, v->prior, gx, gy, gz, idx, tsdf, weight);
            }
        }
    }
    return 0;
}

}  // namespace

extern "C" {

int orc32_solve(const orc_stereo_args* a, float* hyp, float* cost, uint32_t* depths) {
    return solve_impl<float>(a, hyp, cost, depths);
}
int orc64_solve(const orc_stereo_args* a, double* hyp, double* cost, uint32_t* depths) {
    return solve_impl<double>(a, hyp, cost, depths);
}
int orc32_kernel(const orc_stereo_args* a, int32_t kernel, int32_t iteration, int32_t phase,
                 float* hyp, float* cost, uint32_t* depths, uint32_t* filtered) {
    return kernel_impl<float>(a, kernel, iteration, phase, hyp, cost, depths, filtered);
}
int orc64_kernel(const orc_stereo_args* a, int32_t kernel, int32_t iteration, int32_t phase,
                 double* hyp, double* cost, uint32_t* depths, uint32_t* filtered) {
    return kernel_impl<double>(a, kernel, iteration, phase, hyp, cost, depths, filtered);
}
int orc32_plane_cost(const orc_stereo_args* a, const float* planes, float* cost, float* view_costs) {
    return plane_cost_impl<float>(a, planes, cost, view_costs);
}
int orc64_plane_cost(const orc_stereo_args* a, const double* planes, double* cost,
                     double* view_costs) {
    return plane_cost_impl<double>(a, planes, cost, view_costs);
}
int orc32_tsdf_integrate(const orc_tsdf_desc* d, const orc_tsdf_view* v, const uint32_t* depth,
                         float* tsdf, void* weight, int32_t threads) {
    return tsdf_impl<float>(d, v, depth, tsdf, weight, threads);
}
int orc64_tsdf_integrate(const orc_tsdf_desc* d, const orc_tsdf_view* v, const uint32_t* depth,
                         double* tsdf, double* weight, int32_t threads) {
    return tsdf_impl<double>(d, v, depth, tsdf, weight, threads);
}
int orc_tsdf_visible(const orc_tsdf_desc* d, const orc_tsdf_view* v, uint8_t* out) {
    if (d->dense) {
        int nb[3];
        brick_count(d, nb);
        long bricks = (long)nb[0] * nb[1] * nb[2];
        for (long b = 0; b < bricks; b++)
            out[b] = brick_visible(d, v, (int)(b % nb[0]), (int)((b / nb[0]) % nb[1]),
                                   (int)(b / ((long)nb[0] * nb[1])));
    } else {
        for (long b = 0; b < d->count; b++)
            out[b] = brick_visible(d, v, d->coords[b * 4], d->coords[b * 4 + 1], d->coords[b * 4 + 2]);
    }
    return 0;
}
uint32_t orc_pack_sample(float depth, float nx, float ny, float nz, float cost) {
    return pack_sample<float>(depth, V3<float>{nx, ny, nz}, cost);
}
float orc_unpack_depth(uint32_t packed) { return unpack_depth<float>(packed); }
void orc_unpack_normal(uint32_t packed, float* n3) {
    V3<float> n = unpack_normal<float>(packed);
    n3[0] = n.x;
    n3[1] = n.y;
    n3[2] = n.z;
}
uint32_t orc_pcg(uint32_t v) { return l3d_pcg(v); }
float orc_expf(float x) { return l3d_expf(x); }
void orc_sincosf(float a, float* s, float* c) { l3d_sincosf(a, s, c); }
uint32_t orc_f32_to_f16(float f) { return l3d_f32_to_f16(f); }
float orc_f16_to_f32(uint32_t h) { return l3d_f16_to_f32(h); }
uint32_t orc_seed(int32_t ref, int32_t iteration, int32_t phase, int32_t flags) {
    return seed_of(ref, iteration, phase, flags);
}

}  // extern "C"
