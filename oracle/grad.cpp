/*
 * FP64 gradient oracle of the differentiable NCC cost and TSDF integration.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the product library never links or calls it.
 *
 * The reference has no gradients; these functions restate the objectives the product
 * differentiates and obtain their derivatives by forward-mode automatic differentiation (dual
 * numbers) in FP64, so the product's hand-derived adjoint kernels are checked against a
 * derivation that shares none of their algebra.  The tests also check these derivatives against
 * central differences of the FP64 objectives.
 *
 *   NCC objective (frontend/src/app/vision/mvs/patchmatch.wgsl.ts:90-110 prepare_window,
 *   :130-159 view_cost): per reference pixel, the sum over the sources of the bilateral-weighted
 *   1 - NCC of the window, samples bilinear at texel coordinates q.xy / q.z of the homography
 *   H = B + kt u^T (B = K_s R K_r^-1, kt = K_s t, u = K_r^-T n / (d n.ray)).  Per pixel a plane
 *   (d, a, b) with n = (sin a cos b, sin b, -cos a cos b); per view an se(3) increment (v, w)
 *   with R = Exp(w) R0, t = Exp(w) t0 + v.
 *
 *   TSDF integration (frontend/src/app/vision/fusion/tsdf-volume.ts:111-153) with the depth of
 *   valid pixels taken from a continuous map, differentiated with respect to that depth and the
 *   volume state before the update.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

namespace {

/* ---- dual numbers: value + N tangents ---- */
template <int N>
struct Dual {
    double v;
    double d[N];
    Dual() : v(0.0) { std::fill(d, d + N, 0.0); }
    Dual(double x) : v(x) { std::fill(d, d + N, 0.0); }  // NOLINT: constants promote implicitly
};

template <int N> inline Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v + b.v);
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> inline Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v - b.v);
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> inline Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r(-a.v);
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
}
template <int N> inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v * b.v);
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r(a.v / b.v);
    const double ib = 1.0 / b.v;
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N> inline Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N> inline Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N> inline Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N> inline Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N> inline Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r(a.v * b);
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b;
    return r;
}
template <int N> inline Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N> inline Dual<N> operator/(const Dual<N>& a, double b) { return a * (1.0 / b); }
template <int N> inline Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }

template <int N> inline Dual<N> sqrt(const Dual<N>& a) {
    Dual<N> r(std::sqrt(a.v));
    const double h = 0.5 / r.v;
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * h;
    return r;
}
template <int N> inline Dual<N> sin(const Dual<N>& a) {
    Dual<N> r(std::sin(a.v));
    const double c = std::cos(a.v);
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * c;
    return r;
}
template <int N> inline Dual<N> cos(const Dual<N>& a) {
    Dual<N> r(std::cos(a.v));
    const double s = -std::sin(a.v);
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * s;
    return r;
}

inline double val(double x) { return x; }
template <int N> inline double val(const Dual<N>& x) { return x.v; }
using std::cos;
using std::sin;
using std::sqrt;

template <int N> inline Dual<N> seed_dual(double v, int tangent) {
    Dual<N> r(v);
    r.d[tangent] = 1.0;
    return r;
}

/* ---- poses ---- */

/* Exp of so(3): I + A [w]x + B [w]x^2, A = sin t / t, B = (1 - cos t) / t^2, in the square of
 * the angle below 1e-6 (series to t^4), so the derivative at w = 0 is exact. */
template <class S> void exp_so3(const S* w, S* R) {
    const S th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    S A, B;
    if (val(th2) < 1e-6) {
        A = 1.0 - th2 / 6.0 + th2 * th2 / 120.0;
        B = 0.5 - th2 / 24.0 + th2 * th2 / 720.0;
    } else {
        const S th = sqrt(th2);
        A = sin(th) / th;
        B = (1.0 - cos(th)) / th2;
    }
    const S zero(0.0);
    const S K[9] = {zero, -w[2], w[1], w[2], zero, -w[0], -w[1], w[0], zero};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            const S kk = K[r * 3] * K[c] + K[r * 3 + 1] * K[3 + c] + K[r * 3 + 2] * K[6 + c];
            R[r * 3 + c] = (r == c ? 1.0 : 0.0) + A * K[r * 3 + c] + B * kk;
        }
}

/* R = Exp(w) R0, t = Exp(w) t0 + v for a 16-double view (fx fy cx cy | R | t). */
template <class S> void current_pose(const double* view, const S* delta, S* R, S* t) {
    S E[9];
    exp_so3(delta + 3, E);
    const double* R0 = view + 4;
    const double* t0 = view + 13;
    for (int r = 0; r < 3; r++) {
        for (int c = 0; c < 3; c++) R[r * 3 + c] = E[r * 3] * R0[c] + E[r * 3 + 1] * R0[3 + c] + E[r * 3 + 2] * R0[6 + c];
        t[r] = E[r * 3] * t0[0] + E[r * 3 + 1] * t0[1] + E[r * 3 + 2] * t0[2] + delta[r];
    }
}

/* Homography base of a pair: B = K_s R K_r^-1, kt = K_s t with X_s = Rs Rr^T (X_r - tr) + ts. */
template <class S> void pair_homography(const double* vr, const double* vs, const S* dr, const S* ds,
                                        S* B, S* kt) {
    S Rr[9], tr[3], Rs[9], ts[3];
    current_pose(vr, dr, Rr, tr);
    current_pose(vs, ds, Rs, ts);
    S R[9], t[3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            R[r * 3 + c] = Rs[r * 3] * Rr[c * 3] + Rs[r * 3 + 1] * Rr[c * 3 + 1] + Rs[r * 3 + 2] * Rr[c * 3 + 2];
    for (int r = 0; r < 3; r++) t[r] = ts[r] - (R[r * 3] * tr[0] + R[r * 3 + 1] * tr[1] + R[r * 3 + 2] * tr[2]);
    const double fxr = vr[0], fyr = vr[1], cxr = vr[2], cyr = vr[3];
    const double fxs = vs[0], fys = vs[1], cxs = vs[2], cys = vs[3];
    S A[9];
    for (int c = 0; c < 3; c++) {
        A[c] = fxs * R[c] + cxs * R[6 + c];
        A[3 + c] = fys * R[3 + c] + cys * R[6 + c];
        A[6 + c] = R[6 + c];
    }
    for (int r = 0; r < 3; r++) {
        B[r * 3 + 0] = A[r * 3 + 0] / fxr;
        B[r * 3 + 1] = A[r * 3 + 1] / fyr;
        B[r * 3 + 2] = A[r * 3 + 2] - A[r * 3 + 0] * (cxr / fxr) - A[r * 3 + 1] * (cyr / fyr);
    }
    kt[0] = fxs * t[0] + cxs * t[2];
    kt[1] = fys * t[1] + cys * t[2];
    kt[2] = t[2];
}

/* ---- NCC ---- */

struct Image {
    const float* px;
    int W, H;
    double at(int x, int y) const { return (double)px[(size_t)y * W + x]; }
};

struct RefWindow {
    double rv[121], rw[121];
    double sum, mean, var;
};

void view_geometry(const orc_stereo_args* a, int i, int* W, int* H, size_t* off) {
    size_t o = 0;
    for (int j = 0; j < i; j++)
        o += a->sizes ? (size_t)a->sizes[2 * j] * a->sizes[2 * j + 1] : (size_t)a->width * a->height;
    *W = a->sizes ? a->sizes[2 * i] : a->width;
    *H = a->sizes ? a->sizes[2 * i + 1] : a->height;
    *off = o;
}

struct Win {
    int n, dil, half;
    int ox(int i) const { return (i % n) * dil - half; }
    int oy(int i) const { return (i / n) * dil - half; }
    int size() const { return n * n; }
};

/* prepare_window (patchmatch.wgsl.ts:90-110) in FP64 with the shader's f32 constants. */
void ref_window(const Image& img, const Win& win, int x, int y, RefWindow* w) {
    const double c1 = 2.0 * (double)0.06f * (double)0.06f;
    const double c2 = 2.0 * 5.0 * 5.0;
    const double center = img.at(x, y);
    double sw = 0.0, sr = 0.0, srr = 0.0;
    for (int i = 0; i < win.size(); i++) {
        const int ox = win.ox(i), oy = win.oy(i);
        const double v = img.at(std::min(std::max(x + ox, 0), img.W - 1),
                                std::min(std::max(y + oy, 0), img.H - 1));
        const double dc = v - center;
        const double wt = std::exp(-(dc * dc) / c1 - (double)(ox * ox + oy * oy) / c2);
        w->rv[i] = v;
        w->rw[i] = wt;
        sw += wt;
        sr += wt * v;
        srr += wt * v * v;
    }
    w->sum = sw;
    w->mean = sr / sw;
    w->var = std::max(srr / sw - w->mean * w->mean, 0.0);
}

/* view_cost of one (pixel, source) pair: 2 when a sample is invalid, 1 without texture. */
/* margin: smallest distance from a sample to the source's border; cells: hash of the texel
 * cells the samples fall in (the bilinear interpolant is smooth while they stay put). */
template <class S>
S pair_cost(const RefWindow& rw, const Win& win, const Image& src, double px, double py,
            const S* u, const S* B, const S* kt, double* margin = nullptr,
            uint64_t* cells = nullptr) {
    S h[9];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) h[r * 3 + c] = B[r * 3 + c] + kt[r] * u[c];
    S ss(0.0), sss(0.0), srs(0.0);
    for (int i = 0; i < win.size(); i++) {
        const double xi = px + win.ox(i), yi = py + win.oy(i);
        const S qz = h[6] * xi + h[7] * yi + h[8];
        if (!(val(qz) > 1e-6)) return S(2.0);
        const S uu = (h[0] * xi + h[1] * yi + h[2]) / qz;
        const S vv = (h[3] * xi + h[4] * yi + h[5]) / qz;
        if (!(val(uu) >= 0.0 && val(vv) >= 0.0 && val(uu) <= src.W - 1 && val(vv) <= src.H - 1))
            return S(2.0);
        if (margin)
            *margin = std::min({*margin, val(uu), val(vv), src.W - 1 - val(uu), src.H - 1 - val(vv)});
        const double x0 = std::floor(val(uu)), y0 = std::floor(val(vv));
        const S fx = uu - x0, fy = vv - y0;
        const int ix0 = (int)x0, iy0 = (int)y0;
        if (cells) *cells = (*cells ^ ((uint64_t)(ix0 * 73856093u) + (uint64_t)iy0 * 19349663ull + (uint64_t)i)) * 1099511628211ull;
        const int ix1 = std::min(ix0 + 1, src.W - 1), iy1 = std::min(iy0 + 1, src.H - 1);
        const double a = src.at(ix0, iy0), b = src.at(ix1, iy0);
        const double c = src.at(ix0, iy1), e = src.at(ix1, iy1);
        const S top = a + fx * (b - a), bot = c + fx * (e - c);
        const S s = top + fy * (bot - top);
        ss = ss + rw.rw[i] * s;
        sss = sss + rw.rw[i] * s * s;
        srs = srs + (rw.rw[i] * rw.rv[i]) * s;
    }
    const S ms = ss / rw.sum;
    S vs = sss / rw.sum - ms * ms;
    if (val(vs) < 0.0) vs = S(0.0);
    const S den = sqrt(rw.var * vs);
    if (val(den) < 1e-5) return S(1.0);
    const S cov = srs / rw.sum - rw.mean * ms;
    const S c = 1.0 - cov / den;
    if (val(c) < 0.0) return S(0.0);
    if (val(c) > 2.0) return S(2.0);
    return c;
}

/* u = K_r^-T n / (d n.ray); false for d <= 0 or n . ray >= -1e-3. */
template <class S>
bool plane_u(const double* vr, double px, double py, const S& d, const S& al, const S& be, S* u) {
    const S sa = sin(al), ca = cos(al), sb = sin(be), cb = cos(be);
    const S nx = sa * cb, ny = sb, nz = -(ca * cb);
    const double fx = vr[0], fy = vr[1], cx = vr[2], cy = vr[3];
    const S m0 = nx / fx, m1 = ny / fy;
    const S m2 = nz - nx * (cx / fx) - ny * (cy / fy);
    const S mu = m0 * px + m1 * py + m2;
    if (!(val(d) > 0.0) || !(val(mu) < -1e-3)) return false;
    const S rho = d * mu;
    u[0] = m0 / rho;
    u[1] = m1 / rho;
    u[2] = m2 / rho;
    return true;
}

int ncc_impl(const orc_stereo_args* a, const double* planes, const double* deltas,
             const double* weights, double* cost, double* grad_planes, double* grad_deltas,
             double* margin, uint64_t* cells) {
    if (!a || !planes || a->n_sources <= 0 || a->n_sources > 8) return 1;
    const int nsrc = a->n_sources;
    int W, H;
    size_t roff;
    view_geometry(a, a->ref, &W, &H, &roff);
    const Image ref{a->images + roff, W, H};
    Win win;
    win.n = a->win_n > 0 ? a->win_n : 6;
    win.dil = a->win_dil > 0 ? a->win_dil : 2;
    win.half = ((win.n - 1) * win.dil) / 2;
    std::vector<Image> srcs(nsrc);
    for (int k = 0; k < nsrc; k++) {
        int w, h;
        size_t o;
        view_geometry(a, a->sources[k], &w, &h, &o);
        srcs[k] = Image{a->images + o, w, h};
    }
    const double* vr = a->views + (size_t)a->ref * ORC_VIEW_DOUBLES;
    std::vector<double> zero(6 * (size_t)a->n_views, 0.0);
    const double* del = deltas ? deltas : zero.data();
    /* constant homographies for the cost and plane passes */
    double Bc[8][9], ktc[8][3];
    for (int k = 0; k < nsrc; k++) {
        const double* vs = a->views + (size_t)a->sources[k] * ORC_VIEW_DOUBLES;
        pair_homography<double>(vr, vs, del + 6 * a->ref, del + 6 * a->sources[k], Bc[k], ktc[k]);
    }
    int threads = a->threads;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#else
    threads = 1;
#endif
    std::vector<double> gacc((size_t)threads * 12 * nsrc, 0.0);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
#endif
    for (int y = 0; y < H; y++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        RefWindow rw;
        for (int x = 0; x < W; x++) {
            const size_t i = (size_t)y * W + x;
            ref_window(ref, win, x, y, &rw);
            const double px = x, py = y;
            const double wgt = weights ? weights[i] : 1.0;
            if (!grad_planes) {
                /* cost only, plain FP64 */
                double u[3];
                const bool ok = plane_u<double>(vr, px, py, planes[i * 3], planes[i * 3 + 1],
                                                planes[i * 3 + 2], u);
                double total = 0.0, mg = 1e30;
                uint64_t cl = 1469598103934665603ull;
                for (int k = 0; k < nsrc; k++) {
                    double c = 2.0;
                    if (ok) c = pair_cost<double>(rw, win, srcs[k], px, py, u, Bc[k], ktc[k], &mg, &cl);
                    if (c == 2.0 || c == 1.0) mg = -1.0;
                    total += c;
                }
                if (cost) cost[i] = total;
                if (margin) margin[i] = ok ? mg : -1.0;
                if (cells) cells[i] = cl;
            }
            if (grad_planes) {
            /* cost and plane gradient: tangents (d, a, b) */
            const Dual<3> d = seed_dual<3>(planes[i * 3], 0);
            const Dual<3> al = seed_dual<3>(planes[i * 3 + 1], 1);
            const Dual<3> be = seed_dual<3>(planes[i * 3 + 2], 2);
            Dual<3> u[3];
            const bool ok = plane_u(vr, px, py, d, al, be, u);
            Dual<3> total(0.0);
            for (int k = 0; k < nsrc; k++) {
                if (!ok) {
                    total = total + 2.0;
                    continue;
                }
                Dual<3> B[9], kt[3];
                for (int j = 0; j < 9; j++) B[j] = Bc[k][j];
                for (int j = 0; j < 3; j++) kt[j] = ktc[k][j];
                total = total + pair_cost(rw, win, srcs[k], px, py, u, B, kt);
            }
            if (cost) cost[i] = total.v;
            for (int j = 0; j < 3; j++) grad_planes[i * 3 + j] = wgt * total.d[j];
            }
            if (!grad_deltas) continue;
            /* pose gradient: tangents (reference increment, source increment) */
            double uc[3];
            if (!plane_u<double>(vr, px, py, planes[i * 3], planes[i * 3 + 1], planes[i * 3 + 2], uc))
                continue;
            Dual<12> u12[3];
            for (int j = 0; j < 3; j++) u12[j] = uc[j];
            for (int k = 0; k < nsrc; k++) {
                Dual<12> dr[6], ds[6];
                for (int j = 0; j < 6; j++) {
                    dr[j] = seed_dual<12>(del[6 * a->ref + j], j);
                    ds[j] = seed_dual<12>(del[6 * a->sources[k] + j], 6 + j);
                }
                const double* vs = a->views + (size_t)a->sources[k] * ORC_VIEW_DOUBLES;
                Dual<12> B[9], kt[3];
                pair_homography(vr, vs, dr, ds, B, kt);
                const Dual<12> c = pair_cost(rw, win, srcs[k], px, py, u12, B, kt);
                double* g = gacc.data() + ((size_t)tid * nsrc + k) * 12;
                for (int j = 0; j < 12; j++) g[j] += wgt * c.d[j];
            }
        }
    }
    if (grad_deltas) {
        for (int t = 0; t < threads; t++)
            for (int k = 0; k < nsrc; k++) {
                const double* g = gacc.data() + ((size_t)t * nsrc + k) * 12;
                for (int j = 0; j < 6; j++) {
                    grad_deltas[6 * a->ref + j] += g[j];
                    grad_deltas[6 * a->sources[k] + j] += g[6 + j];
                }
            }
    }
    return 0;
}

/* ---- TSDF ---- */

/* unpack_normal (depth-packing.wgsl.ts:3-19) in FP64 */
void normal_of(uint32_t packed, double* n) {
    double ex = ((double)((packed >> 16) & 63u) / 63.0) * 2.0 - 1.0;
    double ey = ((double)((packed >> 22) & 63u) / 63.0) * 2.0 - 1.0;
    double ez = (1.0 - std::fabs(ex)) - std::fabs(ey);
    if (ez < 0.0) {
        double sx = ex >= 0.0 ? 1.0 : -1.0, sy = ey >= 0.0 ? 1.0 : -1.0;
        double nx = (1.0 - std::fabs(ey)) * sx, ny = (1.0 - std::fabs(ex)) * sy;
        ex = nx;
        ey = ny;
    }
    const double il = 1.0 / std::sqrt(ex * ex + ey * ey + ez * ez);
    n[0] = ex * il;
    n[1] = ey * il;
    n[2] = ez * il;
}

/* One voxel: tangents (depth of its pixel, T0, W0). */
void tsdf_voxel(const orc_tsdf_desc* d, const orc_tsdf_view* v, const uint32_t* packed,
                const double* depth, int gx, int gy, int gz, size_t idx, const double* tsdf_in,
                const double* weight_in, double* tsdf_out, double* weight_out, const double* gT,
                const double* gW, double* grad_depth, double* grad_tsdf_in, double* grad_weight_in) {
    const double T0v = tsdf_in[idx], W0v = weight_in[idx];
    const double gt = gT ? gT[idx] : 0.0, gw = gW ? gW[idx] : 0.0;
    auto passthrough = [&]() {
        if (tsdf_out) tsdf_out[idx] = T0v;
        if (weight_out) weight_out[idx] = W0v;
        if (grad_tsdf_in) grad_tsdf_in[idx] = gt;
        if (grad_weight_in) grad_weight_in[idx] = d->weight_q8 ? 0.0 : gw;
    };
    const double wx = (gx + 0.5) * d->voxel + d->origin[0];
    const double wy = (gy + 0.5) * d->voxel + d->origin[1];
    const double wz = (gz + 0.5) * d->voxel + d->origin[2];
    const double* R = v->R;
    const double cam[3] = {R[0] * wx + R[1] * wy + R[2] * wz + v->t[0],
                           R[3] * wx + R[4] * wy + R[5] * wz + v->t[1],
                           R[6] * wx + R[7] * wy + R[8] * wz + v->t[2]};
    /* the shader's f32 constants, as in the FP64 integrate oracle */
    if (!(cam[2] > (double)0.01f)) return passthrough();
    const double rx = std::rint(v->k[0] * cam[0] / cam[2] + v->k[2]);
    const double ry = std::rint(v->k[1] * cam[1] / cam[2] + v->k[3]);
    if (!(rx >= 0.0 && ry >= 0.0 && rx < d->width && ry < d->height)) return passthrough();
    const size_t pix = (size_t)ry * d->width + (size_t)rx;
    const uint32_t pk = packed[pix];
    const double dpk = (double)orc_unpack_depth(pk);
    Dual<3> dep(0.0), w(0.0);
    bool stereo = dpk > 0.0;
    if (stereo) {
        dep = seed_dual<3>(depth[pix], 0);
        double n[3];
        normal_of(pk, n);
        const double cl = std::sqrt(cam[0] * cam[0] + cam[1] * cam[1] + cam[2] * cam[2]);
        const double cosang = std::fabs((n[0] * cam[0] + n[1] * cam[1] + n[2] * cam[2]) / cl);
        w = std::max((double)0.2f, cosang);
        if (v->confidence > 0.0) {
            const double c = (double)(pk >> 28) / 8.0;
            Dual<3> r = v->confidence / dep;
            if (r.v <= 0.5) r = Dual<3>(0.5);
            else if (r.v >= 2.0) r = Dual<3>(2.0);
            w = w * (std::max((double)0.15f, (1.0 - c) * (1.0 - c)) * r * r);
        }
    } else {
        dep = v->prior ? (double)v->prior[pix] : 0.0;
        w = d->prior_weight;
    }
    if (!(dep.v > 0.0)) return passthrough();
    const Dual<3> sdf = dep - cam[2];
    if (sdf.v < -d->truncation) return passthrough();
    Dual<3> obs = sdf / d->truncation;
    if (obs.v > 1.0) obs = Dual<3>(1.0);
    const Dual<3> T0 = seed_dual<3>(T0v, 1);
    const Dual<3> W0 = seed_dual<3>(W0v, 2);
    Dual<3> T1, W1;
    if (d->weight_q8) {
        const double wi = std::rint(w.v * 256.0);
        if (wi == 0.0) return passthrough();
        const Dual<3> wf(wi / 256.0);
        const Dual<3> W0c(W0v);  /* integer weights: no tangent */
        T1 = (T0 * W0c + obs * wf) / (W0c + wf);
        W1 = std::min(std::rint(W0v * 256.0) + wi, std::rint(d->max_weight * 256.0)) / 256.0;
    } else {
        T1 = (T0 * W0 + obs * w) / (W0 + w);
        const Dual<3> sum = W0 + w;
        W1 = sum.v < d->max_weight ? sum : Dual<3>(d->max_weight);
    }
    if (tsdf_out) tsdf_out[idx] = T1.v;
    if (weight_out) weight_out[idx] = W1.v;
    if (grad_depth && stereo) {
        const double gd = gt * T1.d[0] + gw * W1.d[0];
#ifdef _OPENMP
#pragma omp atomic
#endif
        grad_depth[pix] += gd;
    }
    if (grad_tsdf_in) grad_tsdf_in[idx] = gt * T1.d[1] + gw * W1.d[1];
    if (grad_weight_in) grad_weight_in[idx] = d->weight_q8 ? 0.0 : gt * T1.d[2] + gw * W1.d[2];
}

int tsdf_depth_impl(const orc_tsdf_desc* d, const orc_tsdf_view* v, const uint32_t* packed,
                    const double* depth, const double* tsdf_in, const double* weight_in,
                    double* tsdf_out, double* weight_out, const double* gT, const double* gW,
                    double* grad_depth, double* grad_tsdf_in, double* grad_weight_in,
                    int threads) {
    if (!d || !v || !packed || !depth || !tsdf_in || !weight_in) return 1;
    long bricks;
    int nb[3] = {0, 0, 0};
    if (d->dense) {
        for (int i = 0; i < 3; i++) nb[i] = (d->dims[i] + 7) / 8;
        bricks = (long)nb[0] * nb[1] * nb[2];
    } else {
        bricks = d->count;
    }
    std::vector<uint8_t> vis((size_t)bricks);
    orc_tsdf_visible(d, v, vis.data());
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
    for (long b = 0; b < bricks; b++) {
        int bx, by, bz;
        if (d->dense) {
            bx = (int)(b % nb[0]);
            by = (int)((b / nb[0]) % nb[1]);
            bz = (int)(b / ((long)nb[0] * nb[1]));
        } else {
            bx = d->coords[b * 4];
            by = d->coords[b * 4 + 1];
            bz = d->coords[b * 4 + 2];
        }
        for (int l = 0; l < 512; l++) {
            const int gx = bx * 8 + (l & 7), gy = by * 8 + ((l >> 3) & 7), gz = bz * 8 + (l >> 6);
            size_t idx;
            if (d->dense) {
                if (gx >= d->dims[0] || gy >= d->dims[1] || gz >= d->dims[2]) continue;
                idx = ((size_t)gz * d->dims[1] + gy) * d->dims[0] + gx;
            } else {
                idx = (size_t)b * 512 + l;
            }
            if (vis[b]) {
                tsdf_voxel(d, v, packed, depth, gx, gy, gz, idx, tsdf_in, weight_in, tsdf_out,
                           weight_out, gT, gW, grad_depth, grad_tsdf_in, grad_weight_in);
            } else {
                if (tsdf_out) tsdf_out[idx] = tsdf_in[idx];
                if (weight_out) weight_out[idx] = weight_in[idx];
                if (grad_tsdf_in) grad_tsdf_in[idx] = gT ? gT[idx] : 0.0;
                if (grad_weight_in) grad_weight_in[idx] = (gW && !d->weight_q8) ? gW[idx] : 0.0;
            }
        }
    }
    return 0;
}

}  // namespace

extern "C" {

int orc64_ncc_grad(const orc_stereo_args* a, const double* planes, const double* deltas,
                   const double* weights, double* cost, double* grad_planes, double* grad_deltas,
                   double* margin, uint64_t* cells) {
    return ncc_impl(a, planes, deltas, weights, cost, grad_planes, grad_deltas, margin, cells);
}

int orc64_tsdf_depth(const orc_tsdf_desc* d, const orc_tsdf_view* v, const uint32_t* packed,
                     const double* depth, const double* tsdf_in, const double* weight_in,
                     double* tsdf_out, double* weight_out, const double* grad_tsdf_out,
                     const double* grad_weight_out, double* grad_depth, double* grad_tsdf_in,
                     double* grad_weight_in, int32_t threads) {
    return tsdf_depth_impl(d, v, packed, depth, tsdf_in, weight_in, tsdf_out, weight_out,
                           grad_tsdf_out, grad_weight_out, grad_depth, grad_tsdf_in, grad_weight_in,
                           threads);
}

}  // extern "C"
