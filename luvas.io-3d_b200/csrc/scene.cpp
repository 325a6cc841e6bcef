/*
 * Seeded synthetic scenes for the dense-reconstruction path (host code, OpenMP).
 *
 * The reference renders its verification scenes with a GLSL ray caster in WebGL
 * (frontend/tools/scene-renderer.ts) and keeps analytic JS twins of the same scene for ground
 * truth (frontend/tools/synthetic-scene.ts).  This file is the CPU ray caster of the two scenes
 * the dense path is measured on:
 *
 *   sphere scene  unit sphere centred at the origin resting on the plane y = -1, both textured
 *                 by a solid 3-octave value noise in [0, 1]; the sky is a flat 0.5.
 *   room scene    the inside of a 4 x 3 x 2.5 m box (x in [-2, 2], y in [-1.25, 1.25] with the
 *                 floor at y = -1.25, z in [-1.5, 1.5]) holding axis-aligned textured cuboids.
 *
 * Texture: value noise on an integer lattice with smoothstep interpolation; lattice values come
 * from the PCG hash of the lattice coordinates and the seed.  Octave o uses frequency
 * FREQ[o] per metre and amplitude AMP[o]; the amplitudes sum to 1 so the texture stays in [0, 1].
 *
 * Images are 2 x 2 supersampled (sub-pixel offsets +-0.25); ground-truth depth is the camera-z
 * depth of the pixel-centre ray (0 where the ray escapes).  Cameras use computer-vision axes
 * (x right, y down, z forward) with x_cam = R X + t.  Gaussian pixel noise (Box-Muller on the
 * same hash) is added when sigma > 0.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "l3d_fmath.h"

namespace {

const double FREQ[3] = {24.0, 57.0, 131.0};
const double AMP[3] = {0.5, 0.3, 0.2};

inline double lattice(int64_t x, int64_t y, int64_t z, uint32_t seed) {
    uint32_t h = l3d_pcg((uint32_t)x * 0x8da6b343u ^ seed);
    h = l3d_pcg(h ^ (uint32_t)y * 0xd8163841u);
    h = l3d_pcg(h ^ (uint32_t)z * 0xcb1ab31fu);
    return (double)(h >> 8) / 16777216.0;
}

inline double smooth(double t) { return t * t * (3.0 - 2.0 * t); }

double value_noise(double x, double y, double z, uint32_t seed) {
    double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    int64_t ix = (int64_t)fx, iy = (int64_t)fy, iz = (int64_t)fz;
    double wx = smooth(x - fx), wy = smooth(y - fy), wz = smooth(z - fz);
    double c[2][2][2];
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2; b++)
            for (int d = 0; d < 2; d++) c[a][b][d] = lattice(ix + a, iy + b, iz + d, seed);
    double x00 = c[0][0][0] + (c[1][0][0] - c[0][0][0]) * wx;
    double x10 = c[0][1][0] + (c[1][1][0] - c[0][1][0]) * wx;
    double x01 = c[0][0][1] + (c[1][0][1] - c[0][0][1]) * wx;
    double x11 = c[0][1][1] + (c[1][1][1] - c[0][1][1]) * wx;
    double y0 = x00 + (x10 - x00) * wy;
    double y1 = x01 + (x11 - x01) * wy;
    return y0 + (y1 - y0) * wz;
}

double texture(const double* p, uint32_t seed) {
    double v = 0.0;
    for (int o = 0; o < 3; o++)
        v += AMP[o] * value_noise(p[0] * FREQ[o] + 17.0 * o, p[1] * FREQ[o] + 31.0 * o,
                                  p[2] * FREQ[o] + 7.0 * o, seed + 0x9e3779b9u * (uint32_t)o);
    return v;
}

struct Hit {
    double t;
    int object;   /* -1: none */
};

/* ---- sphere scene ---- */
Hit trace_sphere(const double* o, const double* d) {
    Hit best = {INFINITY, -1};
    /* sphere |x| = 1 */
    double b = o[0] * d[0] + o[1] * d[1] + o[2] * d[2];
    double c = o[0] * o[0] + o[1] * o[1] + o[2] * o[2] - 1.0;
    double h = b * b - c;
    if (h > 0) {
        double s = std::sqrt(h);
        double t = -b - s;
        if (t <= 1e-9) t = -b + s;
        if (t > 1e-9) best = {t, 0};
    }
    /* plane y = -1 */
    if (d[1] < 0) {
        double t = (-1.0 - o[1]) / d[1];
        if (t > 1e-9 && t < best.t) best = {t, 1};
    }
    return best;
}

/* ---- room scene ---- */
struct Box {
    double lo[3], hi[3];
};

Hit trace_boxes(const double* o, const double* d, const Box* boxes, int n) {
    Hit best = {INFINITY, -1};
    /* the room: the ray starts inside, take the exit distance */
    {
        const Box& r = boxes[0];
        double tmax = INFINITY;
        for (int k = 0; k < 3; k++) {
            if (d[k] == 0) continue;
            double t0 = (r.lo[k] - o[k]) / d[k], t1 = (r.hi[k] - o[k]) / d[k];
            tmax = std::fmin(tmax, std::fmax(t0, t1));
        }
        if (tmax > 1e-9) best = {tmax, 0};
    }
    for (int i = 1; i < n; i++) {
        const Box& b = boxes[i];
        double enter = -INFINITY, leave = INFINITY;
        for (int k = 0; k < 3; k++) {
            double inv = 1.0 / d[k];
            double t0 = (b.lo[k] - o[k]) * inv, t1 = (b.hi[k] - o[k]) * inv;
            enter = std::fmax(enter, std::fmin(t0, t1));
            leave = std::fmin(leave, std::fmax(t0, t1));
        }
        if (enter > 1e-9 && enter < leave && enter < best.t) best = {enter, i};
    }
    return best;
}

inline double gauss(uint32_t a, uint32_t b) {
    double u1 = ((double)(l3d_pcg(a) >> 8) + 0.5) / 16777216.0;
    double u2 = (double)(l3d_pcg(b ^ 0x68bc21ebu) >> 8) / 16777216.0;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

template <typename Trace>
void render(const double* views, const int32_t* sizes, int n_views, uint32_t seed,
            double sigma, float* images, float* depth, Trace trace) {
    std::vector<size_t> offsets(n_views + 1, 0);
    for (int v = 0; v < n_views; v++)
        offsets[v + 1] = offsets[v] + (size_t)sizes[2 * v] * sizes[2 * v + 1];
    for (int v = 0; v < n_views; v++) {
        const double* cam = views + (size_t)v * 16;
        const double* R = cam + 4;
        const double* t = cam + 13;
        /* camera centre C = -R^T t */
        double C[3];
        for (int j = 0; j < 3; j++) C[j] = -(R[j] * t[0] + R[3 + j] * t[1] + R[6 + j] * t[2]);
        const int W = sizes[2 * v], H = sizes[2 * v + 1];
        float* img = images + offsets[v];
        float* dep = depth ? depth + offsets[v] : nullptr;
#pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < H; y++) {
            for (int x = 0; x < W; x++) {
                double acc = 0.0;
                for (int s = 0; s <= 4; s++) {
                    double u = x + (s == 4 ? 0.0 : ((s & 1) ? 0.25 : -0.25));
                    double w = y + (s == 4 ? 0.0 : ((s & 2) ? 0.25 : -0.25));
                    double rc[3] = {(u - cam[2]) / cam[0], (w - cam[3]) / cam[1], 1.0};
                    double d[3];
                    for (int j = 0; j < 3; j++) d[j] = R[j] * rc[0] + R[3 + j] * rc[1] + R[6 + j] * rc[2];
                    double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                    for (int j = 0; j < 3; j++) d[j] /= len;
                    Hit h = trace(C, d);
                    if (s == 4) {
                        /* camera-z depth of the centre ray */
                        if (dep) dep[(size_t)y * W + x] = h.object < 0 ? 0.0f : (float)(h.t / len);
                        break;
                    }
                    double value = 0.5;
                    if (h.object >= 0) {
                        double p[3] = {C[0] + d[0] * h.t, C[1] + d[1] * h.t, C[2] + d[2] * h.t};
                        value = texture(p, seed + 0x51ed270bu * (uint32_t)h.object);
                    }
                    acc += value;
                }
                double value = acc * 0.25;
                if (sigma > 0) {
                    uint32_t key = (uint32_t)(offsets[v] + (size_t)y * W + x);
                    value += sigma * gauss(key * 2654435761u ^ seed, key ^ (seed * 40503u));
                }
                img[(size_t)y * W + x] = (float)value;
            }
        }
    }
}

}  // namespace

extern "C" {

/* Renders the sphere scene.  views: n_views * 16 doubles (fx fy cx cy | R | t); sizes: n_views
 * pairs (width, height); images and depth (nullable) are concatenated per view. */
int l3d_scene_sphere(const double* views, const int32_t* sizes, int32_t n_views, uint32_t seed,
                     double sigma, float* images, float* depth) {
    if (!views || !sizes || n_views <= 0 || !images) return 1;
    render(views, sizes, n_views, seed, sigma, images, depth,
           [](const double* o, const double* d) { return trace_sphere(o, d); });
    return 0;
}

/* Renders the room scene with n_boxes cuboids (boxes: n_boxes * 6 doubles lo.xyz hi.xyz). */
int l3d_scene_room(const double* views, const int32_t* sizes, int32_t n_views, uint32_t seed,
                   double sigma, const double* boxes, int32_t n_boxes, float* images, float* depth) {
    if (!views || !sizes || n_views <= 0 || !images || n_boxes < 0) return 1;
    std::vector<Box> all(n_boxes + 1);
    all[0] = {{-2.0, -1.25, -1.5}, {2.0, 1.25, 1.5}};
    for (int i = 0; i < n_boxes; i++)
        for (int k = 0; k < 3; k++) {
            all[i + 1].lo[k] = boxes[i * 6 + k];
            all[i + 1].hi[k] = boxes[i * 6 + 3 + k];
        }
    const Box* b = all.data();
    int n = n_boxes + 1;
    render(views, sizes, n_views, seed, sigma, images, depth,
           [b, n](const double* o, const double* d) { return trace_boxes(o, d, b, n); });
    return 0;
}

}  // extern "C"
