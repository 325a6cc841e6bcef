/*
 * CPU oracle of the dense point cloud: depth-map fusion into the cell-averaging accumulator.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the product library never links or calls it.
 *
 * Restates, in the reference's order and number formats:
 *   frontend/src/app/vision/fusion/depth-fusion.ts:42-74        addDepthMap (decode, world point,
 *                                                                rotated normal, thumbnail colour)
 *   frontend/src/app/vision/fusion/point-accumulator.ts:16-147  PointAccumulator (open-addressing
 *                                                                hash on the integer cell, f32
 *                                                                sums, growth at 60 % load,
 *                                                                coarsen by re-binning cell means,
 *                                                                cloud(minSupport))
 *   frontend/src/app/vision/mvs/depth-maps.ts:66-85              unpackDepthSample
 * JavaScript numbers are doubles; Float32Array / Uint32Array / Int32Array elements round or wrap
 * on store, which the restatement reproduces (f32 sums: sums = f32(double(sums) + x)).
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

constexpr int32_t EMPTY = 0x7fffffff;

/* Math.imul(a, b): the low 32 bits of the product as int32 */
inline int32_t imul(int32_t a, int32_t b) {
    return (int32_t)((uint32_t)a * (uint32_t)b);
}

uint32_t hash3(int32_t x, int32_t y, int32_t z) {
    return (uint32_t)(imul(x, 73856093) ^ imul(y, 19349663) ^ imul(z, 83492791));
}

/* ToInt32 of a finite double (Int32Array store) */
inline int32_t to_int32(double v) {
    double t = std::trunc(v);
    double m = std::fmod(t, 4294967296.0);
    if (m < 0) m += 4294967296.0;
    uint32_t u = (uint32_t)m;
    return (int32_t)u;
}

/* ToUint8 of a double (Uint8Array store) */
inline uint8_t to_uint8(double v) {
    if (!std::isfinite(v)) return 0;
    double t = std::trunc(v);
    double m = std::fmod(t, 256.0);
    if (m < 0) m += 256.0;
    return (uint8_t)m;
}

struct Accumulator {
    double cell;
    int32_t capacity = 1 << 16;
    std::vector<int32_t> keys;
    std::vector<float> sums;
    std::vector<uint32_t> counts;
    int32_t used = 0;

    explicit Accumulator(double c) : cell(c) {
        keys.assign((size_t)capacity * 3, EMPTY);
        sums.assign((size_t)capacity * 9, 0.0f);
        counts.assign((size_t)capacity, 0u);
    }

    int32_t slot_of(int32_t ix, int32_t iy, int32_t iz) {
        if ((double)used * 10 > (double)capacity * 6) rebuild(capacity * 2, cell);
        const int32_t mask = capacity - 1;
        int32_t slot = (int32_t)(hash3(ix, iy, iz) & (uint32_t)mask);
        for (;;) {
            const size_t k = (size_t)slot * 3;
            if (keys[k] == EMPTY) {
                keys[k] = ix;
                keys[k + 1] = iy;
                keys[k + 2] = iz;
                used++;
                return slot;
            }
            if (keys[k] == ix && keys[k + 1] == iy && keys[k + 2] == iz) return slot;
            slot = (slot + 1) & mask;
        }
    }

    void add(double x, double y, double z, double nx, double ny, double nz, double r, double g,
             double b) {
        const int32_t slot = slot_of(to_int32(std::floor(x / cell)), to_int32(std::floor(y / cell)),
                                     to_int32(std::floor(z / cell)));
        float* s = &sums[(size_t)slot * 9];
        const double v[9] = {x, y, z, nx, ny, nz, r, g, b};
        for (int i = 0; i < 9; i++) s[i] = (float)((double)s[i] + v[i]);
        counts[slot]++;
    }

    void rebuild(int32_t cap, double c) {
        std::vector<int32_t> ok = std::move(keys);
        std::vector<float> os = std::move(sums);
        std::vector<uint32_t> oc = std::move(counts);
        const int32_t old = capacity;
        capacity = cap;
        cell = c;
        keys.assign((size_t)cap * 3, EMPTY);
        sums.assign((size_t)cap * 9, 0.0f);
        counts.assign((size_t)cap, 0u);
        used = 0;
        for (int32_t s = 0; s < old; s++) {
            if (ok[(size_t)s * 3] == EMPTY) continue;
            const double n = (double)oc[s];
            const float* src = &os[(size_t)s * 9];
            const int32_t slot = slot_of(to_int32(std::floor((double)src[0] / n / c)),
                                         to_int32(std::floor((double)src[1] / n / c)),
                                         to_int32(std::floor((double)src[2] / n / c)));
            float* dst = &sums[(size_t)slot * 9];
            for (int i = 0; i < 9; i++) dst[i] = (float)((double)dst[i] + (double)src[i]);
            counts[slot] += oc[s];
        }
    }
};

/* unpackDepthSample (depth-maps.ts:66-85) */
bool unpack_sample(uint32_t value, double* out) {
    if (value == 0) return false;
    const double d = (double)orc_f16_to_f32(value & 0xffffu);
    if (!(d > 0)) return false;
    const double ex = ((double)((value >> 16) & 63u) / 63.0) * 2.0 - 1.0;
    const double ey = ((double)((value >> 22) & 63u) / 63.0) * 2.0 - 1.0;
    double nx = ex, ny = ey;
    const double nz = 1.0 - std::fabs(ex) - std::fabs(ey);
    if (nz < 0) {
        nx = (1.0 - std::fabs(ey)) * (ex >= 0 ? 1.0 : -1.0);
        ny = (1.0 - std::fabs(ex)) * (ey >= 0 ? 1.0 : -1.0);
    }
    double length = std::sqrt(nx * nx + ny * ny + nz * nz);
    if (!(length != 0.0)) length = 1.0;
    out[0] = d;
    out[1] = nx / length;
    out[2] = ny / length;
    out[3] = nz / length;
    return true;
}

}  // namespace

struct orc_cloud {
    Accumulator acc;
    explicit orc_cloud(double c) : acc(c) {}
};

extern "C" {

orc_cloud* orc_cloud_create(double cell) { return new orc_cloud(cell); }
void orc_cloud_destroy(orc_cloud* c) { delete c; }

void orc_cloud_add_point(orc_cloud* c, const double* p9) {
    c->acc.add(p9[0], p9[1], p9[2], p9[3], p9[4], p9[5], p9[6], p9[7], p9[8]);
}

/* addDepthMap (depth-fusion.ts:42-74): view = fx fy cx cy | R (world -> camera) | t */
void orc_cloud_add_map(orc_cloud* c, const uint32_t* packed, int32_t width, int32_t height,
                       const double* view, const uint8_t* rgb, int32_t tw, int32_t th) {
    const double fx = view[0], fy = view[1], cx = view[2], cy = view[3];
    const double* R = view + 4;
    const double* t = view + 13;
    const double sx = (double)tw / width, sy = (double)th / height;
    double s[4];
    for (int32_t y = 0; y < height; y++)
        for (int32_t x = 0; x < width; x++) {
            if (!unpack_sample(packed[(size_t)y * width + x], s)) continue;
            const double d = s[0];
            const double pc[3] = {((x - cx) / fx) * d, ((y - cy) / fy) * d, d};
            const double v[3] = {pc[0] - t[0], pc[1] - t[1], pc[2] - t[2]};
            /* fromCamera / applyTransposed3 (camera.ts:57-59, mat3.ts:32-38) */
            const double wx = R[0] * v[0] + R[3] * v[1] + R[6] * v[2];
            const double wy = R[1] * v[0] + R[4] * v[1] + R[7] * v[2];
            const double wz = R[2] * v[0] + R[5] * v[1] + R[8] * v[2];
            const double nx = R[0] * s[1] + R[3] * s[2] + R[6] * s[3];
            const double ny = R[1] * s[1] + R[4] * s[2] + R[7] * s[3];
            const double nz = R[2] * s[1] + R[5] * s[2] + R[8] * s[3];
            const int32_t txp = std::min(tw - 1, (int32_t)std::floor((x + 0.5) * sx));
            const int32_t typ = std::min(th - 1, (int32_t)std::floor((y + 0.5) * sy));
            const size_t i = ((size_t)typ * tw + txp) * 3;
            c->acc.add(wx, wy, wz, nx, ny, nz, rgb[i], rgb[i + 1], rgb[i + 2]);
        }
}

void orc_cloud_coarsen(orc_cloud* c, double factor) {
    c->acc.rebuild(c->acc.capacity, c->acc.cell * factor);
}

int32_t orc_cloud_size(const orc_cloud* c) { return c->acc.used; }
double orc_cloud_cell(const orc_cloud* c) { return c->acc.cell; }

/* cloud(minSupport) (point-accumulator.ts:114-143) in slot order, plus each point's cell. */
int32_t orc_cloud_read(const orc_cloud* c, int32_t min_support, float* pos, float* nrm,
                       uint8_t* col, uint16_t* support, int32_t* cells) {
    const Accumulator& a = c->acc;
    int32_t p = 0;
    for (int32_t s = 0; s < a.capacity; s++) {
        if (a.keys[(size_t)s * 3] == EMPTY || a.counts[s] < (uint32_t)min_support) continue;
        if (pos) {
            const double n = (double)a.counts[s];
            const float* o = &a.sums[(size_t)s * 9];
            for (int i = 0; i < 3; i++) pos[p * 3 + i] = (float)((double)o[i] / n);
            double length = std::sqrt((double)o[3] * o[3] + (double)o[4] * o[4] + (double)o[5] * o[5]);
            if (!(length != 0.0)) length = 1.0;
            for (int i = 0; i < 3; i++) nrm[p * 3 + i] = (float)((double)o[3 + i] / length);
            for (int i = 0; i < 3; i++) col[p * 3 + i] = to_uint8((double)o[6 + i] / n);
            support[p] = (uint16_t)std::min<uint32_t>(65535u, a.counts[s]);
            for (int i = 0; i < 3; i++) cells[p * 3 + i] = a.keys[(size_t)s * 3 + i];
        }
        p++;
    }
    return p;
}

}  // extern "C"
