/*
 * CPU oracle of the image preparation steps in front of the stereo stage.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the product library never links or calls it.
 *
 * Restates, in the reference's order and number formats (JavaScript doubles; Float32Array and
 * Uint8Array stores round or truncate):
 *   frontend/src/app/vision/image/gray-image.ts:12-46     rgbaToGray (integer area path, or
 *                                                         f32 luma + resampleArea)
 *   frontend/src/app/vision/image/gray-image.ts:49-82     downsampleRgb (thumbnails)
 *   frontend/src/app/vision/image/gray-image.ts:166-187   downsampleGray
 *   frontend/src/app/vision/image/gray-image.ts:193-239   resampleArea, coverage
 *   frontend/src/app/vision/mvs/depth-maps.ts:9-42        upsampleDepth (phone prior)
 * Math.round is round-half-up: floor(x), plus one when x - floor(x) >= 0.5.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "oracle.h"

namespace {

inline double js_round(double x) {
    const double f = std::floor(x);
    return (x - f >= 0.5) ? f + 1.0 : f;
}

/* ToUint8 of a finite double */
inline uint8_t to_u8(double v) {
    const double t = std::trunc(v);
    double m = std::fmod(t, 256.0);
    if (m < 0) m += 256.0;
    return (uint8_t)m;
}

struct Cover {
    int first;
    std::vector<double> w;
};

/* coverage (gray-image.ts:226-239) */
std::vector<Cover> coverage(int source, int target) {
    const double scale = (double)source / target;
    std::vector<Cover> out((size_t)target);
    for (int t = 0; t < target; t++) {
        const double start = t * scale;
        const double end = std::min((double)source, (t + 1) * scale);
        const int first = (int)std::floor(start);
        out[t].first = first;
        for (int i = first; i < end; i++)
            out[t].w.push_back((std::min(end, (double)(i + 1)) - std::max(start, (double)i)) / scale);
    }
    return out;
}

/* resampleArea (gray-image.ts:193-221) of a source readable as double */
template <typename T>
void resample_area(const T* src, int width, int height, int tw, int th, uint8_t* out) {
    const std::vector<Cover> cols = coverage(width, tw), rows = coverage(height, th);
    std::vector<float> temp((size_t)tw * height);
    for (int y = 0; y < height; y++)
        for (int x = 0; x < tw; x++) {
            double sum = 0;
            for (size_t k = 0; k < cols[x].w.size(); k++)
                sum += cols[x].w[k] * (double)src[(size_t)y * width + cols[x].first + k];
            temp[(size_t)y * tw + x] = (float)sum;
        }
    for (int y = 0; y < th; y++)
        for (int x = 0; x < tw; x++) {
            double sum = 0;
            for (size_t k = 0; k < rows[y].w.size(); k++)
                sum += rows[y].w[k] * (double)temp[(size_t)(rows[y].first + k) * tw + x];
            out[(size_t)y * tw + x] = to_u8(std::min(255.0, js_round(sum)));
        }
}

}  // namespace

extern "C" {

void orc_rgba_to_gray(const uint8_t* rgba, int32_t width, int32_t height, int32_t tw, int32_t th,
                      uint8_t* out) {
    if (width % tw != 0 || height % th != 0) {
        std::vector<float> luma((size_t)width * height);
        for (size_t i = 0; i < luma.size(); i++)
            luma[i] = (float)((77.0 * rgba[i * 4] + 150.0 * rgba[i * 4 + 1] + 29.0 * rgba[i * 4 + 2]) / 256.0);
        resample_area(luma.data(), width, height, tw, th, out);
        return;
    }
    const double sx = (double)width / tw, sy = (double)height / th;
    for (int y = 0; y < th; y++) {
        const int y0 = (int)std::floor(y * sy);
        const int y1 = std::max(y0 + 1, (int)std::floor((y + 1) * sy));
        for (int x = 0; x < tw; x++) {
            const int x0 = (int)std::floor(x * sx);
            const int x1 = std::max(x0 + 1, (int)std::floor((x + 1) * sx));
            double sum = 0;
            for (int yy = y0; yy < y1; yy++)
                for (int xx = x0; xx < x1; xx++) {
                    const size_t i = ((size_t)yy * width + xx) * 4;
                    sum += 77.0 * rgba[i] + 150.0 * rgba[i + 1] + 29.0 * rgba[i + 2];
                }
            out[(size_t)y * tw + x] = to_u8(js_round(sum / (256.0 * (y1 - y0) * (x1 - x0))));
        }
    }
}

void orc_downsample_rgb(const uint8_t* rgba, int32_t width, int32_t height, int32_t tw, int32_t th,
                        uint8_t* out) {
    const double sx = (double)width / tw, sy = (double)height / th;
    for (int y = 0; y < th; y++) {
        const int y0 = (int)std::floor(y * sy);
        const int y1 = std::max(y0 + 1, (int)std::floor((y + 1) * sy));
        for (int x = 0; x < tw; x++) {
            const int x0 = (int)std::floor(x * sx);
            const int x1 = std::max(x0 + 1, (int)std::floor((x + 1) * sx));
            double r = 0, g = 0, b = 0;
            for (int yy = y0; yy < y1; yy++)
                for (int xx = x0; xx < x1; xx++) {
                    const size_t i = ((size_t)yy * width + xx) * 4;
                    r += rgba[i];
                    g += rgba[i + 1];
                    b += rgba[i + 2];
                }
            const double n = (double)(y1 - y0) * (x1 - x0);
            const size_t o = ((size_t)y * tw + x) * 3;
            out[o] = to_u8(r / n);
            out[o + 1] = to_u8(g / n);
            out[o + 2] = to_u8(b / n);
        }
    }
}

void orc_downsample_gray(const uint8_t* gray, int32_t width, int32_t height, int32_t tw, int32_t th,
                         uint8_t* out) {
    if (width % tw != 0 || height % th != 0) {
        resample_area(gray, width, height, tw, th, out);
        return;
    }
    const double sx = (double)width / tw, sy = (double)height / th;
    for (int y = 0; y < th; y++) {
        const int y0 = (int)std::floor(y * sy);
        const int y1 = std::max(y0 + 1, (int)std::floor((y + 1) * sy));
        for (int x = 0; x < tw; x++) {
            const int x0 = (int)std::floor(x * sx);
            const int x1 = std::max(x0 + 1, (int)std::floor((x + 1) * sx));
            double sum = 0;
            for (int yy = y0; yy < y1; yy++)
                for (int xx = x0; xx < x1; xx++) sum += gray[(size_t)yy * width + xx];
            out[(size_t)y * tw + x] = to_u8(js_round(sum / ((double)(y1 - y0) * (x1 - x0))));
        }
    }
}

void orc_upsample_depth(const float* grid, int32_t gw, int32_t gh, int32_t width, int32_t height,
                        float* out) {
    for (int y = 0; y < height; y++) {
        const double gy = std::min((double)(gh - 1), std::max(0.0, ((y + 0.5) / height) * gh - 0.5));
        const int y0 = (int)std::floor(gy);
        const int y1 = std::min(gh - 1, y0 + 1);
        const double wy = gy - y0;
        for (int x = 0; x < width; x++) {
            const double gx = std::min((double)(gw - 1), std::max(0.0, ((x + 0.5) / width) * gw - 0.5));
            const int x0 = (int)std::floor(gx);
            const int x1 = std::min(gw - 1, x0 + 1);
            const double wx = gx - x0;
            const double d[4] = {grid[(size_t)y0 * gw + x0], grid[(size_t)y0 * gw + x1],
                                 grid[(size_t)y1 * gw + x0], grid[(size_t)y1 * gw + x1]};
            const double w[4] = {(1 - wx) * (1 - wy), wx * (1 - wy), (1 - wx) * wy, wx * wy};
            double sum = 0, weight = 0;
            for (int k = 0; k < 4; k++)
                if (d[k] > 0) {
                    sum += d[k] * w[k];
                    weight += w[k];
                }
            out[(size_t)y * width + x] = weight > 0.5 ? (float)(sum / weight) : 0.0f;
        }
    }
}

}  // extern "C"
