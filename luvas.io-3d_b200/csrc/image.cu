/*
 * Image preparation on the device, in front of the stereo stage: RGBA -> gray with area
 * downsampling, RGB thumbnails, gray downsampling, and upsampling of the phone's depth grid into a
 * stereo prior.
 *
 *   frontend/src/app/vision/image/gray-image.ts:12-46    rgbaToGray
 *   frontend/src/app/vision/image/gray-image.ts:49-82    downsampleRgb
 *   frontend/src/app/vision/image/gray-image.ts:166-187  downsampleGray
 *   frontend/src/app/vision/image/gray-image.ts:193-239  resampleArea, coverage
 *   frontend/src/app/vision/mvs/depth-maps.ts:9-42       upsampleDepth
 * One thread per output pixel (per row-pass pixel for the separable area filter).  Arithmetic
 * follows the reference: integer luma sums, FP64 weights and sums, f32 intermediate rows,
 * round-half-up (floor, plus one when the fraction is at least 1/2) and truncating byte stores.
 * The area filter's per-pixel coverage tables (first source pixel and weights) are computed on
 * the host in FP64 like the reference's coverage().
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "l3d_internal.h"

namespace {

__device__ __forceinline__ double js_round(double x) {
    const double f = floor(x);
    return (x - f >= 0.5) ? f + 1.0 : f;
}

__device__ __forceinline__ uint8_t to_u8(double v) {
    const double t = trunc(v);
    return (uint8_t)(t - 256.0 * floor(t / 256.0));
}

__device__ __forceinline__ void block_bounds(int t, double s, int* a, int* b) {
    *a = (int)floor(t * s);
    *b = max(*a + 1, (int)floor((t + 1) * s));
}

/* rgbaToGray, integer-ratio path (gray-image.ts:26-45) */
__global__ void k_gray_blocks(const uint8_t* __restrict__ rgba, int W, int H, int tw, int th,
                              uint8_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tw * th) return;
    const int x = i % tw, y = i / tw;
    int x0, x1, y0, y1;
    block_bounds(x, (double)W / tw, &x0, &x1);
    block_bounds(y, (double)H / th, &y0, &y1);
    double sum = 0.0;
    for (int yy = y0; yy < y1; yy++)
        for (int xx = x0; xx < x1; xx++) {
            const uint8_t* p = rgba + ((size_t)yy * W + xx) * 4;
            sum += (double)(77 * p[0] + 150 * p[1] + 29 * p[2]);
        }
    out[i] = to_u8(js_round(sum / (256.0 * (y1 - y0) * (x1 - x0))));
}

/* source pixel as the area filter reads it: u8 gray, f32, or the f32 luma of an RGBA pixel
 * (rgbaToGray's Float32Array store, gray-image.ts:20-23) computed on the fly */
template <int KIND>
__device__ __forceinline__ double area_src(const void* __restrict__ src, long long i) {
    if (KIND == 0) return (double)((const uint8_t*)src)[i];
    if (KIND == 1) return (double)((const float*)src)[i];
    const uint8_t* p = (const uint8_t*)src + i * 4;
    return (double)(float)((double)(77 * p[0] + 150 * p[1] + 29 * p[2]) / 256.0);
}

/* resampleArea pass 1 (gray-image.ts:203-212): rows of the source -> f32 temp (tw per row).
 * cover: per target column, first source pixel and `k` weights (stride `kmax`). */
template <int KIND>
__global__ void k_area_rows(const void* __restrict__ src, int W, int H, int tw,
                            const int* __restrict__ first, const int* __restrict__ count,
                            const double* __restrict__ weights, int kmax, float* __restrict__ temp) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)tw * H) return;
    const int x = (int)(i % tw);
    const long long y = i / tw;
    const long long row = y * W + first[x];
    const double* w = weights + (size_t)x * kmax;
    double sum = 0.0;
    for (int k = 0; k < count[x]; k++) sum += w[k] * area_src<KIND>(src, row + k);
    temp[i] = (float)sum;
}

/* resampleArea pass 2 (gray-image.ts:213-220): columns of the temp -> bytes */
__global__ void k_area_cols(const float* __restrict__ temp, int tw, int th,
                            const int* __restrict__ first, const int* __restrict__ count,
                            const double* __restrict__ weights, int kmax, uint8_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tw * th) return;
    const int x = i % tw, y = i / tw;
    const double* w = weights + (size_t)y * kmax;
    double sum = 0.0;
    for (int k = 0; k < count[y]; k++) sum += w[k] * (double)temp[(size_t)(first[y] + k) * tw + x];
    out[i] = to_u8(fmin(255.0, js_round(sum)));
}

/* downsampleRgb (gray-image.ts:49-82) */
__global__ void k_rgb_blocks(const uint8_t* __restrict__ rgba, int W, int H, int tw, int th,
                             uint8_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tw * th) return;
    const int x = i % tw, y = i / tw;
    int x0, x1, y0, y1;
    block_bounds(x, (double)W / tw, &x0, &x1);
    block_bounds(y, (double)H / th, &y0, &y1);
    double r = 0.0, g = 0.0, b = 0.0;
    for (int yy = y0; yy < y1; yy++)
        for (int xx = x0; xx < x1; xx++) {
            const uint8_t* p = rgba + ((size_t)yy * W + xx) * 4;
            r += p[0];
            g += p[1];
            b += p[2];
        }
    const double n = (double)(y1 - y0) * (x1 - x0);
    out[(size_t)i * 3] = to_u8(r / n);
    out[(size_t)i * 3 + 1] = to_u8(g / n);
    out[(size_t)i * 3 + 2] = to_u8(b / n);
}

/* downsampleGray, integer-ratio path (gray-image.ts:170-186) */
__global__ void k_gray_down_blocks(const uint8_t* __restrict__ gray, int W, int H, int tw, int th,
                                   uint8_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tw * th) return;
    const int x = i % tw, y = i / tw;
    int x0, x1, y0, y1;
    block_bounds(x, (double)W / tw, &x0, &x1);
    block_bounds(y, (double)H / th, &y0, &y1);
    double sum = 0.0;
    for (int yy = y0; yy < y1; yy++)
        for (int xx = x0; xx < x1; xx++) sum += gray[(size_t)yy * W + xx];
    out[i] = to_u8(js_round(sum / ((double)(y1 - y0) * (x1 - x0))));
}

/* upsampleDepth (depth-maps.ts:9-42) */
__global__ void k_upsample_depth(const float* __restrict__ grid, int gw, int gh, int W, int H,
                                 float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H) return;
    const int x = i % W, y = i / W;
    const double gy = fmin((double)(gh - 1), fmax(0.0, ((y + 0.5) / H) * gh - 0.5));
    const int y0 = (int)floor(gy);
    const int y1 = min(gh - 1, y0 + 1);
    const double wy = gy - y0;
    const double gx = fmin((double)(gw - 1), fmax(0.0, ((x + 0.5) / W) * gw - 0.5));
    const int x0 = (int)floor(gx);
    const int x1 = min(gw - 1, x0 + 1);
    const double wx = gx - x0;
    const double d[4] = {grid[(size_t)y0 * gw + x0], grid[(size_t)y0 * gw + x1],
                         grid[(size_t)y1 * gw + x0], grid[(size_t)y1 * gw + x1]};
    const double w[4] = {(1 - wx) * (1 - wy), wx * (1 - wy), (1 - wx) * wy, wx * wy};
    double sum = 0.0, weight = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (d[k] > 0.0) {
            sum += d[k] * w[k];
            weight += w[k];
        }
    out[i] = weight > 0.5 ? (float)(sum / weight) : 0.0f;
}

inline unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

cudaError_t l3d_launch_gray_blocks(const uint8_t* rgba, int W, int H, int tw, int th, uint8_t* out,
                                   cudaStream_t s) {
    k_gray_blocks<<<blocks_for((long long)tw * th), 256, 0, s>>>(rgba, W, H, tw, th, out);
    return cudaGetLastError();
}
cudaError_t l3d_launch_area(const void* src, int src_kind, int W, int H, int tw, int th,
                            const L3dAreaCover& cols, const L3dAreaCover& rows, float* temp,
                            uint8_t* out, cudaStream_t s) {
    const long long n1 = (long long)tw * H;
    if (src_kind == 2)
        k_area_rows<2><<<blocks_for(n1), 256, 0, s>>>(src, W, H, tw, cols.first, cols.count,
                                                      cols.weights, cols.kmax, temp);
    else if (src_kind == 1)
        k_area_rows<1><<<blocks_for(n1), 256, 0, s>>>(src, W, H, tw, cols.first, cols.count,
                                                      cols.weights, cols.kmax, temp);
    else
        k_area_rows<0><<<blocks_for(n1), 256, 0, s>>>(src, W, H, tw, cols.first, cols.count,
                                                      cols.weights, cols.kmax, temp);
    k_area_cols<<<blocks_for((long long)tw * th), 256, 0, s>>>(temp, tw, th, rows.first, rows.count,
                                                               rows.weights, rows.kmax, out);
    return cudaGetLastError();
}
cudaError_t l3d_launch_rgb_blocks(const uint8_t* rgba, int W, int H, int tw, int th, uint8_t* out,
                                  cudaStream_t s) {
    k_rgb_blocks<<<blocks_for((long long)tw * th), 256, 0, s>>>(rgba, W, H, tw, th, out);
    return cudaGetLastError();
}
cudaError_t l3d_launch_gray_down_blocks(const uint8_t* gray, int W, int H, int tw, int th, uint8_t* out,
                                        cudaStream_t s) {
    k_gray_down_blocks<<<blocks_for((long long)tw * th), 256, 0, s>>>(gray, W, H, tw, th, out);
    return cudaGetLastError();
}
cudaError_t l3d_launch_upsample_depth(const float* grid, int gw, int gh, int W, int H, float* out,
                                      cudaStream_t s) {
    k_upsample_depth<<<blocks_for((long long)W * H), 256, 0, s>>>(grid, gw, gh, W, H, out);
    return cudaGetLastError();
}
