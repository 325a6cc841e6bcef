/*
 * Throughput probe of the texture unit: bilinear samples per second of a block-linear CUDA
 * array read through a texture object configured like the batched forms' source images
 * (clamp-to-edge, unnormalised coordinates): hardware-filtered fetches (the fast form), texture
 * gathers with exact FP32 weights (the exact form), four point fetches, or four loads from
 * linear memory (the plain form's path).
 *
 * The fast propagate kernel is bound by the texture data pipe, not by FP32 issue or HBM; this
 * probe measures the sample rate that pipe sustains on the running device, so that the kernel's
 * achieved rate can be quoted as a fraction of a measured peak.  Each thread block is laid out
 * like k_fast_propagate (128 threads, hardware quads on 2 x 2 pixel blocks of a 16 x 8 tile) and
 * samples a 6 x 6 window dilated by 2 at a fractional offset, so every fetch filters four texels.
 * `checker` places the pixels of one red/black colour (every other column, alternating by row),
 * as the propagate kernel does; otherwise the tile's pixels are adjacent.
 */
#include <cuda_runtime.h>

#include "l3d_internal.h"

namespace {

constexpr int PROBE_TX = 16, PROBE_TY = 8;

/* MODE 0: hardware bilinear (tex2D, linear filtering).  MODE 1: texture gather (tld4) of the
 * footprint at its centre + exact FP32 weights.  MODE 2: four point-sampled fetches + exact
 * weights.  MODE 3: four loads from linear memory (L1/L2) + exact weights. */
template <bool CHECKER, int MODE>
__global__ void __launch_bounds__(128) k_texture_rate(cudaTextureObject_t tex, const float* __restrict__ img,
                                                      int W, int H, int tiles_x, int reps,
                                                      float* __restrict__ out) {
    const int q = threadIdx.x >> 2, j = threadIdx.x & 3;
    const int tx = (q % (PROBE_TX / 2)) * 2 + (j & 1);
    const int ty = (q / (PROBE_TX / 2)) * 2 + (j >> 1);
    const int y = (blockIdx.x / tiles_x) * PROBE_TY + ty;
    const int px = (blockIdx.x % tiles_x) * PROBE_TX + tx;
    const int x = CHECKER ? px * 2 + (y & 1) : px;
    float acc = 0.0f;
    for (int r = 0; r < reps; r++) {
        /* a different sub-texel offset and a small shift per repetition */
        const float u0 = (float)(x + (r & 7)) + 0.5f + 0.3125f + 0.0625f * (float)(r & 3);
        const float v0 = (float)(y + ((r >> 3) & 3)) + 0.5f + 0.1875f;
#pragma unroll
        for (int oy = 0; oy < 6; oy++)
#pragma unroll
            for (int ox = 0; ox < 6; ox++) {
                const float u = u0 + (float)(2 * ox - 5), v = v0 + (float)(2 * oy - 5);
                if (MODE == 0) {
                    acc += tex2D<float>(tex, u, v);
                } else {
                    /* texel coordinates (texel centres at integers) */
                    const float uu = u - 0.5f, vv = v - 0.5f;
                    const float fx0 = floorf(uu), fy0 = floorf(vv);
                    const float fx = uu - fx0, fy = vv - fy0;
                    float a, b, c, e;
                    if (MODE == 1) {
                        const float4 g = tex2Dgather<float4>(tex, fx0 + 1.0f, fy0 + 1.0f, 0);
                        a = g.w; b = g.z; c = g.x; e = g.y;
                    } else if (MODE == 2) {
                        a = tex2D<float>(tex, fx0 + 0.5f, fy0 + 0.5f);
                        b = tex2D<float>(tex, fx0 + 1.5f, fy0 + 0.5f);
                        c = tex2D<float>(tex, fx0 + 0.5f, fy0 + 1.5f);
                        e = tex2D<float>(tex, fx0 + 1.5f, fy0 + 1.5f);
                    } else {
                        const int ix0 = min(max((int)fx0, 0), W - 1), iy0 = min(max((int)fy0, 0), H - 1);
                        const int ix1 = min(ix0 + 1, W - 1), iy1 = min(iy0 + 1, H - 1);
                        a = __ldg(img + (long long)iy0 * W + ix0);
                        b = __ldg(img + (long long)iy0 * W + ix1);
                        c = __ldg(img + (long long)iy1 * W + ix0);
                        e = __ldg(img + (long long)iy1 * W + ix1);
                    }
                    const float top = fmaf(fx, b - a, a);
                    const float bot = fmaf(fx, e - c, c);
                    acc += fmaf(fy, bot - top, top);
                }
            }
    }
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

}  // namespace

long long l3d_texture_rate_blocks(int width, int height, int checker) {
    const int cols = checker ? width / 2 : width;
    return (long long)(cols / PROBE_TX) * (height / PROBE_TY);
}

cudaError_t l3d_launch_texture_rate(cudaTextureObject_t tex, const float* img, int width, int height,
                                    int checker, int mode, int reps, float* out, cudaStream_t s) {
    const int cols = checker ? width / 2 : width;
    const int tiles_x = cols / PROBE_TX;
    const unsigned blocks = (unsigned)l3d_texture_rate_blocks(width, height, checker);
#define L3D_PROBE(C, M) k_texture_rate<C, M><<<blocks, 128, 0, s>>>(tex, img, width, height, tiles_x, reps, out)
    switch (mode * 2 + (checker ? 1 : 0)) {
        case 0: L3D_PROBE(false, 0); break;
        case 1: L3D_PROBE(true, 0); break;
        case 2: L3D_PROBE(false, 1); break;
        case 3: L3D_PROBE(true, 1); break;
        case 4: L3D_PROBE(false, 2); break;
        case 5: L3D_PROBE(true, 2); break;
        case 6: L3D_PROBE(false, 3); break;
        case 7: L3D_PROBE(true, 3); break;
        default: return cudaErrorInvalidValue;
    }
#undef L3D_PROBE
    return cudaGetLastError();
}
