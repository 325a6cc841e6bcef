/*
 * Throughput probe of the texture unit: bilinear samples per second of a block-linear CUDA
 * array read through a texture object configured like the fast form's source images
 * (clamp-to-edge, linear filtering, unnormalised coordinates).
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

template <bool CHECKER>
__global__ void __launch_bounds__(128) k_texture_rate(cudaTextureObject_t tex, int tiles_x, int reps,
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
            for (int ox = 0; ox < 6; ox++)
                acc += tex2D<float>(tex, u0 + (float)(2 * ox - 5), v0 + (float)(2 * oy - 5));
    }
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

}  // namespace

long long l3d_texture_rate_blocks(int width, int height, int checker) {
    const int cols = checker ? width / 2 : width;
    return (long long)(cols / PROBE_TX) * (height / PROBE_TY);
}

cudaError_t l3d_launch_texture_rate(cudaTextureObject_t tex, int width, int height, int checker,
                                    int reps, float* out, cudaStream_t s) {
    const int cols = checker ? width / 2 : width;
    const int tiles_x = cols / PROBE_TX;
    const long long blocks = l3d_texture_rate_blocks(width, height, checker);
    if (checker)
        k_texture_rate<true><<<(unsigned)blocks, 128, 0, s>>>(tex, tiles_x, reps, out);
    else
        k_texture_rate<false><<<(unsigned)blocks, 128, 0, s>>>(tex, tiles_x, reps, out);
    return cudaGetLastError();
}
