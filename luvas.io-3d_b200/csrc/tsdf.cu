/*
 * TSDF integration of packed depth maps (frontend/src/app/vision/fusion/tsdf-volume.ts).
 *
 *   k_visible      visibleBricks (tsdf-volume.ts:220-234) on the device: one thread per
 *                  (brick, view) evaluates the reference's FP64 frustum test, in the reference's
 *                  operation order (built with --fmad=false, so no FP64 contraction).
 *   k_integrate    one view per launch (TsdfVolume.integrate, tsdf-volume.ts:240-268).  A thread
 *                  owns four consecutive voxels along x (inside one 8^3 brick): it computes the
 *                  four observations from the L2-resident depth map first (the four depth loads
 *                  in flight together, normals from the decoded-normal table) and touches the
 *                  volume only when one of them updates, with one 128-bit tsdf access and one
 *                  64-bit (Q8.8) or 128-bit (f32) weight access; culled bricks read nothing but
 *                  their mask byte.
 *   k_count_updates
 *                  the visible voxel-views and voxel-updates of a many-view integration, without
 *                  its writes (the algorithmic bytes of the one-view-per-launch form).
 *   k_depth_tiles, k_super_behind, k_visible_depth
 *                  the depth-aware half of the brick cull (see brick_behind_depths), first for
 *                  blocks of 4^3 bricks, then for the bricks of the blocks not dropped.
 *   k_integrate_many, k_integrate_many_list
 *                  many views per sweep: the same thread keeps its four voxels in registers,
 *                  applies every view in order and writes back once; per-voxel results equal the
 *                  per-view launches bit for bit (the per-voxel update order is unchanged).  The
 *                  list form visits only the bricks some view keeps (k_brick_any, a prefix sum,
 *                  k_brick_list_fill).
 *   k_integrate_list
 *                  one view over the bricks it keeps (k_visible_one_list), grid-stride.
 *
 * Per-voxel arithmetic (tsdf-volume.ts:111-153), fixed order shared with the FP32 restatement:
 *   world = fma(i + 0.5, voxel, origin); cam = R world + t (fma chain); pixel =
 *   rint(fma(f * cam, 1 / cam.z, c)); weight w = max(0.2, |n . normalize(cam)|) x confidence
 *   factor, or the prior weight; tsdf <- fma(tsdf, w0, obs * w) / (w0 + w);
 *   weight <- min(w0 + w, max).  Q8.8 weights: w is rounded to a multiple of 1/256 first, so
 *   weights stay exact integers.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include <cuda_fp16.h>

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
__device__ __forceinline__ float maxw(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float minw(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float clampw(float v, float lo, float hi) { return minw(maxw(v, lo), hi); }

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

/* Observation of one voxel in one view; false when the voxel is not updated. */
__device__ __forceinline__ bool observe(const L3dTsdfGrid& g, const L3dTsdfView& v,
                                        const uint32_t* __restrict__ depth,
                                        const float* __restrict__ prior, int gx, int gy, int gz,
                                        float* obs, float* wout) {
    float wx = fmaf((float)gx + 0.5f, g.voxel, g.origin[0]);
    float wy = fmaf((float)gy + 0.5f, g.voxel, g.origin[1]);
    float wz = fmaf((float)gz + 0.5f, g.voxel, g.origin[2]);
    const float* R = v.R;
    float3 cam = make_float3(fmaf(R[2], wz, fmaf(R[1], wy, fmaf(R[0], wx, v.t[0]))),
                             fmaf(R[5], wz, fmaf(R[4], wy, fmaf(R[3], wx, v.t[1]))),
                             fmaf(R[8], wz, fmaf(R[7], wy, fmaf(R[6], wx, v.t[2]))));
    if (!(cam.z > 0.01f)) return false;
    float iz = 1.0f / cam.z;
    float rx = rintf(fmaf(v.k[0] * cam.x, iz, v.k[2]));
    float ry = rintf(fmaf(v.k[1] * cam.y, iz, v.k[3]));
    if (!(rx >= 0.0f && ry >= 0.0f && rx < (float)v.W && ry < (float)v.H)) return false;
    long long i = (long long)(int)ry * v.W + (int)rx;
    uint32_t packed = __ldg(depth + i);
    float d = l3d_f16_to_f32(packed & 0xffffu);
    float w;
    if (d > 0.0f) {
        float3 n = unpack_normal(packed);
        float3 cn = normalize3f(cam);
        w = maxw(0.2f, fabsf(dot3f(n, cn)));
        if (v.conf > 0.0f) {
            float c = (float)(packed >> 28) / 8.0f;
            float r = clampw(v.conf / d, 0.5f, 2.0f);
            w = w * ((maxw(0.15f, (1.0f - c) * (1.0f - c)) * r) * r);
        }
    } else {
        d = prior ? __ldg(prior + i) : 0.0f;
        w = g.prior_weight;
    }
    if (!(d > 0.0f)) return false;
    float sdf = d - cam.z;
    if (sdf < -g.mu) return false;
    *obs = minw(1.0f, sdf / g.mu);
    *wout = w;
    return true;
}

/* observe() with the same results, reordered for the many-view sweep and split in two.
 * lut_pixel gives the camera point and the depth-map index of every voxel of a quad first, so
 * that their depth loads are in flight together; lut_observe finishes from the loaded sample,
 * with the depth and the truncation test before the weight (most voxels of a view lie behind
 * the surface or outside the truncation band) and the decoded normal from `normals`, a table of
 * unpack_normal over all 4096 normal codes computed with the same arithmetic.  The voxel's world
 * position (fma(i + 0.5, voxel, origin), the same for every view) comes from the caller, and the
 * f16 depth is widened by the hardware conversion, which gives l3d_f16_to_f32's value for every
 * non-NaN half (a NaN fails the d > 0 test either way). */
__device__ __forceinline__ bool lut_pixel(const L3dTsdfView& v, float wx, float wy, float wz,
                                          float3* cam_out, int* pix) {
    const float* R = v.R;
    float3 cam = make_float3(fmaf(R[2], wz, fmaf(R[1], wy, fmaf(R[0], wx, v.t[0]))),
                             fmaf(R[5], wz, fmaf(R[4], wy, fmaf(R[3], wx, v.t[1]))),
                             fmaf(R[8], wz, fmaf(R[7], wy, fmaf(R[6], wx, v.t[2]))));
    *cam_out = cam;
    if (!(cam.z > 0.01f)) return false;
    float iz = 1.0f / cam.z;
    float rx = rintf(fmaf(v.k[0] * cam.x, iz, v.k[2]));
    float ry = rintf(fmaf(v.k[1] * cam.y, iz, v.k[3]));
    if (!(rx >= 0.0f && ry >= 0.0f && rx < (float)v.W && ry < (float)v.H)) return false;
    *pix = (int)ry * v.W + (int)rx;
    return true;
}

__device__ __forceinline__ bool lut_observe(const L3dTsdfGrid& g, const L3dTsdfView& v,
                                            const float* __restrict__ prior,
                                            const float4* __restrict__ normals, float3 cam, int i,
                                            uint32_t packed, float* obs, float* wout) {
    float d = __half2float(__ushort_as_half((unsigned short)(packed & 0xffffu)));
    const bool stereo = d > 0.0f;
    if (!stereo) d = prior ? __ldg(prior + i) : 0.0f;
    if (!(d > 0.0f)) return false;
    float sdf = d - cam.z;
    if (sdf < -g.mu) return false;
    float w;
    if (stereo) {
        float4 n4 = __ldg(normals + ((packed >> 16) & 4095u));
        float3 cn = normalize3f(cam);
        w = maxw(0.2f, fabsf(dot3f(make_float3(n4.x, n4.y, n4.z), cn)));
        if (v.conf > 0.0f) {
            float c = (float)(packed >> 28) / 8.0f;
            float r = clampw(v.conf / d, 0.5f, 2.0f);
            w = w * ((maxw(0.15f, (1.0f - c) * (1.0f - c)) * r) * r);
        }
    } else {
        w = g.prior_weight;
    }
    *obs = minw(1.0f, sdf / g.mu);
    *wout = w;
    return true;
}

__global__ void k_normal_table(float4* normals) {
    const uint32_t code = blockIdx.x * blockDim.x + threadIdx.x;
    if (code >= 4096u) return;
    float3 n = unpack_normal(code << 16);
    normals[code] = make_float4(n.x, n.y, n.z, 0.0f);
}

__device__ __forceinline__ void apply_f32(float& t, float& w0, float obs, float w, float maxw_) {
    t = fmaf(t, w0, obs * w) / (w0 + w);
    w0 = minw(w0 + w, maxw_);
}

__device__ __forceinline__ void apply_q8(float& t, uint32_t& w0i, float obs, float w, unsigned maxq) {
    uint32_t wi = (uint32_t)rintf(w * 256.0f);
    if (wi == 0u) return;
    float w0 = (float)w0i * 0.00390625f;
    float wf = (float)wi * 0.00390625f;
    t = fmaf(t, w0, obs * wf) / (w0 + wf);
    w0i = min(w0i + wi, maxq);
}

/* Voxel coordinates and storage index of the first voxel of quad q (VEC consecutive x).
 * Brick pools and (BRICKS) dense grids run in brick-major order: quad q is quad q % (512 / VEC)
 * of brick q / (512 / VEC), so the 32 threads of a warp stay inside one 8^3 brick (one mask
 * entry, one set of views, converged branches) and touch 32-byte row segments of it; quads of a
 * ragged grid's partial bricks that fall outside the grid are skipped.  Otherwise dense grids
 * run in voxel-index order. */
template <int VEC, bool BRICKS = true>
__device__ __forceinline__ bool quad_coords(const L3dTsdfGrid& g, const int32_t* coords,
                                            long long q, int* gx, int* gy, int* gz,
                                            long long* idx, long long* brick) {
    if (g.dense && BRICKS) {
        long long b = q / (512 / VEC);
        if (b >= g.bricks) return false;
        int local = (int)(q - b * (512 / VEC)) * VEC;
        const long long bxy = (long long)g.nb[0] * g.nb[1];
        const int bz = (int)(b / bxy);
        const int rest = (int)(b - (long long)bz * bxy);
        const int by = rest / g.nb[0], bx = rest - by * g.nb[0];
        *gx = bx * 8 + (local & 7);
        *gy = by * 8 + ((local >> 3) & 7);
        *gz = bz * 8 + (local >> 6);
        if (*gx >= g.dims[0] || *gy >= g.dims[1] || *gz >= g.dims[2]) return false;
        *idx = ((long long)*gz * g.dims[1] + *gy) * g.dims[0] + *gx;
        *brick = b;
    } else if (g.dense) {
        long long qx = g.dims[0] / VEC;
        long long rest = q / qx;
        *gx = (int)(q - rest * qx) * VEC;
        *gy = (int)(rest % g.dims[1]);
        *gz = (int)(rest / g.dims[1]);
        if (*gz >= g.dims[2]) return false;
        *idx = ((long long)*gz * g.dims[1] + *gy) * g.dims[0] + *gx;
        *brick = ((long long)(*gz >> 3) * g.nb[1] + (*gy >> 3)) * g.nb[0] + (*gx >> 3);
    } else {
        long long b = q / (512 / VEC);
        if (b >= g.bricks) return false;
        int local = (int)(q - b * (512 / VEC)) * VEC;
        const int32_t* c = coords + b * 4;
        *gx = c[0] * 8 + (local & 7);
        *gy = c[1] * 8 + ((local >> 3) & 7);
        *gz = c[2] * 8 + (local >> 6);
        *idx = b * 512 + local;
        *brick = b;
    }
    return true;
}

/* visibleBricks (tsdf-volume.ts:220-234) for brick b of view v, FP64, reference order. */
__device__ __forceinline__ uint8_t brick_visible(const L3dTsdfGrid& g, const L3dTsdfView& v,
                                                 const int32_t* __restrict__ coords, long long b) {
    int bx, by, bz;
    if (g.dense) {
        bx = (int)(b % g.nb[0]);
        by = (int)((b / g.nb[0]) % g.nb[1]);
        bz = (int)(b / ((long long)g.nb[0] * g.nb[1]));
    } else {
        bx = coords[b * 4];
        by = coords[b * 4 + 1];
        bz = coords[b * 4 + 2];
    }
    double side = g.voxel_d * 8.0;
    double c0 = g.origin_d[0] + (bx + 0.5) * side;
    double c1 = g.origin_d[1] + (by + 0.5) * side;
    double c2 = g.origin_d[2] + (bz + 0.5) * side;
    double radius = g.voxel_d * 8.0 * 0.87 + g.trunc_d;
    const double* R = v.Rd;
    double p0 = R[0] * c0 + R[1] * c1 + R[2] * c2 + v.td[0];
    double p1 = R[3] * c0 + R[4] * c1 + R[5] * c2 + v.td[1];
    double p2 = R[6] * c0 + R[7] * c1 + R[8] * c2 + v.td[2];
    double u = (v.kd[0] * p0) / p2 + v.kd[2];
    double w = (v.kd[1] * p1) / p2 + v.kd[3];
    double z = p2;
    if (z < 0.02 - radius || z > v.max_depth + radius) return 0;
    double margin = (v.kd[0] * radius) / fmax(0.02, z);
    if (u < -margin || w < -margin || u > v.W + margin || w > v.H + margin) return 0;
    return 1;
}

/* The many-view brick mask is brick-major: brick b's flags for views 0..n-1 are the bytes
 * mask[b * mask_stride(n) + v], the row padded with zeros to a multiple of 16 bytes, so a thread
 * reads a brick's views with 128-bit loads. */
__host__ __device__ __forceinline__ int mask_stride(int n_views) { return (n_views + 15) & ~15; }

__global__ void k_visible(const L3dTsdfGrid g, const L3dTsdfView* __restrict__ views, int n_views,
                          const int32_t* __restrict__ coords, uint8_t* __restrict__ mask) {
    const int stride = mask_stride(n_views);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.bricks * stride) return;
    long long b = t / stride;
    int vi = (int)(t - b * stride);
    mask[t] = vi < n_views ? brick_visible(g, views[vi], coords, b) : 0;
}

/* The depth-aware half of the brick cull.  A voxel of view v is updated only from the depth d
 * of the pixel it rounds to (the packed map's, or the prior where the map has none), and only
 * if d - z >= -mu for its camera depth z.  The voxel centres of brick b span a box; its eight
 * corners bound every centre's camera depth from below (z is affine) and its pixel to the
 * corners' bounding rectangle widened by a pixel (pixels are rounded to the nearest).  If the
 * smallest corner depth exceeds the largest depth over the depth tiles covering that rectangle
 * by more than mu plus a margin, no voxel of the brick updates: the cull changes which voxels
 * are visited, never a result.  The bound is computed in FP32; the margin (0.2 mm plus 1e-6 of
 * the sum of the magnitudes entering the camera depth, about 17 ulp of it) covers the rounding
 * of this computation and of the kernels' own FP32 camera depth and sdf, and the one-pixel
 * widening covers that of the projections.  Bricks with a corner at z <= 0.02 or a footprint
 * wider than 32 x 32 tiles are kept. */
__device__ __forceinline__ bool box_behind_depths(const L3dTsdfGrid& g, const L3dTsdfView& v,
                                                  const float* __restrict__ tiles, float lx, float ly,
                                                  float lz, float span);

__device__ __forceinline__ bool brick_behind_depths(const L3dTsdfGrid& g, const L3dTsdfView& v,
                                                    const int32_t* __restrict__ coords,
                                                    const float* __restrict__ tiles, long long b) {
    int bx, by, bz;
    if (g.dense) {
        bx = (int)(b % g.nb[0]);
        by = (int)((b / g.nb[0]) % g.nb[1]);
        bz = (int)(b / ((long long)g.nb[0] * g.nb[1]));
    } else {
        bx = coords[b * 4];
        by = coords[b * 4 + 1];
        bz = coords[b * 4 + 2];
    }
    return box_behind_depths(g, v, tiles, fmaf((float)(bx * 8) + 0.5f, g.voxel, g.origin[0]),
                             fmaf((float)(by * 8) + 0.5f, g.voxel, g.origin[1]),
                             fmaf((float)(bz * 8) + 0.5f, g.voxel, g.origin[2]), 7.0f * g.voxel);
}

/* brick_behind_depths for the axis-aligned box of voxel centres from (lx, ly, lz) to
 * (lx, ly, lz) + span on each axis. */
__device__ __forceinline__ bool box_behind_depths(const L3dTsdfGrid& g, const L3dTsdfView& v,
                                                  const float* __restrict__ tiles, float lx, float ly,
                                                  float lz, float span) {
    const float* R = v.R;
    const float3 p0 = make_float3(fmaf(R[2], lz, fmaf(R[1], ly, fmaf(R[0], lx, v.t[0]))),
                                  fmaf(R[5], lz, fmaf(R[4], ly, fmaf(R[3], lx, v.t[1]))),
                                  fmaf(R[8], lz, fmaf(R[7], ly, fmaf(R[6], lx, v.t[2]))));
    const float mag = fabsf(lx) + fabsf(ly) + fabsf(lz) + 3.0f * span + fabsf(v.t[0]) +
                      fabsf(v.t[1]) + fabsf(v.t[2]);
    float zmin = 3e38f, umin = 3e38f, umax = -3e38f, vmin = 3e38f, vmax = -3e38f;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const float sx = (c & 1) ? span : 0.0f, sy = (c & 2) ? span : 0.0f, sz = (c & 4) ? span : 0.0f;
        const float px = fmaf(R[2], sz, fmaf(R[1], sy, fmaf(R[0], sx, p0.x)));
        const float py = fmaf(R[5], sz, fmaf(R[4], sy, fmaf(R[3], sx, p0.y)));
        const float pz = fmaf(R[8], sz, fmaf(R[7], sy, fmaf(R[6], sx, p0.z)));
        if (!(pz > 0.02f)) return false;
        const float iz = 1.0f / pz;
        const float u = fmaf(v.k[0] * px, iz, v.k[2]), w = fmaf(v.k[1] * py, iz, v.k[3]);
        zmin = fminf(zmin, pz);
        umin = fminf(umin, u);
        umax = fmaxf(umax, u);
        vmin = fminf(vmin, w);
        vmax = fmaxf(vmax, w);
    }
    const float x0 = fmaxf(floorf(umin) - 1.0f, 0.0f), x1 = fminf(ceilf(umax) + 1.0f, (float)(v.W - 1));
    const float y0 = fmaxf(floorf(vmin) - 1.0f, 0.0f), y1 = fminf(ceilf(vmax) + 1.0f, (float)(v.H - 1));
    if (!(x1 >= x0) || !(y1 >= y0)) return !(isnan(x1) || isnan(y1));  /* nothing projects inside */
    const int tx0 = (int)x0 / L3D_DEPTH_TILE, tx1 = (int)x1 / L3D_DEPTH_TILE;
    const int ty0 = (int)y0 / L3D_DEPTH_TILE, ty1 = (int)y1 / L3D_DEPTH_TILE;
    if (tx1 - tx0 >= 32 || ty1 - ty0 >= 32) return false;
    const int tw = (v.W + L3D_DEPTH_TILE - 1) / L3D_DEPTH_TILE;
    const float* vt = tiles + v.tile_off;
    float dmax = 0.0f;
    for (int ty = ty0; ty <= ty1; ty++)
        for (int tx = tx0; tx <= tx1; tx++) dmax = fmaxf(dmax, __ldg(vt + (long long)ty * tw + tx));
    return zmin - dmax > g.mu + 2e-4f + 1e-6f * (mag + dmax);
}

/* Depth tiles of view v (see l3d_launch_depth_tiles): thread t takes row t % 8 of tile t / 8
 * (eight pixels), and the eight threads of a tile, consecutive lanes of one warp, combine their
 * maxima with shuffles; lane 0 of the group writes the tile. */
__device__ __forceinline__ void depth_tile(const L3dTsdfView& v, const uint32_t* __restrict__ depth,
                                           const float* __restrict__ prior, float* __restrict__ tiles,
                                           long long t) {
    static_assert(L3D_DEPTH_TILE == 8, "eight rows per tile, eight lanes per tile");
    const int tw = (v.W + L3D_DEPTH_TILE - 1) / L3D_DEPTH_TILE, th = (v.H + L3D_DEPTH_TILE - 1) / L3D_DEPTH_TILE;
    const long long tile = t >> 3;
    const int row = (int)(t & 7);
    float m = 0.0f;
    if (tile < (long long)tw * th) {
        const int tx = (int)(tile % tw), ty = (int)(tile / tw);
        const int y = ty * L3D_DEPTH_TILE + row;
        if (y < v.H)
            for (int x = tx * L3D_DEPTH_TILE; x < min(v.W, (tx + 1) * L3D_DEPTH_TILE); x++) {
                const long long i = (long long)y * v.W + x;
                float d = __half2float(__ushort_as_half((unsigned short)(__ldg(depth + i) & 0xffffu)));
                if (!(d > 0.0f)) d = prior ? __ldg(prior + i) : 0.0f;
                if (d > m) m = d;  /* NaN never raises the maximum: such a pixel never updates */
            }
    }
    /* the tile's eight lanes are aligned groups of a warp (blocks are whole warps) */
    for (int o = 4; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (row == 0 && tile < (long long)tw * th) tiles[v.tile_off + tile] = m;
}

__global__ void k_depth_tiles(const L3dTsdfView* __restrict__ views, int n_views,
                              const uint32_t* const* __restrict__ depths, const float* __restrict__ priors,
                              float* __restrict__ tiles, long long max_tiles) {
    const int vi = blockIdx.y;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;  /* every lane takes part */
    const L3dTsdfView& v = views[vi];
    depth_tile(v, depths[vi], v.has_prior ? priors + v.prior_off : nullptr, tiles, t);
}

__global__ void k_depth_tiles_one(const L3dTsdfView v, const uint32_t* __restrict__ depth,
                                  const float* __restrict__ prior, float* __restrict__ tiles) {
    depth_tile(v, depth, v.has_prior ? prior : nullptr, tiles, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

/* Super-bricks of a dense grid: blocks of L3D_SUPER^3 bricks.  super[s * n_views + v] = 1 if
 * the voxel centres of super-brick s (the grid's edge cut off) are behind view v's depths by the
 * test of brick_behind_depths: then so is every brick inside it, and k_visible_depth drops those
 * bricks without their own tests. */
constexpr int L3D_SUPER = 4;
__host__ __device__ __forceinline__ int super_count(const L3dTsdfGrid& g, int axis) {
    return (g.nb[axis] + L3D_SUPER - 1) / L3D_SUPER;
}

__global__ void k_super_behind(const L3dTsdfGrid g, const L3dTsdfView* __restrict__ views, int n_views,
                               const float* __restrict__ tiles, uint8_t* __restrict__ super) {
    const long long n = (long long)super_count(g, 0) * super_count(g, 1) * super_count(g, 2);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * n_views) return;
    const long long sb = t / n_views;
    const int vi = (int)(t - sb * n_views);
    const int sx = (int)(sb % super_count(g, 0));
    const int sy = (int)((sb / super_count(g, 0)) % super_count(g, 1));
    const int sz = (int)(sb / ((long long)super_count(g, 0) * super_count(g, 1)));
    constexpr int V = 8 * L3D_SUPER;
    /* the box's far corner: the last voxel of the super-brick inside the grid on each axis */
    const int ex = min(V, g.dims[0] - sx * V) - 1, ey = min(V, g.dims[1] - sy * V) - 1;
    const int ez = min(V, g.dims[2] - sz * V) - 1;
    const int e = max(ex, max(ey, ez));
    super[t] = box_behind_depths(g, views[vi], tiles, fmaf((float)(sx * V) + 0.5f, g.voxel, g.origin[0]),
                                 fmaf((float)(sy * V) + 0.5f, g.voxel, g.origin[1]),
                                 fmaf((float)(sz * V) + 0.5f, g.voxel, g.origin[2]), (float)e * g.voxel)
                   ? 1 : 0;
}

__global__ void k_visible_depth(const L3dTsdfGrid g, const L3dTsdfView* __restrict__ views, int n_views,
                                const int32_t* __restrict__ coords, const float* __restrict__ tiles,
                                const uint8_t* __restrict__ super, uint8_t* __restrict__ mask) {
    const int stride = mask_stride(n_views);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.bricks * stride) return;
    long long b = t / stride;
    int vi = (int)(t - b * stride);
    if (vi >= n_views) {
        mask[t] = 0;
        return;
    }
    if (super) {
        const int bx = (int)(b % g.nb[0]), by = (int)((b / g.nb[0]) % g.nb[1]);
        const int bz = (int)(b / ((long long)g.nb[0] * g.nb[1]));
        const long long sb = ((long long)(bz / L3D_SUPER) * super_count(g, 1) + by / L3D_SUPER) *
                                 super_count(g, 0) + bx / L3D_SUPER;
        if (__ldg(super + sb * n_views + vi)) {
            mask[t] = 0;
            return;
        }
    }
    /* a brick behind the depths needs no frustum test: it is dropped either way */
    mask[t] = (tiles && brick_behind_depths(g, views[vi], coords, tiles, b))
                  ? 0 : brick_visible(g, views[vi], coords, b);
}

__global__ void k_visible_one_depth(const L3dTsdfGrid g, const L3dTsdfView v,
                                    const int32_t* __restrict__ coords, const float* __restrict__ tiles,
                                    uint8_t* __restrict__ mask) {
    long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.bricks) return;
    mask[b] = brick_behind_depths(g, v, coords, tiles, b) ? 0 : brick_visible(g, v, coords, b);
}

/* k_visible_one_depth that also lists the kept bricks: list[0] counts them (zeroed before the
 * launch), list[1..] receives their indices in any order. */
__global__ void k_visible_one_list(const L3dTsdfGrid g, const L3dTsdfView v,
                                   const int32_t* __restrict__ coords, const float* __restrict__ tiles,
                                   uint8_t* __restrict__ mask, int32_t* __restrict__ list) {
    long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.bricks) return;
    const uint8_t m = brick_behind_depths(g, v, coords, tiles, b) ? 0 : brick_visible(g, v, coords, b);
    mask[b] = m;
    if (m) list[1 + atomicAdd(list, 1)] = (int32_t)b;
}

__global__ void k_visible_one(const L3dTsdfGrid g, const L3dTsdfView v,
                              const int32_t* __restrict__ coords, uint8_t* __restrict__ mask) {
    long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.bricks) return;
    mask[b] = brick_visible(g, v, coords, b);
}

/* One view per launch.  LUT: the normal of a depth sample comes from the 4096-entry normal
 * table and a quad's four depth loads are issued together (lut_pixel / lut_observe, the sweep's
 * path, equal to observe() bit for bit); otherwise observe() decodes each normal. */
template <int VEC, bool Q8, bool LUT>
__device__ __forceinline__ void integrate_quad(const L3dTsdfGrid& g, const L3dTsdfView& v,
                                               const int32_t* __restrict__ coords,
                                               const uint8_t* __restrict__ mask,
                                               const uint32_t* __restrict__ depth,
                                               const float* __restrict__ prior,
                                               const float4* __restrict__ normals,
                                               float* __restrict__ tsdf, void* __restrict__ weight,
                                               long long q) {
    int gx, gy, gz;
    long long idx, brick;
    if (!quad_coords<VEC>(g, coords, q, &gx, &gy, &gz, &idx, &brick)) return;
    if (mask && !mask[brick]) return;
    float obs[VEC], w[VEC];
    bool ok[VEC];
    bool any = false;
    if (LUT) {
        const float wy = fmaf((float)gy + 0.5f, g.voxel, g.origin[1]);
        const float wz = fmaf((float)gz + 0.5f, g.voxel, g.origin[2]);
        const float* pr = v.has_prior ? prior : nullptr;
        float3 cam[VEC];
        int pix[VEC];
        uint32_t packed[VEC];
#pragma unroll
        for (int j = 0; j < VEC; j++)
            ok[j] = lut_pixel(v, fmaf((float)(gx + j) + 0.5f, g.voxel, g.origin[0]), wy, wz, &cam[j], &pix[j]);
#pragma unroll
        for (int j = 0; j < VEC; j++) packed[j] = ok[j] ? __ldg(depth + pix[j]) : 0u;
#pragma unroll
        for (int j = 0; j < VEC; j++) {
            ok[j] = ok[j] && lut_observe(g, v, pr, normals, cam[j], pix[j], packed[j], &obs[j], &w[j]);
            any |= ok[j];
        }
    } else {
#pragma unroll
        for (int j = 0; j < VEC; j++) {
            ok[j] = observe(g, v, depth, v.has_prior ? prior : nullptr, gx + j, gy, gz, &obs[j], &w[j]);
            any |= ok[j];
        }
    }
    if (!any) return;
    if (VEC == 4) {
        float4 t4 = *(const float4*)(tsdf + idx);
        float t[4] = {t4.x, t4.y, t4.z, t4.w};
        if (Q8) {
            ushort4 w4 = *(const ushort4*)((const uint16_t*)weight + idx);
            uint32_t wq[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (ok[j]) apply_q8(t[j], wq[j], obs[j], w[j], g.max_q);
            *(ushort4*)((uint16_t*)weight + idx) =
                make_ushort4((uint16_t)wq[0], (uint16_t)wq[1], (uint16_t)wq[2], (uint16_t)wq[3]);
        } else {
            float4 w4 = *(const float4*)((const float*)weight + idx);
            float ww[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (ok[j]) apply_f32(t[j], ww[j], obs[j], w[j], g.max_weight);
            *(float4*)((float*)weight + idx) = make_float4(ww[0], ww[1], ww[2], ww[3]);
        }
        *(float4*)(tsdf + idx) = make_float4(t[0], t[1], t[2], t[3]);
    } else {
        float t = tsdf[idx];
        if (Q8) {
            uint32_t wq = ((const uint16_t*)weight)[idx];
            apply_q8(t, wq, obs[0], w[0], g.max_q);
            ((uint16_t*)weight)[idx] = (uint16_t)wq;
        } else {
            float ww = ((const float*)weight)[idx];
            apply_f32(t, ww, obs[0], w[0], g.max_weight);
            ((float*)weight)[idx] = ww;
        }
        tsdf[idx] = t;
    }
}

template <int VEC, bool Q8, bool LUT>
__global__ void __launch_bounds__(256) k_integrate(const L3dTsdfGrid g, const L3dTsdfView v,
                                                   const int32_t* __restrict__ coords,
                                                   const uint8_t* __restrict__ mask,
                                                   const uint32_t* __restrict__ depth,
                                                   const float* __restrict__ prior,
                                                   const float4* __restrict__ normals,
                                                   float* __restrict__ tsdf, void* __restrict__ weight,
                                                   long long quads) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= quads) return;
    integrate_quad<VEC, Q8, LUT>(g, v, coords, mask, depth, prior, normals, tsdf, weight, q);
}

/* One view over its kept bricks only: list[0] bricks listed at list[1..] (by
 * k_visible_one_list, in any order; each brick's voxels are updated independently), a
 * grid-stride loop over their quads. */
template <int VEC, bool Q8>
__global__ void __launch_bounds__(256) k_integrate_list(const L3dTsdfGrid g, const L3dTsdfView v,
                                                        const int32_t* __restrict__ coords,
                                                        const int32_t* __restrict__ list,
                                                        const uint32_t* __restrict__ depth,
                                                        const float* __restrict__ prior,
                                                        const float4* __restrict__ normals,
                                                        float* __restrict__ tsdf,
                                                        void* __restrict__ weight) {
    constexpr int PER = 512 / VEC;
    const long long n = (long long)__ldg(list) * PER;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long b = __ldg(list + 1 + i / PER);
        integrate_quad<VEC, Q8, true>(g, v, coords, nullptr, depth, prior, normals, tsdf, weight,
                                      b * PER + i % PER);
    }
}

/* One quad of the many-view sweep: its voxels stay in registers while every view that keeps
 * its brick is applied in view order; written back once. */
template <int VEC, bool Q8>
__device__ __forceinline__ void sweep_quad(const L3dTsdfGrid& g, const L3dTsdfView* __restrict__ views,
                                           int n_views, const int32_t* __restrict__ coords,
                                           const uint8_t* __restrict__ mask,
                                           const uint32_t* const* __restrict__ depths,
                                           const float* __restrict__ priors,
                                           const float4* __restrict__ normals,
                                           float* __restrict__ tsdf, void* __restrict__ weight,
                                           long long q) {
    int gx, gy, gz;
    long long idx, brick;
    if (!quad_coords<VEC>(g, coords, q, &gx, &gy, &gz, &idx, &brick)) return;
    /* the brick's row of the mask, 16 views per 128-bit load; a brick no view keeps is left
     * without touching the volume */
    const int stride = mask_stride(n_views);
    const uint4* mrow = (const uint4*)(mask + brick * stride);
    uint32_t any = 0u;
    for (int k = 0; k < stride / 16; k++) {
        const uint4 m = __ldg(mrow + k);
        any |= m.x | m.y | m.z | m.w;
    }
    if (!any) return;
    float t[VEC];
    float wf[VEC];
    uint32_t wq[VEC];
    float wx[VEC];
#pragma unroll
    for (int j = 0; j < VEC; j++) wx[j] = fmaf((float)(gx + j) + 0.5f, g.voxel, g.origin[0]);
    const float wy = fmaf((float)gy + 0.5f, g.voxel, g.origin[1]);
    const float wz = fmaf((float)gz + 0.5f, g.voxel, g.origin[2]);
    /* the quad's volume values are loaded up front (one 128-bit tsdf load, one 64-bit Q8.8 or
     * 128-bit f32 weight load), so their latency overlaps the first view's projection; they are
     * written back only when a view updated them */
    if (VEC == 4) {
        const float4 t4 = *(const float4*)(tsdf + idx);
        t[0] = t4.x; t[1] = t4.y; t[2] = t4.z; t[3] = t4.w;
        if (Q8) {
            const ushort4 w4 = *(const ushort4*)((const uint16_t*)weight + idx);
            wq[0] = w4.x; wq[1] = w4.y; wq[2] = w4.z; wq[3] = w4.w;
        } else {
            const float4 w4 = *(const float4*)((const float*)weight + idx);
            wf[0] = w4.x; wf[1] = w4.y; wf[2] = w4.z; wf[3] = w4.w;
        }
    } else {
        t[0] = tsdf[idx];
        if (Q8) wq[0] = ((const uint16_t*)weight)[idx];
        else wf[0] = ((const float*)weight)[idx];
    }
    bool loaded = false;
    /* the views that keep the brick, 16 at a time, in view order: a mask byte is 0 or 1, so
     * (word * 0x10204080) >> 28 gathers a 32-bit word's four flags into four bits */
    for (int w0 = 0; w0 < n_views; w0 += 16) {
      const uint4 m = __ldg(mrow + w0 / 16);
      uint32_t seen = ((m.x * 0x10204080u) >> 28) | (((m.y * 0x10204080u) >> 28) << 4) |
                      (((m.z * 0x10204080u) >> 28) << 8) | (((m.w * 0x10204080u) >> 28) << 12);
      while (seen) {
        const int vi = w0 + __ffs(seen) - 1;
        seen &= seen - 1u;
        const L3dTsdfView& v = views[vi];
        const uint32_t* depth = depths[vi];
        const float* prior = v.has_prior ? priors + v.prior_off : nullptr;
        float3 cam[VEC];
        int pix[VEC];
        bool in[VEC];
        uint32_t packed[VEC];
#pragma unroll
        for (int j = 0; j < VEC; j++) in[j] = lut_pixel(v, wx[j], wy, wz, &cam[j], &pix[j]);
#pragma unroll
        for (int j = 0; j < VEC; j++) packed[j] = in[j] ? __ldg(depth + pix[j]) : 0u;
#pragma unroll
        for (int j = 0; j < VEC; j++) {
            float obs, w;
            if (!in[j] || !lut_observe(g, v, prior, normals, cam[j], pix[j], packed[j], &obs, &w)) continue;
            loaded = true;
            if (Q8) apply_q8(t[j], wq[j], obs, w, g.max_q);
            else apply_f32(t[j], wf[j], obs, w, g.max_weight);
        }
      }
    }
    if (!loaded) return;
    if (VEC == 4) {
        *(float4*)(tsdf + idx) = make_float4(t[0], t[1], t[2], t[3]);
        if (Q8)
            *(ushort4*)((uint16_t*)weight + idx) =
                make_ushort4((uint16_t)wq[0], (uint16_t)wq[1], (uint16_t)wq[2], (uint16_t)wq[3]);
        else
            *(float4*)((float*)weight + idx) = make_float4(wf[0], wf[1], wf[2], wf[3]);
    } else {
        tsdf[idx] = t[0];
        if (Q8) ((uint16_t*)weight)[idx] = (uint16_t)wq[0];
        else ((float*)weight)[idx] = wf[0];
    }
}

template <int VEC, bool Q8>
__global__ void __launch_bounds__(256, 4) k_integrate_many(const L3dTsdfGrid g,
                                                        const L3dTsdfView* __restrict__ views,
                                                        int n_views,
                                                        const int32_t* __restrict__ coords,
                                                        const uint8_t* __restrict__ mask,
                                                        const uint32_t* const* __restrict__ depths,
                                                        const float* __restrict__ priors,
                                                        const float4* __restrict__ normals,
                                                        float* __restrict__ tsdf,
                                                        void* __restrict__ weight,
                                                        long long q_begin, long long q_end) {
    const long long q = q_begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= q_end) return;
    sweep_quad<VEC, Q8>(g, views, n_views, coords, mask, depths, priors, normals, tsdf, weight, q);
}

/* The sweep over the bricks some view keeps: list holds them in ascending order
 * (l3d_launch_tsdf_brick_list), prefix[b] is the number of kept bricks below brick b, so the
 * kept bricks of [b_begin, b_end) are list[prefix[b_begin] .. prefix[b_end]).  A grid-stride
 * loop over their quads; each quad is still one thread's, so results equal k_integrate_many's. */
template <int VEC, bool Q8>
__global__ void __launch_bounds__(256, 4) k_integrate_many_list(const L3dTsdfGrid g,
                                                             const L3dTsdfView* __restrict__ views,
                                                             int n_views,
                                                             const int32_t* __restrict__ coords,
                                                             const uint8_t* __restrict__ mask,
                                                             const uint32_t* const* __restrict__ depths,
                                                             const float* __restrict__ priors,
                                                             const float4* __restrict__ normals,
                                                             float* __restrict__ tsdf,
                                                             void* __restrict__ weight,
                                                             const uint32_t* __restrict__ prefix,
                                                             const int32_t* __restrict__ list,
                                                             long long b_begin, long long b_end) {
    constexpr int PER = 512 / VEC;
    /* the view table in shared memory, copied once per block (the blocks loop over the list) */
    extern __shared__ __align__(16) unsigned char sweep_smem[];
    L3dTsdfView* sv = reinterpret_cast<L3dTsdfView*>(sweep_smem);
    {
        const int words = n_views * (int)(sizeof(L3dTsdfView) / 8);
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(views);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(sweep_smem);
        for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = __ldg(src + k);
        __syncthreads();
    }
    const long long first = __ldg(prefix + b_begin);
    const long long n = ((long long)__ldg(prefix + b_end) - first) * PER;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long b = __ldg(list + first + i / PER);
        sweep_quad<VEC, Q8>(g, sv, n_views, coords, mask, depths, priors, normals, tsdf, weight,
                            b * PER + i % PER);
    }
}
static_assert(sizeof(L3dTsdfView) % 8 == 0, "the view table is copied in 8-byte words");

/* flags[b] = 1 if some view keeps brick b (its mask row is not all zero), for b < bricks;
 * flags[bricks] = 0, so that an exclusive scan of bricks + 1 flags ends with the total. */
__global__ void k_brick_any(const uint8_t* __restrict__ mask, int stride, long long bricks,
                            uint32_t* __restrict__ flags) {
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b > bricks) return;
    uint32_t any = 0u;
    if (b < bricks) {
        const uint4* row = (const uint4*)(mask + b * stride);
        for (int k = 0; k < stride / 16; k++) {
            const uint4 m = __ldg(row + k);
            any |= m.x | m.y | m.z | m.w;
        }
    }
    flags[b] = any ? 1u : 0u;
}

__global__ void k_brick_list_fill(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ prefix,
                                  long long bricks, int32_t* __restrict__ list) {
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b < bricks && flags[b]) list[prefix[b]] = (int32_t)b;
}

/* The work of a many-view integration without its writes: per voxel, the views whose brick
 * culling keeps it (visible) and the views that update it (lut_observe true), summed over the
 * volume into counts[0] (visible voxel-views) and counts[1] (voxel-updates). */
template <int VEC>
__global__ void __launch_bounds__(256) k_count_updates(const L3dTsdfGrid g,
                                                       const L3dTsdfView* __restrict__ views,
                                                       int n_views, const int32_t* __restrict__ coords,
                                                       const uint8_t* __restrict__ mask,
                                                       const uint32_t* const* __restrict__ depths,
                                                       const float* __restrict__ priors,
                                                       const float4* __restrict__ normals,
                                                       long long quads,
                                                       unsigned long long* __restrict__ counts) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long vis = 0, upd = 0;
    int gx, gy, gz;
    long long idx, brick;
    if (q < quads && quad_coords<VEC>(g, coords, q, &gx, &gy, &gz, &idx, &brick)) {
        const float wy = fmaf((float)gy + 0.5f, g.voxel, g.origin[1]);
        const float wz = fmaf((float)gz + 0.5f, g.voxel, g.origin[2]);
        for (int vi = 0; vi < n_views; vi++) {
            if (!mask[brick * mask_stride(n_views) + vi]) continue;
            vis += VEC;
            const L3dTsdfView& v = views[vi];
            const float* prior = v.has_prior ? priors + v.prior_off : nullptr;
#pragma unroll
            for (int j = 0; j < VEC; j++) {
                float3 cam;
                int pix;
                float obs, w;
                if (lut_pixel(v, fmaf((float)(gx + j) + 0.5f, g.voxel, g.origin[0]), wy, wz, &cam, &pix) &&
                    lut_observe(g, v, prior, normals, cam, pix, __ldg(depths[vi] + pix), &obs, &w))
                    upd++;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        vis += __shfl_down_sync(0xffffffffu, vis, o);
        upd += __shfl_down_sync(0xffffffffu, upd, o);
    }
    if ((threadIdx.x & 31) == 0 && (vis || upd)) {
        atomicAdd(counts, vis);
        atomicAdd(counts + 1, upd);
    }
}

/* ---- differentiable integration: depth from an FP32 map ---- */

/* observe() with the stereo depth read from an FP32 map (validity, normal and cost still come
 * from the packed map), plus the derivatives of the observation and of its weight with respect
 * to that depth.  *pix is the map index whose depth was used, or -1 for a prior observation
 * (which does not depend on the map).  With depthf[i] == unpack_depth(packed[i]) the results
 * equal observe()'s bit for bit. */
__device__ __forceinline__ bool observe_diff(const L3dTsdfGrid& g, const L3dTsdfView& v,
                                             const uint32_t* __restrict__ depth,
                                             const float* __restrict__ depthf,
                                             const float* __restrict__ prior, int gx, int gy,
                                             int gz, float* obs, float* wout, long long* pix,
                                             float* dobs, float* dw) {
    float wx = fmaf((float)gx + 0.5f, g.voxel, g.origin[0]);
    float wy = fmaf((float)gy + 0.5f, g.voxel, g.origin[1]);
    float wz = fmaf((float)gz + 0.5f, g.voxel, g.origin[2]);
    const float* R = v.R;
    float3 cam = make_float3(fmaf(R[2], wz, fmaf(R[1], wy, fmaf(R[0], wx, v.t[0]))),
                             fmaf(R[5], wz, fmaf(R[4], wy, fmaf(R[3], wx, v.t[1]))),
                             fmaf(R[8], wz, fmaf(R[7], wy, fmaf(R[6], wx, v.t[2]))));
    if (!(cam.z > 0.01f)) return false;
    float iz = 1.0f / cam.z;
    float rx = rintf(fmaf(v.k[0] * cam.x, iz, v.k[2]));
    float ry = rintf(fmaf(v.k[1] * cam.y, iz, v.k[3]));
    if (!(rx >= 0.0f && ry >= 0.0f && rx < (float)v.W && ry < (float)v.H)) return false;
    long long i = (long long)(int)ry * v.W + (int)rx;
    uint32_t packed = __ldg(depth + i);
    float d = l3d_f16_to_f32(packed & 0xffffu);
    float w, dwdd = 0.0f;
    if (d > 0.0f) {
        d = __ldg(depthf + i);
        float3 n = unpack_normal(packed);
        float3 cn = normalize3f(cam);
        w = maxw(0.2f, fabsf(dot3f(n, cn)));
        if (v.conf > 0.0f) {
            float c = (float)(packed >> 28) / 8.0f;
            float q = v.conf / d;
            float r = clampw(q, 0.5f, 2.0f);
            float m = maxw(0.15f, (1.0f - c) * (1.0f - c));
            /* w m r^2 with r = conf / d inside the clamp: dr/dd = -conf / d^2 = -r / d */
            if (q > 0.5f && q < 2.0f) dwdd = w * m * 2.0f * r * (-q / d);
            w = w * ((m * r) * r);
        }
        *pix = i;
    } else {
        d = prior ? __ldg(prior + i) : 0.0f;
        w = g.prior_weight;
        *pix = -1;
    }
    if (!(d > 0.0f)) return false;
    float sdf = d - cam.z;
    if (sdf < -g.mu) return false;
    float ratio = sdf / g.mu;
    *obs = minw(1.0f, ratio);
    *dobs = (1.0f < ratio) ? 0.0f : 1.0f / g.mu;
    *wout = w;
    *dw = dwdd;
    return true;
}

/* Out-of-place integration of one view: (tsdf_in, weight_in) -> (tsdf_out, weight_out), every
 * voxel written (in place when the pointers are equal).  Same culling and arithmetic as
 * k_integrate. */
template <bool Q8>
__global__ void __launch_bounds__(256) k_integrate_depth(const L3dTsdfGrid g, const L3dTsdfView v,
                                                         const int32_t* __restrict__ coords,
                                                         const uint8_t* __restrict__ mask,
                                                         const uint32_t* __restrict__ depth,
                                                         const float* __restrict__ depthf,
                                                         const float* __restrict__ prior,
                                                         const float* tsdf_in, const void* weight_in,
                                                         float* tsdf_out, void* weight_out,
                                                         long long voxels) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= voxels) return;
    int gx, gy, gz;
    long long idx, brick;
    if (!quad_coords<1, false>(g, coords, q, &gx, &gy, &gz, &idx, &brick)) return;
    float t = tsdf_in[idx];
    float ww = 0.0f;
    uint32_t wq = 0;
    if (Q8) wq = ((const uint16_t*)weight_in)[idx];
    else ww = ((const float*)weight_in)[idx];
    float obs, w, dobs, dw;
    long long pix;
    if (mask[brick] &&
        observe_diff(g, v, depth, depthf, v.has_prior ? prior : nullptr, gx, gy, gz, &obs, &w, &pix,
                     &dobs, &dw)) {
        if (Q8) apply_q8(t, wq, obs, w, g.max_q);
        else apply_f32(t, ww, obs, w, g.max_weight);
    }
    tsdf_out[idx] = t;
    if (Q8) ((uint16_t*)weight_out)[idx] = (uint16_t)wq;
    else ((float*)weight_out)[idx] = ww;
}

/* Adjoint of k_integrate_depth.  Per voxel, with the state (T0, W0) before the update and the
 * observation o(d) with weight w(d):
 *   T1 = (T0 W0 + o w) / (W0 + w),  W1 = min(W0 + w, max)
 *   dT1/dT0 = W0 / (W0 + w),  dT1/dW0 = (T0 - T1) / (W0 + w)
 *   dT1/dd  = (w do/dd + (o - T1) dw/dd) / (W0 + w),  dW1/dd = dw/dd, dW1/dW0 = 1 (below max)
 * gT, gW are the loss gradients with respect to T1 and W1 (gW may be NULL).  The depth gradient
 * is added into grad_depth with atomics (many voxels see one pixel); grad_tsdf_in and
 * grad_weight_in (either may be NULL) are written for every voxel.  Q8.8 weights are integers:
 * dw/dd and the weight gradients are zero there. */
template <bool Q8>
__global__ void __launch_bounds__(256) k_integrate_depth_grad(
        const L3dTsdfGrid g, const L3dTsdfView v, const int32_t* __restrict__ coords,
        const uint8_t* __restrict__ mask, const uint32_t* __restrict__ depth,
        const float* __restrict__ depthf, const float* __restrict__ prior,
        const float* __restrict__ tsdf_in, const void* __restrict__ weight_in,
        const float* __restrict__ gT, const float* __restrict__ gW, float* __restrict__ grad_depth,
        float* __restrict__ grad_tsdf_in, float* __restrict__ grad_weight_in, long long voxels) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= voxels) return;
    int gx, gy, gz;
    long long idx, brick;
    if (!quad_coords<1, false>(g, coords, q, &gx, &gy, &gz, &idx, &brick)) return;
    const float gt = gT[idx];
    const float gw = (!Q8 && gW) ? gW[idx] : 0.0f;
    float g_t0 = gt, g_w0 = gw;
    float obs, w, dobs, dw;
    long long pix;
    if (mask[brick] &&
        observe_diff(g, v, depth, depthf, v.has_prior ? prior : nullptr, gx, gy, gz, &obs, &w, &pix,
                     &dobs, &dw)) {
        const float t0 = tsdf_in[idx];
        float w0, wu;
        bool updated = true;
        if (Q8) {
            uint32_t wi = (uint32_t)rintf(w * 256.0f);
            updated = wi != 0u;
            w0 = (float)((const uint16_t*)weight_in)[idx] * 0.00390625f;
            wu = (float)wi * 0.00390625f;
            dw = 0.0f;
        } else {
            w0 = ((const float*)weight_in)[idx];
            wu = w;
        }
        if (updated) {
            const float den = w0 + wu;
            const float t1 = fmaf(t0, w0, obs * wu) / den;
            const float below = (!Q8 && (w0 + wu < g.max_weight)) ? 1.0f : 0.0f;
            g_t0 = gt * (w0 / den);
            g_w0 = Q8 ? 0.0f : fmaf(gt, (t0 - t1) / den, gw * below);
            if (pix >= 0 && grad_depth) {
                float gd = gt * (fmaf(wu, dobs, (obs - t1) * dw) / den) + gw * below * dw;
                if (gd != 0.0f) atomicAdd(grad_depth + pix, gd);
            }
        }
    }
    if (grad_tsdf_in) grad_tsdf_in[idx] = g_t0;
    if (grad_weight_in) grad_weight_in[idx] = Q8 ? 0.0f : g_w0;
}

__global__ void k_fill(float* tsdf, void* weight, long long voxels, int q8) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= voxels) return;
    tsdf[i] = 1.0f;
    if (q8) ((uint16_t*)weight)[i] = 0;
    else ((float*)weight)[i] = 0.0f;
}

inline bool vec4_ok(const L3dTsdfGrid& g) { return !g.dense || (g.dims[0] % 4 == 0); }

/* Threads of the integration kernels (brick-major order, see quad_coords). */
inline long long quad_count(const L3dTsdfGrid& g, int vec) {
    return g.bricks * (512 / vec);
}

/* Threads of the per-voxel kernels in voxel-index order. */
inline long long voxel_count(const L3dTsdfGrid& g) {
    if (g.dense) return (long long)g.dims[0] * g.dims[1] * g.dims[2];
    return g.bricks * 512;
}

}  // namespace

cudaError_t l3d_launch_tsdf_visible(const L3dTsdfGrid& g, const L3dTsdfView* views_dev, int n_views,
                                    const int32_t* coords, uint8_t* mask, cudaStream_t stream) {
    long long n = g.bricks * mask_stride(n_views);
    if (n == 0 || n_views == 0) return cudaSuccess;
    k_visible<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(g, views_dev, n_views, coords, mask);
    return cudaGetLastError();
}

long long l3d_depth_tile_count(int W, int H) {
    return (long long)((W + L3D_DEPTH_TILE - 1) / L3D_DEPTH_TILE) * ((H + L3D_DEPTH_TILE - 1) / L3D_DEPTH_TILE);
}

cudaError_t l3d_launch_depth_tiles(const L3dTsdfView* views_dev, int n_views,
                                   const uint32_t* const* depth_ptrs_dev, const float* priors,
                                   float* tiles, long long max_tiles, cudaStream_t stream) {
    if (n_views <= 0 || max_tiles <= 0) return cudaSuccess;
    dim3 grid((unsigned)((max_tiles * 8 + 127) / 128), (unsigned)n_views);
    k_depth_tiles<<<grid, 128, 0, stream>>>(views_dev, n_views, depth_ptrs_dev, priors, tiles, max_tiles);
    return cudaGetLastError();
}

long long l3d_tsdf_super_flags(const L3dTsdfGrid& g, int n_views) {
    if (!g.dense) return 0;
    return (long long)super_count(g, 0) * super_count(g, 1) * super_count(g, 2) * n_views;
}

cudaError_t l3d_launch_tsdf_visible_depth(const L3dTsdfGrid& g, const L3dTsdfView* views_dev, int n_views,
                                          const int32_t* coords, const float* tiles, uint8_t* super,
                                          uint8_t* mask, cudaStream_t stream) {
    long long n = g.bricks * mask_stride(n_views);
    if (n == 0 || n_views == 0) return cudaSuccess;
    const long long ns = l3d_tsdf_super_flags(g, n_views);
    const bool use_super = super && tiles && ns > 0;
    if (use_super) {
        k_super_behind<<<(unsigned)((ns + 255) / 256), 256, 0, stream>>>(g, views_dev, n_views, tiles, super);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    k_visible_depth<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(g, views_dev, n_views, coords, tiles,
                                                                   use_super ? super : nullptr, mask);
    return cudaGetLastError();
}

cudaError_t l3d_launch_tsdf_view(const L3dTsdfGrid& g, const L3dTsdfView& v, const int32_t* coords,
                                 uint8_t* mask, const uint32_t* depth, const float* prior,
                                 const float4* normals, float* tiles, int32_t* list, float* tsdf,
                                 void* weight, int q8, cudaStream_t stream) {
    if (g.bricks == 0) return cudaSuccess;
    if (tiles && list && normals) {
        /* kept bricks only: tiles, the listing cull, a grid-stride sweep of the listed bricks */
        const long long nt = l3d_depth_tile_count(v.W, v.H);
        L3dTsdfView vt = v;
        vt.tile_off = 0;
        cudaError_t e = cudaMemsetAsync(list, 0, sizeof(int32_t), stream);
        if (e != cudaSuccess) return e;
        k_depth_tiles_one<<<(unsigned)((nt * 8 + 127) / 128), 128, 0, stream>>>(vt, depth, prior, tiles);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        k_visible_one_list<<<(unsigned)((g.bricks + 255) / 256), 256, 0, stream>>>(g, vt, coords, tiles, mask, list);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const unsigned blocks = (unsigned)std::min<long long>(148 * 8, (g.bricks * 128 + 255) / 256);
        if (vec4_ok(g)) {
            if (q8) k_integrate_list<4, true><<<blocks, 256, 0, stream>>>(g, v, coords, list, depth, prior, normals, tsdf, weight);
            else k_integrate_list<4, false><<<blocks, 256, 0, stream>>>(g, v, coords, list, depth, prior, normals, tsdf, weight);
        } else {
            if (q8) k_integrate_list<1, true><<<blocks, 256, 0, stream>>>(g, v, coords, list, depth, prior, normals, tsdf, weight);
            else k_integrate_list<1, false><<<blocks, 256, 0, stream>>>(g, v, coords, list, depth, prior, normals, tsdf, weight);
        }
        return cudaGetLastError();
    }
    if (tiles) {
        const long long nt = l3d_depth_tile_count(v.W, v.H);
        L3dTsdfView vt = v;
        vt.tile_off = 0;
        k_depth_tiles_one<<<(unsigned)((nt * 8 + 127) / 128), 128, 0, stream>>>(vt, depth, prior, tiles);
        k_visible_one_depth<<<(unsigned)((g.bricks + 255) / 256), 256, 0, stream>>>(g, vt, coords, tiles, mask);
    } else {
        k_visible_one<<<(unsigned)((g.bricks + 255) / 256), 256, 0, stream>>>(g, v, coords, mask);
    }
    const int vec = vec4_ok(g) ? 4 : 1;
    long long quads = quad_count(g, vec);
    if (quads == 0) return cudaSuccess;
    unsigned blocks = (unsigned)((quads + 255) / 256);
#define L3D_INTEGRATE(V, Q, L) \
    k_integrate<V, Q, L><<<blocks, 256, 0, stream>>>(g, v, coords, mask, depth, prior, normals, tsdf, weight, quads)
    if (normals) {
        if (vec == 4) {
            if (q8) L3D_INTEGRATE(4, true, true);
            else L3D_INTEGRATE(4, false, true);
        } else {
            if (q8) L3D_INTEGRATE(1, true, true);
            else L3D_INTEGRATE(1, false, true);
        }
    } else {
        if (vec == 4) {
            if (q8) L3D_INTEGRATE(4, true, false);
            else L3D_INTEGRATE(4, false, false);
        } else {
            if (q8) L3D_INTEGRATE(1, true, false);
            else L3D_INTEGRATE(1, false, false);
        }
    }
#undef L3D_INTEGRATE
    return cudaGetLastError();
}

cudaError_t l3d_launch_tsdf_count(const L3dTsdfGrid& g, const L3dTsdfView* views_dev, int n_views,
                                  const int32_t* coords, const uint8_t* mask,
                                  const uint32_t* const* depth_ptrs_dev, const float* priors,
                                  const float4* normals, unsigned long long* counts,
                                  cudaStream_t stream) {
    const int vec = vec4_ok(g) ? 4 : 1;
    long long quads = quad_count(g, vec);
    if (quads == 0 || n_views == 0) return cudaSuccess;
    unsigned blocks = (unsigned)((quads + 255) / 256);
    if (vec == 4)
        k_count_updates<4><<<blocks, 256, 0, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, quads, counts);
    else
        k_count_updates<1><<<blocks, 256, 0, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, quads, counts);
    return cudaGetLastError();
}

cudaError_t l3d_launch_normal_table(float4* normals, cudaStream_t stream) {
    k_normal_table<<<16, 256, 0, stream>>>(normals);
    return cudaGetLastError();
}

long long l3d_tsdf_sweep_units(const L3dTsdfGrid& g, long long* layer_units, long long* layer_voxels) {
    const int vec = vec4_ok(g) ? 4 : 1;
    if (g.dense) {
        if (layer_units) *layer_units = (long long)g.nb[0] * g.nb[1] * (512 / vec);
        if (layer_voxels) *layer_voxels = 8ll * g.dims[0] * g.dims[1];
    } else {
        if (layer_units) *layer_units = 512 / vec;
        if (layer_voxels) *layer_voxels = 512;
    }
    return quad_count(g, vec);
}

cudaError_t l3d_launch_tsdf_many_range(const L3dTsdfGrid& g, const L3dTsdfView* views_dev,
                                       int n_views, const int32_t* coords, const uint8_t* mask,
                                       const uint32_t* const* depth_ptrs_dev, const float* priors,
                                       const float4* normals, float* tsdf, void* weight, int q8,
                                       long long q_begin, long long q_end, cudaStream_t stream) {
    const int vec = vec4_ok(g) ? 4 : 1;
    q_end = q_end < quad_count(g, vec) ? q_end : quad_count(g, vec);
    if (q_end <= q_begin || n_views == 0) return cudaSuccess;
    unsigned blocks = (unsigned)((q_end - q_begin + 255) / 256);
    if (vec == 4) {
        if (q8) k_integrate_many<4, true><<<blocks, 256, 0, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, tsdf, weight, q_begin, q_end);
        else k_integrate_many<4, false><<<blocks, 256, 0, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, tsdf, weight, q_begin, q_end);
    } else {
        if (q8) k_integrate_many<1, true><<<blocks, 256, 0, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, tsdf, weight, q_begin, q_end);
        else k_integrate_many<1, false><<<blocks, 256, 0, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, tsdf, weight, q_begin, q_end);
    }
    return cudaGetLastError();
}

cudaError_t l3d_launch_tsdf_brick_list(const L3dTsdfGrid& g, int n_views, const uint8_t* mask,
                                      uint32_t* flags, uint32_t* prefix, int32_t* list,
                                      uint32_t* scratch, cudaStream_t stream) {
    if (g.bricks == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((g.bricks + 1 + 255) / 256);
    k_brick_any<<<blocks, 256, 0, stream>>>(mask, mask_stride(n_views), g.bricks, flags);
    cudaError_t e = l3d_scan_exclusive(flags, prefix, g.bricks + 1, scratch, nullptr, stream);
    if (e != cudaSuccess) return e;
    k_brick_list_fill<<<blocks, 256, 0, stream>>>(flags, prefix, g.bricks, list);
    return cudaGetLastError();
}

cudaError_t l3d_launch_tsdf_many_list(const L3dTsdfGrid& g, const L3dTsdfView* views_dev,
                                      int n_views, const int32_t* coords, const uint8_t* mask,
                                      const uint32_t* const* depth_ptrs_dev, const float* priors,
                                      const float4* normals, float* tsdf, void* weight, int q8,
                                      const uint32_t* prefix, const int32_t* list,
                                      long long q_begin, long long q_end, cudaStream_t stream) {
    const int vec = vec4_ok(g) ? 4 : 1;
    const long long per = 512 / vec;
    q_end = q_end < quad_count(g, vec) ? q_end : quad_count(g, vec);
    if (q_end <= q_begin || n_views == 0) return cudaSuccess;
    const long long b0 = q_begin / per, b1 = (q_end + per - 1) / per;
    /* a grid-stride loop: four resident blocks per SM */
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        sms = 148;
    const unsigned blocks = (unsigned)(4 * sms);
    const size_t smem = (size_t)n_views * sizeof(L3dTsdfView);
    if (smem > 48 * 1024)  /* more than ~200 views: the sweep of every quad, views from global memory */
        return l3d_launch_tsdf_many_range(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors,
                                          normals, tsdf, weight, q8, q_begin, q_end, stream);
    if (vec == 4) {
        if (q8) k_integrate_many_list<4, true><<<blocks, 256, smem, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, tsdf, weight, prefix, list, b0, b1);
        else k_integrate_many_list<4, false><<<blocks, 256, smem, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, tsdf, weight, prefix, list, b0, b1);
    } else {
        if (q8) k_integrate_many_list<1, true><<<blocks, 256, smem, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, tsdf, weight, prefix, list, b0, b1);
        else k_integrate_many_list<1, false><<<blocks, 256, smem, stream>>>(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors, normals, tsdf, weight, prefix, list, b0, b1);
    }
    return cudaGetLastError();
}

cudaError_t l3d_launch_tsdf_many(const L3dTsdfGrid& g, const L3dTsdfView* views_dev, int n_views,
                                 const int32_t* coords, const uint8_t* mask,
                                 const uint32_t* const* depth_ptrs_dev, const float* priors,
                                 const float4* normals, float* tsdf, void* weight, int q8,
                                 cudaStream_t stream) {
    return l3d_launch_tsdf_many_range(g, views_dev, n_views, coords, mask, depth_ptrs_dev, priors,
                                      normals, tsdf, weight, q8, 0, l3d_tsdf_sweep_units(g, nullptr, nullptr),
                                      stream);
}

cudaError_t l3d_launch_tsdf_depth(const L3dTsdfGrid& g, const L3dTsdfView& v, const int32_t* coords,
                                  uint8_t* mask, const uint32_t* depth, const float* depthf,
                                  const float* prior, const float* tsdf_in, const void* weight_in,
                                  float* tsdf_out, void* weight_out, const float* grad_tsdf_out,
                                  const float* grad_weight_out, float* grad_depth,
                                  float* grad_tsdf_in, float* grad_weight_in, int q8,
                                  cudaStream_t stream) {
    if (g.bricks == 0) return cudaSuccess;
    k_visible_one<<<(unsigned)((g.bricks + 255) / 256), 256, 0, stream>>>(g, v, coords, mask);
    const long long voxels = voxel_count(g);
    if (voxels == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((voxels + 255) / 256);
    if (grad_tsdf_out) {
        if (q8) k_integrate_depth_grad<true><<<blocks, 256, 0, stream>>>(g, v, coords, mask, depth, depthf, prior, tsdf_in, weight_in, grad_tsdf_out, grad_weight_out, grad_depth, grad_tsdf_in, grad_weight_in, voxels);
        else k_integrate_depth_grad<false><<<blocks, 256, 0, stream>>>(g, v, coords, mask, depth, depthf, prior, tsdf_in, weight_in, grad_tsdf_out, grad_weight_out, grad_depth, grad_tsdf_in, grad_weight_in, voxels);
    } else {
        if (q8) k_integrate_depth<true><<<blocks, 256, 0, stream>>>(g, v, coords, mask, depth, depthf, prior, tsdf_in, weight_in, tsdf_out, weight_out, voxels);
        else k_integrate_depth<false><<<blocks, 256, 0, stream>>>(g, v, coords, mask, depth, depthf, prior, tsdf_in, weight_in, tsdf_out, weight_out, voxels);
    }
    return cudaGetLastError();
}

cudaError_t l3d_launch_tsdf_fill(float* tsdf, void* weight, long long voxels, int q8,
                                 cudaStream_t stream) {
    if (voxels == 0) return cudaSuccess;
    k_fill<<<(unsigned)((voxels + 255) / 256), 256, 0, stream>>>(tsdf, weight, voxels, q8);
    return cudaGetLastError();
}
