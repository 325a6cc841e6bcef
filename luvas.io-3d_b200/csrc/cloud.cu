/*
 * Dense point cloud: packed depth maps fused into cell-averaged points on the device.
 *
 * frontend/src/app/vision/fusion/depth-fusion.ts:42-74 decodes every valid sample of a filtered
 * depth map into a world point, a world normal and a thumbnail colour, and
 * frontend/src/app/vision/fusion/point-accumulator.ts:16-147 averages them per cell of a grid
 * (open-addressing hash on the integer cell, growth at 60 % load, coarsening that re-bins cell
 * means into a larger cell).  Here one thread decodes one pixel and adds it to a device hash
 * table with atomics:
 *   - keys: the integer cell packed into 63 bits (21 bits per axis, biased by 2^20), claimed with
 *     atomicCAS on linear probes from the reference's hash; cells beyond +-2^20 set an error flag;
 *   - sums: nine FP64 sums per slot (position, normal, colour), added with FP64 atomics (the
 *     reference keeps f32 sums; FP64 makes the result independent of the order of the adds up
 *     to rounding at the last bit);
 *   - counts: u32 per slot; `used`: the number of claimed slots.
 * Decoding and the world transform run in FP64 in the reference's operation order.  Probing is
 * bounded by the table size (the host keeps the load under 60 %, so a free slot always exists);
 * a probe that runs out sets an error flag instead of looping.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "l3d_fmath.h"
#include "l3d_internal.h"

namespace {

constexpr unsigned long long kEmpty = ~0ull;
constexpr int kBias = 1 << 20;

__device__ __forceinline__ uint32_t cell_hash(int x, int y, int z) {
    return ((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349663u) ^ ((uint32_t)z * 83492791u);
}

__device__ __forceinline__ bool pack_key(double fx, double fy, double fz, unsigned long long* key,
                                         int* ix, int* iy, int* iz) {
    if (!(fabs(fx) < (double)kBias && fabs(fy) < (double)kBias && fabs(fz) < (double)kBias))
        return false;
    *ix = (int)fx;
    *iy = (int)fy;
    *iz = (int)fz;
    *key = (unsigned long long)(*ix + kBias) | ((unsigned long long)(*iy + kBias) << 21) |
           ((unsigned long long)(*iz + kBias) << 42);
    return true;
}

/* Slot of the cell (claimed when new), or -1 after setting an error flag. */
__device__ int claim(const L3dCloudTable& t, double cx, double cy, double cz, unsigned* used,
                     int* err) {
    unsigned long long key;
    int ix, iy, iz;
    if (!pack_key(floor(cx), floor(cy), floor(cz), &key, &ix, &iy, &iz)) {
        atomicOr(err, L3D_CLOUD_ERR_RANGE);
        return -1;
    }
    const unsigned mask = (unsigned)t.capacity - 1u;
    unsigned slot = cell_hash(ix, iy, iz) & mask;
    for (int probe = 0; probe < t.capacity; probe++) {
        const unsigned long long k = __ldcg(t.keys + slot);
        if (k == key) return (int)slot;
        if (k == kEmpty) {
            const unsigned long long prev = atomicCAS(t.keys + slot, kEmpty, key);
            if (prev == kEmpty) {
                atomicAdd(used, 1u);
                return (int)slot;
            }
            if (prev == key) return (int)slot;
        }
        slot = (slot + 1u) & mask;
    }
    atomicOr(err, L3D_CLOUD_ERR_FULL);
    return -1;
}

__device__ __forceinline__ void accumulate(const L3dCloudTable& t, int slot, const double* v,
                                           unsigned n) {
    double* s = t.sums + (size_t)slot * 9;
#pragma unroll
    for (int i = 0; i < 9; i++) atomicAdd(s + i, v[i]);
    atomicAdd(t.counts + slot, n);
}

__device__ void sample_of(const L3dCloudView& v, uint32_t value, double d, int x, int y, int W,
                          int H, const uint8_t* __restrict__ rgb, double* p);

/* addDepthMap (depth-fusion.ts:42-74) for one pixel; unpackDepthSample (depth-maps.ts:66-85).
 * Neighbouring pixels mostly land in the same cell: the lanes of a warp that share a cell add
 * their samples up first (in lane order), and one of them claims the cell and adds the sum, so
 * the table sees one set of atomics per cell and warp instead of one per pixel. */
__global__ void k_cloud_add_map(const L3dCloudTable t, double cell, const uint32_t* __restrict__ packed,
                                int W, int H, const L3dCloudView v, const uint8_t* __restrict__ rgb,
                                unsigned* used, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t value = i < W * H ? __ldg(packed + i) : 0u;
    const double d = value ? (double)l3d_f16_to_f32(value & 0xffffu) : 0.0;
    double p[9];
    unsigned long long key = 0;
    bool valid = d > 0.0;
    if (valid) {
        sample_of(v, value, d, i % W, i / W, W, H, rgb, p);
        int ix, iy, iz;
        valid = pack_key(floor(p[0] / cell), floor(p[1] / cell), floor(p[2] / cell), &key, &ix, &iy, &iz);
        if (!valid) atomicOr(err, L3D_CLOUD_ERR_RANGE);
    }
    const unsigned active = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    const unsigned group = __match_any_sync(active, key);
    double s[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        double acc = 0.0;
        for (unsigned m = group; m; m &= m - 1u) acc += __shfl_sync(group, p[k], __ffs(m) - 1);
        s[k] = acc;
    }
    if ((int)(threadIdx.x & 31u) != __ffs(group) - 1) return;
    const int slot = claim(t, p[0] / cell, p[1] / cell, p[2] / cell, used, err);
    if (slot >= 0) accumulate(t, slot, s, (unsigned)__popc(group));
}

/* The world sample of one valid pixel (depth d > 0): position, normal, thumbnail colour. */
__device__ void sample_of(const L3dCloudView& v, uint32_t value, double d, int x, int y, int W,
                          int H, const uint8_t* __restrict__ rgb, double* p) {
    const double ex = ((double)((value >> 16) & 63u) / 63.0) * 2.0 - 1.0;
    const double ey = ((double)((value >> 22) & 63u) / 63.0) * 2.0 - 1.0;
    double nx = ex, ny = ey;
    const double nz = 1.0 - fabs(ex) - fabs(ey);
    if (nz < 0.0) {
        nx = (1.0 - fabs(ey)) * (ex >= 0.0 ? 1.0 : -1.0);
        ny = (1.0 - fabs(ex)) * (ey >= 0.0 ? 1.0 : -1.0);
    }
    double len = sqrt(nx * nx + ny * ny + nz * nz);
    if (!(len != 0.0)) len = 1.0;
    nx /= len;
    ny /= len;
    const double nzn = nz / len;
    /* fromCamera (camera.ts:57-59): R^T (x_cam - t) */
    const double* R = v.R;
    const double a0 = ((x - v.k[2]) / v.k[0]) * d - v.t[0];
    const double a1 = ((y - v.k[3]) / v.k[1]) * d - v.t[1];
    const double a2 = d - v.t[2];
    p[0] = R[0] * a0 + R[3] * a1 + R[6] * a2;
    p[1] = R[1] * a0 + R[4] * a1 + R[7] * a2;
    p[2] = R[2] * a0 + R[5] * a1 + R[8] * a2;
    p[3] = R[0] * nx + R[3] * ny + R[6] * nzn;
    p[4] = R[1] * nx + R[4] * ny + R[7] * nzn;
    p[5] = R[2] * nx + R[5] * ny + R[8] * nzn;
    const double sx = (double)v.tw / W, sy = (double)v.th / H;
    const int tx = min(v.tw - 1, (int)floor((x + 0.5) * sx));
    const int ty = min(v.th - 1, (int)floor((y + 0.5) * sy));
    const uint8_t* c = rgb + ((size_t)ty * v.tw + tx) * 3;
    p[6] = c[0];
    p[7] = c[1];
    p[8] = c[2];
}

/* PointAccumulator.add (point-accumulator.ts:29-56) of n samples of 9 doubles. */
__global__ void k_cloud_add_points(const L3dCloudTable t, double cell, const double* __restrict__ pts,
                                   long long n, unsigned* used, int* err) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double p[9];
#pragma unroll
    for (int j = 0; j < 9; j++) p[j] = pts[i * 9 + j];
    const int slot = claim(t, p[0] / cell, p[1] / cell, p[2] / cell, used, err);
    if (slot >= 0) accumulate(t, slot, p, 1u);
}

/* rebuild (point-accumulator.ts:89-111): every occupied slot re-binned by its mean position
 * into the table `to` with cell size `cell`. */
__global__ void k_cloud_rebin(const L3dCloudTable from, const L3dCloudTable to, double cell,
                              unsigned* used, int* err) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= from.capacity || from.keys[s] == kEmpty) return;
    const unsigned n = from.counts[s];
    const double* src = from.sums + (size_t)s * 9;
    double p[9];
#pragma unroll
    for (int j = 0; j < 9; j++) p[j] = src[j];
    const double dn = (double)n;
    const int slot = claim(to, p[0] / dn / cell, p[1] / dn / cell, p[2] / dn / cell, used, err);
    if (slot >= 0) accumulate(to, slot, p, n);
}

/* cloud(minSupport) (point-accumulator.ts:114-143), in three steps on the device: the cell keys
 * and slots of the slots with enough support (arbitrary order), the pairs sorted by key, then
 * the averaged points gathered in key order (cells ascending: z, then y, then x). */
__global__ void k_cloud_emit_keys(const L3dCloudTable t, unsigned min_support, unsigned* count,
                                  unsigned long long* keys, uint32_t* slots) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= t.capacity) return;
    const unsigned long long key = t.keys[s];
    if (key == kEmpty || t.counts[s] < min_support) return;
    const unsigned o = atomicAdd(count, 1u);
    keys[o] = key;
    slots[o] = (uint32_t)s;
}

__global__ void k_cloud_emit_sorted(const L3dCloudTable t, unsigned total,
                                    const unsigned long long* __restrict__ keys,
                                    const uint32_t* __restrict__ slots, float* pos, float* nrm,
                                    uint8_t* col, uint16_t* support, int32_t* cells) {
    const unsigned o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= total) return;
    const uint32_t s = slots[o];
    const unsigned long long key = keys[o];
    const unsigned n = t.counts[s];
    const double* sm = t.sums + (size_t)s * 9;
    const double dn = (double)n;
    for (int j = 0; j < 3; j++) pos[(size_t)o * 3 + j] = (float)(sm[j] / dn);
    double len = sqrt(sm[3] * sm[3] + sm[4] * sm[4] + sm[5] * sm[5]);
    if (!(len != 0.0)) len = 1.0;
    for (int j = 0; j < 3; j++) nrm[(size_t)o * 3 + j] = (float)(sm[3 + j] / len);
    for (int j = 0; j < 3; j++) {
        /* Uint8Array store: truncation, then modulo 256 */
        double c = trunc(sm[6 + j] / dn);
        c = c - 256.0 * floor(c / 256.0);
        col[(size_t)o * 3 + j] = (uint8_t)c;
    }
    support[o] = (uint16_t)min(n, 65535u);
    for (int j = 0; j < 3; j++)
        cells[(size_t)o * 3 + j] = (int32_t)((long long)((key >> (21 * j)) & 0x1FFFFFull) - kBias);
}

/* Bitonic sort of n = 2^m (key, value) pairs, m >= 11, ascending by key.  Stages with a
 * partner distance under 2048 run in shared memory, 2048 pairs per block of 1024 threads. */
constexpr int kSortTile = 2048;

__global__ void k_pad_keys(unsigned long long* keys, unsigned from, unsigned n) {
    const unsigned i = from + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keys[i] = kEmpty;
}

__device__ __forceinline__ void order_pair(unsigned long long* k, uint32_t* v, unsigned i, unsigned l,
                                           bool ascending) {
    const unsigned long long a = k[i], b = k[l];
    if ((a > b) == ascending) {
        k[i] = b;
        k[l] = a;
        const uint32_t t = v[i];
        v[i] = v[l];
        v[l] = t;
    }
}

/* stages (k, j) with j < kSortTile: every k from 2 up to kmax when kfrom == 2 (sorts each tile),
 * or the single k = kfrom with j from kSortTile / 2 down to 1 */
__global__ void __launch_bounds__(1024) k_bitonic_tile(unsigned long long* keys, uint32_t* vals,
                                                       unsigned kfrom, unsigned kmax) {
    __shared__ unsigned long long sk[kSortTile];
    __shared__ uint32_t sv[kSortTile];
    const unsigned base = blockIdx.x * kSortTile;
    for (unsigned i = threadIdx.x; i < kSortTile; i += blockDim.x) {
        sk[i] = keys[base + i];
        sv[i] = vals[base + i];
    }
    __syncthreads();
    for (unsigned k = kfrom; k <= kmax; k <<= 1) {
        for (unsigned j = min(k >> 1, (unsigned)kSortTile >> 1); j > 0; j >>= 1) {
            const unsigned t = threadIdx.x;
            const unsigned i = 2 * j * (t / j) + (t % j);
            order_pair(sk, sv, i, i + j, ((base + i) & k) == 0);
            __syncthreads();
        }
    }
    for (unsigned i = threadIdx.x; i < kSortTile; i += blockDim.x) {
        keys[base + i] = sk[i];
        vals[base + i] = sv[i];
    }
}

/* one stage (k, j) with j >= kSortTile over all n / 2 pairs */
__global__ void k_bitonic_global(unsigned long long* keys, uint32_t* vals, unsigned n, unsigned k,
                                 unsigned j) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n / 2) return;
    const unsigned i = 2 * j * (t / j) + (t % j);
    order_pair(keys, vals, i, i + j, (i & k) == 0);
}

__global__ void k_cloud_clear(L3dCloudTable t) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= t.capacity) return;
    t.keys[s] = kEmpty;
    t.counts[s] = 0u;
    double* sm = t.sums + (size_t)s * 9;
#pragma unroll
    for (int j = 0; j < 9; j++) sm[j] = 0.0;
}

inline unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

cudaError_t l3d_launch_cloud_clear(const L3dCloudTable& t, cudaStream_t stream) {
    k_cloud_clear<<<blocks_for(t.capacity), 256, 0, stream>>>(t);
    return cudaGetLastError();
}

cudaError_t l3d_launch_cloud_add_map(const L3dCloudTable& t, double cell, const uint32_t* packed,
                                     int W, int H, const L3dCloudView& v, const uint8_t* rgb,
                                     unsigned* used, int* err, cudaStream_t stream) {
    if ((long long)W * H == 0) return cudaSuccess;
    k_cloud_add_map<<<blocks_for((long long)W * H), 256, 0, stream>>>(t, cell, packed, W, H, v, rgb,
                                                                      used, err);
    return cudaGetLastError();
}

cudaError_t l3d_launch_cloud_add_points(const L3dCloudTable& t, double cell, const double* pts,
                                        long long n, unsigned* used, int* err, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    k_cloud_add_points<<<blocks_for(n), 256, 0, stream>>>(t, cell, pts, n, used, err);
    return cudaGetLastError();
}

cudaError_t l3d_launch_cloud_rebin(const L3dCloudTable& from, const L3dCloudTable& to, double cell,
                                   unsigned* used, int* err, cudaStream_t stream) {
    k_cloud_rebin<<<blocks_for(from.capacity), 256, 0, stream>>>(from, to, cell, used, err);
    return cudaGetLastError();
}

cudaError_t l3d_launch_cloud_emit_keys(const L3dCloudTable& t, unsigned min_support,
                                       unsigned* count, unsigned long long* keys, uint32_t* slots,
                                       cudaStream_t stream) {
    k_cloud_emit_keys<<<blocks_for(t.capacity), 256, 0, stream>>>(t, min_support, count, keys, slots);
    return cudaGetLastError();
}

unsigned l3d_cloud_sort_length(unsigned total) {
    unsigned n = kSortTile;
    while (n < total) n <<= 1;
    return n;
}

cudaError_t l3d_launch_cloud_sort(unsigned long long* keys, uint32_t* slots, unsigned total,
                                  unsigned n, long long* launches, cudaStream_t stream) {
    if (n < (unsigned)kSortTile || (n & (n - 1))) return cudaErrorInvalidValue;
    long long count = 0;
    if (n > total) {
        k_pad_keys<<<blocks_for(n - total), 256, 0, stream>>>(keys, total, n);
        count++;
    }
    const unsigned tiles = n / kSortTile;
    k_bitonic_tile<<<tiles, 1024, 0, stream>>>(keys, slots, 2, kSortTile);
    count++;
    for (unsigned k = 2 * kSortTile; k <= n; k <<= 1) {
        for (unsigned j = k >> 1; j >= (unsigned)kSortTile; j >>= 1, count++)
            k_bitonic_global<<<blocks_for(n / 2), 256, 0, stream>>>(keys, slots, n, k, j);
        k_bitonic_tile<<<tiles, 1024, 0, stream>>>(keys, slots, k, k);
        count++;
    }
    if (launches) *launches += count;
    return cudaGetLastError();
}

cudaError_t l3d_launch_cloud_emit_sorted(const L3dCloudTable& t, unsigned total,
                                         const unsigned long long* keys, const uint32_t* slots,
                                         float* pos, float* nrm, uint8_t* col, uint16_t* support,
                                         int32_t* cells, cudaStream_t stream) {
    if (total == 0) return cudaSuccess;
    k_cloud_emit_sorted<<<blocks_for(total), 256, 0, stream>>>(t, total, keys, slots, pos, nrm, col,
                                                              support, cells);
    return cudaGetLastError();
}
