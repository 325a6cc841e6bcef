/*
 * Exclusive prefix sum of u32 counts on the device (stream compaction for surface extraction,
 * the brick grid and component removal).  Each block scans 1024 elements (256 threads x 4) with
 * warp shuffles and writes its total; the block totals are scanned the same way, recursively,
 * and added back.  Deterministic: the result does not depend on scheduling.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "l3d_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPer = 4;
constexpr int kTile = kThreads * kPer;

__global__ void __launch_bounds__(kThreads) k_scan_block(const uint32_t* in, uint32_t* out,
                                                        long long n, uint32_t* block_sums) {
    __shared__ uint32_t warp_sums[kThreads / 32];
    const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kPer;
    uint32_t v[kPer];
    uint32_t local = 0;
#pragma unroll
    for (int i = 0; i < kPer; i++) {
        v[i] = (base + i < n) ? in[base + i] : 0u;
        local += v[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = local;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kThreads / 32 ? warp_sums[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, off);
            if (lane >= off) wi += t;
        }
        if (lane < kThreads / 32) warp_sums[lane] = wi - w;   /* exclusive warp offsets */
        if (lane == kThreads / 32 - 1 && block_sums) block_sums[blockIdx.x] = wi;
    }
    __syncthreads();
    uint32_t run = warp_sums[warp] + incl - local;
#pragma unroll
    for (int i = 0; i < kPer; i++) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

__global__ void k_scan_add(uint32_t* out, long long n, const uint32_t* offsets) {
    const long long i = (long long)blockIdx.x * kTile + threadIdx.x;
    const uint32_t o = offsets[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        const long long j = i + (long long)k * kThreads;
        if (j < n) out[j] += o;
    }
}

/* total = exclusive[n - 1] + in[n - 1], read before an in-place scan overwrote `in` */
__global__ void k_scan_last(const uint32_t* in, long long n, uint32_t* last) { *last = in[n - 1]; }
__global__ void k_scan_total(const uint32_t* out, long long n, const uint32_t* last, uint32_t* total) {
    *total = out[n - 1] + *last;
}

long long blocks_of(long long n) { return (n + kTile - 1) / kTile; }

}  // namespace

size_t l3d_scan_scratch(long long n) {
    size_t words = 1;  /* the last input element */
    for (long long m = blocks_of(n); m > 1; m = blocks_of(m)) words += (size_t)m;
    return (words + 1) * sizeof(uint32_t);
}

int l3d_scan_launches(long long n, bool total) {
    if (n <= 0) return 0;
    int depth = 0;
    for (long long m = n; blocks_of(m) > 1; m = blocks_of(m)) depth++;
    return 1 + (depth + 1) + depth + (total ? 1 : 0);  /* last, block scans, add-backs, total */
}

cudaError_t l3d_scan_exclusive(const uint32_t* in, uint32_t* out, long long n, uint32_t* scratch,
                               uint32_t* total, cudaStream_t stream) {
    if (n <= 0) {
        if (total) return cudaMemsetAsync(total, 0, sizeof(uint32_t), stream);
        return cudaSuccess;
    }
    uint32_t* last = scratch;
    k_scan_last<<<1, 1, 0, stream>>>(in, n, last);
    /* levels: out (n), then block sums of each level in scratch */
    const uint32_t* src = in;
    uint32_t* dst = out;
    long long m = n;
    uint32_t* level = scratch + 1;
    struct Level { uint32_t* data; long long n; };
    Level stack[8];
    int depth = 0;
    for (;;) {
        const long long b = blocks_of(m);
        uint32_t* sums = b > 1 ? level : nullptr;
        k_scan_block<<<(unsigned)b, kThreads, 0, stream>>>(src, dst, m, sums);
        if (b == 1) break;
        if (depth >= 8) return cudaErrorInvalidValue;
        stack[depth++] = {dst, m};
        src = level;
        dst = level;  /* scanned in place */
        m = b;
        level += b;
    }
    /* add each level's scanned block sums back into the level below */
    for (int d = depth - 1; d >= 0; d--) {
        const uint32_t* offs = d == depth - 1 ? dst : stack[d + 1].data;
        k_scan_add<<<(unsigned)blocks_of(stack[d].n), kThreads, 0, stream>>>(stack[d].data, stack[d].n, offs);
    }
    if (total) k_scan_total<<<1, 1, 0, stream>>>(out, n, last, total);
    return cudaGetLastError();
}
