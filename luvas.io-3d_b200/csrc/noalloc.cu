/*
 * Allocation-free TSDF integration of one depth map (l3d_tsdf_integrate_noalloc).
 *
 * Some callers cannot let this library allocate device memory: their device memory belongs to
 * another allocator (a framework's caching allocator, or a pool sized once at start-up and
 * handed out in slices), or they run inside a pipeline where cudaMalloc/cudaFree would stall
 * every stream on the device.  For them this entry point integrates a depth map into a volume
 * whose buffers the caller owns, without creating a handle and without any allocation.
 *
 * The only extra device memory the integration needs is one visibility flag per 8^3 brick.  It
 * lives in the static array below, sized for L3D_NOALLOC_MAX_BRICKS bricks (1 MiB), which every
 * GPU that loads this library keeps until the process exits.  Host code cannot use the array's
 * name as a device address, so the first call on each device looks its address up with
 * cudaGetSymbolAddress (with that device current) and caches it; later calls reuse it.
 *
 * Every call shares the array.  Each call rewrites the flags of all bricks of its volume before
 * the integration reads them, so nothing needs clearing; but two calls whose kernels overlap on
 * the GPU (different streams, no ordering between them) race on the flags.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/luvas3d.h"
#include "l3d_internal.h"

namespace {

static __device__ __align__(256) uint8_t g_brick_flags[L3D_NOALLOC_MAX_BRICKS];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_flags_ptr[kMaxDevices] = {nullptr};

int noalloc_fail(int code, const char* msg) {
    l3d_set_error(msg);  /* reported by l3d_last_error() like every other entry point */
    return code;
}

/* Device address of g_brick_flags on the current device (set up once per device). */
int flags_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return L3D_ECUDA;
    if (dev < 0 || dev >= kMaxDevices) return L3D_EINVAL;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_flags_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_brick_flags);
        if (e != cudaSuccess || !p) return L3D_ECUDA;
        g_flags_ptr[dev] = p;
    }
    *out = g_flags_ptr[dev];
    return L3D_OK;
}

}  // namespace

extern "C" int l3d_tsdf_integrate_noalloc(const l3d_tsdf_desc* d, const int32_t* coords_dev,
                                          const uint32_t* depth_dev, const float* prior_dev,
                                          const l3d_integration_view* view, float* tsdf_dev,
                                          void* weight_dev, void* stream) {
    if (!d || !view || !depth_dev || !tsdf_dev || !weight_dev)
        return noalloc_fail(L3D_EINVAL, "NULL descriptor, view, depth map or volume buffer");
    if (!(d->voxel > 0.0) || !(d->truncation > 0.0) || !(d->max_weight > 0.0))
        return noalloc_fail(L3D_EINVAL, "voxel, truncation and max_weight must be positive");
    if (d->width <= 0 || d->height <= 0)
        return noalloc_fail(L3D_EINVAL, "depth map size must be positive");
    if (d->weight_type != L3D_WEIGHT_F32 && d->weight_type != L3D_WEIGHT_Q8)
        return noalloc_fail(L3D_EINVAL, "unknown weight type");
    if (d->weight_type == L3D_WEIGHT_Q8 && !(d->max_weight * 256.0 <= 65535.0))
        return noalloc_fail(L3D_EINVAL, "Q8.8 weights need max_weight <= 255.99");
    if (!(view->intrinsics.fx != 0.0) || !(view->intrinsics.fy != 0.0))
        return noalloc_fail(L3D_EINVAL, "zero focal length");
    if (((uintptr_t)tsdf_dev & 15u) || ((uintptr_t)weight_dev & 15u))
        return noalloc_fail(L3D_EINVAL, "tsdf and weight buffers must be 16-byte aligned");
    L3dTsdfGrid g;
    std::memset(&g, 0, sizeof(g));
    if (d->dense) {
        for (int i = 0; i < 3; i++) {
            if (d->dims[i] <= 0) return noalloc_fail(L3D_EINVAL, "dense dims must be positive");
            g.dims[i] = d->dims[i];
            g.nb[i] = (d->dims[i] + 7) / 8;
        }
        g.bricks = (long long)g.nb[0] * g.nb[1] * g.nb[2];
    } else {
        if (d->count <= 0 || !coords_dev)
            return noalloc_fail(L3D_EINVAL, "a brick pool needs device coords and count > 0");
        g.bricks = d->count;
    }
    if (g.bricks > L3D_NOALLOC_MAX_BRICKS) {
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "volume has %lld bricks; the allocation-free integrate handles at most %d "
                      "(use l3d_tsdf_create / l3d_tsdf_integrate)",
                      g.bricks, (int)L3D_NOALLOC_MAX_BRICKS);
        return noalloc_fail(L3D_EINVAL, msg);
    }
    for (int i = 0; i < 3; i++) {
        g.origin[i] = (float)d->origin[i];
        g.origin_d[i] = d->origin[i];
    }
    g.voxel = (float)d->voxel;
    g.mu = (float)d->truncation;
    g.prior_weight = (float)d->prior_weight;
    g.max_weight = (float)d->max_weight;
    g.max_q = (unsigned)rintf(g.max_weight * 256.0f);
    g.voxel_d = d->voxel;
    g.trunc_d = d->truncation;
    g.dense = d->dense ? 1 : 0;
    g.W = d->width;
    g.H = d->height;

    L3dTsdfView v;
    std::memset(&v, 0, sizeof(v));
    const double k[4] = {view->intrinsics.fx, view->intrinsics.fy, view->intrinsics.cx,
                         view->intrinsics.cy};
    for (int i = 0; i < 4; i++) {
        v.k[i] = (float)k[i];
        v.kd[i] = k[i];
    }
    for (int i = 0; i < 9; i++) {
        v.R[i] = (float)view->pose.R[i];
        v.Rd[i] = view->pose.R[i];
    }
    for (int i = 0; i < 3; i++) {
        v.t[i] = (float)view->pose.t[i];
        v.td[i] = view->pose.t[i];
    }
    v.conf = (float)view->confidence;
    v.has_prior = prior_dev != nullptr;
    v.W = d->width;
    v.H = d->height;
    v.max_depth = view->max_depth;

    void* flags = nullptr;
    int rc = flags_address(&flags);
    if (rc) return noalloc_fail(rc, "could not look up the brick-flag array on this device");
    cudaError_t e = l3d_launch_tsdf_view(g, v, d->dense ? nullptr : coords_dev, (uint8_t*)flags,
                                         depth_dev, prior_dev, nullptr, nullptr, nullptr, tsdf_dev, weight_dev,
                                         d->weight_type == L3D_WEIGHT_Q8, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        char msg[256];
        std::snprintf(msg, sizeof(msg), "integrate launch: %s", cudaGetErrorString(e));
        return noalloc_fail(L3D_ECUDA, msg);
    }
    return L3D_OK;
}
