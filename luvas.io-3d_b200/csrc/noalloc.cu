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
 * the GPU (different streams, no ordering between them) race on the flags.  The cached address
 * belongs to the device's context: after cudaDeviceReset the process must not call this entry
 * point again on that device (the address would be stale).
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
    if (!(view->intrinsics.fx != 0.0) || !(view->intrinsics.fy != 0.0))
        return noalloc_fail(L3D_EINVAL, "zero focal length");
    if (((uintptr_t)tsdf_dev & 15u) || ((uintptr_t)weight_dev & 15u))
        return noalloc_fail(L3D_EINVAL, "tsdf and weight buffers must be 16-byte aligned");
    /* the grid and view constants of the handle API (l3d_tsdf_create / l3d_tsdf_integrate) */
    L3dTsdfGrid g;
    char why[256];
    if (!l3d_tsdf_grid_of(d, coords_dev != nullptr, &g, why, sizeof(why))) return noalloc_fail(L3D_EINVAL, why);
    if (g.bricks > L3D_NOALLOC_MAX_BRICKS) {
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "volume has %lld bricks; the allocation-free integrate handles at most %d "
                      "(use l3d_tsdf_create / l3d_tsdf_integrate)",
                      g.bricks, (int)L3D_NOALLOC_MAX_BRICKS);
        return noalloc_fail(L3D_EINVAL, msg);
    }
    L3dTsdfView v = l3d_tsdf_view_of(*view);
    v.has_prior = prior_dev != nullptr;  /* the prior is the caller's device map, not view->prior */
    v.W = d->width;
    v.H = d->height;

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
