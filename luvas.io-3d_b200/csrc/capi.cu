/*
 * C ABI of libluvas3d.so (declared in include/luvas3d.h): handle management, argument checks,
 * dispatch parameters and the solve / filter / integrate schedules.
 *
 * The host side replaces DenseStereo and TsdfVolume (frontend/src/app/vision/mvs/dense-stereo.ts,
 * frontend/src/app/vision/fusion/tsdf-volume.ts).  Differences from the WebGPU host, by design:
 * whole-image launches instead of 20 ms row bands with a host wait per band
 * (dense-stereo.ts:269-298), brick culling on the device instead of a CPU loop
 * (tsdf-volume.ts:220-234), and stream-ordered asynchronous calls instead of awaits.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/luvas3d.h"
#include "l3d_internal.h"

/* Fast-form kernel variant: window rows through the texture unit (0..6; the others use software
 * bilinear on the pair image) + 8 for the 2x2 quad lane mapping (+16 gathers, +32 shared-memory
 * window: see l3d_stereo_set_variant). */
#define L3D_FAST_DEFAULT_VARIANT 14

/* Voxel ranges the sweep of l3d_tsdf_integrate_many_read is split into, each read back as soon
 * as it is done. */
#define L3D_TSDF_READ_SLABS 8

namespace {

thread_local std::string g_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? L3D_ENOMEM : L3D_ECUDA, "%s: %s (%s)", what,
                cudaGetErrorString(e), cudaGetErrorName(e));
}

#define L3D_CUDA(call, what)                          \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

size_t dtype_size(int dtype) {
    switch (dtype) {
        case L3D_DTYPE_U8: return 1;
        case L3D_DTYPE_F32: return 4;
        case L3D_DTYPE_F16:
        case L3D_DTYPE_BF16: return 2;
        default: return 0;
    }
}

/* Scratch buffers and tables that come and go with each call are stream-ordered allocations
 * from a memory pool of the library's own on each device, which keeps up to
 * L3D_POOL_KEEP_BYTES of freed memory mapped for the next call: handing memory back to the
 * driver at every synchronisation and mapping it again costs milliseconds per GB. */
#define L3D_POOL_KEEP_BYTES (16ull << 30)
#define L3D_POOL_DEVICES 64
std::mutex pool_mu;
cudaMemPool_t pools[L3D_POOL_DEVICES] = {};

/* The pool of device `dev`, created on first use when `create` is set (*out stays NULL
 * otherwise). */
cudaError_t device_pool(int dev, bool create, cudaMemPool_t* out) {
    *out = nullptr;
    std::lock_guard<std::mutex> lock(pool_mu);
    if (!pools[dev] && create) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t created;
        cudaError_t e = cudaMemPoolCreate(&created, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = L3D_POOL_KEEP_BYTES;
        if ((e = cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
            cudaMemPoolDestroy(created);
            return e;
        }
        pools[dev] = created;
    }
    *out = pools[dev];
    return cudaSuccess;
}

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= L3D_POOL_DEVICES) return cudaMallocAsync(p, bytes, s);
    cudaMemPool_t pool;
    if ((e = device_pool(dev, true, &pool)) != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) return cudaSuccess;
    return cudaMalloc((void**)p, count * sizeof(T));
}

}  // namespace

/* ---- TSDF descriptor and view conversions shared by the handle API and the allocation-free
 * entry point (noalloc.cu), so both integrate with the same grid and view constants ---- */

bool l3d_tsdf_grid_of(const l3d_tsdf_desc* d, bool pool_coords_given, L3dTsdfGrid* out, char* why,
                      size_t why_size) {
    auto bad = [&](const char* msg) {
        std::snprintf(why, why_size, "%s", msg);
        return false;
    };
    if (!(d->voxel > 0.0) || !(d->truncation > 0.0) || !(d->max_weight > 0.0))
        return bad("voxel, truncation and max_weight must be positive");
    if (d->width <= 0 || d->height <= 0) return bad("depth map size must be positive");
    if (d->weight_type != L3D_WEIGHT_F32 && d->weight_type != L3D_WEIGHT_Q8)
        return bad("unknown weight type");
    if (d->weight_type == L3D_WEIGHT_Q8 && !(d->max_weight * 256.0 <= 65535.0))
        return bad("Q8.8 weights need max_weight <= 255.99");
    L3dTsdfGrid g;
    std::memset(&g, 0, sizeof(g));
    if (d->dense) {
        for (int i = 0; i < 3; i++) {
            if (d->dims[i] <= 0) return bad("dense dims must be positive");
            g.dims[i] = d->dims[i];
            g.nb[i] = (d->dims[i] + 7) / 8;
        }
        g.bricks = (long long)g.nb[0] * g.nb[1] * g.nb[2];
    } else {
        if (d->count <= 0 || !pool_coords_given) return bad("brick pool needs coords and count > 0");
        g.bricks = d->count;
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
    *out = g;
    return true;
}

L3dTsdfView l3d_tsdf_view_of(const l3d_integration_view& v) {
    L3dTsdfView o;
    std::memset(&o, 0, sizeof(o));
    const double k[4] = {v.intrinsics.fx, v.intrinsics.fy, v.intrinsics.cx, v.intrinsics.cy};
    for (int i = 0; i < 4; i++) {
        o.k[i] = (float)k[i];
        o.kd[i] = k[i];
    }
    for (int i = 0; i < 9; i++) {
        o.R[i] = (float)v.pose.R[i];
        o.Rd[i] = v.pose.R[i];
    }
    for (int i = 0; i < 3; i++) {
        o.t[i] = (float)v.pose.t[i];
        o.td[i] = v.pose.t[i];
    }
    o.conf = (float)v.confidence;
    o.has_prior = v.prior != nullptr;
    o.max_depth = v.max_depth;
    return o;
}

/* ------------------------------------------------------------------ stereo handle ---------- */

struct l3d_stereo {
    int W = 0, H = 0, V = 0;           /* W, H: size of view 0 (every view's size when uniform) */
    long long P = 0;                   /* largest view's pixel count */
    std::vector<int> Wv, Hv;           /* per-view image size */
    std::vector<long long> offv;       /* per-view offset in the concatenated per-view arrays */
    long long Ptot = 0;                /* sum of the views' pixel counts */
    bool uniform = true;
    int hyp_ref = 0;                   /* view whose planes the single-view buffers hold */
    int filtered_ref = 0;              /* view of the last filter() */
    std::vector<l3d_view> views;
    l3d_stereo_opts opts{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t done = nullptr;        /* recorded after work other handles consume */
    int n_maps = 0;
    void* images = nullptr;            /* V * P of the storage type */
    uint32_t* depths = nullptr;        /* n_maps * P */
    float4* hyp = nullptr;
    float* cost = nullptr;
    float* prior = nullptr;
    uint32_t* filtered = nullptr;
    uint32_t* filtered_all = nullptr;  /* lazily: V * P */
    float4* hyp_all = nullptr;         /* lazily: V * P */
    float* cost_all = nullptr;
    float* prior_all = nullptr;
    void* staging = nullptr;           /* host image upload staging */
    size_t staging_bytes = 0;
    float4* planes = nullptr;          /* plane_cost scratch */
    float* plane_out = nullptr;
    long long launches = 0;
    /* fast form */
    std::vector<cudaArray_t> arrays;   /* per view (F16/F32 storage): texture-sampled copy */
    std::vector<cudaTextureObject_t> texs;
    L3dFastView* fviews_dev = nullptr; /* capacity fview_cap */
    int* tile_start_dev = nullptr;
    L3dFastView* fviews_host = nullptr;  /* pinned staging */
    int* tile_start_host = nullptr;
    int fview_cap = 0;
    cudaEvent_t staged = nullptr;      /* after the last copy out of the pinned staging */
    uint32_t* pairs = nullptr;         /* fast form: half2(texel, right neighbour) per pixel */
    int variant = L3D_FAST_DEFAULT_VARIANT;
    /* CUDA graphs of batched solves, keyed by the request (fast form, no priors) */
    struct Graph {
        std::vector<int64_t> key;
        cudaGraphExec_t exec = nullptr;
        L3dFastView* views = nullptr;  /* the batch's own view table */
        int* tile_start = nullptr;
    };
    bool graphs = false;
    std::vector<Graph> graph_cache;
    /* differentiable NCC: FP64 view table and per-call pair scratch, allocated on first use */
    L3dGradView* grad_views = nullptr;
    L3dGradPair* grad_pairs = nullptr;
    double* grad_sums = nullptr;
};

namespace {

/* DenseStereo.params (dense-stereo.ts:314-355) for one dispatch, FP64 -> f32.  The homography
 * base B = K_s R K_r^-1 and kt = K_s t are composed in FP64 here. */
void relative_pose(const l3d_pose& a, const l3d_pose& b, double* R, double* t) {
    /* relativePose (geometry/camera.ts:73-77), reference summation order */
    const double* Ra = a.R;
    const double* Rb = b.R;
    double At[9] = {Ra[0], Ra[3], Ra[6], Ra[1], Ra[4], Ra[7], Ra[2], Ra[5], Ra[8]};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            R[r * 3 + c] = Rb[r * 3] * At[c] + Rb[r * 3 + 1] * At[3 + c] + Rb[r * 3 + 2] * At[6 + c];
    for (int r = 0; r < 3; r++) {
        double rt = R[r * 3] * a.t[0] + R[r * 3 + 1] * a.t[1] + R[r * 3 + 2] * a.t[2];
        t[r] = b.t[r] - rt;
    }
}

uint32_t seed_of(int ref, int iteration, int phase, int flags) {
    uint32_t s = (uint32_t)(ref + 1) * 0x9e3779b1u;
    return s + (uint32_t)iteration * 97u + (uint32_t)phase * 13u + (uint32_t)flags * 7u;
}

L3dParams build_params(const l3d_stereo* s, int ref, const int32_t* sources, int n, double min_depth,
                       double max_depth, int iteration, int phase, double step, int flags,
                       int needed, int coarse_w, int coarse_h) {
    L3dParams p;
    std::memset(&p, 0, sizeof(p));
    const l3d_view& rv = s->views[ref];
    const double kr[4] = {rv.intrinsics.fx, rv.intrinsics.fy, rv.intrinsics.cx, rv.intrinsics.cy};
    for (int i = 0; i < 4; i++) p.k[i] = (float)kr[i];
    p.kinv[0] = 1.0f / p.k[0];
    p.kinv[1] = 1.0f / p.k[1];
    p.kinv[2] = (-p.k[2]) / p.k[0];
    p.kinv[3] = (-p.k[3]) / p.k[1];
    p.W = s->Wv[ref];
    p.H = s->Hv[ref];
    p.ref = ref;
    p.n = std::min(n, L3D_MAX_SOURCES);
    p.range[0] = (float)(1.0 / min_depth);
    p.range[1] = (float)(1.0 / max_depth);
    p.range[2] = (float)step;
    p.range[3] = (float)0.2;                 /* GEOMETRIC_WEIGHT, dense-stereo.ts:46 */
    p.iter = (unsigned)iteration;
    p.phase = (unsigned)phase;
    p.seed = seed_of(ref, iteration, phase, flags);
    p.flags = (unsigned)flags;
    p.needed = (unsigned)needed;
    if (coarse_w > 0 && coarse_h > 0) {
        /* scaleIntrinsics (geometry/camera.ts:28-36) */
        double sx = (double)coarse_w / p.W, sy = (double)coarse_h / p.H;
        p.ck[0] = (float)(kr[0] * sx);
        p.ck[1] = (float)(kr[1] * sy);
        p.ck[2] = (float)((kr[2] + 0.5) * sx - 0.5);
        p.ck[3] = (float)((kr[3] + 0.5) * sy - 0.5);
        p.cW = coarse_w;
        p.cH = coarse_h;
    }
    p.ref_off = s->offv[ref];
    p.ref_dep_off = s->n_maps > 1 ? s->offv[ref] : 0;
    for (int k = 0; k < p.n; k++) {
        const l3d_view& v = s->views[sources[k]];
        const double kv[4] = {v.intrinsics.fx, v.intrinsics.fy, v.intrinsics.cx, v.intrinsics.cy};
        double R[9], t[3];
        relative_pose(rv.pose, v.pose, R, t);
        L3dSrc& o = p.src[k];
        for (int i = 0; i < 4; i++) o.k[i] = (float)kv[i];
        for (int i = 0; i < 9; i++) o.R[i] = (float)R[i];
        for (int i = 0; i < 3; i++) o.t[i] = (float)t[i];
        double A[9];
        for (int c = 0; c < 3; c++) {
            A[0 * 3 + c] = kv[0] * R[0 * 3 + c] + kv[2] * R[2 * 3 + c];
            A[1 * 3 + c] = kv[1] * R[1 * 3 + c] + kv[3] * R[2 * 3 + c];
            A[2 * 3 + c] = R[2 * 3 + c];
        }
        for (int r = 0; r < 3; r++) {
            o.B[r * 3 + 0] = (float)(A[r * 3 + 0] / kr[0]);
            o.B[r * 3 + 1] = (float)(A[r * 3 + 1] / kr[1]);
            o.B[r * 3 + 2] =
                (float)(A[r * 3 + 2] - A[r * 3 + 0] * kr[2] / kr[0] - A[r * 3 + 1] * kr[3] / kr[1]);
        }
        o.kt[0] = (float)(kv[0] * t[0] + kv[2] * t[2]);
        o.kt[1] = (float)(kv[1] * t[1] + kv[3] * t[2]);
        o.kt[2] = (float)t[2];
        o.layer = sources[k];
        o.W = s->Wv[sources[k]];
        o.H = s->Hv[sources[k]];
        o.img_off = s->offv[sources[k]];
        o.dep_off = s->n_maps > 1 ? s->offv[sources[k]] : 0;
    }
    return p;
}

L3dStereoDev dev_of(const l3d_stereo* s) {
    L3dStereoDev d;
    d.images = (const float*)s->images;
    d.images_lp = s->images;
    d.hyp = s->hyp;
    d.cost = s->cost;
    d.prior = nullptr;
    d.depths = s->depths;
    d.filtered = s->filtered;
    d.coarse = s->opts.coarse ? s->opts.coarse->hyp : nullptr;
    return d;
}

int check_sources(const l3d_stereo* s, const int32_t* src, int n) {
    if (n < 0) return fail(L3D_EINVAL, "negative source count");
    if (n > 0 && !src) return fail(L3D_EINVAL, "sources is NULL");
    for (int k = 0; k < std::min(n, L3D_MAX_SOURCES); k++)
        if (src[k] < 0 || src[k] >= s->V)
            return fail(L3D_EINVAL, "source layer %d out of range [0, %d)", src[k], s->V);
    return L3D_OK;
}

int check_solve(const l3d_stereo* s, int ref, const l3d_solve_opts* o) {
    if (!s) return fail(L3D_EINVAL, "stereo handle is NULL");
    if (!o) return fail(L3D_EINVAL, "solve options are NULL");
    if (ref < 0 || ref >= s->V) return fail(L3D_EINVAL, "reference layer %d out of range [0, %d)", ref, s->V);
    int rc = check_sources(s, o->sources, o->n_sources);
    if (rc) return rc;
    if (!(o->min_depth > 0.0) || !(o->max_depth > o->min_depth))
        return fail(L3D_EINVAL, "depth range must satisfy 0 < min_depth < max_depth");
    if (o->iterations < 0) return fail(L3D_EINVAL, "negative iteration count");
    if ((o->geometric || o->pack) && s->n_maps == 1 && s->V > 1)
        return fail(L3D_ESTATE, "handle was created without per-view depth maps");
    if (o->from_coarse && !s->opts.coarse)
        return fail(L3D_ESTATE, "from_coarse needs a coarse level");
    return L3D_OK;
}

int upload_prior(l3d_stereo* s, int ref, const float* prior, float* dst) {
    const size_t n = (size_t)s->Wv[ref] * s->Hv[ref];
    L3D_CUDA(cudaMemcpyAsync(dst, prior, n * sizeof(float), cudaMemcpyHostToDevice, s->stream),
             "prior upload");
    return L3D_OK;
}

int launch(l3d_stereo* s, int kernel, const L3dParams& p, const L3dStereoDev& d) {
    cudaError_t e = l3d_launch_plain(kernel, p, d, s->opts.window, s->opts.dilation, s->stream);
    s->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return L3D_OK;
}

/* One reference view through the schedule of DenseStereo.solve (dense-stereo.ts:185-239),
 * on hypothesis buffers hyp/cost. */
int solve_one(l3d_stereo* s, int ref, const l3d_solve_opts* o, float4* hyp, float* cost,
              float* prior_dev) {
    int n = std::min(o->n_sources, L3D_MAX_SOURCES);
    if (n == 0) return L3D_OK;                            /* dense-stereo.ts:187 */
    const int flags = o->geometric ? 1 : 0;
    L3dStereoDev d = dev_of(s);
    d.hyp = hyp;
    d.cost = cost;
    if (o->prior && !o->geometric) {
        int rc = upload_prior(s, ref, o->prior, prior_dev);
        if (rc) return rc;
        d.prior = prior_dev;
    }
    int cw = 0, ch = 0;
    if (s->opts.coarse) {
        cw = s->opts.coarse->W;
        ch = s->opts.coarse->H;
    }
    const bool coarse = o->from_coarse && s->opts.coarse;
    if (coarse) {
        /* the coarse level's planes are written on its own stream */
        const l3d_stereo* c = s->opts.coarse;
        L3D_CUDA(cudaEventRecord(c->done, c->stream), "event record");
        L3D_CUDA(cudaStreamWaitEvent(s->stream, c->done, 0), "stream wait");
    }
    L3dParams p = build_params(s, ref, o->sources, n, o->min_depth, o->max_depth, 0, 0, 1.0, flags,
                               0, cw, ch);
    int rc = launch(s, coarse ? L3D_K_INIT_COARSE : L3D_K_INIT, p, d);
    if (rc) return rc;
    for (int it = 0; it < o->iterations; it++) {
        double step = std::pow(0.5, it);
        for (int phase = 0; phase < 2; phase++) {
            p = build_params(s, ref, o->sources, n, o->min_depth, o->max_depth, it, phase, step,
                             flags, 0, cw, ch);
            rc = launch(s, L3D_K_PROPAGATE, p, d);
            if (rc) return rc;
        }
    }
    if (o->pack) {
        p = build_params(s, ref, o->sources, n, o->min_depth, o->max_depth, 0, 0, 0.0, flags, 0,
                         cw, ch);
        rc = launch(s, L3D_K_PACK, p, d);
        if (rc) return rc;
    }
    return L3D_OK;
}

/* ---- fast form ---- */

bool fast_tex(const l3d_stereo* s) { return s->opts.storage != L3D_DTYPE_BF16; }
/* fast or exact form: every reference view of a batch in one launch per kernel */
bool batched(const l3d_stereo* s) { return s->opts.form != L3D_FORM_PLAIN; }

int fast_capacity(l3d_stereo* s, int n) {
    if (s->fview_cap >= n) return L3D_OK;
    cudaStreamSynchronize(s->stream);
    cudaFree(s->fviews_dev);
    cudaFree(s->tile_start_dev);
    cudaFreeHost(s->fviews_host);
    cudaFreeHost(s->tile_start_host);
    s->fviews_dev = nullptr;
    s->tile_start_dev = nullptr;
    s->fviews_host = nullptr;
    s->tile_start_host = nullptr;
    s->fview_cap = 0;
    L3D_CUDA(cudaMalloc(&s->fviews_dev, (size_t)n * sizeof(L3dFastView)), "view table");
    L3D_CUDA(cudaMalloc(&s->tile_start_dev, (size_t)(n + 1) * sizeof(int)), "view table");
    L3D_CUDA(cudaMallocHost(&s->fviews_host, (size_t)n * sizeof(L3dFastView)), "view staging");
    L3D_CUDA(cudaMallocHost(&s->tile_start_host, (size_t)(n + 1) * sizeof(int)), "view staging");
    s->fview_cap = n;
    return L3D_OK;
}

/* The parameters of one reference view for the fast kernels: DenseStereo.params
 * (dense-stereo.ts:314-355) with the homography base shifted by half a texel for the texture
 * unit (Bt = S B, ktt = S kt, S = [[1, 0, .5], [0, 1, .5], [0, 0, 1]]), composed in FP64. */
L3dFastView fast_view(const l3d_stereo* s, int ref, const l3d_solve_opts* o, long long pix_off) {
    L3dParams p = build_params(s, ref, o->sources, std::min(o->n_sources, L3D_MAX_SOURCES),
                               o->min_depth, o->max_depth, 0, 0, 1.0, o->geometric ? 1 : 0, 0, 0, 0);
    L3dFastView v;
    std::memset(&v, 0, sizeof(v));
    for (int i = 0; i < 4; i++) {
        v.k[i] = p.k[i];
        v.kinv[i] = p.kinv[i];
        v.range[i] = p.range[i];
    }
    v.W = s->Wv[ref];
    v.H = s->Hv[ref];
    v.ref = ref;
    v.n = p.n;
    v.flags = p.flags;
    v.iterations = o->iterations;
    v.tiles_x = ((v.W + 1) / 2 + 15) / 16;
    v.pix_off = pix_off;
    v.ref_img_off = s->offv[ref];
    v.ref_dep_off = p.ref_dep_off;
    v.ref_tex = fast_tex(s) ? (unsigned long long)s->texs[ref] : 0ull;
    v.has_prior = o->prior != nullptr && !o->geometric;
    v.pack = o->pack ? 1 : 0;
    const l3d_view& rv = s->views[ref];
    if (o->from_coarse && s->opts.coarse) {
        /* scaleIntrinsics (geometry/camera.ts:28-36) to the coarse level, in FP64 */
        const l3d_stereo* c = s->opts.coarse;
        const int cw = c->Wv[ref], ch = c->Hv[ref];
        const double sx = (double)cw / v.W, sy = (double)ch / v.H;
        v.ck[0] = (float)(rv.intrinsics.fx * sx);
        v.ck[1] = (float)(rv.intrinsics.fy * sy);
        v.ck[2] = (float)((rv.intrinsics.cx + 0.5) * sx - 0.5);
        v.ck[3] = (float)((rv.intrinsics.cy + 0.5) * sy - 0.5);
        v.cW = cw;
        v.cH = ch;
        v.has_coarse = 1;
        v.has_prior = 0;
        v.flags &= ~1u;
    }
    const double kr[4] = {rv.intrinsics.fx, rv.intrinsics.fy, rv.intrinsics.cx, rv.intrinsics.cy};
    for (int k = 0; k < p.n; k++) {
        const L3dSrc& ps = p.src[k];
        L3dFastSrc& f = v.src[k];
        const l3d_view& sv = s->views[o->sources[k]];
        const double kv[4] = {sv.intrinsics.fx, sv.intrinsics.fy, sv.intrinsics.cx, sv.intrinsics.cy};
        double R[9], t[3];
        relative_pose(rv.pose, sv.pose, R, t);
        double A[9], B[9], kt[3];
        for (int c = 0; c < 3; c++) {
            A[0 * 3 + c] = kv[0] * R[0 * 3 + c] + kv[2] * R[2 * 3 + c];
            A[1 * 3 + c] = kv[1] * R[1 * 3 + c] + kv[3] * R[2 * 3 + c];
            A[2 * 3 + c] = R[2 * 3 + c];
        }
        for (int r = 0; r < 3; r++) {
            B[r * 3 + 0] = A[r * 3 + 0] / kr[0];
            B[r * 3 + 1] = A[r * 3 + 1] / kr[1];
            B[r * 3 + 2] = A[r * 3 + 2] - A[r * 3 + 0] * kr[2] / kr[0] - A[r * 3 + 1] * kr[3] / kr[1];
        }
        kt[0] = kv[0] * t[0] + kv[2] * t[2];
        kt[1] = kv[1] * t[1] + kv[3] * t[2];
        kt[2] = t[2];
        if (s->opts.form == L3D_FORM_EXACT) {
            /* texel coordinates: the plain form's B and kt, rounded to f32 as it rounds them */
            for (int i = 0; i < 9; i++) f.Bt[i] = ps.B[i];
            for (int i = 0; i < 3; i++) f.ktt[i] = ps.kt[i];
        } else {
            for (int c = 0; c < 3; c++) {
                f.Bt[0 * 3 + c] = (float)(B[0 * 3 + c] + 0.5 * B[2 * 3 + c]);
                f.Bt[1 * 3 + c] = (float)(B[1 * 3 + c] + 0.5 * B[2 * 3 + c]);
                f.Bt[2 * 3 + c] = (float)B[2 * 3 + c];
            }
            f.ktt[0] = (float)(kt[0] + 0.5 * kt[2]);
            f.ktt[1] = (float)(kt[1] + 0.5 * kt[2]);
            f.ktt[2] = (float)kt[2];
        }
        for (int i = 0; i < 4; i++) f.k[i] = ps.k[i];
        for (int i = 0; i < 9; i++) f.R[i] = ps.R[i];
        for (int i = 0; i < 3; i++) f.t[i] = ps.t[i];
        f.W = ps.W;
        f.H = ps.H;
        f.img_off = ps.img_off;
        f.dep_off = ps.dep_off;
        f.tex = fast_tex(s) ? (unsigned long long)s->texs[o->sources[k]] : 0ull;
    }
    return v;
}

/* Uploads the view table of a batch (pinned staging guarded by an event) and returns the
 * device-side description for the fast launchers. */
int fast_batch(l3d_stereo* s, int n, const int32_t* refs, const l3d_solve_opts* opts, float4* hyp,
               float* cost, float* prior, bool per_view_offsets, L3dFastDev* out) {
    int rc = fast_capacity(s, n);
    if (rc) return rc;
    L3D_CUDA(cudaEventSynchronize(s->staged), "staging wait");
    int tiles = 0;
    for (int i = 0; i < n; i++) {
        long long off = per_view_offsets ? s->offv[refs[i]] : 0;
        L3dFastView v = fast_view(s, refs[i], &opts[i], off);
        /* batched coarse planes sit at the coarse level's per-view offsets */
        if (v.has_coarse && per_view_offsets) v.coarse_off = s->opts.coarse->offv[refs[i]];
        v.tile_start = tiles;
        s->fviews_host[i] = v;
        s->tile_start_host[i] = tiles;
        tiles += v.tiles_x * ((v.H + 7) / 8);
        if (v.has_prior) {
            L3D_CUDA(cudaMemcpyAsync(prior + off, opts[i].prior, (size_t)v.W * v.H * sizeof(float),
                                     cudaMemcpyHostToDevice, s->stream), "prior upload");
        }
    }
    s->tile_start_host[n] = tiles;
    L3D_CUDA(cudaMemcpyAsync(s->fviews_dev, s->fviews_host, (size_t)n * sizeof(L3dFastView),
                             cudaMemcpyHostToDevice, s->stream), "view table upload");
    L3D_CUDA(cudaMemcpyAsync(s->tile_start_dev, s->tile_start_host, (size_t)(n + 1) * sizeof(int),
                             cudaMemcpyHostToDevice, s->stream), "view table upload");
    L3D_CUDA(cudaEventRecord(s->staged, s->stream), "event record");
    L3dFastDev d;
    d.views = s->fviews_dev;
    d.tile_start = s->tile_start_dev;
    d.n_views = n;
    d.total_tiles = tiles;
    d.images = s->images;
    d.pairs = s->pairs;
    d.storage = s->opts.storage;
    d.hyp = hyp;
    d.cost = cost;
    d.prior = prior;
    d.depths = s->depths;
    d.coarse = nullptr;
    d.exact = s->opts.form == L3D_FORM_EXACT ? 1 : 0;
    d.comp = s->opts.compensated ? 1 : 0;
    *out = d;
    return L3D_OK;
}

int fast_launch(l3d_stereo* s, int kernel, const L3dFastDev& d, int it, int phase) {
    cudaError_t e = l3d_launch_fast(kernel, d, it, phase, s->variant, s->stream);
    s->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return L3D_OK;
}

int fast_pack(l3d_stereo* s, const L3dFastDev& d) {
    cudaError_t e = l3d_launch_fast_pack(d, s->P, s->stream);
    s->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return L3D_OK;
}

/* The schedule of DenseStereo.solve for every view of a batch at once: init, iterations x
 * (colour 0, colour 1), pack. */
/* The launches of one batched solve (init, iterations x two colours, pack). */
int fast_schedule(l3d_stereo* s, const L3dFastDev& d, int max_it, bool any_pack) {
    int rc;
    if ((rc = fast_launch(s, L3D_K_INIT, d, 0, 0))) return rc;
    for (int it = 0; it < max_it; it++)
        for (int phase = 0; phase < 2; phase++)
            if ((rc = fast_launch(s, L3D_K_PROPAGATE, d, it, phase))) return rc;
    if (any_pack && (rc = fast_pack(s, d))) return rc;
    return L3D_OK;
}

/* Request key of a batched solve: everything that shapes the launches and their parameters. */
std::vector<int64_t> graph_key(const l3d_stereo* s, const std::vector<int32_t>& r,
                               const std::vector<l3d_solve_opts>& o) {
    std::vector<int64_t> k;
    k.push_back(s->variant);
    for (size_t i = 0; i < r.size(); i++) {
        const l3d_solve_opts& q = o[i];
        k.push_back(r[i]);
        k.push_back(q.n_sources);
        for (int j = 0; j < std::min(q.n_sources, L3D_MAX_SOURCES); j++) k.push_back(q.sources[j]);
        int64_t a, b;
        std::memcpy(&a, &q.min_depth, 8);
        std::memcpy(&b, &q.max_depth, 8);
        k.push_back(a);
        k.push_back(b);
        k.push_back(q.geometric * 4 + q.pack * 2);
        k.push_back(q.iterations);
    }
    return k;
}

void free_graph(l3d_stereo::Graph& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    cudaFree(g.views);
    cudaFree(g.tile_start);
    g.exec = nullptr;
    g.views = nullptr;
    g.tile_start = nullptr;
}

/* Captures the batch's launches into a CUDA graph on first use and replays it afterwards.  The
 * graph owns a copy of the view table, so replays need no host staging. */
int fast_solve_graph(l3d_stereo* s, const std::vector<int32_t>& r, const std::vector<l3d_solve_opts>& o,
                     int max_it, bool any_pack) {
    std::vector<int64_t> key = graph_key(s, r, o);
    for (auto& g : s->graph_cache)
        if (g.key == key) {
            L3D_CUDA(cudaGraphLaunch(g.exec, s->stream), "graph launch");
            s->launches += 2 + 2 * max_it;
            return L3D_OK;
        }
    const int n = (int)r.size();
    L3dFastDev d;
    int rc = fast_batch(s, n, r.data(), o.data(), s->hyp_all, s->cost_all, s->prior_all, true, &d);
    if (rc) return rc;
    l3d_stereo::Graph g;
    g.key = key;
    L3D_CUDA(cudaMalloc(&g.views, (size_t)n * sizeof(L3dFastView)), "graph view table");
    L3D_CUDA(cudaMalloc(&g.tile_start, (size_t)(n + 1) * sizeof(int)), "graph view table");
    L3D_CUDA(cudaMemcpyAsync(g.views, d.views, (size_t)n * sizeof(L3dFastView), cudaMemcpyDeviceToDevice,
                             s->stream), "graph view table");
    L3D_CUDA(cudaMemcpyAsync(g.tile_start, d.tile_start, (size_t)(n + 1) * sizeof(int),
                             cudaMemcpyDeviceToDevice, s->stream), "graph view table");
    d.views = g.views;
    d.tile_start = g.tile_start;
    cudaGraph_t graph = nullptr;
    L3D_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    rc = fast_schedule(s, d, max_it, any_pack);
    cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        free_graph(g);
        return rc;
    }
    if (e != cudaSuccess) {
        free_graph(g);
        return cuda_fail(e, "graph capture");
    }
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        free_graph(g);
        return cuda_fail(e, "graph instantiation");
    }
    if (s->graph_cache.size() >= 8) {  /* keep the eight most recent batches */
        free_graph(s->graph_cache.front());
        s->graph_cache.erase(s->graph_cache.begin());
    }
    s->graph_cache.push_back(g);
    L3D_CUDA(cudaGraphLaunch(g.exec, s->stream), "graph launch");
    return L3D_OK;
}

int fast_solve(l3d_stereo* s, int n, const int32_t* refs, const l3d_solve_opts* opts, bool all) {
    int nn = 0;
    std::vector<int32_t> r;
    std::vector<l3d_solve_opts> o;
    int max_it = 0;
    bool any_pack = false;
    for (int i = 0; i < n; i++) {
        if (std::min(opts[i].n_sources, L3D_MAX_SOURCES) == 0) continue;  /* dense-stereo.ts:187 */
        r.push_back(refs[i]);
        o.push_back(opts[i]);
        max_it = std::max(max_it, opts[i].iterations);
        any_pack |= opts[i].pack != 0;
        nn++;
    }
    if (nn == 0) return L3D_OK;
    bool any_prior = false, any_coarse = false;
    for (auto& q : o) {
        any_prior |= q.prior != nullptr && !q.geometric;
        any_coarse |= q.from_coarse != 0;
    }
    /* coarse-to-fine: a single view starts from the coarse level's last solve of that view, a
     * batch from the coarse level's batched planes of its views */
    const float4* coarse = nullptr;
    if (any_coarse) {
        const l3d_stereo* c = s->opts.coarse;
        if (all) {
            if (!c->hyp_all) return fail(L3D_ESTATE, "the coarse level has no batched planes (solve_all it first)");
            coarse = c->hyp_all;
        } else {
            if (c->hyp_ref != r[0]) return fail(L3D_ESTATE, "the coarse level's planes are of view %d, not %d", c->hyp_ref, r[0]);
            coarse = c->hyp;
        }
        L3D_CUDA(cudaEventRecord(c->done, c->stream), "event record");
        L3D_CUDA(cudaStreamWaitEvent(s->stream, c->done, 0), "stream wait");
    }
    if (all && s->graphs && !any_prior && !any_coarse) return fast_solve_graph(s, r, o, max_it, any_pack);
    L3dFastDev d;
    int rc = all ? fast_batch(s, nn, r.data(), o.data(), s->hyp_all, s->cost_all, s->prior_all, true, &d)
                 : fast_batch(s, nn, r.data(), o.data(), s->hyp, s->cost, s->prior, false, &d);
    if (rc) return rc;
    d.coarse = coarse;
    return fast_schedule(s, d, max_it, any_pack);
}

}  // namespace

void l3d_set_error(const char* msg) { g_error = msg ? msg : ""; }

extern "C" {

size_t l3d_last_error(char* buf, size_t size) {
    if (buf && size) {
        size_t n = std::min(size - 1, g_error.size());
        std::memcpy(buf, g_error.data(), n);
        buf[n] = 0;
    }
    return g_error.size();
}

void l3d_stereo_opts_default(l3d_stereo_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->depth_maps = 1;
    o->storage = L3D_DTYPE_F32;
    o->form = L3D_FORM_PLAIN;
    o->window = 6;
    o->dilation = 2;
}

int l3d_stereo_create(int32_t width, int32_t height, int32_t n_views, const l3d_view* views,
                      const l3d_stereo_opts* opts, l3d_stereo** out) {
    if (!out) return fail(L3D_EINVAL, "out is NULL");
    *out = nullptr;
    if (n_views <= 0 || !views) return fail(L3D_EINVAL, "need at least one view");
    std::vector<int32_t> sizes(2 * (size_t)n_views);
    for (int i = 0; i < n_views; i++) {
        sizes[2 * i] = width;
        sizes[2 * i + 1] = height;
    }
    return l3d_stereo_create_sized(n_views, views, sizes.data(), opts, out);
}

int l3d_stereo_create_sized(int32_t n_views, const l3d_view* views, const int32_t* sizes,
                            const l3d_stereo_opts* opts, l3d_stereo** out) {
    if (!out) return fail(L3D_EINVAL, "out is NULL");
    *out = nullptr;
    if (n_views <= 0 || !views || !sizes) return fail(L3D_EINVAL, "need at least one view and its size");
    long long ptot = 0, pmax = 0;
    for (int i = 0; i < n_views; i++) {
        const int w = sizes[2 * i], h = sizes[2 * i + 1];
        if (w <= 0 || h <= 0) return fail(L3D_EINVAL, "image size must be positive");
        if ((long long)w * h >= (1ll << 31)) return fail(L3D_EINVAL, "image too large");
        ptot += (long long)w * h;
        pmax = std::max(pmax, (long long)w * h);
    }
    const int width = sizes[0], height = sizes[1];
    l3d_stereo_opts o;
    if (opts) o = *opts;
    else l3d_stereo_opts_default(&o);
    if (!((o.window == 6 && o.dilation == 2) || (o.window == 11 && o.dilation == 1)))
        return fail(L3D_EINVAL, "window %d / dilation %d not supported (6/2 or 11/1)", o.window, o.dilation);
    if (o.form != L3D_FORM_PLAIN && o.form != L3D_FORM_FAST && o.form != L3D_FORM_EXACT)
        return fail(L3D_EINVAL, "unknown form %d", o.form);
    if (o.form == L3D_FORM_PLAIN && o.storage != L3D_DTYPE_F32)
        return fail(L3D_EINVAL, "the plain form stores images as F32");
    if (o.form == L3D_FORM_EXACT && o.storage != L3D_DTYPE_F32)
        return fail(L3D_EINVAL, "the exact form stores images as F32");
    if (o.compensated != 0 && o.compensated != 1)
        return fail(L3D_EINVAL, "compensated must be 0 or 1");
    if (o.compensated && o.form == L3D_FORM_PLAIN)
        return fail(L3D_EINVAL, "compensated sums are a fast- and exact-form option (the plain form is "
                                "the oracle's uncompensated order)");
    if (o.storage != L3D_DTYPE_F32 && o.storage != L3D_DTYPE_F16 && o.storage != L3D_DTYPE_BF16 &&
        o.storage != L3D_DTYPE_U8)
        return fail(L3D_EINVAL, "image storage must be U8, F32, F16 or BF16");
    if (o.form != L3D_FORM_PLAIN && !(o.window == 6 && o.dilation == 2))
        return fail(L3D_EINVAL, "the fast and exact forms use the reference window (6 samples, dilation 2)");
    for (int i = 0; i < n_views; i++) {
        const l3d_intrinsics& k = views[i].intrinsics;
        if (!(k.fx != 0.0) || !(k.fy != 0.0) || !std::isfinite(k.fx) || !std::isfinite(k.fy))
            return fail(L3D_EINVAL, "view %d has a zero or non-finite focal length", i);
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "no CUDA device");
    l3d_stereo* s = new (std::nothrow) l3d_stereo();
    if (!s) return fail(L3D_ENOMEM, "host allocation failed");
    s->W = width;
    s->H = height;
    s->V = n_views;
    s->P = pmax;
    s->Ptot = ptot;
    s->Wv.resize(n_views);
    s->Hv.resize(n_views);
    s->offv.resize(n_views);
    long long acc = 0;
    for (int i = 0; i < n_views; i++) {
        s->Wv[i] = sizes[2 * i];
        s->Hv[i] = sizes[2 * i + 1];
        s->offv[i] = acc;
        acc += (long long)s->Wv[i] * s->Hv[i];
        s->uniform = s->uniform && s->Wv[i] == width && s->Hv[i] == height;
    }
    if (o.coarse && (!s->uniform || !o.coarse->uniform)) {
        delete s;
        return fail(L3D_EINVAL, "coarse-to-fine levels need views of one size");
    }
    s->views.assign(views, views + n_views);
    s->opts = o;
    s->n_maps = o.depth_maps ? n_views : 1;
    auto cleanup = [&](int rc) {
        l3d_stereo_destroy(s);
        return rc;
    };
    if (o.stream) {
        s->stream = (cudaStream_t)o.stream;
    } else {
        e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "stream creation"));
        s->own_stream = true;
    }
    e = cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "event creation"));
    e = cudaEventCreateWithFlags(&s->staged, cudaEventDisableTiming);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "event creation"));
    size_t esize = dtype_size(o.storage);
    if (o.form != L3D_FORM_PLAIN && o.storage != L3D_DTYPE_BF16) {
        /* texture-sampled copies: block-linear CUDA arrays with clamp-to-edge addressing and
         * unnormalised coordinates (texel centres at +0.5); hardware bilinear filtering for
         * the fast form, texture gathers (point filtering) for the exact form */
        const bool gather = o.form == L3D_FORM_EXACT;
        cudaChannelFormatDesc ch = o.storage == L3D_DTYPE_F16  ? cudaCreateChannelDescHalf()
                                   : o.storage == L3D_DTYPE_U8 ? cudaCreateChannelDesc<unsigned char>()
                                                               : cudaCreateChannelDesc<float>();
        s->arrays.assign(n_views, nullptr);
        s->texs.assign(n_views, 0);
        for (int i = 0; i < n_views; i++) {
            if ((e = cudaMallocArray(&s->arrays[i], &ch, s->Wv[i], s->Hv[i],
                                     cudaArrayTextureGather)) != cudaSuccess)
                return cleanup(cuda_fail(e, "image array allocation"));
            cudaResourceDesc res;
            std::memset(&res, 0, sizeof(res));
            res.resType = cudaResourceTypeArray;
            res.res.array.array = s->arrays[i];
            cudaTextureDesc td;
            std::memset(&td, 0, sizeof(td));
            td.addressMode[0] = cudaAddressModeClamp;
            td.addressMode[1] = cudaAddressModeClamp;
            td.filterMode = gather ? cudaFilterModePoint : cudaFilterModeLinear;
            /* U8 texels read as value / 255 (the r8unorm format of the reference's textures) */
            td.readMode = o.storage == L3D_DTYPE_U8 ? cudaReadModeNormalizedFloat
                                                    : cudaReadModeElementType;
            td.normalizedCoords = 0;
            if ((e = cudaCreateTextureObject(&s->texs[i], &res, &td, nullptr)) != cudaSuccess)
                return cleanup(cuda_fail(e, "texture creation"));
        }
        if (!gather) {
            if ((e = dalloc(&s->pairs, (size_t)s->Ptot)) != cudaSuccess)
                return cleanup(cuda_fail(e, "pair image allocation"));
            if ((e = cudaMemsetAsync(s->pairs, 0, (size_t)s->Ptot * 4, s->stream)) != cudaSuccess)
                return cleanup(cuda_fail(e, "device clear"));
        }
    }
    const size_t depth_len = s->n_maps > 1 ? (size_t)s->Ptot : (size_t)s->P;
    if ((e = cudaMalloc(&s->images, (size_t)s->Ptot * esize)) != cudaSuccess ||
        (e = dalloc(&s->depths, depth_len)) != cudaSuccess ||
        (e = dalloc(&s->hyp, (size_t)s->P)) != cudaSuccess ||
        (e = dalloc(&s->cost, (size_t)s->P)) != cudaSuccess ||
        (e = dalloc(&s->prior, (size_t)s->P)) != cudaSuccess ||
        (e = dalloc(&s->filtered, (size_t)s->P)) != cudaSuccess)
        return cleanup(cuda_fail(e, "device allocation"));
    /* zero-initialised like WebGPU buffers */
    if ((e = cudaMemsetAsync(s->images, 0, (size_t)s->Ptot * esize, s->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(s->depths, 0, depth_len * 4, s->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(s->hyp, 0, (size_t)s->P * 16, s->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(s->cost, 0, (size_t)s->P * 4, s->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(s->prior, 0, (size_t)s->P * 4, s->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(s->filtered, 0, (size_t)s->P * 4, s->stream)) != cudaSuccess)
        return cleanup(cuda_fail(e, "device clear"));
    *out = s;
    return L3D_OK;
}

int l3d_stereo_set_image(l3d_stereo* s, int32_t layer, int32_t dtype, const void* pixels,
                         int64_t row_stride_bytes) {
    if (!s || !pixels) return fail(L3D_EINVAL, "NULL handle or pixels");
    if (layer < 0 || layer >= s->V) return fail(L3D_EINVAL, "layer %d out of range [0, %d)", layer, s->V);
    size_t es = dtype_size(dtype);
    if (!es) return fail(L3D_EINVAL, "unknown dtype %d", dtype);
    const int W = s->Wv[layer], H = s->Hv[layer];
    size_t row = (size_t)W * es;
    size_t stride = row_stride_bytes ? (size_t)row_stride_bytes : row;
    if (stride < row) return fail(L3D_EINVAL, "row stride smaller than a row");
    size_t need = row * H;
    if (s->staging_bytes < need) {
        if (s->staging) {
            cudaStreamSynchronize(s->stream);
            cudaFree(s->staging);
            s->staging = nullptr;
            s->staging_bytes = 0;
        }
        L3D_CUDA(cudaMalloc(&s->staging, need), "staging allocation");
        s->staging_bytes = need;
    }
    L3D_CUDA(cudaMemcpy2DAsync(s->staging, row, pixels, stride, row, H, cudaMemcpyHostToDevice,
                               s->stream),
             "image upload");
    size_t out_es = dtype_size(s->opts.storage);
    void* dst = (char*)s->images + (size_t)s->offv[layer] * out_es;
    cudaError_t e = l3d_launch_convert(s->staging, dtype, (int64_t)row, W, H, dst,
                                       s->opts.storage, s->stream);
    s->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "image conversion");
    if (!s->arrays.empty()) {
        size_t rb = (size_t)W * out_es;
        L3D_CUDA(cudaMemcpy2DToArrayAsync(s->arrays[layer], 0, 0, dst, rb, rb, H,
                                          cudaMemcpyDeviceToDevice, s->stream),
                 "image array copy");
    }
    if (s->pairs) {
        e = l3d_launch_make_pairs(dst, s->opts.storage, W, H, s->pairs + s->offv[layer], s->stream);
        s->launches++;
        if (e != cudaSuccess) return cuda_fail(e, "pair image");
    }
    return L3D_OK;
}

int l3d_stereo_solve(l3d_stereo* s, int32_t ref, const l3d_solve_opts* o) {
    int rc = check_solve(s, ref, o);
    if (rc) return rc;
    s->hyp_ref = ref;
    if (batched(s)) return fast_solve(s, 1, &ref, o, false);
    return solve_one(s, ref, o, s->hyp, s->cost, s->prior);
}

int l3d_stereo_solve_all(l3d_stereo* s, int32_t n_refs, const int32_t* refs,
                         const l3d_solve_opts* opts) {
    if (!s || n_refs < 0 || (n_refs > 0 && (!refs || !opts)))
        return fail(L3D_EINVAL, "bad arguments to solve_all");
    for (int i = 0; i < n_refs; i++) {
        int rc = check_solve(s, refs[i], &opts[i]);
        if (rc) return rc;
    }
    for (int i = 0; i < n_refs; i++)
        for (int j = 0; j < i; j++)
            if (refs[i] == refs[j]) return fail(L3D_EINVAL, "reference layer %d appears twice", refs[i]);
    if (!s->hyp_all) {
        L3D_CUDA(dalloc(&s->hyp_all, (size_t)s->Ptot), "hyp_all allocation");
        L3D_CUDA(dalloc(&s->cost_all, (size_t)s->Ptot), "cost_all allocation");
        L3D_CUDA(dalloc(&s->prior_all, (size_t)s->Ptot), "prior_all allocation");
    }
    if (batched(s)) return fast_solve(s, n_refs, refs, opts, true);
    for (int i = 0; i < n_refs; i++) {
        int r = refs[i];
        int rc = solve_one(s, r, &opts[i], s->hyp_all + s->offv[r], s->cost_all + s->offv[r],
                           s->prior_all + s->offv[r]);
        if (rc) return rc;
    }
    return L3D_OK;
}

int l3d_stereo_dispatch(l3d_stereo* s, int32_t kernel, int32_t ref, const l3d_solve_opts* o,
                        int32_t iteration, int32_t phase) {
    if (kernel == L3D_KERNEL_CONSISTENCY) return fail(L3D_EINVAL, "use l3d_stereo_filter");
    int rc = check_solve(s, ref, o);
    if (rc) return rc;
    if (kernel < L3D_KERNEL_INIT || kernel > L3D_KERNEL_PACK)
        return fail(L3D_EINVAL, "unknown kernel %d", kernel);
    if (kernel == L3D_KERNEL_INIT_COARSE && !s->opts.coarse)
        return fail(L3D_ESTATE, "init_coarse needs a coarse level");
    if (phase != 0 && phase != 1) return fail(L3D_EINVAL, "phase must be 0 or 1");
    s->hyp_ref = ref;
    int n = std::min(o->n_sources, L3D_MAX_SOURCES);
    if (batched(s)) {
        if (kernel == L3D_KERNEL_INIT_COARSE)
            return fail(L3D_EINVAL, "the fast and exact forms start from the coarse level in init (from_coarse)");
        l3d_solve_opts one = *o;
        one.iterations = iteration + 1;
        one.pack = 1;
        L3dFastDev fd;
        if ((rc = fast_batch(s, 1, &ref, &one, s->hyp, s->cost, s->prior, false, &fd))) return rc;
        if (kernel == L3D_KERNEL_PACK) return fast_pack(s, fd);
        return fast_launch(s, kernel == L3D_KERNEL_INIT ? L3D_K_INIT : L3D_K_PROPAGATE, fd, iteration, phase);
    }
    L3dStereoDev d = dev_of(s);
    if (kernel == L3D_KERNEL_INIT_COARSE) {
        const l3d_stereo* c = s->opts.coarse;
        L3D_CUDA(cudaEventRecord(c->done, c->stream), "event record");
        L3D_CUDA(cudaStreamWaitEvent(s->stream, c->done, 0), "stream wait");
    }
    if (kernel == L3D_KERNEL_INIT && o->prior && !o->geometric) {
        rc = upload_prior(s, ref, o->prior, s->prior);
        if (rc) return rc;
        d.prior = s->prior;
    }
    int cw = s->opts.coarse ? s->opts.coarse->W : 0, ch = s->opts.coarse ? s->opts.coarse->H : 0;
    double step = kernel == L3D_KERNEL_PACK ? 0.0 : std::pow(0.5, iteration);
    L3dParams p = build_params(s, ref, o->sources, n, o->min_depth, o->max_depth, iteration, phase,
                               step, o->geometric ? 1 : 0, 0, cw, ch);
    return launch(s, kernel, p, d);
}

int l3d_stereo_filter(l3d_stereo* s, int32_t ref, const int32_t* checks, int32_t n, int32_t needed) {
    if (!s) return fail(L3D_EINVAL, "stereo handle is NULL");
    if (ref < 0 || ref >= s->V) return fail(L3D_EINVAL, "reference layer %d out of range", ref);
    int rc = check_sources(s, checks, n);
    if (rc) return rc;
    if (s->n_maps == 1 && s->V > 1) return fail(L3D_ESTATE, "handle was created without per-view depth maps");
    /* DenseStereo.filter (dense-stereo.ts:250-263): range 0.01 - 100 m, no flags */
    L3dParams p = build_params(s, ref, checks, std::min(n, L3D_MAX_SOURCES), 0.01, 100.0, 0, 0, 0.0,
                               0, needed, 0, 0);
    s->filtered_ref = ref;
    return launch(s, L3D_K_CONSISTENCY, p, dev_of(s));
}

int l3d_stereo_filter_all(l3d_stereo* s, int32_t n_refs, const int32_t* refs, const int32_t* checks,
                          const int32_t* needed) {
    if (!s || n_refs < 0 || (n_refs > 0 && (!refs || !checks || !needed)))
        return fail(L3D_EINVAL, "bad arguments to filter_all");
    if (s->n_maps == 1 && s->V > 1) return fail(L3D_ESTATE, "handle was created without per-view depth maps");
    if (!s->filtered_all) L3D_CUDA(dalloc(&s->filtered_all, (size_t)s->Ptot), "filtered_all allocation");
    for (int i = 0; i < n_refs; i++) {
        int r = refs[i];
        if (r < 0 || r >= s->V) return fail(L3D_EINVAL, "reference layer %d out of range", r);
        int32_t src[L3D_MAX_SOURCES];
        int n = 0;
        for (int k = 0; k < L3D_MAX_SOURCES; k++)
            if (checks[i * L3D_MAX_SOURCES + k] >= 0) src[n++] = checks[i * L3D_MAX_SOURCES + k];
        int rc = check_sources(s, src, n);
        if (rc) return rc;
        L3dParams p = build_params(s, r, src, n, 0.01, 100.0, 0, 0, 0.0, 0, needed[i], 0, 0);
        L3dStereoDev d = dev_of(s);
        d.filtered = s->filtered_all + s->offv[r];
        rc = launch(s, L3D_K_CONSISTENCY, p, d);
        if (rc) return rc;
    }
    return L3D_OK;
}

static int read_dev(l3d_stereo* s, void* dst, const void* src, size_t bytes, const char* what) {
    L3D_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->stream), what);
    L3D_CUDA(cudaStreamSynchronize(s->stream), what);
    return L3D_OK;
}

int l3d_stereo_read_filtered(l3d_stereo* s, uint32_t* out) {
    if (!s || !out) return fail(L3D_EINVAL, "NULL argument");
    const int r = s->filtered_ref;
    return read_dev(s, out, s->filtered, (size_t)s->Wv[r] * s->Hv[r] * 4, "read filtered");
}

int l3d_stereo_read_filtered_layer(l3d_stereo* s, int32_t layer, uint32_t* out) {
    if (!s || !out) return fail(L3D_EINVAL, "NULL argument");
    if (layer < 0 || layer >= s->V) return fail(L3D_EINVAL, "layer out of range");
    if (!s->filtered_all) return fail(L3D_ESTATE, "no filter_all has run");
    return read_dev(s, out, s->filtered_all + s->offv[layer], (size_t)s->Wv[layer] * s->Hv[layer] * 4,
                    "read filtered layer");
}

int l3d_stereo_read_filtered_all_async(l3d_stereo* s, uint32_t* out) {
    if (!s || !out) return fail(L3D_EINVAL, "NULL argument");
    if (!s->filtered_all) return fail(L3D_ESTATE, "no filter_all has run");
    L3D_CUDA(cudaMemcpyAsync(out, s->filtered_all, (size_t)s->Ptot * 4, cudaMemcpyDeviceToHost, s->stream),
             "read filtered maps");
    return L3D_OK;
}

int l3d_stereo_read_depth(l3d_stereo* s, int32_t ref, uint32_t* out) {
    if (!s || !out) return fail(L3D_EINVAL, "NULL argument");
    if (ref < 0 || ref >= s->n_maps) return fail(L3D_EINVAL, "depth map %d out of range", ref);
    return read_dev(s, out, s->depths + (s->n_maps > 1 ? s->offv[ref] : 0),
                    (size_t)s->Wv[ref] * s->Hv[ref] * 4, "read depth");
}

int l3d_stereo_read_hyp(l3d_stereo* s, float* hyp4, float* cost) {
    if (!s) return fail(L3D_EINVAL, "NULL handle");
    if (hyp4) {
        int rc = read_dev(s, hyp4, s->hyp, (size_t)s->Wv[s->hyp_ref] * s->Hv[s->hyp_ref] * 16,
                          "read hypotheses");
        if (rc) return rc;
    }
    if (cost)
        return read_dev(s, cost, s->cost, (size_t)s->Wv[s->hyp_ref] * s->Hv[s->hyp_ref] * 4, "read costs");
    return L3D_OK;
}

int l3d_stereo_read_hyp_layer(l3d_stereo* s, int32_t layer, float* hyp4, float* cost) {
    if (!s) return fail(L3D_EINVAL, "NULL handle");
    if (layer < 0 || layer >= s->V) return fail(L3D_EINVAL, "layer out of range");
    if (!s->hyp_all) return fail(L3D_ESTATE, "no solve_all has run");
    if (hyp4) {
        int rc = read_dev(s, hyp4, s->hyp_all + s->offv[layer], (size_t)s->Wv[layer] * s->Hv[layer] * 16,
                          "read hypotheses");
        if (rc) return rc;
    }
    if (cost)
        return read_dev(s, cost, s->cost_all + s->offv[layer], (size_t)s->Wv[layer] * s->Hv[layer] * 4,
                        "read costs");
    return L3D_OK;
}

int l3d_stereo_write_hyp(l3d_stereo* s, const float* hyp4, const float* cost) {
    if (!s) return fail(L3D_EINVAL, "NULL handle");
    const size_t n = (size_t)s->Wv[s->hyp_ref] * s->Hv[s->hyp_ref];
    if (hyp4) L3D_CUDA(cudaMemcpyAsync(s->hyp, hyp4, n * 16, cudaMemcpyHostToDevice, s->stream), "write hypotheses");
    if (cost) L3D_CUDA(cudaMemcpyAsync(s->cost, cost, n * 4, cudaMemcpyHostToDevice, s->stream), "write costs");
    return L3D_OK;
}

int l3d_stereo_write_depth(l3d_stereo* s, int32_t ref, const uint32_t* packed) {
    if (!s || !packed) return fail(L3D_EINVAL, "NULL argument");
    if (ref < 0 || ref >= s->n_maps) return fail(L3D_EINVAL, "depth map %d out of range", ref);
    L3D_CUDA(cudaMemcpyAsync(s->depths + (s->n_maps > 1 ? s->offv[ref] : 0), packed,
                             (size_t)s->Wv[ref] * s->Hv[ref] * 4, cudaMemcpyHostToDevice,
                             s->stream),
             "write depth");
    return L3D_OK;
}

int l3d_stereo_plane_cost(l3d_stereo* s, int32_t ref, const l3d_solve_opts* o, const float* planes,
                          float* cost, float* view_costs) {
    int rc = check_solve(s, ref, o);
    if (rc) return rc;
    if (!planes || !cost) return fail(L3D_EINVAL, "NULL planes or cost");
    if (!s->planes) {
        L3D_CUDA(dalloc(&s->planes, (size_t)s->P), "plane scratch");
        L3D_CUDA(dalloc(&s->plane_out, (size_t)s->P * (1 + L3D_MAX_SOURCES)), "plane scratch");
    }
    const size_t pn = (size_t)s->Wv[ref] * s->Hv[ref];
    L3D_CUDA(cudaMemcpyAsync(s->planes, planes, pn * 16, cudaMemcpyHostToDevice, s->stream), "planes upload");
    if (batched(s)) {
        if (view_costs) return fail(L3D_EINVAL, "the fast and exact forms report the combined cost only");
        L3dFastDev fd;
        l3d_solve_opts one = *o;
        one.prior = nullptr;
        if ((rc = fast_batch(s, 1, &ref, &one, s->hyp, s->cost, s->prior, false, &fd))) return rc;
        cudaError_t e = l3d_launch_fast_plane_cost(fd, s->planes, s->plane_out, s->variant, s->stream);
        s->launches++;
        if (e != cudaSuccess) return cuda_fail(e, "plane cost launch");
        return read_dev(s, cost, s->plane_out, pn * 4, "read plane cost");
    }
    int n = std::min(o->n_sources, L3D_MAX_SOURCES);
    L3dParams p = build_params(s, ref, o->sources, n, o->min_depth, o->max_depth, 0, 0, 1.0,
                               o->geometric ? 1 : 0, 0, 0, 0);
    cudaError_t e = l3d_launch_plane_cost(p, dev_of(s), s->planes, s->plane_out, s->plane_out + s->P,
                                          s->opts.window, s->opts.dilation, s->stream);
    s->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "plane cost launch");
    rc = read_dev(s, cost, s->plane_out, pn * 4, "read plane cost");
    if (rc) return rc;
    if (view_costs)
        return read_dev(s, view_costs, s->plane_out + s->P, pn * 4 * L3D_MAX_SOURCES, "read view costs");
    return L3D_OK;
}

/* Shared body of l3d_ncc_forward / l3d_ncc_backward. */
static int ncc_run(l3d_stereo* s, int32_t ref, const int32_t* sources, int32_t n, const float* planes,
                   const float* deltas, const float* grad_cost, float* cost, float* grad_planes,
                   double* grad_deltas, void* stream) {
    if (!s) return fail(L3D_EINVAL, "stereo handle is NULL");
    if (ref < 0 || ref >= s->V) return fail(L3D_EINVAL, "reference layer %d out of range [0, %d)", ref, s->V);
    if (n <= 0 || n > L3D_MAX_SOURCES)
        return fail(L3D_EINVAL, "source count %d outside [1, %d]", n, L3D_MAX_SOURCES);
    int rc = check_sources(s, sources, n);
    if (rc) return rc;
    for (int k = 0; k < n; k++)
        if (sources[k] == ref) return fail(L3D_EINVAL, "the reference layer %d is listed as a source", ref);
    if (!planes) return fail(L3D_EINVAL, "planes is NULL");
    if (!s->grad_views) {
        std::vector<L3dGradView> table(s->V);
        for (int v = 0; v < s->V; v++) {
            const l3d_view& sv = s->views[v];
            L3dGradView& g = table[v];
            std::memset(&g, 0, sizeof(g));
            g.k[0] = sv.intrinsics.fx;
            g.k[1] = sv.intrinsics.fy;
            g.k[2] = sv.intrinsics.cx;
            g.k[3] = sv.intrinsics.cy;
            for (int i = 0; i < 9; i++) g.R[i] = sv.pose.R[i];
            for (int i = 0; i < 3; i++) g.t[i] = sv.pose.t[i];
            g.W = s->Wv[v];
            g.H = s->Hv[v];
            g.img_off = s->offv[v];
        }
        L3D_CUDA(dalloc(&s->grad_pairs, L3D_MAX_SOURCES), "gradient scratch");
        L3D_CUDA(dalloc(&s->grad_sums, 6 * L3D_MAX_SOURCES), "gradient scratch");
        L3D_CUDA(dalloc(&s->grad_views, (size_t)s->V), "gradient view table");
        L3D_CUDA(cudaMemcpy(s->grad_views, table.data(), table.size() * sizeof(L3dGradView),
                            cudaMemcpyHostToDevice),
                 "gradient view table upload");
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    const bool other = st != s->stream;
    if (other) {
        /* after the handle's queued work (image uploads) */
        L3D_CUDA(cudaEventRecord(s->done, s->stream), "event record");
        L3D_CUDA(cudaStreamWaitEvent(st, s->done, 0), "stream wait");
    }
    L3dGradDev d;
    std::memset(&d, 0, sizeof(d));
    d.images = s->images;
    d.storage = s->opts.storage;
    d.elem = (int)dtype_size(s->opts.storage);
    d.window = s->opts.window;
    d.dilation = s->opts.dilation;
    d.W = s->Wv[ref];
    d.H = s->Hv[ref];
    d.ref_img_off = s->offv[ref];
    const l3d_intrinsics& ki = s->views[ref].intrinsics;
    const float k[4] = {(float)ki.fx, (float)ki.fy, (float)ki.cx, (float)ki.cy};
    d.kinv[0] = 1.0f / k[0];
    d.kinv[1] = 1.0f / k[1];
    d.kinv[2] = (-k[2]) / k[0];
    d.kinv[3] = (-k[3]) / k[1];
    L3dGradJob job;
    std::memset(&job, 0, sizeof(job));
    job.ref = ref;
    job.n = n;
    for (int i = 0; i < n; i++) job.src[i] = sources[i];
    cudaError_t e = l3d_launch_ncc_grad(d, s->grad_views, deltas, job, s->grad_pairs, s->grad_sums,
                                        planes, grad_cost, cost, grad_planes, grad_deltas, st);
    s->launches += grad_deltas ? 3 : 2;
    if (e != cudaSuccess) return cuda_fail(e, "NCC gradient launch");
    if (other) {
        /* later handle work (image uploads) waits for these reads */
        L3D_CUDA(cudaEventRecord(s->done, st), "event record");
        L3D_CUDA(cudaStreamWaitEvent(s->stream, s->done, 0), "stream wait");
    }
    return L3D_OK;
}

int l3d_ncc_forward(l3d_stereo* s, int32_t ref, const int32_t* sources, int32_t n_sources,
                    const float* planes, const float* pose_deltas, float* cost, void* stream) {
    if (!cost) return fail(L3D_EINVAL, "cost is NULL");
    return ncc_run(s, ref, sources, n_sources, planes, pose_deltas, nullptr, cost, nullptr, nullptr,
                   stream);
}

int l3d_ncc_backward(l3d_stereo* s, int32_t ref, const int32_t* sources, int32_t n_sources,
                     const float* planes, const float* pose_deltas, const float* grad_cost,
                     float* cost, float* grad_planes, double* grad_deltas, void* stream) {
    if (!grad_planes && !grad_deltas) return fail(L3D_EINVAL, "no gradient output requested");
    return ncc_run(s, ref, sources, n_sources, planes, pose_deltas, grad_cost, cost, grad_planes,
                   grad_deltas, stream);
}

int l3d_stereo_buffers_get(const l3d_stereo* s, l3d_stereo_buffers* out) {
    if (!s || !out) return fail(L3D_EINVAL, "NULL argument");
    out->images = s->images;
    out->depths = s->depths;
    out->hyp = (float*)s->hyp;
    out->cost = s->cost;
    out->filtered = s->filtered;
    out->filtered_all = s->filtered_all;
    out->hyp_all = (float*)s->hyp_all;
    out->cost_all = s->cost_all;
    return L3D_OK;
}

int l3d_stereo_stream(const l3d_stereo* s, void** stream) {
    if (!s || !stream) return fail(L3D_EINVAL, "NULL argument");
    *stream = (void*)s->stream;
    return L3D_OK;
}

int l3d_stereo_synchronize(l3d_stereo* s) {
    if (!s) return fail(L3D_EINVAL, "NULL handle");
    L3D_CUDA(cudaStreamSynchronize(s->stream), "synchronize");
    return L3D_OK;
}

int64_t l3d_stereo_launches(const l3d_stereo* s) { return s ? s->launches : -1; }

int l3d_stereo_view_size(const l3d_stereo* s, int32_t layer, int32_t* width, int32_t* height) {
    if (!s || !width || !height) return fail(L3D_EINVAL, "NULL argument");
    if (layer < 0 || layer >= s->V) return fail(L3D_EINVAL, "layer %d out of range", layer);
    *width = s->Wv[layer];
    *height = s->Hv[layer];
    return L3D_OK;
}

int l3d_stereo_set_variant(l3d_stereo* s, int32_t variant) {
    if (!s) return fail(L3D_EINVAL, "NULL handle");
    if (!batched(s)) return fail(L3D_ESTATE, "variants select fast- and exact-form kernels");
    const int rows = variant & 7, rest = variant & ~63;
    const bool gather = (variant & 16) != 0, shared_window = (variant & 32) != 0;
    if (rest || !(rows == 6 || rows == 4 || rows == 3 || rows == 2))
        return fail(L3D_EINVAL, "variant %d: texture rows must be 6, 4, 3 or 2 (+8 for quads, +16 "
                                "for gathers, +32 for a shared-memory window)", variant);
    if (rows != 6 && (s->opts.form == L3D_FORM_EXACT || s->opts.compensated || gather || shared_window))
        return fail(L3D_EINVAL, "variant %d: the exact form, compensated sums, gathers and the "
                                "shared-memory window sample all six rows through the texture unit",
                    variant);
    if (gather && (s->opts.form != L3D_FORM_FAST || s->opts.storage == L3D_DTYPE_BF16))
        return fail(L3D_EINVAL, "variant %d: gathers with exact weights are a fast-form option for "
                                "texture storage (U8, F16, F32); the exact form always gathers", variant);
    if (shared_window && (s->opts.form != L3D_FORM_FAST || s->opts.storage == L3D_DTYPE_BF16))
        return fail(L3D_EINVAL, "variant %d: the shared-memory window is a fast-form option for "
                                "texture storage (U8, F16, F32); the exact form always keeps its "
                                "window in shared memory", variant);
    s->variant = variant;
    return L3D_OK;
}

int32_t l3d_stereo_variant(const l3d_stereo* s) { return s ? s->variant : -1; }

int l3d_stereo_set_graphs(l3d_stereo* s, int32_t enable) {
    if (!s) return fail(L3D_EINVAL, "NULL handle");
    if (!batched(s)) return fail(L3D_ESTATE, "graph replay is a fast- and exact-form feature");
    s->graphs = enable != 0;
    if (!s->graphs) {
        cudaStreamSynchronize(s->stream);
        for (auto& g : s->graph_cache) free_graph(g);
        s->graph_cache.clear();
    }
    return L3D_OK;
}

int l3d_stereo_autotune(l3d_stereo* s, int32_t n_refs, const int32_t* refs,
                        const l3d_solve_opts* opts, int32_t* best_variant, float* best_ms) {
    if (!s) return fail(L3D_EINVAL, "NULL handle");
    if (!batched(s)) return fail(L3D_ESTATE, "the autotuner picks fast- and exact-form variants");
    if (s->opts.storage == L3D_DTYPE_BF16) {
        if (best_variant) *best_variant = s->variant;
        return L3D_OK;  /* one sampler only */
    }
    const bool six_only = s->opts.form == L3D_FORM_EXACT || s->opts.compensated || !s->pairs ||
                          (s->variant & 16);
    /* +32 (the window in shared memory) is a fast-form option; BF16 returned above */
    const bool shwin = s->opts.form == L3D_FORM_FAST;
    std::vector<int> candidates = six_only ? std::vector<int>{6, 14} : std::vector<int>{6, 14, 4, 12};
    if (shwin) {
        candidates.push_back(6 | 32);
        candidates.push_back(14 | 32);
    }
    /* up to three iterations: the first propagates random planes, the later ones the converging
     * planes whose neighbouring pixels agree, and the variants rank differently on the two */
    std::vector<l3d_solve_opts> one(opts, opts + n_refs);
    for (auto& q : one) {
        q.iterations = std::max(1, std::min(q.iterations, 3));
        q.prior = nullptr;
        q.pack = 0;
    }
    cudaEvent_t a, b;
    L3D_CUDA(cudaEventCreate(&a), "event");
    L3D_CUDA(cudaEventCreate(&b), "event");
    const bool graphs = s->graphs;
    s->graphs = false;
    /* gathers change the weights, so they are the caller's accuracy choice, kept as set */
    const int keep = s->variant & 16;
    int best = s->variant;
    float best_t = 3.0e38f;
    int rc = L3D_OK;
    for (int c : candidates) {
        const int v = c | keep;
        s->variant = v;
        for (int rep = 0; rep < 2 && rc == L3D_OK; rep++) {  /* the first run warms the caches */
            cudaEventRecord(a, s->stream);
            rc = l3d_stereo_solve_all(s, n_refs, refs, one.data());
            cudaEventRecord(b, s->stream);
        }
        if (rc) break;
        if (cudaEventSynchronize(b) != cudaSuccess) {
            rc = cuda_fail(cudaGetLastError(), "autotune");
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best_t) {
            best_t = ms;
            best = v;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    s->graphs = graphs;
    s->variant = best;
    if (rc) return rc;
    if (best_variant) *best_variant = best;
    if (best_ms) *best_ms = best_t;
    return L3D_OK;
}

void l3d_stereo_destroy(l3d_stereo* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    cudaFree(s->images);
    cudaFree(s->depths);
    cudaFree(s->hyp);
    cudaFree(s->cost);
    cudaFree(s->prior);
    cudaFree(s->filtered);
    cudaFree(s->filtered_all);
    cudaFree(s->hyp_all);
    cudaFree(s->cost_all);
    cudaFree(s->prior_all);
    cudaFree(s->staging);
    cudaFree(s->planes);
    cudaFree(s->plane_out);
    for (auto& g : s->graph_cache) free_graph(g);
    for (cudaTextureObject_t t : s->texs)
        if (t) cudaDestroyTextureObject(t);
    for (cudaArray_t a : s->arrays)
        if (a) cudaFreeArray(a);
    cudaFree(s->pairs);
    cudaFree(s->grad_views);
    cudaFree(s->grad_pairs);
    cudaFree(s->grad_sums);
    cudaFree(s->fviews_dev);
    cudaFree(s->tile_start_dev);
    cudaFreeHost(s->fviews_host);
    cudaFreeHost(s->tile_start_host);
    if (s->staged) cudaEventDestroy(s->staged);
    if (s->done) cudaEventDestroy(s->done);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

}  // extern "C"

/* ------------------------------------------------------------------ TSDF handle ------------ */

struct l3d_tsdf {
    L3dTsdfGrid g{};
    int q8 = 0;
    long long voxels = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t done = nullptr;
    cudaEvent_t staged = nullptr;     /* after the last copy out of the pinned staging tables */
    float* tsdf = nullptr;
    void* weight = nullptr;
    int32_t* coords = nullptr;
    uint8_t* mask = nullptr;          /* bricks * mask_views */
    int mask_views = 0;
    L3dTsdfView* views = nullptr;     /* device, capacity view_cap */
    int view_cap = 0;
    const uint32_t** depth_ptrs = nullptr;  /* device, capacity view_cap */
    uint32_t* maps = nullptr;         /* uploaded host maps, map_cap * P */
    long long map_cap = 0;
    float* priors = nullptr;          /* uploaded priors, prior_cap * P */
    long long prior_cap = 0;
    float4* normals = nullptr;        /* decoded normal per 12-bit normal code */
    float* tiles = nullptr;           /* depth tiles of the depth-aware brick cull, tile_cap */
    int32_t* list = nullptr;          /* 1 + bricks: kept bricks of a one-view integration */
    uint32_t* sweep = nullptr;        /* the sweep's brick list: flags, prefix (bricks + 1 each),
                                         list (bricks), scan scratch */
    uint8_t* super = nullptr;         /* super-brick flags of the visibility pass, super_cap */
    long long super_cap = 0;
    cudaEvent_t read_done = nullptr;  /* after the copies of an asynchronous read-back */
    bool read_pending = false;
    long long tile_cap = 0;
    L3dTsdfView* views_host = nullptr;      /* pinned staging for views */
    const uint32_t** ptrs_host = nullptr;   /* pinned staging for depth pointers */
    long long launches = 0;
    cudaStream_t copy = nullptr;      /* read-back stream of integrate_many_read */
    cudaEvent_t slab_done[L3D_TSDF_READ_SLABS] = {};
};

namespace {

L3dTsdfView make_view(const l3d_integration_view& v) { return l3d_tsdf_view_of(v); }

int ensure_views(l3d_tsdf* t, int n) {
    if (t->view_cap >= n) return L3D_OK;
    cudaStreamSynchronize(t->stream);
    cudaFree(t->views);
    cudaFree(t->depth_ptrs);
    cudaFreeHost(t->views_host);
    cudaFreeHost(t->ptrs_host);
    t->views = nullptr;
    t->depth_ptrs = nullptr;
    t->views_host = nullptr;
    t->ptrs_host = nullptr;
    t->view_cap = 0;
    L3D_CUDA(cudaMalloc(&t->views, (size_t)n * sizeof(L3dTsdfView)), "view table");
    L3D_CUDA(cudaMalloc(&t->depth_ptrs, (size_t)n * sizeof(void*)), "view table");
    L3D_CUDA(cudaMallocHost(&t->views_host, (size_t)n * sizeof(L3dTsdfView)), "view staging");
    L3D_CUDA(cudaMallocHost(&t->ptrs_host, (size_t)n * sizeof(void*)), "view staging");
    t->view_cap = n;
    return L3D_OK;
}

int ensure_mask(l3d_tsdf* t, int n) {
    if (t->mask_views >= n) return L3D_OK;
    cudaStreamSynchronize(t->stream);
    cudaFree(t->mask);
    t->mask = nullptr;
    t->mask_views = 0;
    /* brick-major rows of n flags padded to 16 bytes (one flag per brick for one view) */
    L3D_CUDA(cudaMalloc(&t->mask, (size_t)t->g.bricks * (size_t)((n + 15) & ~15)), "brick mask");
    t->mask_views = n;
    return L3D_OK;
}

/* Depth tiles of the depth-aware brick cull, sized in tiles. */
int ensure_tiles(l3d_tsdf* t, long long n) {
    if (t->tile_cap >= n) return L3D_OK;
    L3D_CUDA(cudaStreamSynchronize(t->stream), "depth tiles: wait");
    L3D_CUDA(cudaFree(t->tiles), "depth tiles: free");
    t->tiles = nullptr;
    t->tile_cap = 0;
    L3D_CUDA(cudaMalloc(&t->tiles, (size_t)n * sizeof(float)), "depth tiles");
    t->tile_cap = n;
    return L3D_OK;
}

/* The sweep's list of the bricks some view keeps (allocated once: its size is the grid's). */
long long sweep_words(const l3d_tsdf* t) {
    return 3 * (t->g.bricks + 1) + (long long)((l3d_scan_scratch(t->g.bricks + 1) + 3) / 4);
}
int ensure_sweep(l3d_tsdf* t) {
    if (t->sweep || t->g.bricks == 0) return L3D_OK;
    L3D_CUDA(cudaMalloc(&t->sweep, (size_t)sweep_words(t) * 4), "sweep brick list");
    return L3D_OK;
}
uint32_t* sweep_flags(l3d_tsdf* t) { return t->sweep; }
uint32_t* sweep_prefix(l3d_tsdf* t) { return t->sweep + (t->g.bricks + 1); }
int32_t* sweep_list(l3d_tsdf* t) { return (int32_t*)(t->sweep + 2 * (t->g.bricks + 1)); }
uint32_t* sweep_scratch(l3d_tsdf* t) { return t->sweep + 3 * (t->g.bricks + 1); }

/* Work that writes the volume waits (on the device) for an asynchronous read-back of it. */
int after_read(l3d_tsdf* t) {
    if (t->read_pending) L3D_CUDA(cudaStreamWaitEvent(t->stream, t->read_done, 0), "stream wait");
    return L3D_OK;
}

int ensure_super(l3d_tsdf* t, int n_views) {
    const long long n = l3d_tsdf_super_flags(t->g, n_views);
    if (t->super_cap >= n) return L3D_OK;
    L3D_CUDA(cudaStreamSynchronize(t->stream), "super-brick flags: wait");
    L3D_CUDA(cudaFree(t->super), "super-brick flags: free");
    t->super = nullptr;
    t->super_cap = 0;
    L3D_CUDA(cudaMalloc(&t->super, (size_t)n), "super-brick flags");
    t->super_cap = n;
    return L3D_OK;
}

/* Upload buffers, sized in elements (u32 maps / f32 priors). */
int ensure_maps(l3d_tsdf* t, long long elems) {
    if (t->map_cap >= elems) return L3D_OK;
    cudaStreamSynchronize(t->stream);
    cudaFree(t->maps);
    t->maps = nullptr;
    t->map_cap = 0;
    L3D_CUDA(cudaMalloc(&t->maps, (size_t)elems * 4), "depth map upload buffer");
    t->map_cap = elems;
    return L3D_OK;
}

int ensure_priors(l3d_tsdf* t, long long elems) {
    if (t->prior_cap >= elems) return L3D_OK;
    cudaStreamSynchronize(t->stream);
    cudaFree(t->priors);
    t->priors = nullptr;
    t->prior_cap = 0;
    L3D_CUDA(cudaMalloc(&t->priors, (size_t)elems * 4), "prior upload buffer");
    t->prior_cap = elems;
    return L3D_OK;
}

int check_view(const l3d_integration_view* v) {
    if (!v) return fail(L3D_EINVAL, "integration view is NULL");
    if (!(v->intrinsics.fx != 0.0) || !(v->intrinsics.fy != 0.0))
        return fail(L3D_EINVAL, "zero focal length");
    return L3D_OK;
}

/* Orders the TSDF stream after the stereo handle's queued work (the filtered maps). */
int after_stereo(l3d_tsdf* t, const l3d_stereo* s) {
    L3D_CUDA(cudaEventRecord(s->done, s->stream), "event record");
    L3D_CUDA(cudaStreamWaitEvent(t->stream, s->done, 0), "stream wait");
    return L3D_OK;
}
/* Orders the stereo stream after the TSDF kernels that read its maps. */
int before_stereo(l3d_tsdf* t, const l3d_stereo* s) {
    L3D_CUDA(cudaEventRecord(t->done, t->stream), "event record");
    L3D_CUDA(cudaStreamWaitEvent(s->stream, t->done, 0), "stream wait");
    return L3D_OK;
}

}  // namespace

extern "C" {

int l3d_tsdf_create(const l3d_tsdf_desc* d, l3d_tsdf** out) {
    if (!out) return fail(L3D_EINVAL, "out is NULL");
    *out = nullptr;
    if (!d) return fail(L3D_EINVAL, "descriptor is NULL");
    L3dTsdfGrid g;
    char why[256];
    if (!l3d_tsdf_grid_of(d, d->coords != nullptr, &g, why, sizeof(why))) return fail(L3D_EINVAL, "%s", why);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "no CUDA device");
    l3d_tsdf* t = new (std::nothrow) l3d_tsdf();
    if (!t) return fail(L3D_ENOMEM, "host allocation failed");
    t->g = g;
    t->q8 = d->weight_type == L3D_WEIGHT_Q8;
    t->voxels = g.dense ? (long long)g.dims[0] * g.dims[1] * g.dims[2] : g.bricks * 512;
    auto cleanup = [&](int rc) {
        l3d_tsdf_destroy(t);
        return rc;
    };
    if (d->stream) {
        t->stream = (cudaStream_t)d->stream;
    } else {
        e = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "stream creation"));
        t->own_stream = true;
    }
    if ((e = cudaEventCreateWithFlags(&t->done, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&t->staged, cudaEventDisableTiming)) != cudaSuccess)
        return cleanup(cuda_fail(e, "event creation"));
    if ((e = cudaMalloc(&t->tsdf, (size_t)t->voxels * 4)) != cudaSuccess ||
        (e = cudaMalloc(&t->weight, (size_t)t->voxels * (t->q8 ? 2 : 4))) != cudaSuccess)
        return cleanup(cuda_fail(e, "volume allocation"));
    if (!g.dense) {
        if ((e = cudaMalloc(&t->coords, (size_t)g.bricks * 16)) != cudaSuccess)
            return cleanup(cuda_fail(e, "coords allocation"));
        if ((e = cudaMemcpyAsync(t->coords, d->coords, (size_t)g.bricks * 16, cudaMemcpyHostToDevice,
                                 t->stream)) != cudaSuccess)
            return cleanup(cuda_fail(e, "coords upload"));
        if ((e = cudaStreamSynchronize(t->stream)) != cudaSuccess)
            return cleanup(cuda_fail(e, "coords upload"));
    }
    if ((e = cudaMalloc(&t->normals, 4096 * sizeof(float4))) != cudaSuccess)
        return cleanup(cuda_fail(e, "normal table allocation"));
    if ((e = l3d_launch_normal_table(t->normals, t->stream)) != cudaSuccess)
        return cleanup(cuda_fail(e, "normal table"));
    t->launches++;
    int rc = l3d_tsdf_reset(t);
    if (rc) return cleanup(rc);
    *out = t;
    return L3D_OK;
}

int l3d_tsdf_reset(l3d_tsdf* t) {
    if (!t) return fail(L3D_EINVAL, "NULL handle");
    int rc = after_read(t);
    if (rc) return rc;
    cudaError_t e = l3d_launch_tsdf_fill(t->tsdf, t->weight, t->voxels, t->q8, t->stream);
    t->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "volume fill");
    return L3D_OK;
}

/* Body of l3d_tsdf_integrate and l3d_tsdf_integrate_layer: layer < 0 takes the stereo handle's
 * last filter() map, layer >= 0 its filter_all map of that layer. */
static int integrate_one(l3d_tsdf* t, const l3d_stereo* src, int layer, const uint32_t* packed,
                         const l3d_integration_view* view) {
    if (!t) return fail(L3D_EINVAL, "NULL handle");
    int rc = check_view(view);
    if (rc) return rc;
    if ((src == nullptr) == (packed == nullptr))
        return fail(L3D_EINVAL, "give exactly one of a stereo handle or a packed map");
    if (src && layer >= 0) {
        if (layer >= src->V) return fail(L3D_EINVAL, "layer %d out of range [0, %d)", layer, src->V);
        if (!src->filtered_all) return fail(L3D_ESTATE, "stereo handle has no filter_all output");
    }
    /* a stereo handle's filtered map has the size of the view it was filtered for */
    const int ml = src ? (layer >= 0 ? layer : src->filtered_ref) : 0;
    const int mw = src ? src->Wv[ml] : t->g.W;
    const int mh = src ? src->Hv[ml] : t->g.H;
    const long long P = (long long)mw * mh;
    if ((rc = ensure_mask(t, 1)) || (rc = after_read(t))) return rc;
    L3dTsdfView v = make_view(*view);
    v.W = mw;
    v.H = mh;
    const uint32_t* depth;
    if (src) {
        if ((rc = after_stereo(t, src))) return rc;
        depth = layer >= 0 ? src->filtered_all + src->offv[layer] : src->filtered;
    } else {
        if ((rc = ensure_maps(t, P))) return rc;
        L3D_CUDA(cudaMemcpyAsync(t->maps, packed, P * 4, cudaMemcpyHostToDevice, t->stream), "map upload");
        depth = t->maps;
    }
    const float* prior = nullptr;
    if (view->prior) {
        if ((rc = ensure_priors(t, P))) return rc;
        L3D_CUDA(cudaMemcpyAsync(t->priors, view->prior, P * 4, cudaMemcpyHostToDevice, t->stream), "prior upload");
        prior = t->priors;
    }
    /* visibility of this view's bricks, then the integration: two launches */
    if ((rc = ensure_tiles(t, l3d_depth_tile_count(mw, mh)))) return rc;
    if (!t->list) L3D_CUDA(cudaMalloc(&t->list, (size_t)(t->g.bricks + 1) * sizeof(int32_t)), "brick list");
    L3D_CUDA(cudaGetLastError(), "before the integrate launch");
    cudaError_t e = l3d_launch_tsdf_view(t->g, v, t->coords, t->mask, depth, prior, t->normals, t->tiles,
                                         t->list, t->tsdf, t->weight, t->q8, t->stream);
    t->launches += 3;
    if (e != cudaSuccess) return cuda_fail(e, "integrate launch");
    if (src && (rc = before_stereo(t, src))) return rc;
    return L3D_OK;
}

int l3d_tsdf_integrate(l3d_tsdf* t, const l3d_stereo* src, const uint32_t* packed,
                       const l3d_integration_view* view) {
    return integrate_one(t, src, -1, packed, view);
}

int l3d_tsdf_integrate_layer(l3d_tsdf* t, const l3d_stereo* src, int32_t layer,
                             const l3d_integration_view* view) {
    if (!src) return fail(L3D_EINVAL, "stereo handle is NULL");
    if (layer < 0) return fail(L3D_EINVAL, "layer %d out of range", layer);
    return integrate_one(t, src, layer, nullptr, view);
}

/* Body of l3d_tsdf_integrate_many and l3d_tsdf_integrate_many_read: with output buffers the
 * sweep runs as L3D_TSDF_READ_SLABS launches over consecutive voxel ranges, and each range is
 * copied out on the copy stream as soon as its launch is done. */
static int integrate_many(l3d_tsdf* t, const l3d_stereo* src, const int32_t* layers,
                          const uint32_t* packed, int32_t n, const l3d_integration_view* views,
                          float* tsdf_out, void* weight_out, int64_t* counts_out = nullptr,
                          bool wait = true) {
    if (!t) return fail(L3D_EINVAL, "NULL handle");
    if (!counts_out) {
        int rc0 = after_read(t);
        if (rc0) return rc0;
    }
    if (n < 0 || (n > 0 && !views)) return fail(L3D_EINVAL, "bad view list");
    if (n == 0) return L3D_OK;
    if ((src == nullptr) == (packed == nullptr))
        return fail(L3D_EINVAL, "give exactly one of a stereo handle or packed maps");
    const long long P = (long long)t->g.W * t->g.H;
    if (src) {
        if (!layers) return fail(L3D_EINVAL, "layers is NULL");
        if (!src->filtered_all) return fail(L3D_ESTATE, "stereo handle has no filter_all output");
        for (int i = 0; i < n; i++)
            if (layers[i] < 0 || layers[i] >= src->V) return fail(L3D_EINVAL, "layer %d out of range", layers[i]);
    }
    /* map size and prior offset per view (maps from a stereo handle keep their view's size) */
    std::vector<int> mw(n), mh(n);
    std::vector<long long> poff(n);
    long long ptotal = 0;
    for (int i = 0; i < n; i++) {
        mw[i] = src ? src->Wv[layers[i]] : t->g.W;
        mh[i] = src ? src->Hv[layers[i]] : t->g.H;
        poff[i] = ptotal;
        ptotal += (long long)mw[i] * mh[i];
    }
    int rc;
    for (int i = 0; i < n; i++)
        if ((rc = check_view(&views[i]))) return rc;
    if ((rc = ensure_views(t, n)) || (rc = ensure_mask(t, n))) return rc;
    bool any_prior = false;
    for (int i = 0; i < n; i++) any_prior |= views[i].prior != nullptr;
    if (src) {
        if ((rc = after_stereo(t, src))) return rc;
    } else {
        if ((rc = ensure_maps(t, (long long)n * P))) return rc;
        L3D_CUDA(cudaMemcpyAsync(t->maps, packed, (size_t)n * P * 4, cudaMemcpyHostToDevice, t->stream), "map upload");
    }
    if (any_prior) {
        if ((rc = ensure_priors(t, ptotal))) return rc;
        for (int i = 0; i < n; i++)
            if (views[i].prior)
                L3D_CUDA(cudaMemcpyAsync(t->priors + poff[i], views[i].prior, (size_t)mw[i] * mh[i] * 4,
                                         cudaMemcpyHostToDevice, t->stream), "prior upload");
    }
    /* depth tiles per view for the depth-aware brick cull (the update count reports what
     * visibleBricks alone keeps, and what the depth-aware cull keeps of it) */
    std::vector<long long> toff(n);
    long long ttotal = 0, tmax = 0;
    for (int i = 0; i < n; i++) {
        toff[i] = ttotal;
        const long long nt = l3d_depth_tile_count(mw[i], mh[i]);
        ttotal += nt;
        tmax = std::max(tmax, nt);
    }
    if ((rc = ensure_tiles(t, ttotal)) || (rc = ensure_super(t, n)) ||
        (!counts_out && (rc = ensure_sweep(t))))
        return rc;
    /* the pinned staging tables are reused: wait until the previous call's copies have run */
    L3D_CUDA(cudaEventSynchronize(t->staged), "staging wait");
    for (int i = 0; i < n; i++) {
        t->views_host[i] = make_view(views[i]);
        t->views_host[i].W = mw[i];
        t->views_host[i].H = mh[i];
        t->views_host[i].prior_off = poff[i];
        t->views_host[i].tile_off = toff[i];
        t->ptrs_host[i] = src ? src->filtered_all + src->offv[layers[i]] : t->maps + (size_t)i * P;
    }
    L3D_CUDA(cudaMemcpyAsync(t->views, t->views_host, (size_t)n * sizeof(L3dTsdfView), cudaMemcpyHostToDevice, t->stream), "view upload");
    L3D_CUDA(cudaMemcpyAsync(t->depth_ptrs, t->ptrs_host, (size_t)n * sizeof(void*), cudaMemcpyHostToDevice, t->stream), "view upload");
    L3D_CUDA(cudaEventRecord(t->staged, t->stream), "event record");
    cudaError_t e;
    if (counts_out) {
        /* visibleBricks alone: visible voxel-views and updates; then the depth-aware mask: the
         * voxel-views it keeps (the updates are the same, which the count checks) */
        unsigned long long* counts = nullptr;
        unsigned long long host[4] = {0, 0, 0, 0};
        L3D_CUDA(pool_alloc((void**)&counts, 4 * sizeof(unsigned long long), t->stream), "count buffer");
        e = cudaMemsetAsync(counts, 0, 4 * sizeof(unsigned long long), t->stream);
        if (e == cudaSuccess) e = l3d_launch_tsdf_visible(t->g, t->views, n, t->coords, t->mask, t->stream);
        if (e == cudaSuccess)
            e = l3d_launch_tsdf_count(t->g, t->views, n, t->coords, t->mask, t->depth_ptrs, t->priors,
                                      t->normals, counts, t->stream);
        if (e == cudaSuccess)
            e = l3d_launch_depth_tiles(t->views, n, t->depth_ptrs, t->priors, t->tiles, tmax, t->stream);
        if (e == cudaSuccess)
            e = l3d_launch_tsdf_visible_depth(t->g, t->views, n, t->coords, t->tiles, t->super, t->mask, t->stream);
        if (e == cudaSuccess)
            e = l3d_launch_tsdf_count(t->g, t->views, n, t->coords, t->mask, t->depth_ptrs, t->priors,
                                      t->normals, counts + 2, t->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(host, counts, sizeof(host), cudaMemcpyDeviceToHost, t->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
        t->launches += 5 + (l3d_tsdf_super_flags(t->g, n) > 0 ? 1 : 0);
        cudaFreeAsync(counts, t->stream);
        if (e != cudaSuccess) return cuda_fail(e, "update count");
        if (host[3] != host[1])
            return fail(L3D_ECUDA, "update count: the depth-aware cull dropped %llu updates",
                        (unsigned long long)(host[1] - host[3]));
        counts_out[0] = (int64_t)host[0];
        counts_out[1] = (int64_t)host[1];
        counts_out[2] = (int64_t)host[2];
        if (src && (rc = before_stereo(t, src))) return rc;
        return L3D_OK;
    }
    e = l3d_launch_depth_tiles(t->views, n, t->depth_ptrs, t->priors, t->tiles, tmax, t->stream);
    if (e == cudaSuccess)
        e = l3d_launch_tsdf_visible_depth(t->g, t->views, n, t->coords, t->tiles, t->super, t->mask, t->stream);
    /* the sweep visits only the bricks some view keeps */
    if (e == cudaSuccess)
        e = l3d_launch_tsdf_brick_list(t->g, n, t->mask, sweep_flags(t), sweep_prefix(t), sweep_list(t),
                                       sweep_scratch(t), t->stream);
    t->launches += 4 + (l3d_tsdf_super_flags(t->g, n) > 0 ? 1 : 0) + l3d_scan_launches(t->g.bricks + 1, false);
    if (e != cudaSuccess) return cuda_fail(e, "visibility launch");
    if (!tsdf_out && !weight_out) {
        e = l3d_launch_tsdf_many_list(t->g, t->views, n, t->coords, t->mask, t->depth_ptrs, t->priors,
                                      t->normals, t->tsdf, t->weight, t->q8, sweep_prefix(t),
                                      sweep_list(t), 0, l3d_tsdf_sweep_units(t->g, nullptr, nullptr),
                                      t->stream);
        t->launches++;
        if (e != cudaSuccess) return cuda_fail(e, "integrate launch");
    } else {
        if (!t->copy) {
            L3D_CUDA(cudaStreamCreateWithFlags(&t->copy, cudaStreamNonBlocking), "stream creation");
            for (cudaEvent_t& ev : t->slab_done)
                L3D_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event creation");
        }
        long long lu = 1, lv = 1;
        const long long units = l3d_tsdf_sweep_units(t->g, &lu, &lv);
        const long long layers = units / lu;
        const long long per = (layers + L3D_TSDF_READ_SLABS - 1) / L3D_TSDF_READ_SLABS;
        /* every launch first, so that a copy into pageable memory (which blocks the host until
         * it is done) does not hold back the next launch; each slab is whole layers, so its
         * voxels are one contiguous range */
        for (int i = 0; i < L3D_TSDF_READ_SLABS; i++) {
            const long long q0 = std::min(layers, i * per) * lu;
            const long long q1 = std::min(layers, i * per + per) * lu;
            e = l3d_launch_tsdf_many_list(t->g, t->views, n, t->coords, t->mask, t->depth_ptrs,
                                          t->priors, t->normals, t->tsdf, t->weight, t->q8,
                                          sweep_prefix(t), sweep_list(t), q0, q1, t->stream);
            t->launches += q1 > q0 ? 1 : 0;
            if (e != cudaSuccess) return cuda_fail(e, "integrate launch");
            L3D_CUDA(cudaEventRecord(t->slab_done[i], t->stream), "event record");
        }
        const size_t wsize = t->q8 ? 2 : 4;
        if (!wait && !t->read_done)
            L3D_CUDA(cudaEventCreateWithFlags(&t->read_done, cudaEventDisableTiming), "event creation");
        for (int i = 0; i < L3D_TSDF_READ_SLABS; i++) {
            const long long v0 = std::min(t->voxels, std::min(layers, i * per) * lv);
            const long long v1 = std::min(t->voxels, std::min(layers, i * per + per) * lv);
            if (v1 <= v0) continue;
            L3D_CUDA(cudaStreamWaitEvent(t->copy, t->slab_done[i], 0), "stream wait");
            if (tsdf_out)
                L3D_CUDA(cudaMemcpyAsync(tsdf_out + v0, t->tsdf + v0, (size_t)(v1 - v0) * 4,
                                         cudaMemcpyDeviceToHost, t->copy), "read tsdf");
            if (weight_out)
                L3D_CUDA(cudaMemcpyAsync((char*)weight_out + v0 * wsize, (char*)t->weight + v0 * wsize,
                                         (size_t)(v1 - v0) * wsize, cudaMemcpyDeviceToHost, t->copy),
                         "read weight");
        }
        if (wait) {
            L3D_CUDA(cudaStreamSynchronize(t->copy), "read");
            t->read_pending = false;
        } else {
            L3D_CUDA(cudaEventRecord(t->read_done, t->copy), "event record");
            t->read_pending = true;
        }
    }
    if (src && (rc = before_stereo(t, src))) return rc;
    return L3D_OK;
}

int l3d_tsdf_count_updates(l3d_tsdf* t, const l3d_stereo* src, const int32_t* layers,
                           const uint32_t* packed, int32_t n, const l3d_integration_view* views,
                           int64_t* visible, int64_t* updates, int64_t* kept) {
    if (!visible || !updates) return fail(L3D_EINVAL, "visible and updates must not be NULL");
    int64_t c[3] = {0, 0, 0};
    int rc = integrate_many(t, src, layers, packed, n, views, nullptr, nullptr, c);
    *visible = c[0];
    *updates = c[1];
    if (kept) *kept = c[2];
    return rc;
}

int l3d_tsdf_integrate_many(l3d_tsdf* t, const l3d_stereo* src, const int32_t* layers,
                            const uint32_t* packed, int32_t n, const l3d_integration_view* views) {
    return integrate_many(t, src, layers, packed, n, views, nullptr, nullptr);
}

int l3d_tsdf_integrate_many_read(l3d_tsdf* t, const l3d_stereo* src, const int32_t* layers,
                                 const uint32_t* packed, int32_t n,
                                 const l3d_integration_view* views, float* tsdf, void* weight) {
    if (!tsdf && !weight) return fail(L3D_EINVAL, "no output buffer");
    return integrate_many(t, src, layers, packed, n, views, tsdf, weight);
}

int l3d_tsdf_integrate_many_read_async(l3d_tsdf* t, const l3d_stereo* src, const int32_t* layers,
                                       const uint32_t* packed, int32_t n,
                                       const l3d_integration_view* views, float* tsdf, void* weight) {
    if (!tsdf && !weight) return fail(L3D_EINVAL, "no output buffer");
    return integrate_many(t, src, layers, packed, n, views, tsdf, weight, nullptr, false);
}

/* Shared body of l3d_tsdf_forward_depth / l3d_tsdf_backward. */
static int tsdf_depth_run(l3d_tsdf* t, const l3d_integration_view* view, int32_t width,
                          int32_t height, const uint32_t* packed, const float* depth,
                          const float* prior, const float* tsdf_in, const void* weight_in,
                          float* tsdf_out, void* weight_out, const float* grad_tsdf_out,
                          const float* grad_weight_out, float* grad_depth, float* grad_tsdf_in,
                          float* grad_weight_in, void* stream) {
    if (!t) return fail(L3D_EINVAL, "NULL handle");
    int rc = check_view(view);
    if (rc) return rc;
    if (width <= 0 || height <= 0) return fail(L3D_EINVAL, "depth map size must be positive");
    if (!packed || !depth || !tsdf_in || !weight_in)
        return fail(L3D_EINVAL, "NULL packed map, depth map or input volume");
    if ((rc = ensure_mask(t, 1))) return rc;
    L3dTsdfView v = make_view(*view);
    v.has_prior = prior != nullptr;
    v.W = width;
    v.H = height;
    cudaStream_t st = stream ? (cudaStream_t)stream : t->stream;
    const bool other = st != t->stream;
    if (other) {
        L3D_CUDA(cudaEventRecord(t->done, t->stream), "event record");
        L3D_CUDA(cudaStreamWaitEvent(st, t->done, 0), "stream wait");
    }
    /* the caller's buffers may be the handle's own volume: after its pending read-back */
    if (t->read_pending) L3D_CUDA(cudaStreamWaitEvent(st, t->read_done, 0), "stream wait");
    cudaError_t e = l3d_launch_tsdf_depth(t->g, v, t->coords, t->mask, packed, depth, prior, tsdf_in,
                                          weight_in, tsdf_out, weight_out, grad_tsdf_out,
                                          grad_weight_out, grad_depth, grad_tsdf_in, grad_weight_in,
                                          t->q8, st);
    t->launches += 2;
    if (e != cudaSuccess) return cuda_fail(e, "differentiable integrate launch");
    if (other) {
        /* the brick mask is shared with the handle's own integrations */
        L3D_CUDA(cudaEventRecord(t->done, st), "event record");
        L3D_CUDA(cudaStreamWaitEvent(t->stream, t->done, 0), "stream wait");
    }
    return L3D_OK;
}

int l3d_tsdf_forward_depth(l3d_tsdf* t, const l3d_integration_view* view, int32_t width,
                           int32_t height, const uint32_t* packed_dev, const float* depth_dev,
                           const float* prior_dev, const float* tsdf_in, const void* weight_in,
                           float* tsdf_out, void* weight_out, void* stream) {
    if (!tsdf_out || !weight_out) return fail(L3D_EINVAL, "NULL output volume");
    return tsdf_depth_run(t, view, width, height, packed_dev, depth_dev, prior_dev, tsdf_in,
                          weight_in, tsdf_out, weight_out, nullptr, nullptr, nullptr, nullptr,
                          nullptr, stream);
}

int l3d_tsdf_backward(l3d_tsdf* t, const l3d_integration_view* view, int32_t width, int32_t height,
                      const uint32_t* packed_dev, const float* depth_dev, const float* prior_dev,
                      const float* tsdf_in, const void* weight_in, const float* grad_tsdf_out,
                      const float* grad_weight_out, float* grad_depth, float* grad_tsdf_in,
                      float* grad_weight_in, void* stream) {
    if (!grad_tsdf_out) return fail(L3D_EINVAL, "grad_tsdf_out is NULL");
    if (!grad_depth && !grad_tsdf_in && !grad_weight_in)
        return fail(L3D_EINVAL, "no gradient output requested");
    return tsdf_depth_run(t, view, width, height, packed_dev, depth_dev, prior_dev, tsdf_in,
                          weight_in, nullptr, nullptr, grad_tsdf_out, grad_weight_out, grad_depth,
                          grad_tsdf_in, grad_weight_in, stream);
}

int l3d_tsdf_read(l3d_tsdf* t, float* tsdf, void* weight) {
    if (!t) return fail(L3D_EINVAL, "NULL handle");
    int rc = l3d_tsdf_wait_read(t);
    if (rc) return rc;
    if (tsdf) L3D_CUDA(cudaMemcpyAsync(tsdf, t->tsdf, (size_t)t->voxels * 4, cudaMemcpyDeviceToHost, t->stream), "read tsdf");
    if (weight)
        L3D_CUDA(cudaMemcpyAsync(weight, t->weight, (size_t)t->voxels * (t->q8 ? 2 : 4), cudaMemcpyDeviceToHost, t->stream), "read weight");
    L3D_CUDA(cudaStreamSynchronize(t->stream), "read");
    return L3D_OK;
}

int64_t l3d_tsdf_voxels(const l3d_tsdf* t) { return t ? t->voxels : -1; }

int l3d_tsdf_device_buffers(const l3d_tsdf* t, float** tsdf, void** weight) {
    if (!t) return fail(L3D_EINVAL, "NULL handle");
    if (tsdf) *tsdf = t->tsdf;
    if (weight) *weight = t->weight;
    return L3D_OK;
}

int l3d_tsdf_stream(const l3d_tsdf* t, void** stream) {
    if (!t || !stream) return fail(L3D_EINVAL, "NULL argument");
    *stream = (void*)t->stream;
    return L3D_OK;
}

int l3d_tsdf_wait_read(l3d_tsdf* t) {
    if (!t) return fail(L3D_EINVAL, "NULL handle");
    if (t->read_pending) {
        L3D_CUDA(cudaEventSynchronize(t->read_done), "read");
        t->read_pending = false;
    }
    return L3D_OK;
}

int l3d_tsdf_synchronize(l3d_tsdf* t) {
    if (!t) return fail(L3D_EINVAL, "NULL handle");
    L3D_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
    return l3d_tsdf_wait_read(t);
}

int64_t l3d_tsdf_launches(const l3d_tsdf* t) { return t ? t->launches : -1; }

void l3d_tsdf_destroy(l3d_tsdf* t) {
    if (!t) return;
    if (t->stream) cudaStreamSynchronize(t->stream);
    cudaFree(t->tsdf);
    cudaFree(t->weight);
    cudaFree(t->coords);
    cudaFree(t->mask);
    cudaFree(t->views);
    cudaFree(t->depth_ptrs);
    cudaFree(t->maps);
    cudaFree(t->priors);
    cudaFree(t->normals);
    cudaFree(t->tiles);
    cudaFree(t->list);
    cudaFree(t->sweep);
    cudaFree(t->super);
    cudaFreeHost(t->views_host);
    cudaFreeHost(t->ptrs_host);
    if (t->done) cudaEventDestroy(t->done);
    if (t->staged) cudaEventDestroy(t->staged);
    if (t->copy) cudaStreamSynchronize(t->copy);
    if (t->read_done) cudaEventDestroy(t->read_done);
    for (cudaEvent_t ev : t->slab_done)
        if (ev) cudaEventDestroy(ev);
    if (t->copy) cudaStreamDestroy(t->copy);
    if (t->own_stream && t->stream) cudaStreamDestroy(t->stream);
    delete t;
}

}  // extern "C"

/* ------------------------------------------------------------------ dense point cloud ------ */

struct l3d_cloud {
    double cell = 0.0;
    L3dCloudTable t{};
    unsigned* counters = nullptr;     /* [0] used slots, [1] emitted points */
    int* err = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t done = nullptr;
    uint8_t* thumb = nullptr;         /* uploaded thumbnail */
    size_t thumb_cap = 0;
    uint32_t* map = nullptr;          /* uploaded packed map */
    size_t map_cap = 0;
    double* pts = nullptr;            /* uploaded samples */
    size_t pts_cap = 0;
    long long launches = 0;
    long long used_bound = 0;         /* host-side upper bound of the used slots */
};

namespace {

/* Tables are stream-ordered allocations: growing or coarsening the table does not wait for the
 * whole device. */
void free_table(L3dCloudTable& t, cudaStream_t s) {
    if (t.keys) cudaFreeAsync(t.keys, s);
    if (t.sums) cudaFreeAsync(t.sums, s);
    if (t.counts) cudaFreeAsync(t.counts, s);
    t = L3dCloudTable{};
}

int alloc_table(l3d_cloud* c, int capacity, L3dCloudTable* out) {
    L3dCloudTable t{};
    t.capacity = capacity;
    cudaError_t e;
    if ((e = pool_alloc((void**)&t.keys, (size_t)capacity * 8, c->stream)) != cudaSuccess ||
        (e = pool_alloc((void**)&t.sums, (size_t)capacity * 9 * 8, c->stream)) != cudaSuccess ||
        (e = pool_alloc((void**)&t.counts, (size_t)capacity * 4, c->stream)) != cudaSuccess) {
        free_table(t, c->stream);
        return cuda_fail(e, "point table allocation");
    }
    if ((e = l3d_launch_cloud_clear(t, c->stream)) != cudaSuccess) {
        free_table(t, c->stream);
        return cuda_fail(e, "point table clear");
    }
    c->launches++;
    *out = t;
    return L3D_OK;
}

/* Waits for the queued work and reports a device-side error of the table. */
int cloud_state(l3d_cloud* c, unsigned* used) {
    unsigned h[2];
    int err = 0;
    L3D_CUDA(cudaMemcpyAsync(h, c->counters, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "read counters");
    L3D_CUDA(cudaMemcpyAsync(&err, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "read error flag");
    L3D_CUDA(cudaStreamSynchronize(c->stream), "synchronize");
    if (err & L3D_CLOUD_ERR_RANGE)
        return fail(L3D_EINVAL, "a point lies more than 2^20 cells from the origin (cell %g m)", c->cell);
    if (err & L3D_CLOUD_ERR_FULL) return fail(L3D_ECUDA, "point table overflow");
    if (used) *used = h[0];
    c->used_bound = h[0];
    return L3D_OK;
}

/* rebuild (point-accumulator.ts:89-111) into a table of `capacity` slots with cell `cell`. */
int cloud_rebuild(l3d_cloud* c, int capacity, double cell) {
    L3dCloudTable nt;
    int rc = alloc_table(c, capacity, &nt);
    if (rc) return rc;
    L3D_CUDA(cudaMemsetAsync(c->counters, 0, sizeof(unsigned), c->stream), "reset counter");
    cudaError_t e = l3d_launch_cloud_rebin(c->t, nt, cell, c->counters, c->err, c->stream);
    c->launches++;
    if (e != cudaSuccess) {
        free_table(nt, c->stream);
        return cuda_fail(e, "rebin launch");
    }
    free_table(c->t, c->stream);
    c->t = nt;
    c->cell = cell;
    return L3D_OK;
}

/* Grows the table (grow(), point-accumulator.ts:77-79) until `extra` new cells keep the load
 * at or under 60 %. */
int cloud_reserve(l3d_cloud* c, long long extra) {
    /* every sample adds at most one cell: while the bound kept on the host leaves room, the
     * table state need not be read back (no host round trip) */
    if ((c->used_bound + extra) * 10 <= (long long)c->t.capacity * 6) {
        c->used_bound += extra;
        return L3D_OK;
    }
    unsigned used = 0;
    int rc = cloud_state(c, &used);
    if (rc) return rc;
    long long cap = c->t.capacity;
    while (((long long)used + extra) * 10 > cap * 6) cap *= 2;
    if (cap > (1ll << 30)) return fail(L3D_ENOMEM, "point table would exceed 2^30 slots");
    if (cap != c->t.capacity && (rc = cloud_rebuild(c, (int)cap, c->cell))) return rc;
    c->used_bound = (long long)used + extra;
    return L3D_OK;
}

template <typename T>
int ensure_upload(T** p, size_t* cap, size_t n, cudaStream_t stream, const char* what) {
    if (*cap >= n) return L3D_OK;
    if (*p) cudaFreeAsync(*p, stream);
    *p = nullptr;
    *cap = 0;
    L3D_CUDA(pool_alloc((void**)p, std::max<size_t>(n, 1) * sizeof(T), stream), what);
    *cap = n;
    return L3D_OK;
}

}  // namespace

extern "C" {

int l3d_cloud_create(double cell, void* stream, l3d_cloud** out) {
    if (!out) return fail(L3D_EINVAL, "out is NULL");
    *out = nullptr;
    if (!(cell > 0.0)) return fail(L3D_EINVAL, "cell must be positive");
    l3d_cloud* c = new (std::nothrow) l3d_cloud();
    if (!c) return fail(L3D_ENOMEM, "host allocation failed");
    c->cell = cell;
    auto cleanup = [&](int rc) {
        l3d_cloud_destroy(c);
        return rc;
    };
    cudaError_t e;
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess)
            return cleanup(cuda_fail(e, "stream creation"));
        c->own_stream = true;
    }
    if ((e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming)) != cudaSuccess)
        return cleanup(cuda_fail(e, "event creation"));
    if ((e = pool_alloc((void**)&c->counters, 2 * sizeof(unsigned), c->stream)) != cudaSuccess ||
        (e = pool_alloc((void**)&c->err, sizeof(int), c->stream)) != cudaSuccess)
        return cleanup(cuda_fail(e, "counter allocation"));
    if ((e = cudaMemsetAsync(c->counters, 0, 2 * sizeof(unsigned), c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->err, 0, sizeof(int), c->stream)) != cudaSuccess)
        return cleanup(cuda_fail(e, "counter clear"));
    int rc = alloc_table(c, 1 << 16, &c->t);
    if (rc) return cleanup(rc);
    *out = c;
    return L3D_OK;
}

int l3d_cloud_add(l3d_cloud* c, const l3d_stereo* src, const uint32_t* packed, int32_t width,
                  int32_t height, const l3d_view* view, const uint8_t* thumb_rgb, int32_t thumb_w,
                  int32_t thumb_h) {
    if (!c || !view || !thumb_rgb) return fail(L3D_EINVAL, "NULL handle, view or thumbnail");
    if ((src == nullptr) == (packed == nullptr))
        return fail(L3D_EINVAL, "give exactly one of a stereo handle or a packed map");
    if (thumb_w <= 0 || thumb_h <= 0) return fail(L3D_EINVAL, "thumbnail size must be positive");
    if (!(view->intrinsics.fx != 0.0) || !(view->intrinsics.fy != 0.0))
        return fail(L3D_EINVAL, "zero focal length");
    /* a stereo handle's filtered map has the size of the view it was filtered for */
    const int W = src ? src->Wv[src->filtered_ref] : width;
    const int H = src ? src->Hv[src->filtered_ref] : height;
    if (W <= 0 || H <= 0) return fail(L3D_EINVAL, "depth map size must be positive");
    int rc = cloud_reserve(c, (long long)W * H);
    if (rc) return rc;
    const size_t tb = (size_t)thumb_w * thumb_h * 3;
    if ((rc = ensure_upload(&c->thumb, &c->thumb_cap, tb, c->stream, "thumbnail buffer"))) return rc;
    L3D_CUDA(cudaMemcpyAsync(c->thumb, thumb_rgb, tb, cudaMemcpyHostToDevice, c->stream), "thumbnail upload");
    const uint32_t* map;
    if (src) {
        L3D_CUDA(cudaEventRecord(src->done, src->stream), "event record");
        L3D_CUDA(cudaStreamWaitEvent(c->stream, src->done, 0), "stream wait");
        map = src->filtered;
    } else {
        if ((rc = ensure_upload(&c->map, &c->map_cap, (size_t)W * H, c->stream, "map buffer"))) return rc;
        L3D_CUDA(cudaMemcpyAsync(c->map, packed, (size_t)W * H * 4, cudaMemcpyHostToDevice, c->stream),
                 "map upload");
        map = c->map;
    }
    L3dCloudView v;
    std::memset(&v, 0, sizeof(v));
    v.k[0] = view->intrinsics.fx;
    v.k[1] = view->intrinsics.fy;
    v.k[2] = view->intrinsics.cx;
    v.k[3] = view->intrinsics.cy;
    for (int i = 0; i < 9; i++) v.R[i] = view->pose.R[i];
    for (int i = 0; i < 3; i++) v.t[i] = view->pose.t[i];
    v.tw = thumb_w;
    v.th = thumb_h;
    cudaError_t e = l3d_launch_cloud_add_map(c->t, c->cell, map, W, H, v, c->thumb, c->counters,
                                             c->err, c->stream);
    c->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "point add launch");
    if (src) {
        /* the stereo handle's later work (the next filter) waits for this read */
        L3D_CUDA(cudaEventRecord(c->done, c->stream), "event record");
        L3D_CUDA(cudaStreamWaitEvent(src->stream, c->done, 0), "stream wait");
    }
    return L3D_OK;
}

int l3d_cloud_add_points(l3d_cloud* c, int64_t n, const double* samples) {
    if (!c) return fail(L3D_EINVAL, "NULL handle");
    if (n < 0 || (n > 0 && !samples)) return fail(L3D_EINVAL, "bad sample list");
    if (n == 0) return L3D_OK;
    int rc = cloud_reserve(c, n);
    if (rc) return rc;
    if ((rc = ensure_upload(&c->pts, &c->pts_cap, (size_t)n * 9, c->stream, "sample buffer"))) return rc;
    L3D_CUDA(cudaMemcpyAsync(c->pts, samples, (size_t)n * 9 * 8, cudaMemcpyHostToDevice, c->stream),
             "sample upload");
    cudaError_t e = l3d_launch_cloud_add_points(c->t, c->cell, c->pts, n, c->counters, c->err, c->stream);
    c->launches++;
    if (e != cudaSuccess) return cuda_fail(e, "point add launch");
    return L3D_OK;
}

int l3d_cloud_coarsen(l3d_cloud* c, double factor) {
    if (!c) return fail(L3D_EINVAL, "NULL handle");
    if (!(factor > 0.0)) return fail(L3D_EINVAL, "factor must be positive");
    int rc = cloud_state(c, nullptr);
    if (rc) return rc;
    return cloud_rebuild(c, c->t.capacity, c->cell * factor);
}

int l3d_cloud_size(l3d_cloud* c, int64_t* size) {
    if (!c || !size) return fail(L3D_EINVAL, "NULL argument");
    unsigned used = 0;
    int rc = cloud_state(c, &used);
    if (rc) return rc;
    *size = used;
    return L3D_OK;
}

int l3d_cloud_cell(const l3d_cloud* c, double* cell) {
    if (!c || !cell) return fail(L3D_EINVAL, "NULL argument");
    *cell = c->cell;
    return L3D_OK;
}

int l3d_cloud_read(l3d_cloud* c, int32_t min_support, int64_t capacity, int64_t* count,
                   float* positions, float* normals, uint8_t* colors, uint16_t* support,
                   int32_t* cells) {
    if (!c || !count) return fail(L3D_EINVAL, "NULL handle or count");
    unsigned used = 0;
    int rc = cloud_state(c, &used);
    if (rc) return rc;
    const unsigned sort_n = l3d_cloud_sort_length(std::max<unsigned>(used, 1u));
    unsigned long long* dkey = nullptr;
    uint32_t* dslot = nullptr;
    float* dpos = nullptr;
    float* dnrm = nullptr;
    uint8_t* dcol = nullptr;
    uint16_t* dsup = nullptr;
    int32_t* dcell = nullptr;
    cudaError_t e;
    auto cleanup = [&]() {
        for (void* q : {(void*)dkey, (void*)dslot, (void*)dpos, (void*)dnrm, (void*)dcol, (void*)dsup,
                        (void*)dcell})
            if (q) cudaFreeAsync(q, c->stream);
    };
    if ((e = pool_alloc((void**)&dkey, (size_t)sort_n * 8, c->stream)) != cudaSuccess ||
        (e = pool_alloc((void**)&dslot, (size_t)sort_n * 4, c->stream)) != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "read buffers");
    }
    unsigned total = 0;
    if ((e = cudaMemsetAsync(c->counters + 1, 0, sizeof(unsigned), c->stream)) != cudaSuccess ||
        (e = l3d_launch_cloud_emit_keys(c->t, (unsigned)std::max(min_support, 0), c->counters + 1, dkey,
                                        dslot, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&total, c->counters + 1, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             c->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "point read");
    }
    c->launches++;
    *count = total;
    if (!positions && !normals && !colors && !support && !cells) {
        cleanup();
        return L3D_OK;
    }
    if (capacity < (int64_t)total) {
        cleanup();
        return fail(L3D_EINVAL, "output holds %lld points, the cloud has %u", (long long)capacity, total);
    }
    /* cells in ascending packed order (z, then y, then x; keys are distinct), sorted and
     * gathered on the device, then copied straight into the caller's arrays */
    const size_t m = std::max<unsigned>(total, 1u);
    if ((e = pool_alloc((void**)&dpos, m * 12, c->stream)) != cudaSuccess ||
        (e = pool_alloc((void**)&dnrm, m * 12, c->stream)) != cudaSuccess ||
        (e = pool_alloc((void**)&dcol, m * 3, c->stream)) != cudaSuccess ||
        (e = pool_alloc((void**)&dsup, m * 2, c->stream)) != cudaSuccess ||
        (e = pool_alloc((void**)&dcell, m * 12, c->stream)) != cudaSuccess ||
        (e = l3d_launch_cloud_sort(dkey, dslot, total, sort_n, &c->launches, c->stream)) != cudaSuccess ||
        (e = l3d_launch_cloud_emit_sorted(c->t, total, dkey, dslot, dpos, dnrm, dcol, dsup, dcell,
                                          c->stream)) != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "point ordering");
    }
    c->launches += total ? 1 : 0;
    struct Out {
        void* host;
        const void* dev;
        size_t bytes;
    } outs[] = {{positions, dpos, (size_t)total * 12}, {normals, dnrm, (size_t)total * 12},
                {colors, dcol, (size_t)total * 3}, {support, dsup, (size_t)total * 2},
                {cells, dcell, (size_t)total * 12}};
    for (const Out& o : outs)
        if (o.host && o.bytes &&
            (e = cudaMemcpyAsync(o.host, o.dev, o.bytes, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess) {
            cleanup();
            return cuda_fail(e, "point download");
        }
    cleanup();
    L3D_CUDA(cudaStreamSynchronize(c->stream), "point download");
    return L3D_OK;
}

int64_t l3d_cloud_launches(const l3d_cloud* c) { return c ? c->launches : -1; }

void l3d_cloud_destroy(l3d_cloud* c) {
    if (!c) return;
    free_table(c->t, c->stream);
    for (void* q : {(void*)c->counters, (void*)c->err, (void*)c->thumb, (void*)c->map, (void*)c->pts})
        if (q) cudaFreeAsync(q, c->stream);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->done) cudaEventDestroy(c->done);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

}  // extern "C"

/* ------------------------------------------------------------------ surface extraction ----- */

struct l3d_mesh {
    float* pos = nullptr;
    float* nrm = nullptr;
    uint32_t* idx = nullptr;
    long long nv = 0, ni = 0;
    long long launches = 0;
};

namespace {

/* Scratch buffers allocated and freed in the order of stream `s` (no device-wide wait), freed
 * when the holder goes out of scope. */
struct DevBufs {
    cudaStream_t s;
    std::vector<void*> ptrs;
    explicit DevBufs(cudaStream_t stream) : s(stream) {}
    ~DevBufs() {
        for (void* p : ptrs) cudaFreeAsync(p, s);
    }
    template <typename T>
    cudaError_t get(T** p, size_t count) {
        *p = nullptr;
        cudaError_t e = pool_alloc((void**)p, std::max<size_t>(count, 1) * sizeof(T), s);
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};

int read_u32(const uint32_t* dev, uint32_t* host, cudaStream_t s) {
    L3D_CUDA(cudaMemcpyAsync(host, dev, 4, cudaMemcpyDeviceToHost, s), "read count");
    L3D_CUDA(cudaStreamSynchronize(s), "synchronize");
    return L3D_OK;
}

/* Mesh buffers come from the library's pool.  Every mesh call waits for its own work before it
 * returns, so a mesh handed back to the caller has nothing pending and is freed on the default
 * stream; error paths free on the stream that may still hold work on the buffers. */
void mesh_free(l3d_mesh* m, cudaStream_t s = 0) {
    if (!m) return;
    for (void* q : {(void*)m->pos, (void*)m->nrm, (void*)m->idx})
        if (q) cudaFreeAsync(q, s);
    delete m;
}

/* extractSurface (surface-nets.ts:47-174) + computeNormals (mesh.ts:9-31) of a volume view with
 * `bricks` bricks. */
int extract_mesh(const L3dSdfView& v, long long bricks, cudaStream_t s, l3d_mesh** out) {
    const long long cells = bricks * 512;
    if (cells >= (1ll << 31)) return fail(L3D_EINVAL, "volume too large for surface extraction");
    DevBufs tmp(s);
    uint32_t *flag, *base, *qcount, *qbase, *scratch, *total;
    int32_t* cell_vertex;
    L3D_CUDA(tmp.get(&flag, cells), "surface buffers");
    L3D_CUDA(tmp.get(&base, cells), "surface buffers");
    L3D_CUDA(tmp.get(&qcount, cells), "surface buffers");
    L3D_CUDA(tmp.get(&qbase, cells), "surface buffers");
    L3D_CUDA(tmp.get(&cell_vertex, cells), "surface buffers");
    L3D_CUDA(tmp.get(&scratch, l3d_scan_scratch(std::max(cells, 1ll)) / 4 + 1), "scan scratch");
    L3D_CUDA(tmp.get(&total, 2), "scan total");
    l3d_mesh* m = new (std::nothrow) l3d_mesh();
    if (!m) return fail(L3D_ENOMEM, "host allocation failed");
    auto bail = [&](int rc) {
        mesh_free(m, s);
        return rc;
    };
    cudaError_t e;
    uint32_t nv = 0, nq = 0;
    if ((e = l3d_launch_sn_flag(v, cells, flag, s)) != cudaSuccess ||
        (e = l3d_scan_exclusive(flag, base, cells, scratch, total, s)) != cudaSuccess)
        return bail(cuda_fail(e, "surface vertices"));
    int rc = read_u32(total, &nv, s);
    if (rc) return bail(rc);
    double* pos_d;
    if ((e = tmp.get(&pos_d, (size_t)nv * 3)) != cudaSuccess ||
        (e = pool_alloc((void**)&m->pos, std::max<size_t>(nv, 1) * 12, s)) != cudaSuccess ||
        (e = pool_alloc((void**)&m->nrm, std::max<size_t>(nv, 1) * 12, s)) != cudaSuccess)
        return bail(cuda_fail(e, "vertex buffers"));
    if ((e = l3d_launch_sn_vertex(v, cells, flag, base, cell_vertex, pos_d, m->pos, s)) != cudaSuccess ||
        (e = l3d_launch_sn_count(v, cells, cell_vertex, qcount, s)) != cudaSuccess ||
        (e = l3d_scan_exclusive(qcount, qbase, cells, scratch, total, s)) != cudaSuccess)
        return bail(cuda_fail(e, "surface quads"));
    if ((rc = read_u32(total, &nq, s))) return bail(rc);
    const long long faces = 2ll * nq;
    if ((e = pool_alloc((void**)&m->idx, std::max<long long>(faces * 3, 1) * 4, s)) != cudaSuccess)
        return bail(cuda_fail(e, "index buffer"));
    if ((e = l3d_launch_sn_emit(v, cells, cell_vertex, qcount, qbase, pos_d, m->idx, s)) != cudaSuccess)
        return bail(cuda_fail(e, "surface triangles"));
    /* normals: faces gathered per vertex in face order */
    double* fn;
    uint32_t *degree, *start, *cursor, *lists;
    if ((e = tmp.get(&fn, (size_t)faces * 3)) != cudaSuccess || (e = tmp.get(&degree, nv)) != cudaSuccess ||
        (e = tmp.get(&start, nv)) != cudaSuccess || (e = tmp.get(&cursor, nv)) != cudaSuccess ||
        (e = tmp.get(&lists, (size_t)faces * 3)) != cudaSuccess)
        return bail(cuda_fail(e, "normal buffers"));
    uint32_t* nscratch;
    if ((e = tmp.get(&nscratch, l3d_scan_scratch(std::max<long long>(nv, 1)) / 4 + 1)) != cudaSuccess)
        return bail(cuda_fail(e, "scan scratch"));
    if ((e = cudaMemsetAsync(degree, 0, std::max<size_t>(nv, 1) * 4, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(cursor, 0, std::max<size_t>(nv, 1) * 4, s)) != cudaSuccess ||
        (e = l3d_launch_face_normals(m->pos, m->idx, faces, fn, degree, s)) != cudaSuccess ||
        (e = l3d_scan_exclusive(degree, start, nv, nscratch, nullptr, s)) != cudaSuccess ||
        (e = l3d_launch_face_lists(m->idx, faces, start, cursor, lists, s)) != cudaSuccess ||
        (e = l3d_launch_vertex_normals(nv, start, degree, lists, fn, m->nrm, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return bail(cuda_fail(e, "vertex normals"));
    m->nv = nv;
    m->ni = faces * 3;
    m->launches = 13;
    *out = m;
    return L3D_OK;
}

/* Grid dims and lookup of a brick pool from its coords (host). */
void pool_lookup(const int32_t* coords, long long count, int dims[3], std::vector<int32_t>& lookup) {
    dims[0] = dims[1] = dims[2] = 1;
    for (long long b = 0; b < count; b++)
        for (int k = 0; k < 3; k++) dims[k] = std::max(dims[k], coords[b * 4 + k] + 1);
    lookup.assign((size_t)dims[0] * dims[1] * dims[2], -1);
    for (long long b = 0; b < count; b++)
        lookup[((size_t)coords[b * 4 + 2] * dims[1] + coords[b * 4 + 1]) * dims[0] + coords[b * 4]] = (int32_t)b;
}

}  // namespace

extern "C" {

int l3d_tsdf_extract_surface(l3d_tsdf* t, double min_weight, l3d_mesh** out) {
    if (!t || !out) return fail(L3D_EINVAL, "NULL handle or out");
    *out = nullptr;
    L3dSdfView v;
    std::memset(&v, 0, sizeof(v));
    v.tsdf = t->tsdf;
    v.weight = t->weight;
    v.q8 = t->q8;
    for (int i = 0; i < 3; i++) v.origin[i] = t->g.origin_d[i];
    v.voxel = t->g.voxel_d;
    v.min_weight = min_weight;
    DevBufs tmp(t->stream);
    long long bricks;
    if (t->g.dense) {
        v.dense = 1;
        for (int i = 0; i < 3; i++) {
            v.dims[i] = t->g.nb[i];
            v.vdims[i] = t->g.dims[i];
        }
        bricks = (long long)v.dims[0] * v.dims[1] * v.dims[2];
    } else {
        bricks = t->g.bricks;
        std::vector<int32_t> coords((size_t)bricks * 4), lookup;
        L3D_CUDA(cudaMemcpyAsync(coords.data(), t->coords, coords.size() * 4, cudaMemcpyDeviceToHost,
                                 t->stream), "read coords");
        L3D_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
        pool_lookup(coords.data(), bricks, v.dims, lookup);
        int32_t* dl;
        L3D_CUDA(tmp.get(&dl, lookup.size()), "lookup buffer");
        L3D_CUDA(cudaMemcpyAsync(dl, lookup.data(), lookup.size() * 4, cudaMemcpyHostToDevice, t->stream),
                 "lookup upload");
        v.lookup = dl;
        v.coords = t->coords;
        for (int i = 0; i < 3; i++) v.vdims[i] = v.dims[i] * 8;
    }
    int rc = extract_mesh(v, bricks, t->stream, out);
    if (!rc) t->launches += (*out)->launches;
    return rc;
}

int l3d_extract_surface(const l3d_sdf_bricks* vol, double min_weight, l3d_mesh** out) {
    if (!vol || !out || !vol->lookup || !vol->tsdf || !vol->weight)
        return fail(L3D_EINVAL, "NULL volume, array or out");
    *out = nullptr;
    if (vol->bricks < 0 || vol->dims[0] <= 0 || vol->dims[1] <= 0 || vol->dims[2] <= 0)
        return fail(L3D_EINVAL, "bad volume dimensions");
    const size_t cells = (size_t)vol->dims[0] * vol->dims[1] * vol->dims[2];
    std::vector<int32_t> coords((size_t)std::max<int64_t>(vol->bricks, 1) * 4, 0);
    for (size_t i = 0; i < cells; i++) {
        const int32_t b = vol->lookup[i];
        if (b < 0) continue;
        if (b >= vol->bricks) return fail(L3D_EINVAL, "lookup entry %d beyond %lld bricks", b, (long long)vol->bricks);
        coords[(size_t)b * 4] = (int32_t)(i % vol->dims[0]);
        coords[(size_t)b * 4 + 1] = (int32_t)((i / vol->dims[0]) % vol->dims[1]);
        coords[(size_t)b * 4 + 2] = (int32_t)(i / ((size_t)vol->dims[0] * vol->dims[1]));
    }
    cudaStream_t s;
    L3D_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream creation");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard{s};
    DevBufs tmp(s);
    int32_t *dl, *dc;
    float *dt, *dw;
    const size_t voxels = (size_t)vol->bricks * 512;
    L3D_CUDA(tmp.get(&dl, cells), "volume upload");
    L3D_CUDA(tmp.get(&dc, coords.size()), "volume upload");
    L3D_CUDA(tmp.get(&dt, voxels), "volume upload");
    L3D_CUDA(tmp.get(&dw, voxels), "volume upload");
    L3D_CUDA(cudaMemcpyAsync(dl, vol->lookup, cells * 4, cudaMemcpyHostToDevice, s), "volume upload");
    L3D_CUDA(cudaMemcpyAsync(dc, coords.data(), coords.size() * 4, cudaMemcpyHostToDevice, s), "volume upload");
    L3D_CUDA(cudaMemcpyAsync(dt, vol->tsdf, voxels * 4, cudaMemcpyHostToDevice, s), "volume upload");
    L3D_CUDA(cudaMemcpyAsync(dw, vol->weight, voxels * 4, cudaMemcpyHostToDevice, s), "volume upload");
    L3dSdfView v;
    std::memset(&v, 0, sizeof(v));
    v.tsdf = dt;
    v.weight = dw;
    v.lookup = dl;
    v.coords = dc;
    for (int i = 0; i < 3; i++) {
        v.dims[i] = vol->dims[i];
        v.vdims[i] = vol->dims[i] * 8;
        v.origin[i] = vol->origin[i];
    }
    v.voxel = vol->voxel;
    v.min_weight = min_weight;
    return extract_mesh(v, vol->bricks, s, out);
}

int l3d_mesh_counts(const l3d_mesh* m, int64_t* vertices, int64_t* indices) {
    if (!m) return fail(L3D_EINVAL, "NULL mesh");
    if (vertices) *vertices = m->nv;
    if (indices) *indices = m->ni;
    return L3D_OK;
}

int l3d_mesh_read(const l3d_mesh* m, float* positions, float* normals, uint32_t* indices) {
    if (!m) return fail(L3D_EINVAL, "NULL mesh");
    if (positions && m->nv) L3D_CUDA(cudaMemcpy(positions, m->pos, m->nv * 12, cudaMemcpyDeviceToHost), "read positions");
    if (normals && m->nv) L3D_CUDA(cudaMemcpy(normals, m->nrm, m->nv * 12, cudaMemcpyDeviceToHost), "read normals");
    if (indices && m->ni) L3D_CUDA(cudaMemcpy(indices, m->idx, m->ni * 4, cudaMemcpyDeviceToHost), "read indices");
    return L3D_OK;
}

int l3d_mesh_remove_small_components(const l3d_mesh* m, double fraction, int32_t min_faces,
                                     l3d_mesh** out) {
    if (!m || !out) return fail(L3D_EINVAL, "NULL mesh or out");
    *out = nullptr;
    const long long nv = m->nv, faces = m->ni / 3;
    cudaStream_t s;
    L3D_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream creation");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard{s};
    DevBufs tmp(s);
    uint32_t *label, *comp, *kept, *first, *face_base, *marks, *rank, *scratch, *total;
    int* changed;
    L3D_CUDA(tmp.get(&label, nv), "component buffers");
    L3D_CUDA(tmp.get(&comp, nv), "component buffers");
    L3D_CUDA(tmp.get(&kept, faces), "component buffers");
    L3D_CUDA(tmp.get(&first, nv), "component buffers");
    L3D_CUDA(tmp.get(&face_base, faces), "component buffers");
    L3D_CUDA(tmp.get(&marks, faces * 3), "component buffers");
    L3D_CUDA(tmp.get(&rank, faces * 3), "component buffers");
    L3D_CUDA(tmp.get(&scratch, l3d_scan_scratch(std::max(faces * 3, 1ll)) / 4 + 1), "scan scratch");
    L3D_CUDA(tmp.get(&total, 2), "scan total");
    L3D_CUDA(tmp.get(&changed, 1), "flag");
    L3D_CUDA(l3d_launch_cc_init(nv, label, s), "component labels");
    /* rounds in batches of 8 between host checks: once the labels have settled a round changes
     * nothing, so the extra rounds of the last batch leave the result as it is */
    int rounds = 0;
    for (;;) {
        if (rounds >= 256) return fail(L3D_ECUDA, "connected components did not settle in 256 rounds");
        int h = 0;
        L3D_CUDA(cudaMemsetAsync(changed, 0, sizeof(int), s), "flag clear");
        for (int k = 0; k < 8; k++, rounds++)
            L3D_CUDA(l3d_launch_cc_round(m->idx, faces, nv, label, changed, s), "component round");
        L3D_CUDA(cudaMemcpyAsync(&h, changed, sizeof(int), cudaMemcpyDeviceToHost, s), "flag read");
        L3D_CUDA(cudaStreamSynchronize(s), "synchronize");
        if (!h) break;
    }
    const double limit = std::max((double)min_faces, (double)faces * fraction);
    uint32_t kf = 0, kv = 0;
    L3D_CUDA(cudaMemsetAsync(comp, 0, std::max<size_t>(nv, 1) * 4, s), "clear");
    L3D_CUDA(cudaMemsetAsync(first, 0xff, std::max<size_t>(nv, 1) * 4, s), "clear");
    L3D_CUDA(cudaMemsetAsync(marks, 0, std::max<size_t>(faces * 3, 1) * 4, s), "clear");
    L3D_CUDA(l3d_launch_cc_count(m->idx, faces, label, comp, s), "component sizes");
    L3D_CUDA(l3d_launch_cc_keep(m->idx, faces, label, comp, limit, kept, first, s), "kept faces");
    L3D_CUDA(l3d_scan_exclusive(kept, face_base, faces, scratch, total, s), "face scan");
    int rc = read_u32(total, &kf, s);
    if (rc) return rc;
    L3D_CUDA(l3d_launch_cc_first_marks(nv, first, marks, s), "vertex order");
    L3D_CUDA(l3d_scan_exclusive(marks, rank, faces * 3, scratch, total, s), "vertex scan");
    if ((rc = read_u32(total, &kv, s))) return rc;
    l3d_mesh* r = new (std::nothrow) l3d_mesh();
    if (!r) return fail(L3D_ENOMEM, "host allocation failed");
    cudaError_t e;
    if ((e = pool_alloc((void**)&r->pos, std::max<size_t>(kv, 1) * 12, s)) != cudaSuccess ||
        (e = pool_alloc((void**)&r->nrm, std::max<size_t>(kv, 1) * 12, s)) != cudaSuccess ||
        (e = pool_alloc((void**)&r->idx, std::max<size_t>(kf, 1) * 12, s)) != cudaSuccess ||
        (e = l3d_launch_cc_emit(m->idx, faces, kept, face_base, first, rank, m->pos, m->nrm, r->idx,
                                r->pos, r->nrm, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        mesh_free(r, s);
        return cuda_fail(e, "component output");
    }
    r->nv = kv;
    r->ni = 3ll * kf;
    r->launches = 2ll * rounds + 9;
    *out = r;
    return L3D_OK;
}

int64_t l3d_mesh_launches(const l3d_mesh* m) { return m ? m->launches : -1; }

void l3d_mesh_destroy(l3d_mesh* m) { mesh_free(m); }

int l3d_brick_grid_build(const double origin[3], double voxel, const double extent[3],
                         const float* points, int64_t n, double radius, int32_t dims[3],
                         int32_t* count, int32_t* coords, int32_t* lookup) {
    if (!origin || !extent || !dims || !count) return fail(L3D_EINVAL, "NULL argument");
    if (!(voxel > 0.0)) return fail(L3D_EINVAL, "voxel must be positive");
    if (n < 0 || (n > 0 && !points)) return fail(L3D_EINVAL, "bad point list");
    /* BrickGrid constructor (tsdf-volume.ts:17-29) */
    const double side = voxel * 8.0;
    L3dBrickGrid g;
    long long cells = 1;
    for (int i = 0; i < 3; i++) {
        const double d = std::ceil(extent[i] / side);
        if (!(d < 1e6)) return fail(L3D_EINVAL, "grid too large");
        g.dims[i] = std::max(1, (int)d);
        g.origin[i] = origin[i];
        dims[i] = g.dims[i];
        cells *= g.dims[i];
    }
    g.voxel = voxel;
    if (cells >= (1ll << 31)) return fail(L3D_EINVAL, "grid of %lld bricks too large", cells);
    cudaStream_t s;
    L3D_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream creation");
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } guard{s};
    DevBufs tmp(s);
    uint8_t* marks;
    float* pts;
    uint32_t *flags, *base, *scratch, *total;
    int32_t *dlook, *dcoords;
    L3D_CUDA(tmp.get(&marks, cells), "grid buffers");
    L3D_CUDA(tmp.get(&pts, (size_t)n * 3), "grid buffers");
    L3D_CUDA(tmp.get(&flags, cells), "grid buffers");
    L3D_CUDA(tmp.get(&base, cells), "grid buffers");
    L3D_CUDA(tmp.get(&dlook, cells), "grid buffers");
    L3D_CUDA(tmp.get(&scratch, l3d_scan_scratch(cells) / 4 + 1), "scan scratch");
    L3D_CUDA(tmp.get(&total, 1), "scan total");
    L3D_CUDA(cudaMemsetAsync(marks, 0, cells, s), "clear marks");
    if (n) L3D_CUDA(cudaMemcpyAsync(pts, points, (size_t)n * 12, cudaMemcpyHostToDevice, s), "point upload");
    L3D_CUDA(l3d_launch_grid_mark(pts, n, g, radius, marks, s), "mark");
    L3D_CUDA(l3d_launch_grid_widen(marks, cells, flags, s), "mark");
    L3D_CUDA(l3d_scan_exclusive(flags, base, cells, scratch, total, s), "brick scan");
    uint32_t c = 0;
    int rc = read_u32(total, &c, s);
    if (rc) return rc;
    *count = (int32_t)c;
    L3D_CUDA(tmp.get(&dcoords, (size_t)c * 4), "coords buffer");
    L3D_CUDA(l3d_launch_grid_build(flags, base, cells, g, dlook, dcoords, s), "build");
    if (lookup) L3D_CUDA(cudaMemcpyAsync(lookup, dlook, cells * 4, cudaMemcpyDeviceToHost, s), "read lookup");
    if (coords && c) L3D_CUDA(cudaMemcpyAsync(coords, dcoords, (size_t)c * 16, cudaMemcpyDeviceToHost, s), "read coords");
    L3D_CUDA(cudaStreamSynchronize(s), "synchronize");
    return L3D_OK;
}

}  // extern "C"

/* ------------------------------------------------------------------ image preparation ------ */

namespace {

/* coverage (gray-image.ts:226-239), flattened for the device */
struct HostCover {
    std::vector<int> first, count;
    std::vector<double> weights;
    int kmax = 1;
};

HostCover host_coverage(int source, int target) {
    HostCover c;
    const double scale = (double)source / target;
    std::vector<std::vector<double>> w((size_t)target);
    for (int t = 0; t < target; t++) {
        const double start = t * scale;
        const double end = std::min((double)source, (t + 1) * scale);
        const int first = (int)std::floor(start);
        c.first.push_back(first);
        for (int i = first; i < end; i++)
            w[t].push_back((std::min(end, (double)(i + 1)) - std::max(start, (double)i)) / scale);
        c.count.push_back((int)w[t].size());
        c.kmax = std::max(c.kmax, (int)w[t].size());
    }
    c.weights.assign((size_t)target * c.kmax, 0.0);
    for (int t = 0; t < target; t++)
        for (size_t k = 0; k < w[t].size(); k++) c.weights[(size_t)t * c.kmax + k] = w[t][k];
    return c;
}

int check_sizes(int w, int h, int tw, int th) {
    if (w <= 0 || h <= 0 || tw <= 0 || th <= 0) return fail(L3D_EINVAL, "sizes must be positive");
    if ((long long)w * h >= (1ll << 31) || (long long)tw * th >= (1ll << 31))
        return fail(L3D_EINVAL, "image too large");
    return L3D_OK;
}

/* Coverage tables of both axes on the device, packed in one block: first/count ints of the
 * columns then the rows, then the columns' and the rows' weights (8-byte aligned). */
struct DeviceCover {
    unsigned char* block = nullptr;
    L3dAreaCover cols{}, rows{};
};

/* `s` != NULL: a stream-ordered block from the pool for one call (freed by the caller on `s`);
 * else a plain allocation kept by the cache. */
int make_device_cover(int w, int h, int tw, int th, cudaStream_t s, bool pooled, DeviceCover* out) {
    const HostCover hc = host_coverage(w, tw), hr = host_coverage(h, th);
    const size_t off_w = (((size_t)2 * tw + (size_t)2 * th) * 4 + 7) & ~(size_t)7;
    std::vector<unsigned char> host(off_w + (hc.weights.size() + hr.weights.size()) * 8);
    int* hi = (int*)host.data();
    std::memcpy(hi, hc.first.data(), (size_t)tw * 4);
    std::memcpy(hi + tw, hc.count.data(), (size_t)tw * 4);
    std::memcpy(hi + 2 * tw, hr.first.data(), (size_t)th * 4);
    std::memcpy(hi + 2 * tw + th, hr.count.data(), (size_t)th * 4);
    double* hw = (double*)(host.data() + off_w);
    std::memcpy(hw, hc.weights.data(), hc.weights.size() * 8);
    std::memcpy(hw + hc.weights.size(), hr.weights.data(), hr.weights.size() * 8);
    unsigned char* block;
    cudaError_t e;
    if (pooled) {
        L3D_CUDA(pool_alloc((void**)&block, host.size(), s), "area filter tables");
        if ((e = cudaMemcpyAsync(block, host.data(), host.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess) {
            cudaFreeAsync(block, s);
            return cuda_fail(e, "area filter tables");
        }
    } else {
        L3D_CUDA(cudaMalloc((void**)&block, host.size()), "area filter tables");
        if ((e = cudaMemcpy(block, host.data(), host.size(), cudaMemcpyHostToDevice)) != cudaSuccess) {
            cudaFree(block);
            return cuda_fail(e, "area filter tables");
        }
    }
    const int* di = (const int*)block;
    const double* dw = (const double*)(block + off_w);
    out->block = block;
    out->cols = L3dAreaCover{di, di + tw, dw, hc.kmax};
    out->rows = L3dAreaCover{di + 2 * tw, di + 2 * tw + th, dw + hc.weights.size(), hr.kmax};
    return L3D_OK;
}

/* The tables of the first few (device, source size, target size) combinations stay on their
 * device for later calls (an app resamples every frame of a capture to the same size); other
 * combinations get tables for one call (*temporary set: free the block on `s` after use). */
constexpr size_t kCoverCacheEntries = 32;

int device_cover(int w, int h, int tw, int th, cudaStream_t s, DeviceCover* out, bool* temporary) {
    *temporary = false;
    static std::mutex mu;
    static std::vector<std::pair<std::array<int, 5>, DeviceCover>> cache;
    int dev = 0;
    L3D_CUDA(cudaGetDevice(&dev), "device query");
    const std::array<int, 5> key{dev, w, h, tw, th};
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& e : cache)
        if (e.first == key) {
            *out = e.second;
            return L3D_OK;
        }
    if (cache.size() >= kCoverCacheEntries) {
        *temporary = true;
        return make_device_cover(w, h, tw, th, s, true, out);
    }
    DeviceCover c;
    int rc = make_device_cover(w, h, tw, th, s, false, &c);
    if (rc) return rc;
    cache.emplace_back(key, c);
    *out = c;
    return L3D_OK;
}

/* resampleArea (gray-image.ts:193-221) of a device source (src_kind as l3d_launch_area), with
 * the coverage tables from the cache and the row-pass buffer from the pool. */
int area_resample(const void* src, int src_kind, int w, int h, int tw, int th, uint8_t* out,
                  cudaStream_t s) {
    DeviceCover c;
    bool temporary = false;
    int rc = device_cover(w, h, tw, th, s, &c, &temporary);
    if (rc) return rc;
    float* temp;
    cudaError_t e = pool_alloc((void**)&temp, (size_t)tw * h * 4, s);
    if (e == cudaSuccess) {
        e = l3d_launch_area(src, src_kind, w, h, tw, th, c.cols, c.rows, temp, out, s);
        cudaFreeAsync(temp, s);
    }
    if (temporary) cudaFreeAsync(c.block, s);
    if (e != cudaSuccess) return cuda_fail(e, "area filter launch");
    return L3D_OK;
}

}  // namespace

extern "C" {

int l3d_image_rgba_to_gray(const uint8_t* rgba, int32_t width, int32_t height, int32_t target_width,
                           int32_t target_height, uint8_t* gray, void* stream) {
    if (!rgba || !gray) return fail(L3D_EINVAL, "NULL image");
    int rc = check_sizes(width, height, target_width, target_height);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (width % target_width == 0 && height % target_height == 0) {
        L3D_CUDA(l3d_launch_gray_blocks(rgba, width, height, target_width, target_height, gray, s), "gray launch");
        return L3D_OK;
    }
    /* the area filter reads the RGBA pixels and forms their f32 luma itself */
    return area_resample(rgba, 2, width, height, target_width, target_height, gray, s);
}

int l3d_image_downsample_rgb(const uint8_t* rgba, int32_t width, int32_t height, int32_t target_width,
                             int32_t target_height, uint8_t* rgb, void* stream) {
    if (!rgba || !rgb) return fail(L3D_EINVAL, "NULL image");
    int rc = check_sizes(width, height, target_width, target_height);
    if (rc) return rc;
    L3D_CUDA(l3d_launch_rgb_blocks(rgba, width, height, target_width, target_height, rgb, (cudaStream_t)stream),
             "rgb launch");
    return L3D_OK;
}

int l3d_image_downsample_gray(const uint8_t* gray, int32_t width, int32_t height, int32_t target_width,
                              int32_t target_height, uint8_t* out, void* stream) {
    if (!gray || !out) return fail(L3D_EINVAL, "NULL image");
    int rc = check_sizes(width, height, target_width, target_height);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (width % target_width == 0 && height % target_height == 0) {
        L3D_CUDA(l3d_launch_gray_down_blocks(gray, width, height, target_width, target_height, out, s),
                 "gray launch");
        return L3D_OK;
    }
    return area_resample(gray, 0, width, height, target_width, target_height, out, s);
}

int l3d_depth_upsample(const float* grid, int32_t grid_width, int32_t grid_height, int32_t width,
                       int32_t height, float* out, void* stream) {
    if (!grid || !out) return fail(L3D_EINVAL, "NULL buffer");
    int rc = check_sizes(grid_width, grid_height, width, height);
    if (rc) return rc;
    L3D_CUDA(l3d_launch_upsample_depth(grid, grid_width, grid_height, width, height, out,
                                       (cudaStream_t)stream), "upsample launch");
    return L3D_OK;
}

/* ------------------------------------------------------------------ texture-rate probe ----- */

int l3d_measure_texture_rate(int32_t dtype, int32_t checker, double* samples_per_second) {
    return l3d_measure_fetch_rate(dtype, checker, L3D_FETCH_FILTERED, samples_per_second);
}

int l3d_measure_fetch_rate(int32_t dtype, int32_t checker, int32_t mode, double* samples_per_second) {
    if (!samples_per_second) return fail(L3D_EINVAL, "NULL output");
    if (dtype != L3D_DTYPE_U8 && dtype != L3D_DTYPE_F16 && dtype != L3D_DTYPE_F32)
        return fail(L3D_EINVAL, "texture-rate probe: dtype must be u8, f16 or f32");
    if (mode < L3D_FETCH_FILTERED || mode > L3D_FETCH_LOADS)
        return fail(L3D_EINVAL, "texture-rate probe: unknown fetch mode %d", mode);
    if (mode == L3D_FETCH_LOADS && dtype != L3D_DTYPE_F32)
        return fail(L3D_EINVAL, "texture-rate probe: loads from linear memory read F32 images");
    *samples_per_second = 0.0;
    const int W = 2048, H = 2048, reps = 32, launches = 3;
    const long long blocks = l3d_texture_rate_blocks(W, H, checker ? 1 : 0);
    cudaChannelFormatDesc ch = dtype == L3D_DTYPE_F16  ? cudaCreateChannelDescHalf()
                               : dtype == L3D_DTYPE_U8 ? cudaCreateChannelDesc<unsigned char>()
                                                       : cudaCreateChannelDesc<float>();
    const size_t es = dtype_size(dtype);
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    void* fill = nullptr;
    float* out = nullptr;
    cudaError_t e = cudaSuccess;
    const char* what = "";
    auto step = [&](cudaError_t r, const char* w) {
        if (e == cudaSuccess && r != cudaSuccess) {
            e = r;
            what = w;
        }
        return e == cudaSuccess;
    };
    if (step(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream creation") &&
        step(cudaEventCreate(&ev[0]), "event creation") && step(cudaEventCreate(&ev[1]), "event creation") &&
        step(cudaMallocArray(&arr, &ch, W, H, mode == L3D_FETCH_GATHER ? cudaArrayTextureGather : 0),
             "array allocation") &&
        step(cudaMalloc(&fill, (size_t)W * H * es), "fill allocation") &&
        step(cudaMalloc((void**)&out, (size_t)blocks * 128 * sizeof(float)), "output allocation") &&
        step(cudaMemsetAsync(fill, 0x3c, (size_t)W * H * es, st), "fill") &&
        step(cudaMemcpy2DToArrayAsync(arr, 0, 0, fill, (size_t)W * es, (size_t)W * es, H,
                                      cudaMemcpyDeviceToDevice, st), "array fill")) {
        cudaResourceDesc res;
        std::memset(&res, 0, sizeof(res));
        res.resType = cudaResourceTypeArray;
        res.res.array.array = arr;
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = cudaAddressModeClamp;
        td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = mode == L3D_FETCH_FILTERED ? cudaFilterModeLinear : cudaFilterModePoint;
        td.readMode = dtype == L3D_DTYPE_U8 ? cudaReadModeNormalizedFloat : cudaReadModeElementType;
        td.normalizedCoords = 0;
        const float* img = (const float*)fill;
        if (step(cudaCreateTextureObject(&tex, &res, &td, nullptr), "texture creation") &&
            step(l3d_launch_texture_rate(tex, img, W, H, checker ? 1 : 0, mode, reps, out, st), "probe launch") &&
            step(cudaEventRecord(ev[0], st), "event record")) {
            for (int i = 0; i < launches; i++)
                if (!step(l3d_launch_texture_rate(tex, img, W, H, checker ? 1 : 0, mode, reps, out, st),
                          "probe launch"))
                    break;
            float ms = 0.0f;
            if (step(cudaEventRecord(ev[1], st), "event record") &&
                step(cudaEventSynchronize(ev[1]), "probe") &&
                step(cudaEventElapsedTime(&ms, ev[0], ev[1]), "event timing") && ms > 0.0f)
                *samples_per_second = (double)launches * blocks * 128 * reps * 36 / (ms * 1e-3);
        }
    }
    if (st) cudaStreamSynchronize(st);
    if (tex) cudaDestroyTextureObject(tex);
    if (arr) cudaFreeArray(arr);
    cudaFree(fill);
    cudaFree(out);
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    if (st) cudaStreamDestroy(st);
    if (e != cudaSuccess) return cuda_fail(e, what);
    return L3D_OK;
}

int l3d_memory_trim(int64_t keep_bytes) {
    if (keep_bytes < 0) return fail(L3D_EINVAL, "keep_bytes must not be negative");
    int dev = 0;
    L3D_CUDA(cudaGetDevice(&dev), "current device");
    if (dev < 0 || dev >= L3D_POOL_DEVICES) return L3D_OK;
    cudaMemPool_t pool;
    L3D_CUDA(device_pool(dev, false, &pool), "memory pool");
    if (!pool) return L3D_OK;
    /* memory freed in stream order returns to the pool once its stream has passed the free */
    L3D_CUDA(cudaDeviceSynchronize(), "synchronize");
    L3D_CUDA(cudaMemPoolTrimTo(pool, (size_t)keep_bytes), "trim the memory pool");
    return L3D_OK;
}

int l3d_memory_reserved(int64_t* reserved, int64_t* used) {
    if (!reserved || !used) return fail(L3D_EINVAL, "reserved and used must not be NULL");
    *reserved = 0;
    *used = 0;
    int dev = 0;
    L3D_CUDA(cudaGetDevice(&dev), "current device");
    if (dev < 0 || dev >= L3D_POOL_DEVICES) return L3D_OK;
    cudaMemPool_t pool;
    L3D_CUDA(device_pool(dev, false, &pool), "memory pool");
    if (!pool) return L3D_OK;
    uint64_t r = 0, u = 0;
    L3D_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r), "pool reserved bytes");
    L3D_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u), "pool used bytes");
    *reserved = (int64_t)r;
    *used = (int64_t)u;
    return L3D_OK;
}

}  // extern "C"

