/*
 * luvas3d - B200-native dense reconstruction (PatchMatch multi-view stereo + TSDF integration).
 *
 * Plain C ABI of libluvas3d.so.  It replaces the WebGPU plumbing behind the scanner's stereo
 * and fusion stage API; every entry point names the reference interface it stands in for
 * (paths inside the reference project, frontend/src/app/vision/...).
 *
 * Conventions
 *   - Every call returns an int status (L3D_OK = 0).  On failure l3d_last_error() gives a
 *     message for the calling thread.  No C++ exception crosses the ABI.
 *   - Handles are opaque.  A handle owns its device memory and one CUDA stream; calls on one
 *     handle are serialised on that stream and must not be made concurrently from two threads.
 *     Different handles may be used from different threads.
 *   - Host buffers are owned by the caller.  Input buffers in pageable memory may be reused as
 *     soon as the call returns.  Input buffers in pinned (page-locked) memory are copied
 *     asynchronously and must stay unchanged until the next synchronising call on the handle
 *     (any l3d_*_read_*, l3d_*_synchronize or destroy).
 *   - solve/filter/integrate enqueue device work and return without waiting (the reference's
 *     Promises resolve when the GPU finishes; here l3d_*_synchronize or a read waits).
 *   - Poses map world to camera in computer-vision axes (x right, y down, z forward):
 *     x_cam = R X + t, R row-major (frontend/src/app/vision/geometry/camera.ts:19-26).
 *   - There is no CPU fallback: when no CUDA device is usable, create calls fail with
 *     L3D_ECUDA.
 */
#ifndef LUVAS3D_H
#define LUVAS3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Version of the structures and calls below.  2: l3d_stereo_opts gained `compensated` (its size
 * changed, so a host built against version 1 must be rebuilt), L3D_FORM_EXACT, variant bits 16
 * and 32, l3d_tsdf_integrate_layer, l3d_tsdf_count_updates (with the kept count),
 * l3d_measure_fetch_rate, l3d_stereo_read_filtered_all_async, l3d_tsdf_integrate_many_read_async
 * and l3d_tsdf_wait_read. */
#define L3D_ABI_VERSION 2

/* Status codes. */
#define L3D_OK 0
#define L3D_EINVAL 1     /* bad argument: null pointer, shape, index or option */
#define L3D_ECUDA 2      /* CUDA runtime error (message carries the CUDA error string) */
#define L3D_ENOMEM 3     /* device or pinned-host allocation failed */
#define L3D_ESTATE 4     /* not valid in the handle's current state */
#define L3D_ETIMEOUT 5   /* a bounded device-side wait gave up */

/* Element types of host images and device image storage. */
#define L3D_DTYPE_U8 0   /* r8unorm: value / 255 (the reference's texture format) */
#define L3D_DTYPE_F32 1
#define L3D_DTYPE_F16 2
#define L3D_DTYPE_BF16 3

/* Kernel forms. */
#define L3D_FORM_PLAIN 0 /* FP32, one reference view per launch, the oracle's operation order */
#define L3D_FORM_FAST 1  /* mixed precision, batched views: FP16 (or U8, BF16, F32) image storage,
                            hardware bilinear filtering, FP32 window sums of values shifted by the
                            window centre (compensated when opts.compensated is set) */
#define L3D_FORM_EXACT 2 /* batched views with the plain form's arithmetic: F32 storage, texture
                            gathers with exact bilinear weights; equal to the plain form and the
                            FP32 oracle bit for bit (to the oracle's compensated mode when
                            opts.compensated is set) */

/* TSDF weight storage. */
#define L3D_WEIGHT_F32 0 /* f32 weights in [0, max_weight] (the reference's storage) */
#define L3D_WEIGHT_Q8 1  /* uint16 weights in Q8.8 fixed point: weight = value / 256 */

/* Single-kernel dispatch ids for l3d_stereo_dispatch (the units DenseStereo.sliced submits). */
#define L3D_KERNEL_INIT 0
#define L3D_KERNEL_INIT_COARSE 1
#define L3D_KERNEL_PROPAGATE 2
#define L3D_KERNEL_PACK 3
#define L3D_KERNEL_CONSISTENCY 4

typedef struct l3d_stereo l3d_stereo;
typedef struct l3d_tsdf l3d_tsdf;

/* Intrinsics (geometry/camera.ts:12-17). */
typedef struct {
    double fx, fy, cx, cy;
} l3d_intrinsics;

/* Pose, world -> camera (geometry/camera.ts:23-26). */
typedef struct {
    double R[9];
    double t[3];
} l3d_pose;

/* StereoView (mvs/dense-stereo.ts:11-14). */
typedef struct {
    l3d_intrinsics intrinsics;
    l3d_pose pose;
} l3d_view;

/* StereoOptions (mvs/dense-stereo.ts:38-42) plus the device layout choices. */
typedef struct {
    const l3d_stereo* coarse; /* CoarseLevel (dense-stereo.ts:32-36): its planes seed from_coarse
                                 solves; it must outlive this handle.  NULL = none */
    int32_t depth_maps;       /* 1: a packed depth map per view (default); 0: one map */
    int32_t storage;          /* device image storage: F32 (plain form); U8, F16, BF16 or F32 (fast) */
    int32_t form;             /* L3D_FORM_PLAIN, L3D_FORM_FAST or L3D_FORM_EXACT */
    int32_t window;           /* samples per window side: 6 (reference, offsets +-1,3,5) or 11 */
    int32_t dilation;         /* spacing of window samples: 2 (reference) or 1 */
    void* stream;             /* cudaStream_t to run on, or NULL to create one */
    int32_t compensated;      /* fast and exact forms: 1 = compensated FP32 window sums for the
                                 NCC means, variances and covariances (exact form: a Neumaier sum
                                 of every term; fast form: FP32 sums of each 6-sample window row
                                 added with Neumaier compensation); 0 = plain FP32 sums */
} l3d_stereo_opts;

/* SolveOptions (mvs/dense-stereo.ts:16-29). */
typedef struct {
    const int32_t* sources;   /* source layers; the first 8 are used (MAX_SOURCES) */
    int32_t n_sources;
    double min_depth, max_depth;
    const float* prior;       /* host, width * height metres (0 = no prior), or NULL */
    int32_t geometric;        /* ACMM pass: start from the packed map, add reprojection error */
    int32_t iterations;
    int32_t from_coarse;      /* start from the coarse level's planes */
    int32_t pack;             /* store the packed depth map (reference default: 1) */
} l3d_solve_opts;

/* Device pointers of a stereo handle, for zero-copy interop (e.g. DLPack / torch). */
typedef struct {
    void* images;             /* n_views * height * width of the storage type */
    uint32_t* depths;         /* depth_maps ? n_views : 1  maps of width * height */
    float* hyp;               /* width * height * 4: normal xyz, depth */
    float* cost;              /* width * height */
    uint32_t* filtered;       /* width * height */
    uint32_t* filtered_all;   /* n_views * width * height, NULL until l3d_stereo_filter_all */
    float* hyp_all;           /* n_views * width * height * 4, NULL until l3d_stereo_solve_all */
    float* cost_all;          /* n_views * width * height, NULL until l3d_stereo_solve_all */
} l3d_stereo_buffers;

/* Brick-sparse or dense TSDF volume: BrickGrid / TsdfVolume (fusion/tsdf-volume.ts:13-65,
 * 158-188).  tsdf starts at 1 and weight at 0 (tsdf-volume.ts:188). */
typedef struct {
    double origin[3];         /* world position of voxel (0,0,0)'s corner */
    double voxel;             /* voxel edge (m) */
    double truncation;        /* mu (m); the reference uses 4 voxels (tsdf-volume.ts:179) */
    double max_weight;        /* MAX_WEIGHT = 96 (tsdf-volume.ts:7) */
    double prior_weight;      /* PRIOR_WEIGHT = 0.12 (tsdf-volume.ts:8) */
    int32_t dense;            /* 1: dense dims[0] x dims[1] x dims[2], x fastest;
                                 0: brick pool, voxel (brick, x, y, z) at brick*512 + x + 8y + 64z */
    int32_t dims[3];
    const int32_t* coords;    /* brick pool: count * 4 int32 (bx, by, bz, pad) (BrickGrid.build) */
    int32_t count;            /* number of bricks in the pool */
    int32_t weight_type;      /* L3D_WEIGHT_F32 or L3D_WEIGHT_Q8 */
    int32_t width, height;    /* size of the depth maps that will be integrated */
    void* stream;             /* cudaStream_t to run on, or NULL to create one */
} l3d_tsdf_desc;

/* IntegrationView (fusion/tsdf-volume.ts:67-79). */
typedef struct {
    l3d_intrinsics intrinsics;
    l3d_pose pose;
    double max_depth;         /* farthest depth worth integrating (m) */
    const float* prior;       /* host, width * height (0 = none), or NULL */
    double confidence;        /* typical scene depth for confidence weighting, 0 = off */
} l3d_integration_view;

/* ---- errors ---- */

/* Copies the calling thread's last error message into buf (always NUL-terminated); returns the
 * message length.  No reference counterpart: the reference throws JS Errors
 * (pipeline/stages/stage-runner.ts:40-49, gpu/gpu-device.ts:92-100). */
size_t l3d_last_error(char* buf, size_t size);

/* ---- stereo: DenseStereo (mvs/dense-stereo.ts:61-370) ---- */

/* Fills the reference defaults: depth_maps 1, storage F32, form PLAIN, window 6, dilation 2. */
void l3d_stereo_opts_default(l3d_stereo_opts* opts);

/* new DenseStereo(device, width, height, views, options) (dense-stereo.ts:80-172). */
int l3d_stereo_create(int32_t width, int32_t height, int32_t n_views, const l3d_view* views,
                      const l3d_stereo_opts* opts, l3d_stereo** out);

/* A DenseStereo whose views have their own image sizes (sizes: n_views (width, height) pairs).
 * No reference counterpart (the reference keeps one texture array of one size); all calls work
 * per view, buffers are concatenated per view.  Coarse-to-fine levels need equal sizes. */
int l3d_stereo_create_sized(int32_t n_views, const l3d_view* views, const int32_t* sizes,
                            const l3d_stereo_opts* opts, l3d_stereo** out);
/* Image size of one view. */
int l3d_stereo_view_size(const l3d_stereo* s, int32_t layer, int32_t* width, int32_t* height);

/* DenseStereo.setImage(layer, gray) (dense-stereo.ts:175-182).  dtype is the host element type;
 * row_stride_bytes = 0 means tightly packed rows. */
int l3d_stereo_set_image(l3d_stereo* s, int32_t layer, int32_t dtype, const void* pixels,
                         int64_t row_stride_bytes);

/* DenseStereo.solve(ref, options) (dense-stereo.ts:185-239): init (or init_coarse), iterations
 * x red/black propagate, pack. */
int l3d_stereo_solve(l3d_stereo* s, int32_t ref, const l3d_solve_opts* opts);

/* The photometric stage for many reference views at once (reconstructor.ts:88-94 loops
 * StereoRun.solve over layers).  opts[i] belongs to refs[i].  Each view's hypotheses live in
 * hyp_all/cost_all; packed maps land in depths[ref] exactly as a sequence of solve() calls
 * would leave them.  Geometric passes read the maps as they were when the call started
 * (Jacobi order), a documented difference from per-view solve() calls (Gauss-Seidel). */
int l3d_stereo_solve_all(l3d_stereo* s, int32_t n_refs, const int32_t* refs,
                         const l3d_solve_opts* opts);

/* One kernel of the schedule over the whole image of view ref, with the dispatch state of
 * (iteration, phase): the unit DenseStereo.sliced submits (dense-stereo.ts:269-289). */
int l3d_stereo_dispatch(l3d_stereo* s, int32_t kernel, int32_t ref, const l3d_solve_opts* opts,
                        int32_t iteration, int32_t phase);

/* DenseStereo.filter(ref, sources, needed) (dense-stereo.ts:250-263): consistency filter of
 * depths[ref] into the filtered map. */
int l3d_stereo_filter(l3d_stereo* s, int32_t ref, const int32_t* checks, int32_t n_checks,
                      int32_t needed);

/* filter() for many views into filtered_all[layer] (the loop of fusion/tsdf-meshing.ts:72-83
 * and depth-fusion.ts:34).  checks: n_refs * 8 layers, -1 padded; needed: n_refs values. */
int l3d_stereo_filter_all(l3d_stereo* s, int32_t n_refs, const int32_t* refs,
                          const int32_t* checks, const int32_t* needed);

/* Reads (block until the handle's queued work is done). */
/* DenseStereo.filteredMap readback (dense-stereo.ts:301-306) of the filtered map. */
int l3d_stereo_read_filtered(l3d_stereo* s, uint32_t* out);
/* filtered_all[layer]. */
int l3d_stereo_read_filtered_layer(l3d_stereo* s, int32_t layer, uint32_t* out);
/* Every view's filter_all map in one copy queued on the handle's stream, without waiting: the
 * maps concatenated in layer order (each of its view's width * height), the same values as
 * l3d_stereo_read_filtered_layer per layer.  `out` (pinned memory overlaps with other work) holds
 * them after l3d_stereo_synchronize; later work on the handle is ordered after the copy. */
int l3d_stereo_read_filtered_all_async(l3d_stereo* s, uint32_t* out);
/* DenseStereo.depthMap(ref) (dense-stereo.ts:309-312). */
int l3d_stereo_read_depth(l3d_stereo* s, int32_t ref, uint32_t* out);
/* DenseStereo.hypotheses (dense-stereo.ts:242-244) and the cost buffer; hyp4 is
 * width * height * 4 floats (normal xyz, depth).  Either pointer may be NULL. */
int l3d_stereo_read_hyp(l3d_stereo* s, float* hyp4, float* cost);
/* hyp_all/cost_all of one layer after solve_all. */
int l3d_stereo_read_hyp_layer(l3d_stereo* s, int32_t layer, float* hyp4, float* cost);

/* State uploads (no reference counterpart; they restore a saved state, e.g. to run one kernel
 * from a known state, like the session snapshot of pipeline/reconstructor.ts:49-51). */
int l3d_stereo_write_hyp(l3d_stereo* s, const float* hyp4, const float* cost);
int l3d_stereo_write_depth(l3d_stereo* s, int32_t ref, const uint32_t* packed);

/* hypothesis_cost of given planes at every pixel of view ref (patchmatch.wgsl.ts:192-233):
 * planes is width * height * 4 floats (normal, depth); view_costs (NULL or width*height*8)
 * receives the per-source costs. */
int l3d_stereo_plane_cost(l3d_stereo* s, int32_t ref, const l3d_solve_opts* opts,
                          const float* planes, float* cost, float* view_costs);

int l3d_stereo_buffers_get(const l3d_stereo* s, l3d_stereo_buffers* out);
/* The handle's cudaStream_t (as void*). */
int l3d_stereo_stream(const l3d_stereo* s, void** stream);
int l3d_stereo_synchronize(l3d_stereo* s);
/* Device kernels launched by this handle since creation (for launch accounting). */
int64_t l3d_stereo_launches(const l3d_stereo* s);

/* Batched-form kernel variant (no reference counterpart; the reference has one WGSL kernel):
 * window rows sampled by the texture unit (6, 4, 3 or 2; the others use software bilinear
 * on the LSU path) + 8 for the 2x2 quad lane mapping + 16 (fast form, 6 rows) for texture
 * gathers weighted with exact FP32 bilinear weights instead of the hardware filter + 32 (fast
 * form, 6 rows) for the reference window kept in shared memory instead of registers (more
 * resident warps; results unchanged).  All variants compute the same algorithm; fast-form
 * results differ only by the texture unit's 8-bit filter weights on the rows it filters.  The
 * exact form and compensated sums take 6 or 14 (the exact form always gathers and always keeps
 * its window in shared memory). */
int l3d_stereo_set_variant(l3d_stereo* s, int32_t variant);
int32_t l3d_stereo_variant(const l3d_stereo* s);

/* Times every variant of the handle's form on up to three iterations of the given batch (it
 * overwrites that batch's hypotheses) and keeps the fastest, the shared-memory window (32)
 * included; the gather bit (16) stays as set.
 * best_variant / best_ms (either may be NULL) report it.
 * No reference counterpart. */
int l3d_stereo_autotune(l3d_stereo* s, int32_t n_refs, const int32_t* refs,
                        const l3d_solve_opts* opts, int32_t* best_variant, float* best_ms);

/* Fast form: when enabled, l3d_stereo_solve_all captures a batch's launches into a CUDA graph on
 * first use and replays the graph for identical requests (batches with priors are launched
 * directly).  No reference counterpart. */
int l3d_stereo_set_graphs(l3d_stereo* s, int32_t enable);
/* DenseStereo.destroy() (dense-stereo.ts:357-370). */
void l3d_stereo_destroy(l3d_stereo* s);

/* ---- TSDF: TsdfVolume (fusion/tsdf-volume.ts:158-291) ---- */

/* new TsdfVolume(device, grid, layout, depthBuffer, width, height) (tsdf-volume.ts:171-217). */
int l3d_tsdf_create(const l3d_tsdf_desc* desc, l3d_tsdf** out);

/* TsdfVolume.integrate(view) (tsdf-volume.ts:240-268): integrates one packed depth map, either
 * the filtered map of stereo (src != NULL, the buffer shared at tsdf-meshing.ts:71) or a host
 * map (packed, width * height u32).  Brick culling (visibleBricks, tsdf-volume.ts:220-234) runs
 * on the device. */
int l3d_tsdf_integrate(l3d_tsdf* t, const l3d_stereo* src, const uint32_t* packed,
                       const l3d_integration_view* view);

/* TsdfVolume.integrate(view) (tsdf-volume.ts:240-268) of the filter_all map of one layer of
 * src: the reference's one-view-per-pass form on the batched filtered maps. */
int l3d_tsdf_integrate_layer(l3d_tsdf* t, const l3d_stereo* src, int32_t layer,
                             const l3d_integration_view* view);

/* The work of integrating n depth maps (arguments as for l3d_tsdf_integrate_many) without doing
 * it: *visible receives the voxel-views that visibleBricks keeps, *updates the voxel-updates the
 * integration applies (the voxels a view's depth sample updates), and *kept (may be NULL) the
 * voxel-views of the bricks the depth-aware cull keeps as well (a brick entirely behind the
 * truncation band of its view's depths is dropped; the call fails if that cull would drop an
 * update).  12 bytes per update (f32 tsdf and Q8.8 weight read and written) are the algorithmic
 * bytes of the one-view-per-pass form.  Synchronises.  No reference counterpart. */
int l3d_tsdf_count_updates(l3d_tsdf* t, const l3d_stereo* src, const int32_t* layers,
                           const uint32_t* packed, int32_t n, const l3d_integration_view* views,
                           int64_t* visible, int64_t* updates, int64_t* kept);

/* Integrates n depth maps in one sweep over the volume (each voxel read and written once);
 * equal, bit for bit, to n integrate() calls in order.  Maps come from src's filtered_all
 * (src != NULL, layers[i]) or from packed (host, n * width * height).  The sweep visits only the
 * bricks that some view keeps (visibleBricks and a depth-aware cull that drops bricks entirely
 * behind a view's truncation band, which cannot be updated), and writes back only the voxels of
 * the four-voxel groups that some view updated. */
int l3d_tsdf_integrate_many(l3d_tsdf* t, const l3d_stereo* src, const int32_t* layers,
                            const uint32_t* packed, int32_t n, const l3d_integration_view* views);

/* integrate_many followed by read(): the same volume, bit for bit, in the same host buffers
 * (weight is float* or uint16_t* as for l3d_tsdf_read; either may be NULL, not both), with the
 * read-back overlapped with the sweep: the sweep runs over consecutive voxel ranges and each
 * range is copied out while the next is integrated.  Returns when the copies are done.  Host
 * buffers from cudaHostAlloc / cudaHostRegister overlap fully; pageable ones still work. */
int l3d_tsdf_integrate_many_read(l3d_tsdf* t, const l3d_stereo* src, const int32_t* layers,
                                 const uint32_t* packed, int32_t n,
                                 const l3d_integration_view* views, float* tsdf, void* weight);

/* TsdfVolume.read() (tsdf-volume.ts:270-277).  weight is float* (F32) or uint16_t* (Q8).
 * Either pointer may be NULL. */
/* l3d_tsdf_integrate_many_read without waiting for the read-back: it returns once the sweep and
 * the copies are queued (the copies run on a second stream as each part of the sweep is done).
 * The host buffers must stay valid and untouched until l3d_tsdf_wait_read (or
 * l3d_tsdf_synchronize / l3d_tsdf_read / l3d_tsdf_destroy) returns; work queued later on the
 * handle that writes the volume waits for the copies on the device, so the next scan's
 * reset and sweep can be queued at once and the read-back overlaps other work (a stereo
 * solve on another handle).  No reference counterpart. */
int l3d_tsdf_integrate_many_read_async(l3d_tsdf* t, const l3d_stereo* src, const int32_t* layers,
                                       const uint32_t* packed, int32_t n,
                                       const l3d_integration_view* views, float* tsdf, void* weight);
/* Blocks until the handle's asynchronous read-back (if any) is in host memory. */
int l3d_tsdf_wait_read(l3d_tsdf* t);
int l3d_tsdf_read(l3d_tsdf* t, float* tsdf, void* weight);
/* Back to the initial state (tsdf 1, weight 0). */
int l3d_tsdf_reset(l3d_tsdf* t);
/* Voxel count (dense: product of dims; pool: count * 512). */
int64_t l3d_tsdf_voxels(const l3d_tsdf* t);
int l3d_tsdf_device_buffers(const l3d_tsdf* t, float** tsdf, void** weight);
int l3d_tsdf_stream(const l3d_tsdf* t, void** stream);
int l3d_tsdf_synchronize(l3d_tsdf* t);
int64_t l3d_tsdf_launches(const l3d_tsdf* t);
/* TsdfVolume.destroy() (tsdf-volume.ts:279-290). */
void l3d_tsdf_destroy(l3d_tsdf* t);

/* ---- Dense point cloud: PointAccumulator (fusion/point-accumulator.ts:16-147) fed by
 * addDepthMap (fusion/depth-fusion.ts:42-74) ----
 *
 * Points are averaged per cell of a grid in a device hash table: position, normal and colour
 * sums in FP64 (the reference keeps f32 sums), a sample count per cell.  Cells must lie within
 * 2^20 cells of the origin on every axis. */
typedef struct l3d_cloud l3d_cloud;

/* new PointAccumulator(cell) (point-accumulator.ts:23); work runs on `stream` (a cudaStream_t,
 * NULL = a stream of its own). */
int l3d_cloud_create(double cell, void* stream, l3d_cloud** out);
/* addDepthMap (depth-fusion.ts:42-74): every valid sample of a packed depth map becomes a world
 * point (FP64), a world normal and the colour of the nearest thumbnail pixel (thumb_rgb: host,
 * thumb_w * thumb_h * 3 bytes), added to its cell.  Give exactly one of `src` (its last
 * l3d_stereo_filter result stays on the device; width and height are ignored) or `packed`
 * (host, width * height).  `view` is the depth map's camera.  The add is queued on the
 * cloud's stream; an add that leaves the table room returns without waiting for the device, so
 * a sample outside the table's range (more than 2^20 cells from the origin) is reported by the
 * next call that reads the table back (size, coarsen, read, or an add that must grow it). */
int l3d_cloud_add(l3d_cloud* c, const l3d_stereo* src, const uint32_t* packed, int32_t width,
                  int32_t height, const l3d_view* view, const uint8_t* thumb_rgb, int32_t thumb_w,
                  int32_t thumb_h);
/* PointAccumulator.add (:29-56) of n samples, host, 9 doubles each: x y z nx ny nz r g b. */
int l3d_cloud_add_points(l3d_cloud* c, int64_t n, const double* samples);
/* coarsen(factor) (:85-87): the cell grows by `factor`; every cell is re-binned by its mean
 * position and cells that fall together merge. */
int l3d_cloud_coarsen(l3d_cloud* c, double factor);
/* size (:25-27): occupied cells (synchronises). */
int l3d_cloud_size(l3d_cloud* c, int64_t* size);
int l3d_cloud_cell(const l3d_cloud* c, double* cell);
/* cloud(minSupport) (:114-143): the averaged points of the cells with at least min_support
 * samples, ordered by cell (z, then y, then x; the reference's order is its hash-slot order).
 * *count receives the number of points; with every output NULL only the count is computed.
 * Outputs (host, `capacity` points): positions and normals 3 floats, colors 3 bytes, support
 * min(samples, 65535), cells 3 int32 (the integer cell of each point; any may be NULL). */
int l3d_cloud_read(l3d_cloud* c, int32_t min_support, int64_t capacity, int64_t* count,
                   float* positions, float* normals, uint8_t* colors, uint16_t* support,
                   int32_t* cells);
int64_t l3d_cloud_launches(const l3d_cloud* c);
void l3d_cloud_destroy(l3d_cloud* c);

/* ---- Surface extraction: extractSurface (fusion/surface-nets.ts:47-174), computeNormals and
 * removeSmallComponents (fusion/mesh.ts:9-87), BrickGrid (fusion/tsdf-volume.ts:13-65) ----
 *
 * The mesh equals the reference's: vertices in its append order (one per sign-changing cell in
 * brick, voxel order), triangles in (brick, voxel, axis) order, positions computed in FP64 and
 * rounded to f32, normals summed in f32 in face order.  Vector lengths use sqrt(x^2+y^2+z^2)
 * where the reference calls Math.hypot. */
typedef struct l3d_mesh l3d_mesh;

/* SdfBricks (surface-nets.ts:4-12), host arrays: lookup over dims[0]*dims[1]*dims[2] grid
 * cells (pool brick or -1), tsdf and weight of `bricks` pool bricks, voxel b*512 + x + 8y + 64z. */
typedef struct {
    double origin[3];
    double voxel;
    int32_t dims[3];
    const int32_t* lookup;
    const float* tsdf;
    const float* weight;
    int64_t bricks;
} l3d_sdf_bricks;

/* extractSurface(volume, minWeight) of a host volume. */
int l3d_extract_surface(const l3d_sdf_bricks* volume, double min_weight, l3d_mesh** out);
/* extractSurface of a TSDF handle's volume in place (brick pool: the grid spans the pool's
 * brick coordinates; dense grid: bricks in dense brick order, voxels outside dims missing). */
int l3d_tsdf_extract_surface(l3d_tsdf* t, double min_weight, l3d_mesh** out);
int l3d_mesh_counts(const l3d_mesh* m, int64_t* vertices, int64_t* indices);
/* Host copies: positions and normals 3 floats per vertex, indices 3 per triangle (any NULL). */
int l3d_mesh_read(const l3d_mesh* m, float* positions, float* normals, uint32_t* indices);
/* removeSmallComponents (mesh.ts:37-87): a new mesh without the connected components of fewer
 * than max(min_faces, faces * fraction) faces, vertices renumbered in order of first use. */
int l3d_mesh_remove_small_components(const l3d_mesh* m, double fraction, int32_t min_faces,
                                     l3d_mesh** out);
int64_t l3d_mesh_launches(const l3d_mesh* m);
void l3d_mesh_destroy(l3d_mesh* m);
/* new BrickGrid(origin, voxel, extent), mark(point, radius) for n host points (3 floats each),
 * build(): dims, the brick count, coords (4 int32 per brick, grid order) and lookup (one per grid
 * cell); with coords and lookup NULL only dims and count are returned. */
int l3d_brick_grid_build(const double origin[3], double voxel, const double extent[3],
                         const float* points, int64_t n, double radius, int32_t dims[3],
                         int32_t* count, int32_t* coords, int32_t* lookup);

/* ---- Image preparation (device pointers; work on `stream`, a cudaStream_t, NULL = the
 * default stream) ---- */

/* rgbaToGray (image/gray-image.ts:12-46): luma (77 R + 150 G + 29 B) / 256 averaged over the
 * source area of each target pixel (integer ratios: whole blocks, rounded half up; other
 * ratios: exact box filter with partial weights). */
int l3d_image_rgba_to_gray(const uint8_t* rgba, int32_t width, int32_t height, int32_t target_width,
                           int32_t target_height, uint8_t* gray, void* stream);
/* downsampleRgb (gray-image.ts:49-82): packed RGB thumbnail, block means truncated. */
int l3d_image_downsample_rgb(const uint8_t* rgba, int32_t width, int32_t height, int32_t target_width,
                             int32_t target_height, uint8_t* rgb, void* stream);
/* downsampleGray (gray-image.ts:166-187): area average of a gray image. */
int l3d_image_downsample_gray(const uint8_t* gray, int32_t width, int32_t height, int32_t target_width,
                              int32_t target_height, uint8_t* out, void* stream);
/* upsampleDepth (mvs/depth-maps.ts:9-42): bilinear upsampling of a phone depth grid (0 = no
 * data) ignoring empty cells; 0 where less than half of the weight has data. */
int l3d_depth_upsample(const float* grid, int32_t grid_width, int32_t grid_height, int32_t width,
                       int32_t height, float* out, void* stream);

/* ---- Differentiation (no reference counterpart) ----
 *
 * The reference has no gradients: its WGSL kernels only evaluate costs.  These entry points give
 * the adjoints that gradient-based plane and pose polishing after PatchMatch needs.  All
 * pointers are device pointers; work goes on `stream` (a cudaStream_t; NULL = the handle's
 * stream; cudaStreamLegacy for the legacy default stream), ordered after the handle's queued
 * work and before its later work.
 *
 * NCC objective of a reference view: per pixel, the sum over the sources of view_cost
 * (mvs/patchmatch.wgsl.ts:130-159, the bilateral-weighted 1 - NCC over the handle's window,
 * exact bilinear samples of the stored images; 2 for a source the window leaves, 1 for a window
 * without texture).  Parameters:
 *   planes       width * height * 3 f32 of the reference view: z-depth d and normal angles
 *                (a, b), n = (sin a cos b, sin b, -cos a cos b); a plane with d <= 0 or
 *                n . ray >= -1e-3 costs 2 per source.
 *   pose_deltas  n_views * 6 f32 se(3) increments (v, w) or NULL (all zero): view i's world ->
 *                camera map becomes X -> Exp(w) (R_i X + t_i) + v.  The handle's poses stay the
 *                FP64 base; the relative poses are composed in FP64 on the device. */
int l3d_ncc_forward(l3d_stereo* s, int32_t ref, const int32_t* sources, int32_t n_sources,
                    const float* planes, const float* pose_deltas, float* cost, void* stream);
/* Adjoint of l3d_ncc_forward: with grad_cost (width * height, NULL = all ones) the gradient of
 * sum(grad_cost * cost), written per pixel into grad_planes (width * height * 3, may be NULL)
 * and ADDED into grad_deltas (n_views * 6 doubles, may be NULL; zero it before the first
 * reference view of a step).  cost (may be NULL) receives the forward values.  The warped
 * samples are recomputed, not stored. */
int l3d_ncc_backward(l3d_stereo* s, int32_t ref, const int32_t* sources, int32_t n_sources,
                     const float* planes, const float* pose_deltas, const float* grad_cost,
                     float* cost, float* grad_planes, double* grad_deltas, void* stream);

/* TSDF integration of one view with its depths taken from an FP32 map (depth_dev), out of place:
 * (tsdf_in, weight_in) -> (tsdf_out, weight_out), every voxel written (in place when the
 * pointers are equal).  packed_dev (width * height) still gives each pixel's validity, normal and
 * cost; with depth_dev equal to the packed depths the result equals l3d_tsdf_integrate bit for
 * bit.  The handle supplies the grid, weight type and brick mask; its own volume is untouched. */
int l3d_tsdf_forward_depth(l3d_tsdf* t, const l3d_integration_view* view, int32_t width,
                           int32_t height, const uint32_t* packed_dev, const float* depth_dev,
                           const float* prior_dev, const float* tsdf_in, const void* weight_in,
                           float* tsdf_out, void* weight_out, void* stream);
/* Adjoint of l3d_tsdf_forward_depth at (depth_dev, tsdf_in, weight_in): given the gradients with
 * respect to tsdf_out and weight_out (f32 weights; NULL = zero), ADDS the depth gradient into
 * grad_depth (width * height) and writes grad_tsdf_in / grad_weight_in (voxel count, f32); any
 * of the three outputs may be NULL.  Q8.8 weights are integers, so their gradients are zero. */
int l3d_tsdf_backward(l3d_tsdf* t, const l3d_integration_view* view, int32_t width, int32_t height,
                      const uint32_t* packed_dev, const float* depth_dev, const float* prior_dev,
                      const float* tsdf_in, const void* weight_in, const float* grad_tsdf_out,
                      const float* grad_weight_out, float* grad_depth, float* grad_tsdf_in,
                      float* grad_weight_in, void* stream);

/* Measures the bilinear sample rate of this device's texture unit on a 2048 x 2048 texture of
 * `dtype` (L3D_DTYPE_U8, _F16 or _F32) set up like the fast form's images, with a 6 x 6 window
 * dilated by 2 per pixel and the propagate kernel's thread layout; `checker` != 0 samples the
 * pixels of one red/black colour.  No counterpart in the reference: it is the measured peak
 * that the fast propagate kernel, bound by the texture pipe, is quoted against.  Allocates and
 * frees its own buffers and stream; blocks until the probe is done. */
int l3d_measure_texture_rate(int32_t dtype, int32_t checker, double* samples_per_second);

/* Fetch modes of l3d_measure_fetch_rate. */
#define L3D_FETCH_FILTERED 0 /* hardware bilinear filtering (the fast form) */
#define L3D_FETCH_GATHER 1   /* one texture gather of the footprint + exact FP32 weights (the
                                exact form) */
#define L3D_FETCH_POINT 2    /* four point-sampled texture fetches + exact FP32 weights */
#define L3D_FETCH_LOADS 3    /* four loads from linear F32 memory + exact FP32 weights (the plain
                                form's path) */

/* l3d_measure_texture_rate for one of the fetch modes above: bilinear samples per second
 * (L3D_FETCH_LOADS needs dtype F32).  No reference counterpart: the measured rates the batched
 * forms' propagate kernels are quoted against. */
int l3d_measure_fetch_rate(int32_t dtype, int32_t checker, int32_t mode, double* samples_per_second);

/* ---- memory ---- */

/* Scratch buffers, point tables and mesh outputs come from a stream-ordered memory pool of the
 * library's own on each device, which keeps up to 16 GB of freed memory mapped for the next
 * call.  l3d_memory_trim waits for the current device's queued work, then hands the pool's
 * unused memory back to the driver until at most keep_bytes stay reserved (0 releases all of
 * it); memory held by live handles stays.  It replaces what GPUBuffer.destroy() does for the
 * reference at once (fusion/tsdf-volume.ts:279-290, mvs/dense-stereo.ts:357-370): a caller
 * that shares the device with another allocator calls it after destroying handles. */
int l3d_memory_trim(int64_t keep_bytes);

/* The current device pool's reserved bytes (mapped: in use plus freed and kept) and the part
 * in use by live allocations; both 0 before the pool's first allocation.  No counterpart in
 * the reference. */
int l3d_memory_reserved(int64_t* reserved, int64_t* used);

/* Largest volume, in 8^3 bricks, that l3d_tsdf_integrate_noalloc accepts (a dense grid has
 * ceil(X/8) * ceil(Y/8) * ceil(Z/8) bricks; 2^20 covers 768^3). */
#define L3D_NOALLOC_MAX_BRICKS (1 << 20)

/* Integrates one packed depth map into a TSDF volume without allocating any device memory.
 * No counterpart in the reference: it exists for callers that cannot let this library call
 * cudaMalloc, because their device memory is owned by another allocator (a framework's caching
 * allocator, a pool sized once at start-up) or because an allocation's device-wide
 * synchronisation would stall the rest of their pipeline.  The caller owns every buffer: desc
 * describes the volume as for l3d_tsdf_create (desc->coords and desc->stream are ignored),
 * coords_dev holds the brick pool's coordinates on the device (NULL for a dense grid),
 * depth_dev the width * height packed map, prior_dev an optional width * height prior (NULL =
 * none; view->prior is ignored), tsdf_dev and weight_dev the volume (16-byte aligned, tsdf 1 and
 * weight 0 for a fresh volume).  The update equals l3d_tsdf_integrate bit for bit.
 * The per-brick visibility flags live in a static device array of L3D_NOALLOC_MAX_BRICKS bytes
 * that every GPU using the library keeps until exit; larger volumes are rejected with
 * L3D_EINVAL.  The first call on each device looks that array's address up (make it before any
 * stream capture); all calls share the array, so calls whose kernels overlap on the GPU race.
 * Work is enqueued on `stream` (a cudaStream_t, NULL = the default stream). */
int l3d_tsdf_integrate_noalloc(const l3d_tsdf_desc* desc, const int32_t* coords_dev,
                               const uint32_t* depth_dev, const float* prior_dev,
                               const l3d_integration_view* view, float* tsdf_dev,
                               void* weight_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif
