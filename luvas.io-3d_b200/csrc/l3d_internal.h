/*
 * Internal types shared by the C-ABI layer and the CUDA kernels of libluvas3d.so.
 */
#ifndef L3D_INTERNAL_H
#define L3D_INTERNAL_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

#include "../../include/luvas3d.h"

#define L3D_MAX_SOURCES 8      /* MAX_SOURCES, mvs/dense-stereo.ts:44 */
#define L3D_FILTER_COST 7u     /* FILTER_COST, mvs/patchmatch.wgsl.ts:43 */

/* One source view of a dispatch: the View block of patchmatch.wgsl.ts:4-10 (k, R rows, t,
 * layer) plus the homography base B = K_s R K_r^-1 and kt = K_s t composed in FP64 on the host
 * and rounded to f32. */
struct L3dSrc {
    float k[4];
    float R[9];
    float t[3];
    float B[9];
    float kt[3];
    int layer;
    int W, H;                  /* source image size */
    long long img_off;         /* element offset of the source image in the image array */
    long long dep_off;         /* element offset of the source's packed depth map */
};

/* The Params block of patchmatch.wgsl.ts:12-26 as DenseStereo.params fills it
 * (dense-stereo.ts:314-355); the band rows are gone (whole-image launches). */
struct L3dParams {
    float k[4];
    float kinv[4];             /* 1/fx, 1/fy, -cx/fx, -cy/fy in f32 */
    int W, H, ref, n;
    float range[4];            /* 1/min depth, 1/max depth, step, geometric weight */
    unsigned iter, phase, seed, flags, needed;
    float ck[4];               /* coarse-level intrinsics */
    int cW, cH;
    long long ref_off;         /* element offset of the reference image */
    long long ref_dep_off;     /* element offset of the reference's packed depth map */
    L3dSrc src[L3D_MAX_SOURCES];
};

/* Per-view constants of the TSDF integrate uniform (tsdf-volume.ts:81-91), in f32, plus the
 * FP64 pose for brick culling. */
struct L3dTsdfView {
    float k[4];
    float R[9];
    float t[3];
    float conf;
    int has_prior;
    int W, H;                  /* this view's depth-map size */
    long long prior_off;       /* element offset of this view's prior in the prior buffer */
    long long tile_off;        /* element offset of this view's depth tiles (depth-aware culling) */
    double kd[4];
    double Rd[9];
    double td[3];
    double max_depth;
};

struct L3dTsdfGrid {
    float origin[3];
    float voxel;
    float mu;
    float prior_weight;
    float max_weight;
    unsigned max_q;            /* rint(max_weight * 256) for Q8.8 weights */
    double origin_d[3];
    double voxel_d;
    double trunc_d;
    int dense;
    int dims[3];
    int nb[3];                 /* bricks per axis (dense) */
    long long bricks;          /* dense: nb product; pool: count */
    int W, H;                  /* depth map size */
};

/* The grid constants of a TSDF descriptor (validated: false with the reason in why) and the
 * constants of an integration view (the pose in f32 for the kernels and FP64 for brick
 * culling), shared by l3d_tsdf_create / l3d_tsdf_integrate and the allocation-free entry point.
 * pool_coords_given: a brick pool's coordinates are supplied (host or device). */
bool l3d_tsdf_grid_of(const l3d_tsdf_desc* d, bool pool_coords_given, L3dTsdfGrid* out, char* why,
                      size_t why_size);
L3dTsdfView l3d_tsdf_view_of(const l3d_integration_view& v);

/* ---- launchers (stereo.cu / stereo_fast.cu / tsdf.cu); each returns cudaGetLastError() ---- */

enum { L3D_K_INIT = 0, L3D_K_INIT_COARSE = 1, L3D_K_PROPAGATE = 2, L3D_K_PACK = 3,
       L3D_K_CONSISTENCY = 4 };

struct L3dStereoDev {
    const float* images;       /* f32 storage (plain form) */
    const void* images_lp;     /* f16/bf16 storage (fast form) */
    float4* hyp;
    float* cost;
    const float* prior;        /* may be NULL */
    uint32_t* depths;
    uint32_t* filtered;
    const float4* coarse;      /* may be NULL */
};

cudaError_t l3d_launch_plain(int kernel, const L3dParams& p, const L3dStereoDev& d, int win,
                             int dil, cudaStream_t stream);

/* ---- fast form: every reference view of a batch in one launch per kernel ---- */

/* One source of one reference view.  Fast evaluator: Bt/ktt are the homography base and K_s t
 * with the texture's half-texel offset folded in (rows 0 and 1 plus 0.5 x row 2), so q.xy / q.z
 * is directly the filtering coordinate.  Exact evaluator: Bt/ktt hold B and kt unshifted (the
 * plain form's values), q.xy / q.z being texel coordinates. */
struct L3dFastSrc {
    float Bt[9];
    float ktt[3];
    float k[4];
    float R[9];
    float t[3];
    int W, H;
    long long img_off;         /* element offset of the source image (linear storage) */
    long long dep_off;         /* element offset of the source's packed depth map */
    unsigned long long tex;    /* cudaTextureObject_t (F16/F32 storage), 0 otherwise */
};

struct L3dFastView {
    float k[4];
    float kinv[4];
    float range[4];            /* 1/min depth, 1/max depth, unused, geometric weight */
    int W, H, ref, n;
    unsigned flags;            /* bit 0: geometric pass */
    int iterations;
    int tiles_x;               /* pixel tiles per row of one colour */
    int tile_start;            /* first tile of this view in the launch */
    long long pix_off;         /* element offset of this view in hyp_all / cost_all / prior_all */
    long long ref_img_off;
    long long ref_dep_off;
    unsigned long long ref_tex;
    int has_prior;
    int pack;                  /* store the packed depth map in the pack launch */
    /* coarse-to-fine start (init_coarse, patchmatch.wgsl.ts:296-333) */
    float ck[4];               /* coarse-level intrinsics */
    int cW, cH;
    long long coarse_off;      /* element offset of this view's planes in L3dFastDev.coarse */
    int has_coarse;
    int pad_;
    L3dFastSrc src[L3D_MAX_SOURCES];
};

struct L3dFastDev {
    const L3dFastView* views;  /* device array */
    const int* tile_start;     /* n_views + 1 prefix sums of tiles per view */
    int n_views;
    int total_tiles;
    const void* images;        /* linear storage (BF16 sampling path) */
    const uint32_t* pairs;     /* pair image (half2 of a texel and its right neighbour) or NULL */
    int storage;               /* L3D_DTYPE_F32/F16 (texture path) or BF16 (loads) */
    float4* hyp;               /* hyp_all */
    float* cost;               /* cost_all */
    const float* prior;        /* prior_all (rows of views with has_prior) */
    uint32_t* depths;
    const float4* coarse;      /* coarse level's planes (views with has_coarse) or NULL */
    int exact;                 /* 1: exact evaluator (FP32 texture gathers, plain arithmetic) */
    int comp;                  /* 1: Neumaier-compensated window sums */
};

/* kernel: L3D_K_INIT or L3D_K_PROPAGATE; iteration/phase select the RNG stream and the
 * refinement step; views with fewer iterations than `iteration + 1` are skipped.  variant:
 * window rows sampled by the texture unit (0..6, the rest from the pair image) + 8 for the 2x2
 * quad lane mapping. */
cudaError_t l3d_launch_fast(int kernel, const L3dFastDev& d, int iteration, int phase,
                            int variant, cudaStream_t stream);
/* pair image of one layer: half2(texel, right neighbour) from the linear storage */
cudaError_t l3d_launch_make_pairs(const void* img, int storage, int W, int H, uint32_t* pairs,
                                  cudaStream_t stream);
/* pack of every view with pack != 0; max_pixels bounds the views' width * height */
cudaError_t l3d_launch_fast_pack(const L3dFastDev& d, long long max_pixels, cudaStream_t stream);
cudaError_t l3d_launch_fast_plane_cost(const L3dFastDev& d, const float4* planes, float* cost,
                                       int variant, cudaStream_t stream);
cudaError_t l3d_launch_plane_cost(const L3dParams& p, const L3dStereoDev& d, const float4* planes,
                                  float* cost, float* view_costs, int win, int dil,
                                  cudaStream_t stream);
cudaError_t l3d_launch_convert(const void* src, int dtype, int64_t row_stride, int W, int H,
                               void* dst, int storage, cudaStream_t stream);

cudaError_t l3d_launch_tsdf_visible(const L3dTsdfGrid& g, const L3dTsdfView* views_dev, int n_views,
                                    const int32_t* coords, uint8_t* mask, cudaStream_t stream);
/* visibility of one view (into mask) followed by its integration: two launches (three with
 * tiles).  normals: the decoded-normal table (l3d_launch_normal_table), or NULL to decode each
 * normal in place; tiles: scratch of l3d_depth_tile_count(v.W, v.H) floats for the depth-aware
 * cull, or NULL for visibleBricks alone; list (with tiles and normals): scratch of 1 + bricks
 * int32 that lists the kept bricks, so that only their quads are launched (same results in
 * every case) */
cudaError_t l3d_launch_tsdf_view(const L3dTsdfGrid& g, const L3dTsdfView& v, const int32_t* coords,
                                 uint8_t* mask, const uint32_t* depth, const float* prior,
                                 const float4* normals, float* tiles, int32_t* list, float* tsdf,
                                 void* weight, int q8, cudaStream_t stream);
/* Depth tiles for the depth-aware brick cull: per view, the largest depth a voxel of that view
 * can be updated from over every L3D_DEPTH_TILE x L3D_DEPTH_TILE pixel tile (decoded f16 depth,
 * or the prior where the map has none), views[i].tile_off elements into `tiles`. */
#define L3D_DEPTH_TILE 8
long long l3d_depth_tile_count(int W, int H);
cudaError_t l3d_launch_depth_tiles(const L3dTsdfView* views_dev, int n_views,
                                   const uint32_t* const* depth_ptrs_dev, const float* priors,
                                   float* tiles, long long max_tiles, cudaStream_t stream);
/* brick mask of n views with the depth-aware cull: visibleBricks and, where `tiles` is given
 * (l3d_launch_depth_tiles first), not provably behind every depth of its footprint by more than
 * the truncation band (such a brick has no voxel that updates) */
cudaError_t l3d_launch_tsdf_visible_depth(const L3dTsdfGrid& g, const L3dTsdfView* views_dev, int n_views,
                                          const int32_t* coords, const float* tiles, uint8_t* super,
                                          uint8_t* mask, cudaStream_t stream);
/* Bytes of the super-brick flags l3d_launch_tsdf_visible_depth uses on a dense grid (0 for a
 * brick pool, which gets no super-brick pass; `super` may then be NULL).  With `super` and
 * `tiles` it first tests blocks of 4^3 bricks per view and skips the bricks of those behind the
 * depths (one launch more). */
long long l3d_tsdf_super_flags(const L3dTsdfGrid& g, int n_views);
/* counts[0] += visible voxel-views, counts[1] += voxel-updates of a many-view integration */
cudaError_t l3d_launch_tsdf_count(const L3dTsdfGrid& g, const L3dTsdfView* views_dev, int n_views,
                                  const int32_t* coords, const uint8_t* mask,
                                  const uint32_t* const* depth_ptrs_dev, const float* priors,
                                  const float4* normals, unsigned long long* counts,
                                  cudaStream_t stream);
/* normals[code] = unpack_normal(code << 16) for the 4096 normal codes */
cudaError_t l3d_launch_normal_table(float4* normals, cudaStream_t stream);
/* The bricks some view keeps (a non-zero mask row), in ascending order: flags (bricks + 1),
 * prefix (bricks + 1: prefix[b] = kept bricks below b, prefix[bricks] = their number), list
 * (bricks), scratch of l3d_scan_scratch(bricks + 1) bytes. */
cudaError_t l3d_launch_tsdf_brick_list(const L3dTsdfGrid& g, int n_views, const uint8_t* mask,
                                      uint32_t* flags, uint32_t* prefix, int32_t* list,
                                      uint32_t* scratch, cudaStream_t stream);
/* The many-view sweep of quads [q_begin, q_end) (whole bricks) over the listed bricks only. */
cudaError_t l3d_launch_tsdf_many_list(const L3dTsdfGrid& g, const L3dTsdfView* views_dev,
                                      int n_views, const int32_t* coords, const uint8_t* mask,
                                      const uint32_t* const* depth_ptrs_dev, const float* priors,
                                      const float4* normals, float* tsdf, void* weight, int q8,
                                      const uint32_t* prefix, const int32_t* list,
                                      long long q_begin, long long q_end, cudaStream_t stream);
cudaError_t l3d_launch_tsdf_many(const L3dTsdfGrid& g, const L3dTsdfView* views_dev, int n_views,
                                 const int32_t* coords, const uint8_t* mask,
                                 const uint32_t* const* depth_ptrs_dev, const float* priors,
                                 const float4* normals, float* tsdf, void* weight, int q8,
                                 cudaStream_t stream);
/* The sweep's work units in launch order (brick-major quads).  They come in layers: a layer is
 * *layer_units units (dense grid: one z-row of bricks; brick pool: one brick) and covers the
 * contiguous voxel-index range of *layer_voxels voxels after the layers before it (the last
 * dense layer may be shorter).  A sweep over units [q_begin, q_end) only (l3d_launch_tsdf_many_
 * range) with whole layers therefore integrates one contiguous voxel range. */
long long l3d_tsdf_sweep_units(const L3dTsdfGrid& g, long long* layer_units, long long* layer_voxels);
cudaError_t l3d_launch_tsdf_many_range(const L3dTsdfGrid& g, const L3dTsdfView* views_dev,
                                       int n_views, const int32_t* coords, const uint8_t* mask,
                                       const uint32_t* const* depth_ptrs_dev, const float* priors,
                                       const float4* normals, float* tsdf, void* weight, int q8,
                                       long long q_begin, long long q_end, cudaStream_t stream);
cudaError_t l3d_launch_tsdf_fill(float* tsdf, void* weight, long long voxels, int q8,
                                 cudaStream_t stream);

/* ---- differentiable NCC (grad.cu) ---- */

/* FP64 base pose and intrinsics of one view, uploaded once per stereo handle. */
struct L3dGradView {
    double k[4];
    double R[9];
    double t[3];
    int W, H;
    long long img_off;         /* element offset of the view's image in the storage */
};

/* One (reference, source) pair, composed on the device from the poses and increments. */
struct L3dGradPair {
    float B[9];
    float kt[3];
    float ks[4];               /* source intrinsics fx, fy, cx, cy */
    int W, H;
    long long img_off;
};

struct L3dGradJob {
    int ref, n;
    int src[L3D_MAX_SOURCES];
};

struct L3dGradDev {
    const void* images;        /* the handle's image storage */
    int storage;               /* L3D_DTYPE_* of the storage */
    int elem;                  /* bytes per texel */
    int window, dilation;      /* 6/2 or 11/1 */
    int W, H;                  /* reference view size */
    long long ref_img_off;
    float kinv[4];             /* 1/fx, 1/fy, -cx/fx, -cy/fy of the reference, f32 */
};

/* Cost per reference pixel (sum over the job's sources) into cost (may be NULL) and, when
 * grad_planes / grad_deltas are given, the gradients: per-pixel (depth, a, b) written into
 * grad_planes, per-view se(3) gradients added into grad_deltas (FP64, 6 per view).  pairs_dev
 * (L3D_MAX_SOURCES entries) and pair_sums (6 * L3D_MAX_SOURCES doubles) are scratch. */
cudaError_t l3d_launch_ncc_grad(const L3dGradDev& d, const L3dGradView* views_dev,
                                const float* deltas, const L3dGradJob& job, L3dGradPair* pairs_dev,
                                double* pair_sums, const float* planes, const float* grad_cost,
                                float* cost, float* grad_planes, double* grad_deltas,
                                cudaStream_t stream);

/* Differentiable TSDF integration of one view with its depth taken from an FP32 map (tsdf.cu):
 * visibility into mask, then either the out-of-place forward (grad_tsdf_out == NULL) or its
 * adjoint.  Two launches. */
cudaError_t l3d_launch_tsdf_depth(const L3dTsdfGrid& g, const L3dTsdfView& v, const int32_t* coords,
                                  uint8_t* mask, const uint32_t* depth, const float* depthf,
                                  const float* prior, const float* tsdf_in, const void* weight_in,
                                  float* tsdf_out, void* weight_out, const float* grad_tsdf_out,
                                  const float* grad_weight_out, float* grad_depth,
                                  float* grad_tsdf_in, float* grad_weight_in, int q8,
                                  cudaStream_t stream);

/* ---- dense point cloud (cloud.cu) ---- */

struct L3dCloudTable {
    unsigned long long* keys;  /* capacity packed cells, ~0 = empty */
    double* sums;              /* capacity x 9: position, normal, colour sums */
    unsigned* counts;          /* capacity */
    int capacity;              /* power of two */
};

/* One view of addDepthMap in FP64: fx fy cx cy, R (world -> camera), t, thumbnail size. */
struct L3dCloudView {
    double k[4];
    double R[9];
    double t[3];
    int tw, th;
};

enum { L3D_CLOUD_ERR_RANGE = 1, L3D_CLOUD_ERR_FULL = 2 };

cudaError_t l3d_launch_cloud_clear(const L3dCloudTable& t, cudaStream_t stream);
cudaError_t l3d_launch_cloud_add_map(const L3dCloudTable& t, double cell, const uint32_t* packed,
                                     int W, int H, const L3dCloudView& v, const uint8_t* rgb,
                                     unsigned* used, int* err, cudaStream_t stream);
cudaError_t l3d_launch_cloud_add_points(const L3dCloudTable& t, double cell, const double* pts,
                                        long long n, unsigned* used, int* err, cudaStream_t stream);
cudaError_t l3d_launch_cloud_rebin(const L3dCloudTable& from, const L3dCloudTable& to, double cell,
                                   unsigned* used, int* err, cudaStream_t stream);
/* cloud read-back: (key, slot) of the slots with at least min_support samples, appended at
 * *count; the pairs sorted by key on the device (n = l3d_cloud_sort_length(total) entries,
 * padded); the points gathered in key order. */
cudaError_t l3d_launch_cloud_emit_keys(const L3dCloudTable& t, unsigned min_support,
                                       unsigned* count, unsigned long long* keys, uint32_t* slots,
                                       cudaStream_t stream);
unsigned l3d_cloud_sort_length(unsigned total);
cudaError_t l3d_launch_cloud_sort(unsigned long long* keys, uint32_t* slots, unsigned total,
                                  unsigned n, long long* launches, cudaStream_t stream);
cudaError_t l3d_launch_cloud_emit_sorted(const L3dCloudTable& t, unsigned total,
                                         const unsigned long long* keys, const uint32_t* slots,
                                         float* pos, float* nrm, uint8_t* col, uint16_t* support,
                                         int32_t* cells, cudaStream_t stream);

/* ---- prefix sums (scan.cu) ---- */

/* Bytes of scratch l3d_scan_exclusive needs for n elements. */
size_t l3d_scan_scratch(long long n);
/* Kernel launches l3d_scan_exclusive makes for n elements (with or without `total`). */
int l3d_scan_launches(long long n, bool total);
/* out[i] = in[0] + ... + in[i-1] (in == out allowed); *total (device, may be NULL) = the sum. */
cudaError_t l3d_scan_exclusive(const uint32_t* in, uint32_t* out, long long n, uint32_t* scratch,
                               uint32_t* total, cudaStream_t stream);

/* ---- surface extraction (mesh.cu) ---- */

/* A TSDF volume as surface extraction reads it: a brick pool (lookup over the grid of dims
 * bricks, coords per pool brick) or a dense grid (bricks in dense brick order). */
struct L3dSdfView {
    const float* tsdf;
    const void* weight;        /* f32, or u16 Q8.8 when q8 */
    const int32_t* lookup;     /* pool: grid cell -> pool brick or -1 */
    const int32_t* coords;     /* pool: 4 int32 per brick */
    int dims[3];               /* grid size in bricks */
    int vdims[3];              /* voxels per axis (dense dims, or dims x 8) */
    int dense;
    int q8;
    double origin[3];
    double voxel;
    double min_weight;
};

struct L3dBrickGrid {
    double origin[3];
    double voxel;
    int dims[3];
};

cudaError_t l3d_launch_sn_flag(const L3dSdfView& v, long long cells, uint32_t* flag, cudaStream_t s);
cudaError_t l3d_launch_sn_vertex(const L3dSdfView& v, long long cells, const uint32_t* flag,
                                 const uint32_t* base, int32_t* cell_vertex, double* pos_d,
                                 float* pos_f, cudaStream_t s);
cudaError_t l3d_launch_sn_count(const L3dSdfView& v, long long cells, const int32_t* cell_vertex,
                                uint32_t* qcount, cudaStream_t s);
cudaError_t l3d_launch_sn_emit(const L3dSdfView& v, long long cells, const int32_t* cell_vertex,
                               const uint32_t* qcount, const uint32_t* qbase, const double* pos_d,
                               uint32_t* indices, cudaStream_t s);
cudaError_t l3d_launch_face_normals(const float* pos, const uint32_t* idx, long long faces, double* fn,
                                    uint32_t* degree, cudaStream_t s);
cudaError_t l3d_launch_face_lists(const uint32_t* idx, long long faces, const uint32_t* start,
                                  uint32_t* cursor, uint32_t* lists, cudaStream_t s);
cudaError_t l3d_launch_vertex_normals(long long vertices, const uint32_t* start, const uint32_t* degree,
                                      uint32_t* lists, const double* fn, float* nrm, cudaStream_t s);
cudaError_t l3d_launch_cc_init(long long vertices, uint32_t* label, cudaStream_t s);
cudaError_t l3d_launch_cc_round(const uint32_t* idx, long long faces, long long vertices, uint32_t* label,
                                int* changed, cudaStream_t s);
cudaError_t l3d_launch_cc_count(const uint32_t* idx, long long faces, const uint32_t* label,
                                uint32_t* comp_faces, cudaStream_t s);
cudaError_t l3d_launch_cc_keep(const uint32_t* idx, long long faces, const uint32_t* label,
                               const uint32_t* comp_faces, double limit, uint32_t* kept,
                               uint32_t* first, cudaStream_t s);
cudaError_t l3d_launch_cc_first_marks(long long vertices, const uint32_t* first, uint32_t* marks,
                                      cudaStream_t s);
cudaError_t l3d_launch_cc_emit(const uint32_t* idx, long long faces, const uint32_t* kept,
                               const uint32_t* face_base, const uint32_t* first, const uint32_t* rank,
                               const float* pos, const float* nrm, uint32_t* out_idx, float* out_pos,
                               float* out_nrm, cudaStream_t s);
cudaError_t l3d_launch_grid_mark(const float* pts, long long n, const L3dBrickGrid& g, double radius,
                                 uint8_t* marks, cudaStream_t s);
cudaError_t l3d_launch_grid_widen(const uint8_t* marks, long long cells, uint32_t* flags, cudaStream_t s);
cudaError_t l3d_launch_grid_build(const uint32_t* flags, const uint32_t* base, long long cells,
                                  const L3dBrickGrid& g, int32_t* lookup, int32_t* coords, cudaStream_t s);

/* ---- image preparation (image.cu) ---- */

/* coverage() of one axis of the area filter: per target pixel the first source pixel and
 * `count` weights (stride kmax). */
struct L3dAreaCover {
    const int* first;
    const int* count;
    const double* weights;
    int kmax;
};

cudaError_t l3d_launch_gray_blocks(const uint8_t* rgba, int W, int H, int tw, int th, uint8_t* out,
                                   cudaStream_t s);
/* src_kind: 0 u8 gray, 1 f32, 2 RGBA (its f32 luma) */
cudaError_t l3d_launch_area(const void* src, int src_kind, int W, int H, int tw, int th,
                            const L3dAreaCover& cols, const L3dAreaCover& rows, float* temp,
                            uint8_t* out, cudaStream_t s);
cudaError_t l3d_launch_rgb_blocks(const uint8_t* rgba, int W, int H, int tw, int th, uint8_t* out,
                                  cudaStream_t s);
cudaError_t l3d_launch_gray_down_blocks(const uint8_t* gray, int W, int H, int tw, int th, uint8_t* out,
                                        cudaStream_t s);
cudaError_t l3d_launch_upsample_depth(const float* grid, int gw, int gh, int W, int H, float* out,
                                      cudaStream_t s);

/* Sets the calling thread's l3d_last_error() message (capi.cu). */
void l3d_set_error(const char* msg);

/* texture-rate probe (probe.cu) */
long long l3d_texture_rate_blocks(int width, int height, int checker);
/* probe launch; mode: 0 hardware bilinear, 1 gather + exact weights, 2 four point fetches,
 * 3 four loads from img (linear F32, width * height) */
cudaError_t l3d_launch_texture_rate(cudaTextureObject_t tex, const float* img, int width, int height,
                                    int checker, int mode, int reps, float* out, cudaStream_t s);

#endif
