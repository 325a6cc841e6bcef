/*
 * CPU oracle of the dense-reconstruction path (PatchMatch MVS + TSDF integration).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg (and its --impl reference arm) load this library, and only as the checker or as the timed
 * CPU baseline.  The product library (libluvas3d.so) never links or calls it.
 *
 * Parity unpinned: the reference implements these stages only as WGSL compute shaders
 * (frontend/src/app/vision/mvs/patchmatch.wgsl.ts, frontend/src/app/vision/fusion/tsdf-volume.ts)
 * run through WebGPU in Chrome, holds no golden vectors for them and cannot run here.  This file
 * restates that WGSL line by line in C++; the known-answer tests under tests/ pin it.
 */
#ifndef L3D_ORACLE_H
#define L3D_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Per-view camera, 16 doubles: fx fy cx cy | R (row-major, world -> camera) | t. */
#define ORC_VIEW_DOUBLES 16

enum { ORC_INIT = 0, ORC_INIT_COARSE = 1, ORC_PROPAGATE = 2, ORC_PACK = 3, ORC_CONSISTENCY = 4 };

typedef struct {
    int32_t width, height, n_views;
    const double* views;       /* n_views * 16 */
    const float* images;       /* every view's image, concatenated, values in [0, 1] */
    int32_t ref;
    const int32_t* sources;    /* n_sources layer indices (at most 8 are used) */
    int32_t n_sources;
    double min_depth, max_depth;
    const float* prior;        /* width * height or NULL */
    int32_t geometric;         /* flags bit 0 */
    int32_t iterations;
    int32_t win_n;             /* samples per window side (6 = reference) */
    int32_t win_dil;           /* sample spacing (2 = reference) */
    int32_t pack;
    int32_t from_coarse;
    const void* coarse_hyp;    /* coarse_w * coarse_h * 4 (same precision as the solve) */
    int32_t coarse_w, coarse_h;
    int32_t needed;            /* consistency: views that must agree */
    int32_t threads;           /* OpenMP threads, <= 0 for the default */
    const int32_t* sizes;      /* n_views (width, height) pairs, or NULL: every view is
                                  width x height.  Images and depth maps are concatenated per view */
    int32_t compensated;       /* 1: window sums as Neumaier-compensated sums (the arithmetic of
                                  the product's compensated mode); 0: the reference's plain sums */
} orc_stereo_args;

/* Full schedule of DenseStereo.solve (dense-stereo.ts:185-239) for one reference view. */
int orc32_solve(const orc_stereo_args* a, float* hyp, float* cost, uint32_t* depths);
int orc64_solve(const orc_stereo_args* a, double* hyp, double* cost, uint32_t* depths);

/* One kernel over the whole image: init, init_coarse, propagate (one colour), pack or
 * consistency.  `iteration` and `phase` fill the dispatch state; step = 0.5^iteration. */
int orc32_kernel(const orc_stereo_args* a, int32_t kernel, int32_t iteration, int32_t phase,
                 float* hyp, float* cost, uint32_t* depths, uint32_t* filtered);
int orc64_kernel(const orc_stereo_args* a, int32_t kernel, int32_t iteration, int32_t phase,
                 double* hyp, double* cost, uint32_t* depths, uint32_t* filtered);

/* hypothesis_cost of a given plane per pixel (planes: P * 4 = n, d); view_costs gets the
 * per-source view_cost (P * 8, unused slots 0) when not NULL. */
int orc32_plane_cost(const orc_stereo_args* a, const float* planes, float* cost, float* view_costs);
int orc64_plane_cost(const orc_stereo_args* a, const double* planes, double* cost,
                     double* view_costs);

/* TSDF integration of one packed depth map (tsdf-volume.ts:103-154 and 425-473). */
typedef struct {
    double origin[3];
    double voxel;
    double truncation;
    double max_weight;
    double prior_weight;
    int32_t dense;             /* 1: dense grid dims[0..2]; 0: brick pool with coords */
    int32_t dims[3];
    const int32_t* coords;     /* brick pool: count * 4 (x, y, z, pad) */
    int32_t count;
    int32_t weight_q8;         /* 1: uint16 weights in Q8.8; 0: f32 weights */
    int32_t width, height;     /* depth map size */
} orc_tsdf_desc;

typedef struct {
    double k[4];
    double R[9];
    double t[3];
    double max_depth;
    double confidence;
    const float* prior;        /* width * height or NULL */
} orc_tsdf_view;

int orc32_tsdf_integrate(const orc_tsdf_desc* d, const orc_tsdf_view* v, const uint32_t* depth,
                         float* tsdf, void* weight, int32_t threads);
int orc64_tsdf_integrate(const orc_tsdf_desc* d, const orc_tsdf_view* v, const uint32_t* depth,
                         double* tsdf, double* weight, int32_t threads);
/* Brick visibility of tsdf-volume.ts:220-234 (FP64); out: count (or dense brick count) bytes. */
int orc_tsdf_visible(const orc_tsdf_desc* d, const orc_tsdf_view* v, uint8_t* out);

/* ---- gradients (grad.cpp): forward-mode dual numbers over FP64 restatements ---- */

/* Summed NCC cost of reference a->ref over a->sources (a->n_sources <= 8) per pixel, for planes
 * (P * 3: z-depth, angles a, b with n = (sin a cos b, sin b, -cos a cos b)) and per-view se(3)
 * increments deltas (n_views * 6: v, w; NULL = zero): cost (P, may be NULL) and the gradient of
 * sum(weights * cost) (weights P, NULL = ones) per pixel in grad_planes (P * 3, may be NULL) and
 * for the poses ADDED into grad_deltas (n_views * 6, may be NULL).  Computed with the cost only
 * (grad_planes NULL): margin (P, may be NULL) receives each pixel's smallest distance in texels
 * from a window sample to a source image's border, -1 where a source costs the constant 2 or 1,
 * and cells (P, may be NULL) a hash of the texel cells its samples fall in (the objective is
 * smooth in a parameter as long as the pixel's hash stays the same).
 * Uses a->views, images, sizes, width, height, win_n, win_dil, threads. */
int orc64_ncc_grad(const orc_stereo_args* a, const double* planes, const double* deltas,
                   const double* weights, double* cost, double* grad_planes, double* grad_deltas,
                   double* margin, uint64_t* cells);

/* TSDF integration of one view with the depth of each valid pixel (packed map says valid) taken
 * from depth (width * height), out of place, and its adjoint: tsdf_out / weight_out (may be
 * NULL); with grad_tsdf_out / grad_weight_out (NULL = zero) the gradient ADDED into grad_depth
 * and written into grad_tsdf_in / grad_weight_in (any may be NULL).  Weights are in units
 * (Q8.8 volumes: value / 256). */
int orc64_tsdf_depth(const orc_tsdf_desc* d, const orc_tsdf_view* v, const uint32_t* packed,
                     const double* depth, const double* tsdf_in, const double* weight_in,
                     double* tsdf_out, double* weight_out, const double* grad_tsdf_out,
                     const double* grad_weight_out, double* grad_depth, double* grad_tsdf_in,
                     double* grad_weight_in, int32_t threads);

/* ---- dense point cloud (cloud.cpp): depth-fusion.ts addDepthMap + PointAccumulator ---- */
typedef struct orc_cloud orc_cloud;
orc_cloud* orc_cloud_create(double cell);
void orc_cloud_destroy(orc_cloud* c);
/* PointAccumulator.add of one sample: x y z nx ny nz r g b */
void orc_cloud_add_point(orc_cloud* c, const double* p9);
/* addDepthMap: packed width * height map, view = 16 doubles (fx fy cx cy | R | t), thumbnail
 * rgb (tw * th * 3 bytes) */
void orc_cloud_add_map(orc_cloud* c, const uint32_t* packed, int32_t width, int32_t height,
                       const double* view, const uint8_t* rgb, int32_t tw, int32_t th);
void orc_cloud_coarsen(orc_cloud* c, double factor);
int32_t orc_cloud_size(const orc_cloud* c);
double orc_cloud_cell(const orc_cloud* c);
/* cloud(minSupport) in slot order; returns the point count, fills the outputs (and each point's
 * integer cell, 3 int32) when pos is not NULL */
int32_t orc_cloud_read(const orc_cloud* c, int32_t min_support, float* pos, float* nrm,
                       uint8_t* col, uint16_t* support, int32_t* cells);

/* ---- surface extraction (mesh.cpp) ---- */

/* SdfBricks (surface-nets.ts:4-12): grid of dims bricks, lookup (dims product) -> pool brick or
 * -1, tsdf and weight of `bricks` pool bricks (512 voxels each, b*512 + x + 8y + 64z). */
typedef struct {
    double origin[3];
    double voxel;
    int32_t dims[3];
    const int32_t* lookup;
    const float* tsdf;
    const float* weight;
    int64_t bricks;
} orc_sdf_bricks;

/* extractSurface + computeNormals; counts always, arrays when not NULL. */
int orc_extract_surface(const orc_sdf_bricks* vol, double min_weight, int64_t* n_vertices,
                        int64_t* n_indices, float* positions, float* normals, uint32_t* indices);
/* removeSmallComponents (mesh.ts:37-87) */
int orc_remove_small_components(int64_t nv, int64_t ni, const float* pos, const float* nrm,
                                const uint32_t* idx, double fraction, int32_t min_faces,
                                int64_t* out_nv, int64_t* out_ni, float* out_pos, float* out_nrm,
                                uint32_t* out_idx);
/* BrickGrid (tsdf-volume.ts:13-65) */
void orc_brick_grid_dims(double voxel, const double* extent, int32_t* dims);
void orc_brick_grid_mark(const double* origin, double voxel, const int32_t* dims, uint8_t* marks,
                         const float* points, int64_t n, double radius);
int32_t orc_brick_grid_build(const int32_t* dims, const uint8_t* marks, int32_t* coords,
                             int32_t* lookup);

/* ---- image preparation (image.cpp): gray-image.ts, depth-maps.ts upsampleDepth ---- */
void orc_rgba_to_gray(const uint8_t* rgba, int32_t width, int32_t height, int32_t tw, int32_t th,
                      uint8_t* out);
void orc_downsample_rgb(const uint8_t* rgba, int32_t width, int32_t height, int32_t tw, int32_t th,
                        uint8_t* out);
void orc_downsample_gray(const uint8_t* gray, int32_t width, int32_t height, int32_t tw, int32_t th,
                         uint8_t* out);
void orc_upsample_depth(const float* grid, int32_t gw, int32_t gh, int32_t width, int32_t height,
                        float* out);

/* Packing helpers (depth-packing.wgsl.ts:3-33) and primitives for unit tests. */
uint32_t orc_pack_sample(float depth, float nx, float ny, float nz, float cost);
float orc_unpack_depth(uint32_t packed);
void orc_unpack_normal(uint32_t packed, float* n3);
uint32_t orc_pcg(uint32_t v);
float orc_expf(float x);
void orc_sincosf(float a, float* s, float* c);
uint32_t orc_f32_to_f16(float f);
float orc_f16_to_f32(uint32_t h);
uint32_t orc_seed(int32_t ref, int32_t iteration, int32_t phase, int32_t flags);

#ifdef __cplusplus
}
#endif
#endif
