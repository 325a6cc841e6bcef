/*
 * Surface extraction on the device: naive surface nets on the TSDF volume in place, area-weighted
 * vertex normals, removal of small connected components, and the brick grid that allocates a
 * volume around a point cloud.
 *
 * frontend/src/app/vision/fusion/surface-nets.ts:47-174 walks the pool brick by brick, voxel by
 * voxel, appending one vertex per cell whose eight corners are observed and change sign, then
 * one quad per sign-changing voxel edge.  Here each pass is one thread per cell and the
 * reference's append order is reproduced with prefix sums: vertex k of the output is the k-th
 * flagged cell in (brick, local voxel) order, and the triangles come in (brick, voxel, axis)
 * order.  Positions are computed in FP64 and rounded to f32 like the reference's number[] ->
 * Float32Array; the quad diagonal is chosen on the FP64 positions.
 *
 * Normals (mesh.ts:9-31): the reference adds each face's FP64 cross product into f32 vertex
 * sums in face order.  Each vertex gathers its faces (a CSR of vertex -> faces, each list sorted
 * by face index) and sums them in that order, so the f32 sums round exactly as the reference's.
 *
 * Components (mesh.ts:37-87): connected components by min-label hooking with pointer jumping
 * (rounds bounded on the host); the kept faces keep their order and vertices are renumbered in
 * order of first use, as the reference's union-find pass does.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "l3d_internal.h"

namespace {

constexpr int BV = 512;

struct Cell {
    int x, y, z;
};

__device__ __forceinline__ void brick_origin(const L3dSdfView& v, long long b, int* x0, int* y0, int* z0) {
    if (v.dense) {
        *x0 = (int)(b % v.dims[0]) * 8;
        *y0 = (int)((b / v.dims[0]) % v.dims[1]) * 8;
        *z0 = (int)(b / ((long long)v.dims[0] * v.dims[1])) * 8;
    } else {
        *x0 = v.coords[b * 4] * 8;
        *y0 = v.coords[b * 4 + 1] * 8;
        *z0 = v.coords[b * 4 + 2] * 8;
    }
}

/* Storage index of voxel (x, y, z), -1 when it does not exist (the reference's slot()). */
__device__ __forceinline__ long long storage_of(const L3dSdfView& v, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= v.vdims[0] || y >= v.vdims[1] || z >= v.vdims[2]) return -1;
    if (v.dense) return ((long long)z * v.vdims[1] + y) * v.vdims[0] + x;
    const int brick = v.lookup[((long long)(z >> 3) * v.dims[1] + (y >> 3)) * v.dims[0] + (x >> 3)];
    if (brick < 0) return -1;
    return (long long)brick * BV + (x & 7) + ((y & 7) << 3) + ((z & 7) << 6);
}

/* Cell index (brick * 512 + local) of voxel (x, y, z), -1 when it does not exist. */
__device__ __forceinline__ long long cell_of(const L3dSdfView& v, int x, int y, int z) {
    if (!v.dense) return storage_of(v, x, y, z);
    if (x < 0 || y < 0 || z < 0 || x >= v.vdims[0] || y >= v.vdims[1] || z >= v.vdims[2]) return -1;
    const long long b = ((long long)(z >> 3) * v.dims[1] + (y >> 3)) * v.dims[0] + (x >> 3);
    return b * BV + (x & 7) + ((y & 7) << 3) + ((z & 7) << 6);
}

__device__ __forceinline__ double weight_at(const L3dSdfView& v, long long s) {
    if (v.q8) return (double)((float)((const uint16_t*)v.weight)[s] * 0.00390625f);
    return (double)((const float*)v.weight)[s];
}

__device__ __forceinline__ bool cell_xyz(const L3dSdfView& v, long long c, int* x, int* y, int* z) {
    const long long b = c / BV;
    const int local = (int)(c - b * BV);
    int x0, y0, z0;
    brick_origin(v, b, &x0, &y0, &z0);
    *x = x0 + (local & 7);
    *y = y0 + ((local >> 3) & 7);
    *z = z0 + (local >> 6);
    return *x < v.vdims[0] && *y < v.vdims[1] && *z < v.vdims[2];
}

__constant__ int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
__constant__ int kEdge[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                                 {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

/* sampleCell (surface-nets.ts:79-88) */
__device__ bool sample_cell(const L3dSdfView& v, int x, int y, int z, double* values) {
    int inside = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const long long s = storage_of(v, x + kCorner[c][0], y + kCorner[c][1], z + kCorner[c][2]);
        if (s < 0 || weight_at(v, s) < v.min_weight) return false;
        values[c] = (double)v.tsdf[s];
        if (values[c] < 0.0) inside++;
    }
    return inside > 0 && inside < 8;
}

__global__ void k_sn_flag(const L3dSdfView v, long long cells, uint32_t* flag) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    int x, y, z;
    double values[8];
    flag[c] = (cell_xyz(v, c, &x, &y, &z) && sample_cell(v, x, y, z, values)) ? 1u : 0u;
}

/* Pass 1 (surface-nets.ts:90-118): the vertex of each flagged cell. */
__global__ void k_sn_vertex(const L3dSdfView v, long long cells, const uint32_t* flag,
                            const uint32_t* base, int32_t* cell_vertex, double* pos_d, float* pos_f) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    if (!flag[c]) {
        cell_vertex[c] = -1;
        return;
    }
    const uint32_t k = base[c];
    cell_vertex[c] = (int32_t)k;
    int x, y, z;
    cell_xyz(v, c, &x, &y, &z);
    double values[8];
    sample_cell(v, x, y, z, values);
    double sx = 0.0, sy = 0.0, sz = 0.0;
    int n = 0;
#pragma unroll
    for (int e = 0; e < 12; e++) {
        const int a = kEdge[e][0], b = kEdge[e][1];
        const double va = values[a], vc = values[b];
        if ((va < 0.0) == (vc < 0.0)) continue;
        const double t = va / (va - vc);
        sx += kCorner[a][0] + (kCorner[b][0] - kCorner[a][0]) * t;
        sy += kCorner[a][1] + (kCorner[b][1] - kCorner[a][1]) * t;
        sz += kCorner[a][2] + (kCorner[b][2] - kCorner[a][2]) * t;
        n++;
    }
    const double p[3] = {v.origin[0] + (x + 0.5 + sx / n) * v.voxel,
                         v.origin[1] + (y + 0.5 + sy / n) * v.voxel,
                         v.origin[2] + (z + 0.5 + sz / n) * v.voxel};
#pragma unroll
    for (int i = 0; i < 3; i++) {
        pos_d[(size_t)k * 3 + i] = p[i];
        pos_f[(size_t)k * 3 + i] = (float)p[i];
    }
}

__device__ __forceinline__ int32_t vertex_at(const L3dSdfView& v, const int32_t* cell_vertex, int x,
                                             int y, int z) {
    const long long c = cell_of(v, x, y, z);
    return c < 0 ? -1 : cell_vertex[c];
}

__device__ __forceinline__ double dist2(const double* p, uint32_t a, uint32_t b) {
    const double dx = p[(size_t)a * 3] - p[(size_t)b * 3];
    const double dy = p[(size_t)a * 3 + 1] - p[(size_t)b * 3 + 1];
    const double dz = p[(size_t)a * 3 + 2] - p[(size_t)b * 3 + 2];
    return dx * dx + dy * dy + dz * dz;
}

/* Pass 2 (surface-nets.ts:120-165): the quads of one voxel; counts them, or writes their two
 * triangles each at out (6 indices per quad). */
__device__ int voxel_quads(const L3dSdfView& v, long long c, const int32_t* cell_vertex,
                           const double* pos_d, uint32_t* out) {
    int x, y, z;
    if (!cell_xyz(v, c, &x, &y, &z)) return 0;
    const long long s0 = storage_of(v, x, y, z);
    if (weight_at(v, s0) < v.min_weight) return 0;
    const double v0 = (double)v.tsdf[s0];
    int quads = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const int ax = a == 0, ay = a == 1, az = a == 2;
        const long long s1 = storage_of(v, x + ax, y + ay, z + az);
        if (s1 < 0 || weight_at(v, s1) < v.min_weight) continue;
        const double v1 = (double)v.tsdf[s1];
        if ((v0 < 0.0) == (v1 < 0.0)) continue;
        const int b = (a + 1) % 3, d = (a + 2) % 3;
        const int ux = b == 0, uy = b == 1, uz = b == 2;
        const int wx = d == 0, wy = d == 1, wz = d == 2;
        const int32_t q0 = vertex_at(v, cell_vertex, x - ux - wx, y - uy - wy, z - uz - wz);
        const int32_t q1 = vertex_at(v, cell_vertex, x - wx, y - wy, z - wz);
        const int32_t q2 = vertex_at(v, cell_vertex, x, y, z);
        const int32_t q3 = vertex_at(v, cell_vertex, x - ux, y - uy, z - uz);
        if (q0 < 0 || q1 < 0 || q2 < 0 || q3 < 0) continue;
        if (out) {
            uint32_t q[4];
            if (v0 < 0.0) {
                q[0] = q0; q[1] = q1; q[2] = q2; q[3] = q3;
            } else {
                q[0] = q0; q[1] = q3; q[2] = q2; q[3] = q1;
            }
            uint32_t* o = out + (size_t)quads * 6;
            if (dist2(pos_d, q[0], q[2]) <= dist2(pos_d, q[1], q[3])) {
                o[0] = q[0]; o[1] = q[1]; o[2] = q[2]; o[3] = q[0]; o[4] = q[2]; o[5] = q[3];
            } else {
                o[0] = q[0]; o[1] = q[1]; o[2] = q[3]; o[3] = q[1]; o[4] = q[2]; o[5] = q[3];
            }
        }
        quads++;
    }
    return quads;
}

__global__ void k_sn_count(const L3dSdfView v, long long cells, const int32_t* cell_vertex,
                           uint32_t* qcount) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    qcount[c] = (uint32_t)voxel_quads(v, c, cell_vertex, nullptr, nullptr);
}

__global__ void k_sn_emit(const L3dSdfView v, long long cells, const int32_t* cell_vertex,
                          const uint32_t* qcount, const uint32_t* qbase, const double* pos_d,
                          uint32_t* indices) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells || qcount[c] == 0u) return;
    voxel_quads(v, c, cell_vertex, pos_d, indices + (size_t)qbase[c] * 6);
}

/* ---- normals ---- */

__global__ void k_face_normals(const float* p, const uint32_t* idx, long long faces, double* fn,
                               uint32_t* degree) {
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= faces) return;
    const size_t a = (size_t)idx[f * 3] * 3, b = (size_t)idx[f * 3 + 1] * 3, c = (size_t)idx[f * 3 + 2] * 3;
    const double e1[3] = {(double)p[b] - p[a], (double)p[b + 1] - p[a + 1], (double)p[b + 2] - p[a + 2]};
    const double e2[3] = {(double)p[c] - p[a], (double)p[c + 1] - p[a + 1], (double)p[c + 2] - p[a + 2]};
    fn[f * 3] = e1[1] * e2[2] - e1[2] * e2[1];
    fn[f * 3 + 1] = e1[2] * e2[0] - e1[0] * e2[2];
    fn[f * 3 + 2] = e1[0] * e2[1] - e1[1] * e2[0];
#pragma unroll
    for (int k = 0; k < 3; k++) atomicAdd(degree + idx[f * 3 + k], 1u);
}

__global__ void k_face_lists(const uint32_t* idx, long long faces, const uint32_t* start,
                             uint32_t* cursor, uint32_t* lists) {
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= faces) return;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const uint32_t v = idx[f * 3 + k];
        lists[start[v] + atomicAdd(cursor + v, 1u)] = (uint32_t)f;
    }
}

/* computeNormals: each vertex sums its faces in face order into f32, then normalises. */
__global__ void k_vertex_normals(long long vertices, const uint32_t* start, const uint32_t* degree,
                                 uint32_t* lists, const double* fn, float* nrm) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= vertices) return;
    uint32_t* l = lists + start[v];
    const uint32_t n = degree[v];
    for (uint32_t i = 1; i < n; i++) {  /* insertion sort: a handful of faces per vertex */
        const uint32_t key = l[i];
        uint32_t j = i;
        while (j > 0 && l[j - 1] > key) {
            l[j] = l[j - 1];
            j--;
        }
        l[j] = key;
    }
    float s[3] = {0.0f, 0.0f, 0.0f};
    for (uint32_t i = 0; i < n; i++) {
        const double* f = fn + (size_t)l[i] * 3;
#pragma unroll
        for (int k = 0; k < 3; k++) s[k] = (float)((double)s[k] + f[k]);
    }
    double length = sqrt((double)s[0] * s[0] + (double)s[1] * s[1] + (double)s[2] * s[2]);
    if (!(length != 0.0)) length = 1.0;
#pragma unroll
    for (int k = 0; k < 3; k++) nrm[v * 3 + k] = (float)((double)s[k] / length);
}

/* ---- components ---- */

__global__ void k_cc_init(long long vertices, uint32_t* label) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < vertices) label[v] = (uint32_t)v;
}

__device__ __forceinline__ uint32_t root_of(const uint32_t* label, uint32_t v) {
    for (int guard = 0; guard < 64; guard++) {  /* labels are compressed every round */
        const uint32_t p = __ldcg(label + v);
        if (p == v) return v;
        v = p;
    }
    return v;
}

/* Hooks the larger roots of a face's vertices onto the smallest. */
__global__ void k_cc_hook(const uint32_t* idx, long long faces, uint32_t* label, int* changed) {
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= faces) return;
    const uint32_t r0 = root_of(label, idx[f * 3]);
    const uint32_t r1 = root_of(label, idx[f * 3 + 1]);
    const uint32_t r2 = root_of(label, idx[f * 3 + 2]);
    const uint32_t m = min(r0, min(r1, r2));
    if (r0 != m && atomicMin(label + r0, m) > m) *changed = 1;
    if (r1 != m && atomicMin(label + r1, m) > m) *changed = 1;
    if (r2 != m && atomicMin(label + r2, m) > m) *changed = 1;
}

/* Points every vertex on the path from v to its root at the root.  Labels only ever point at
 * smaller indices and roots do not move here, so concurrent compressions agree. */
__global__ void k_cc_compress(long long vertices, uint32_t* label, int* changed) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= vertices) return;
    uint32_t root = __ldcg(label + v);
    for (int guard = 0; guard < 1 << 20; guard++) {
        const uint32_t p = __ldcg(label + root);
        if (p == root) break;
        root = p;
    }
    uint32_t x = (uint32_t)v;
    for (int guard = 0; guard < 1 << 20; guard++) {
        const uint32_t p = __ldcg(label + x);
        if (p == root || x == root) break;
        if (atomicMin(label + x, root) > root) *changed = 1;
        x = p;
    }
}

__global__ void k_cc_count(const uint32_t* idx, long long faces, const uint32_t* label,
                           uint32_t* comp_faces) {
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f < faces) atomicAdd(comp_faces + label[idx[f * 3]], 1u);
}

/* kept[f]; first[v] = first corner position (3f + k) of a kept face that uses v */
__global__ void k_cc_keep(const uint32_t* idx, long long faces, const uint32_t* label,
                          const uint32_t* comp_faces, double limit, uint32_t* kept, uint32_t* first) {
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= faces) return;
    const bool k = (double)comp_faces[label[idx[f * 3]]] >= limit;
    kept[f] = k ? 1u : 0u;
    if (k) {
#pragma unroll
        for (int q = 0; q < 3; q++) atomicMin(first + idx[f * 3 + q], (uint32_t)(f * 3 + q));
    }
}

__global__ void k_cc_first_marks(long long vertices, const uint32_t* first, uint32_t* marks) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < vertices && first[v] != 0xffffffffu) marks[first[v]] = 1u;
}

__global__ void k_cc_emit(const uint32_t* idx, long long faces, const uint32_t* kept,
                          const uint32_t* face_base, const uint32_t* first, const uint32_t* rank,
                          const float* pos, const float* nrm, uint32_t* out_idx, float* out_pos,
                          float* out_nrm) {
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= faces || !kept[f]) return;
    const size_t o = (size_t)face_base[f] * 3;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const uint32_t v = idx[f * 3 + q];
        const uint32_t r = rank[first[v]];
        out_idx[o + q] = r;
        if (first[v] == (uint32_t)(f * 3 + q)) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                out_pos[(size_t)r * 3 + k] = pos[(size_t)v * 3 + k];
                out_nrm[(size_t)r * 3 + k] = nrm[(size_t)v * 3 + k];
            }
        }
    }
}

/* ---- brick grid (tsdf-volume.ts:36-64) ---- */

__global__ void k_grid_mark(const float* pts, long long n, L3dBrickGrid g, double radius, uint8_t* marks) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double side = g.voxel * 8.0;
    int lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double p = (double)pts[i * 3 + k];
        lo[k] = (int)fmax(0.0, floor((p - radius - g.origin[k]) / side));
        hi[k] = (int)fmin((double)(g.dims[k] - 1), floor((p + radius - g.origin[k]) / side));
    }
    for (int bz = lo[2]; bz <= hi[2]; bz++)
        for (int by = lo[1]; by <= hi[1]; by++)
            for (int bx = lo[0]; bx <= hi[0]; bx++)
                marks[((long long)bz * g.dims[1] + by) * g.dims[0] + bx] = 1;
}

__global__ void k_grid_widen(const uint8_t* marks, long long cells, uint32_t* flags) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cells) flags[i] = marks[i] ? 1u : 0u;
}

__global__ void k_grid_build(const uint32_t* flags, const uint32_t* base, long long cells, L3dBrickGrid g,
                             int32_t* lookup, int32_t* coords) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    if (!flags[i]) {
        lookup[i] = -1;
        return;
    }
    const uint32_t b = base[i];
    lookup[i] = (int32_t)b;
    if (coords) {
        coords[(size_t)b * 4] = (int32_t)(i % g.dims[0]);
        coords[(size_t)b * 4 + 1] = (int32_t)((i / g.dims[0]) % g.dims[1]);
        coords[(size_t)b * 4 + 2] = (int32_t)(i / ((long long)g.dims[0] * g.dims[1]));
        coords[(size_t)b * 4 + 3] = 0;
    }
}

inline unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

cudaError_t l3d_launch_sn_flag(const L3dSdfView& v, long long cells, uint32_t* flag, cudaStream_t s) {
    if (cells) k_sn_flag<<<blocks_for(cells), 256, 0, s>>>(v, cells, flag);
    return cudaGetLastError();
}
cudaError_t l3d_launch_sn_vertex(const L3dSdfView& v, long long cells, const uint32_t* flag,
                                 const uint32_t* base, int32_t* cell_vertex, double* pos_d,
                                 float* pos_f, cudaStream_t s) {
    if (cells) k_sn_vertex<<<blocks_for(cells), 256, 0, s>>>(v, cells, flag, base, cell_vertex, pos_d, pos_f);
    return cudaGetLastError();
}
cudaError_t l3d_launch_sn_count(const L3dSdfView& v, long long cells, const int32_t* cell_vertex,
                                uint32_t* qcount, cudaStream_t s) {
    if (cells) k_sn_count<<<blocks_for(cells), 256, 0, s>>>(v, cells, cell_vertex, qcount);
    return cudaGetLastError();
}
cudaError_t l3d_launch_sn_emit(const L3dSdfView& v, long long cells, const int32_t* cell_vertex,
                               const uint32_t* qcount, const uint32_t* qbase, const double* pos_d,
                               uint32_t* indices, cudaStream_t s) {
    if (cells) k_sn_emit<<<blocks_for(cells), 256, 0, s>>>(v, cells, cell_vertex, qcount, qbase, pos_d, indices);
    return cudaGetLastError();
}
cudaError_t l3d_launch_face_normals(const float* pos, const uint32_t* idx, long long faces, double* fn,
                                    uint32_t* degree, cudaStream_t s) {
    if (faces) k_face_normals<<<blocks_for(faces), 256, 0, s>>>(pos, idx, faces, fn, degree);
    return cudaGetLastError();
}
cudaError_t l3d_launch_face_lists(const uint32_t* idx, long long faces, const uint32_t* start,
                                  uint32_t* cursor, uint32_t* lists, cudaStream_t s) {
    if (faces) k_face_lists<<<blocks_for(faces), 256, 0, s>>>(idx, faces, start, cursor, lists);
    return cudaGetLastError();
}
cudaError_t l3d_launch_vertex_normals(long long vertices, const uint32_t* start, const uint32_t* degree,
                                      uint32_t* lists, const double* fn, float* nrm, cudaStream_t s) {
    if (vertices) k_vertex_normals<<<blocks_for(vertices), 256, 0, s>>>(vertices, start, degree, lists, fn, nrm);
    return cudaGetLastError();
}
cudaError_t l3d_launch_cc_init(long long vertices, uint32_t* label, cudaStream_t s) {
    if (vertices) k_cc_init<<<blocks_for(vertices), 256, 0, s>>>(vertices, label);
    return cudaGetLastError();
}
cudaError_t l3d_launch_cc_round(const uint32_t* idx, long long faces, long long vertices, uint32_t* label,
                                int* changed, cudaStream_t s) {
    if (faces) k_cc_hook<<<blocks_for(faces), 256, 0, s>>>(idx, faces, label, changed);
    if (vertices) k_cc_compress<<<blocks_for(vertices), 256, 0, s>>>(vertices, label, changed);
    return cudaGetLastError();
}
cudaError_t l3d_launch_cc_count(const uint32_t* idx, long long faces, const uint32_t* label,
                                uint32_t* comp_faces, cudaStream_t s) {
    if (faces) k_cc_count<<<blocks_for(faces), 256, 0, s>>>(idx, faces, label, comp_faces);
    return cudaGetLastError();
}
cudaError_t l3d_launch_cc_keep(const uint32_t* idx, long long faces, const uint32_t* label,
                               const uint32_t* comp_faces, double limit, uint32_t* kept,
                               uint32_t* first, cudaStream_t s) {
    if (faces) k_cc_keep<<<blocks_for(faces), 256, 0, s>>>(idx, faces, label, comp_faces, limit, kept, first);
    return cudaGetLastError();
}
cudaError_t l3d_launch_cc_first_marks(long long vertices, const uint32_t* first, uint32_t* marks,
                                      cudaStream_t s) {
    if (vertices) k_cc_first_marks<<<blocks_for(vertices), 256, 0, s>>>(vertices, first, marks);
    return cudaGetLastError();
}
cudaError_t l3d_launch_cc_emit(const uint32_t* idx, long long faces, const uint32_t* kept,
                               const uint32_t* face_base, const uint32_t* first, const uint32_t* rank,
                               const float* pos, const float* nrm, uint32_t* out_idx, float* out_pos,
                               float* out_nrm, cudaStream_t s) {
    if (faces)
        k_cc_emit<<<blocks_for(faces), 256, 0, s>>>(idx, faces, kept, face_base, first, rank, pos, nrm,
                                                    out_idx, out_pos, out_nrm);
    return cudaGetLastError();
}
cudaError_t l3d_launch_grid_mark(const float* pts, long long n, const L3dBrickGrid& g, double radius,
                                 uint8_t* marks, cudaStream_t s) {
    if (n) k_grid_mark<<<blocks_for(n), 256, 0, s>>>(pts, n, g, radius, marks);
    return cudaGetLastError();
}
cudaError_t l3d_launch_grid_widen(const uint8_t* marks, long long cells, uint32_t* flags, cudaStream_t s) {
    if (cells) k_grid_widen<<<blocks_for(cells), 256, 0, s>>>(marks, cells, flags);
    return cudaGetLastError();
}
cudaError_t l3d_launch_grid_build(const uint32_t* flags, const uint32_t* base, long long cells,
                                  const L3dBrickGrid& g, int32_t* lookup, int32_t* coords, cudaStream_t s) {
    if (cells) k_grid_build<<<blocks_for(cells), 256, 0, s>>>(flags, base, cells, g, lookup, coords);
    return cudaGetLastError();
}
