/*
 * CPU oracle of surface extraction: naive surface nets on a brick TSDF, area-weighted vertex
 * normals, removal of small components, and the brick grid that allocates the volume.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the product library never links or calls it.
 *
 * Restates, in the reference's order and number formats (JavaScript doubles; Float32Array
 * stores round to f32):
 *   frontend/src/app/vision/fusion/surface-nets.ts:47-174   extractSurface
 *   frontend/src/app/vision/fusion/mesh.ts:9-31             computeNormals (f32 normal sums,
 *                                                           faces in order)
 *   frontend/src/app/vision/fusion/mesh.ts:37-87            removeSmallComponents
 *   frontend/src/app/vision/fusion/tsdf-volume.ts:13-65     BrickGrid (dims, mark, build)
 * Vector lengths use sqrt(x^2 + y^2 + z^2) in double where the reference calls Math.hypot.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "oracle.h"

namespace {

constexpr int BRICK = 8;
constexpr int BV = BRICK * BRICK * BRICK;
const int CORNERS[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0},
                           {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
const int EDGES[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                          {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

struct Mesh {
    std::vector<double> pos;      /* the reference's `positions: number[]` */
    std::vector<uint32_t> idx;
    std::vector<float> posf, nrm;
};

double len3(double x, double y, double z) { return std::sqrt(x * x + y * y + z * z); }

/* computeNormals (mesh.ts:9-31) */
void compute_normals(const std::vector<float>& p, const std::vector<uint32_t>& idx,
                     std::vector<float>& n) {
    n.assign(p.size(), 0.0f);
    for (size_t f = 0; f < idx.size(); f += 3) {
        const size_t a = (size_t)idx[f] * 3, b = (size_t)idx[f + 1] * 3, c = (size_t)idx[f + 2] * 3;
        const double e1[3] = {(double)p[b] - p[a], (double)p[b + 1] - p[a + 1], (double)p[b + 2] - p[a + 2]};
        const double e2[3] = {(double)p[c] - p[a], (double)p[c + 1] - p[a + 1], (double)p[c + 2] - p[a + 2]};
        const double nx = e1[1] * e2[2] - e1[2] * e2[1];
        const double ny = e1[2] * e2[0] - e1[0] * e2[2];
        const double nz = e1[0] * e2[1] - e1[1] * e2[0];
        for (size_t v : {a, b, c}) {
            n[v] = (float)((double)n[v] + nx);
            n[v + 1] = (float)((double)n[v + 1] + ny);
            n[v + 2] = (float)((double)n[v + 2] + nz);
        }
    }
    for (size_t v = 0; v < n.size(); v += 3) {
        double length = len3(n[v], n[v + 1], n[v + 2]);
        if (!(length != 0.0)) length = 1.0;
        n[v] = (float)((double)n[v] / length);
        n[v + 1] = (float)((double)n[v + 1] / length);
        n[v + 2] = (float)((double)n[v + 2] / length);
    }
}

/* extractSurface (surface-nets.ts:47-174) */
Mesh extract(const orc_sdf_bricks* vol, double min_weight) {
    const int bx = vol->dims[0], by = vol->dims[1], bz = vol->dims[2];
    const int ext[3] = {bx * BRICK, by * BRICK, bz * BRICK};
    const long long bricks = vol->bricks;
    auto slot = [&](int x, int y, int z) -> long long {
        if (x < 0 || y < 0 || z < 0 || x >= ext[0] || y >= ext[1] || z >= ext[2]) return -1;
        const int brick = vol->lookup[((long long)(z >> 3) * by + (y >> 3)) * bx + (x >> 3)];
        if (brick < 0) return -1;
        return (long long)brick * BV + (x & 7) + ((y & 7) << 3) + ((z & 7) << 6);
    };
    std::vector<int32_t> cell_vertex((size_t)bricks * BV, -1);
    std::vector<int32_t> coord((size_t)bricks * 3, 0);
    const long long nlook = (long long)bx * by * bz;
    for (long long i = 0; i < nlook; i++) {
        const int b = vol->lookup[i];
        if (b < 0) continue;
        coord[(size_t)b * 3] = (int)(i % bx);
        coord[(size_t)b * 3 + 1] = (int)((i / bx) % by);
        coord[(size_t)b * 3 + 2] = (int)(i / ((long long)bx * by));
    }
    double values[8];
    auto sample_cell = [&](int x, int y, int z) -> bool {
        int inside = 0;
        for (int c = 0; c < 8; c++) {
            const long long s = slot(x + CORNERS[c][0], y + CORNERS[c][1], z + CORNERS[c][2]);
            if (s < 0 || (double)vol->weight[s] < min_weight) return false;
            values[c] = vol->tsdf[s];
            if (values[c] < 0) inside++;
        }
        return inside > 0 && inside < 8;
    };
    Mesh m;
    for (long long b = 0; b < bricks; b++) {
        const int x0 = coord[b * 3] * BRICK, y0 = coord[b * 3 + 1] * BRICK, z0 = coord[b * 3 + 2] * BRICK;
        for (int local = 0; local < BV; local++) {
            const int x = x0 + (local & 7), y = y0 + ((local >> 3) & 7), z = z0 + (local >> 6);
            if (!sample_cell(x, y, z)) continue;
            double sx = 0, sy = 0, sz = 0;
            int n = 0;
            for (const auto& e : EDGES) {
                const double va = values[e[0]], vc = values[e[1]];
                if ((va < 0) == (vc < 0)) continue;
                const double t = va / (va - vc);
                sx += CORNERS[e[0]][0] + (CORNERS[e[1]][0] - CORNERS[e[0]][0]) * t;
                sy += CORNERS[e[0]][1] + (CORNERS[e[1]][1] - CORNERS[e[0]][1]) * t;
                sz += CORNERS[e[0]][2] + (CORNERS[e[1]][2] - CORNERS[e[0]][2]) * t;
                n++;
            }
            cell_vertex[b * BV + local] = (int32_t)(m.pos.size() / 3);
            m.pos.push_back(vol->origin[0] + (x + 0.5 + sx / n) * vol->voxel);
            m.pos.push_back(vol->origin[1] + (y + 0.5 + sy / n) * vol->voxel);
            m.pos.push_back(vol->origin[2] + (z + 0.5 + sz / n) * vol->voxel);
        }
    }
    auto vertex_at = [&](int x, int y, int z) -> int32_t {
        const long long s = slot(x, y, z);
        return s < 0 ? -1 : cell_vertex[s];
    };
    auto dist2 = [&](uint32_t a, uint32_t b) {
        const double dx = m.pos[a * 3] - m.pos[b * 3], dy = m.pos[a * 3 + 1] - m.pos[b * 3 + 1];
        const double dz = m.pos[a * 3 + 2] - m.pos[b * 3 + 2];
        return dx * dx + dy * dy + dz * dz;
    };
    const int axes[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (long long b = 0; b < bricks; b++) {
        const int x0 = coord[b * 3] * BRICK, y0 = coord[b * 3 + 1] * BRICK, z0 = coord[b * 3 + 2] * BRICK;
        for (int local = 0; local < BV; local++) {
            const int x = x0 + (local & 7), y = y0 + ((local >> 3) & 7), z = z0 + (local >> 6);
            const long long s0 = b * BV + local;
            if ((double)vol->weight[s0] < min_weight) continue;
            const double v0 = vol->tsdf[s0];
            for (int a = 0; a < 3; a++) {
                const int* ax = axes[a];
                const long long s1 = slot(x + ax[0], y + ax[1], z + ax[2]);
                if (s1 < 0 || (double)vol->weight[s1] < min_weight) continue;
                const double v1 = vol->tsdf[s1];
                if ((v0 < 0) == (v1 < 0)) continue;
                const int* u = axes[(a + 1) % 3];
                const int* w = axes[(a + 2) % 3];
                const int32_t q0 = vertex_at(x - u[0] - w[0], y - u[1] - w[1], z - u[2] - w[2]);
                const int32_t q1 = vertex_at(x - w[0], y - w[1], z - w[2]);
                const int32_t q2 = vertex_at(x, y, z);
                const int32_t q3 = vertex_at(x - u[0], y - u[1], z - u[2]);
                if (q0 < 0 || q1 < 0 || q2 < 0 || q3 < 0) continue;
                uint32_t q[4];
                if (v0 < 0) {
                    q[0] = q0; q[1] = q1; q[2] = q2; q[3] = q3;
                } else {
                    q[0] = q0; q[1] = q3; q[2] = q2; q[3] = q1;
                }
                if (dist2(q[0], q[2]) <= dist2(q[1], q[3])) {
                    for (uint32_t i : {q[0], q[1], q[2], q[0], q[2], q[3]}) m.idx.push_back(i);
                } else {
                    for (uint32_t i : {q[0], q[1], q[3], q[1], q[2], q[3]}) m.idx.push_back(i);
                }
            }
        }
    }
    m.posf.resize(m.pos.size());
    for (size_t i = 0; i < m.pos.size(); i++) m.posf[i] = (float)m.pos[i];
    compute_normals(m.posf, m.idx, m.nrm);
    return m;
}

void copy_out(const std::vector<float>& p, const std::vector<float>& n, const std::vector<uint32_t>& idx,
              int64_t* nv, int64_t* ni, float* pos, float* nrm, uint32_t* ind) {
    *nv = (int64_t)(p.size() / 3);
    *ni = (int64_t)idx.size();
    if (pos) std::memcpy(pos, p.data(), p.size() * 4);
    if (nrm) std::memcpy(nrm, n.data(), n.size() * 4);
    if (ind) std::memcpy(ind, idx.data(), idx.size() * 4);
}

}  // namespace

extern "C" {

int orc_extract_surface(const orc_sdf_bricks* vol, double min_weight, int64_t* n_vertices,
                        int64_t* n_indices, float* positions, float* normals, uint32_t* indices) {
    if (!vol || !n_vertices || !n_indices) return 1;
    Mesh m = extract(vol, min_weight);
    copy_out(m.posf, m.nrm, m.idx, n_vertices, n_indices, positions, normals, indices);
    return 0;
}

/* removeSmallComponents (mesh.ts:37-87) */
int orc_remove_small_components(int64_t nv, int64_t ni, const float* pos, const float* nrm,
                                const uint32_t* idx, double fraction, int32_t min_faces,
                                int64_t* out_nv, int64_t* out_ni, float* out_pos, float* out_nrm,
                                uint32_t* out_idx) {
    std::vector<int32_t> parent((size_t)nv);
    for (int64_t i = 0; i < nv; i++) parent[i] = (int32_t)i;
    auto find = [&](int32_t i) {
        while (parent[i] != i) {
            parent[i] = parent[parent[i]];
            i = parent[i];
        }
        return i;
    };
    for (int64_t f = 0; f < ni; f += 3) {
        const int32_t a = find((int32_t)idx[f]);
        const int32_t b = find((int32_t)idx[f + 1]);
        const int32_t c = find((int32_t)idx[f + 2]);
        parent[b] = a;
        parent[find(c)] = a;
    }
    std::unordered_map<int32_t, int64_t> faces;
    for (int64_t f = 0; f < ni; f += 3) faces[find((int32_t)idx[f])] += 1;
    const double limit = std::max((double)min_faces, (double)(ni / 3) * fraction);
    std::vector<int32_t> remap((size_t)nv, -1);
    std::vector<float> p, n;
    std::vector<uint32_t> kept;
    for (int64_t f = 0; f < ni; f += 3) {
        auto it = faces.find(find((int32_t)idx[f]));
        if ((double)(it == faces.end() ? 0 : it->second) < limit) continue;
        for (int k = 0; k < 3; k++) {
            const uint32_t v = idx[f + k];
            if (remap[v] < 0) {
                remap[v] = (int32_t)(p.size() / 3);
                for (int q = 0; q < 3; q++) {
                    p.push_back(pos[(size_t)v * 3 + q]);
                    n.push_back(nrm[(size_t)v * 3 + q]);
                }
            }
            kept.push_back((uint32_t)remap[v]);
        }
    }
    copy_out(p, n, kept, out_nv, out_ni, out_pos, out_nrm, out_idx);
    return 0;
}

/* BrickGrid constructor (tsdf-volume.ts:17-29) */
void orc_brick_grid_dims(double voxel, const double* extent, int32_t* dims) {
    const double side = voxel * BRICK;
    for (int i = 0; i < 3; i++) dims[i] = std::max(1, (int32_t)std::ceil(extent[i] / side));
}

/* BrickGrid.mark (tsdf-volume.ts:36-51) of n points (3 floats each) */
void orc_brick_grid_mark(const double* origin, double voxel, const int32_t* dims, uint8_t* marks,
                         const float* points, int64_t n, double radius) {
    const double side = voxel * BRICK;
    for (int64_t i = 0; i < n; i++) {
        const double p[3] = {points[i * 3], points[i * 3 + 1], points[i * 3 + 2]};
        int lo[3], hi[3];
        for (int k = 0; k < 3; k++) {
            lo[k] = (int)std::max(0.0, std::floor((p[k] - radius - origin[k]) / side));
            hi[k] = (int)std::min((double)(dims[k] - 1), std::floor((p[k] + radius - origin[k]) / side));
        }
        for (int bz = lo[2]; bz <= hi[2]; bz++)
            for (int by = lo[1]; by <= hi[1]; by++)
                for (int bx = lo[0]; bx <= hi[0]; bx++)
                    marks[((int64_t)bz * dims[1] + by) * dims[0] + bx] = 1;
    }
}

/* BrickGrid.build (tsdf-volume.ts:54-64): returns the brick count; coords (4 per brick) and
 * lookup (one per grid cell) are filled when not NULL. */
int32_t orc_brick_grid_build(const int32_t* dims, const uint8_t* marks, int32_t* coords,
                             int32_t* lookup) {
    const int64_t cells = (int64_t)dims[0] * dims[1] * dims[2];
    int32_t count = 0;
    for (int64_t i = 0; i < cells; i++) {
        if (lookup) lookup[i] = -1;
        if (!marks[i]) continue;
        if (lookup) lookup[i] = count;
        if (coords) {
            coords[count * 4] = (int32_t)(i % dims[0]);
            coords[count * 4 + 1] = (int32_t)((i / dims[0]) % dims[1]);
            coords[count * 4 + 2] = (int32_t)(i / ((int64_t)dims[0] * dims[1]));
            coords[count * 4 + 3] = 0;
        }
        count++;
    }
    return count;
}

}  // extern "C"
