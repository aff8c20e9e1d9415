// Collision-mesh grid build: MeshAccel::generateAccel (PLiB/Geometry/MeshAccel.h:57-165)
// on the device. The per-particle query and force live in the integrate step
// (physics.cuh: mesh_closest, integrate_particle).
//
// The reference evaluates, for every cell centre, the squared distance to every triangle
// (triSDF2) and keeps the triangles below 3 cellSize^2 + searchDistance, in ascending
// triangle order: a count pass, an exclusive scan of the counts, a fill pass. Here one
// warp takes one cell and walks the triangles 32 at a time; a ballot keeps the lane
// order, so each cell's list comes out ascending, as the reference's serial loop writes it.
#include "kernels.h"
#include "physics.cuh"

namespace hidem {

namespace {

constexpr int kMeshWarps = 8;

// FILL = false: sizes[cell] = number of triangles of the cell's list;
// FILL = true:  values[starts[cell] + k] = k-th triangle of the list.
template <class LP, bool FILL>
__global__ void __launch_bounds__(kMeshWarps * 32)
k_mesh_cells(MeshView<LP> m, int ntri, LP cellSize, LP maxDist, int *sizes, const int *starts,
             int *values) {
    const int lane = threadIdx.x & 31;
    const long long w = (long long)blockIdx.x * kMeshWarps + (threadIdx.x >> 5);
    const long long cells = (long long)m.xCount * m.yCount * m.zCount;
    if (w >= cells) return;
    const int z = (int)(w % m.zCount);
    const int y = (int)((w / m.zCount) % m.yCount);
    const int x = (int)(w / ((long long)m.zCount * m.yCount));
    // cell centre as MeshAccel.h:116-118 computes it, in lp
    const LP half = (LP)0.5f * cellSize;
    const LP xPos = ((LP)x * cellSize + half) + m.xLower;
    const LP yPos = ((LP)y * cellSize + half) + m.yLower;
    const LP zPos = ((LP)z * cellSize + half) + m.zLower;
    const int cell = mesh_cell(m, xPos, yPos, zPos);
    if (cell < 0) return;
    const V3f p{(float)xPos, (float)yPos, (float)zPos};
    const int start = FILL ? starts[cell] : 0;
    int count = 0;
    for (int base = 0; base < ntri; base += 32) {
        const int i = base + lane;
        bool hit = false;
        if (i < ntri)
            hit = tri_sdf2<LP>(p, mesh_vertex(m, 3 * i), mesh_vertex(m, 3 * i + 1), mesh_vertex(m, 3 * i + 2)) <
                  maxDist;
        const unsigned mask = __ballot_sync(0xffffffffu, hit);
        if (FILL && hit) values[start + count + __popc(mask & ((1u << lane) - 1u))] = i;
        count += __popc(mask);
    }
    if (!FILL && lane == 0) sizes[cell] = count;
}

// Lower bound of the distance between triangle abc and the box [lo, hi]: the largest
// gap between their projections on the box axes and on the triangle's normal (each gap
// is a lower bound of the distance, by separation along that direction).
__device__ double tri_box_gap(double3 a, double3 b, double3 c, double3 lo, double3 hi) {
    double g = 0.0;
    g = fmax(g, fmax(fmin(fmin(a.x, b.x), c.x) - hi.x, lo.x - fmax(fmax(a.x, b.x), c.x)));
    g = fmax(g, fmax(fmin(fmin(a.y, b.y), c.y) - hi.y, lo.y - fmax(fmax(a.y, b.y), c.y)));
    g = fmax(g, fmax(fmin(fmin(a.z, b.z), c.z) - hi.z, lo.z - fmax(fmax(a.z, b.z), c.z)));
    const double ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z;
    const double vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
    double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
    const double nn = sqrt(nx * nx + ny * ny + nz * nz);
    if (nn > 0.0) {
        nx /= nn;
        ny /= nn;
        nz /= nn;
        const double pa = nx * a.x + ny * a.y + nz * a.z, pb = nx * b.x + ny * b.y + nz * b.z;
        const double pc = nx * c.x + ny * c.y + nz * c.z;
        const double tmin = fmin(fmin(pa, pb), pc), tmax = fmax(fmax(pa, pb), pc);
        const double bmin = fmin(nx * lo.x, nx * hi.x) + fmin(ny * lo.y, ny * hi.y) + fmin(nz * lo.z, nz * hi.z);
        const double bmax = fmax(nx * lo.x, nx * hi.x) + fmax(ny * lo.y, ny * hi.y) + fmax(nz * lo.z, nz * hi.z);
        g = fmax(g, fmax(tmin - bmax, bmin - tmax));
    }
    return g;
}

template <class LP>
__device__ __forceinline__ double3 mesh_vertex_d(const MeshView<LP> &m, int i) {
    return make_double3((double)m.vx[i], (double)m.vy[i], (double)m.vz[i]);
}

// The query lists: per cell, the reference's list (ascending) without the triangles whose
// distance from the cell's box (grown by `margin` for the rounding of the cell
// assignment) exceeds `reach`; triangles flagged in `keep` (ill-conditioned in float,
// whose float distance need not follow the geometry) always stay.
template <class LP, bool FILL>
__global__ void __launch_bounds__(kMeshWarps * 32)
k_mesh_prune(MeshView<LP> m, double cellSize, double margin, double reach, const uint8_t *keep,
             int *qSizes, const int *qStarts, int *qValues) {
    const int lane = threadIdx.x & 31;
    const long long w = (long long)blockIdx.x * kMeshWarps + (threadIdx.x >> 5);
    const long long cells = (long long)m.xCount * m.yCount * m.zCount;
    if (w >= cells) return;
    const int z = (int)(w % m.zCount);
    const int y = (int)((w / m.zCount) % m.yCount);
    const int x = (int)(w / ((long long)m.zCount * m.yCount));
    const double3 lo = make_double3((double)m.xLower + x * cellSize - margin, (double)m.yLower + y * cellSize - margin,
                                    (double)m.zLower + z * cellSize - margin);
    const double3 hi = make_double3((double)m.xLower + (x + 1) * cellSize + margin,
                                    (double)m.yLower + (y + 1) * cellSize + margin,
                                    (double)m.zLower + (z + 1) * cellSize + margin);
    const int start = m.starts[w], size = m.sizes[w];
    const int qStart = FILL ? qStarts[w] : 0;
    int count = 0;
    for (int base = 0; base < size; base += 32) {
        const int k = base + lane;
        bool hit = false;
        int tri = 0;
        if (k < size) {
            tri = m.values[start + k];
            hit = keep[tri] || tri_box_gap(mesh_vertex_d(m, 3 * tri), mesh_vertex_d(m, 3 * tri + 1),
                                           mesh_vertex_d(m, 3 * tri + 2), lo, hi) <= reach;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, hit);
        if (FILL && hit) qValues[qStart + count + __popc(mask & ((1u << lane) - 1u))] = tri;
        count += __popc(mask);
    }
    if (!FILL && lane == 0) qSizes[w] = count;
}

}  // namespace

template <class LP>
void launch_mesh_prune(const MeshView<LP> &m, double cellSize, double margin, double reach,
                       const uint8_t *keep, int *qSizes, const int *qStarts, int *qValues, bool fill,
                       cudaStream_t s) {
    const long long cells = (long long)m.xCount * m.yCount * m.zCount;
    const unsigned blocks = (unsigned)((cells + kMeshWarps - 1) / kMeshWarps);
    if (fill)
        k_mesh_prune<LP, true><<<blocks, kMeshWarps * 32, 0, s>>>(m, cellSize, margin, reach, keep, qSizes, qStarts,
                                                                  qValues);
    else
        k_mesh_prune<LP, false><<<blocks, kMeshWarps * 32, 0, s>>>(m, cellSize, margin, reach, keep, qSizes, qStarts,
                                                                   qValues);
}

template void launch_mesh_prune<float>(const MeshView<float> &, double, double, double, const uint8_t *, int *,
                                       const int *, int *, bool, cudaStream_t);
template void launch_mesh_prune<double>(const MeshView<double> &, double, double, double, const uint8_t *, int *,
                                        const int *, int *, bool, cudaStream_t);

template <class LP>
void launch_mesh_cells(const MeshView<LP> &m, int ntri, LP cellSize, LP maxDist, int *sizes,
                       const int *starts, int *values, bool fill, cudaStream_t s) {
    const long long cells = (long long)m.xCount * m.yCount * m.zCount;
    const unsigned blocks = (unsigned)((cells + kMeshWarps - 1) / kMeshWarps);
    if (fill)
        k_mesh_cells<LP, true><<<blocks, kMeshWarps * 32, 0, s>>>(m, ntri, cellSize, maxDist, sizes, starts, values);
    else
        k_mesh_cells<LP, false><<<blocks, kMeshWarps * 32, 0, s>>>(m, ntri, cellSize, maxDist, sizes, starts, values);
}

template void launch_mesh_cells<float>(const MeshView<float> &, int, float, float, int *, const int *, int *,
                                       bool, cudaStream_t);
template void launch_mesh_cells<double>(const MeshView<double> &, int, double, double, int *, const int *,
                                        int *, bool, cudaStream_t);

}  // namespace hidem
