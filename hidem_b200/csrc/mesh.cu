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

}  // namespace

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
