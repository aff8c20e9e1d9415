// Internal declarations shared by the CUDA translation units of libhidem_b200.
//
// Device data layout (all arrays in device memory of the context's GPU):
//
//  * particles live in "slot" order: binned by neighbour-grid cell (linear cell
//    colour, PLiB/NeighbourGrid.cpp:25-33) and, inside a cell, by input index —
//    the iteration order of NeighbourGrid::generateIterationList (NeighbourGrid.cpp:163-184).
//    One 64-byte (mixed) or 128-byte (fp64) record per slot carries everything a
//    partner read needs: position, the six per-step increments, radius, rotation.
//    Two record buffers alternate between timesteps (the fused step reads one and
//    writes the other), so forces never make a round trip through HBM.
//  * the contact list and the link ends use a warp-blocked ELL layout: slots
//    32w..32w+31 form block w with width W[w] = max row length in the block;
//    entry k of slot s sits at off[w] + 32*k + (s & 31), so a warp reads entry k of
//    its 32 rows as one coalesced 128-byte line.
//  * link ends ("sides", PLiB/Accel/LinkAccelSide.h) carry the history state CT0..CT5,
//    the per-side state mirror (PLiB/Accel/CombinedAccelSmem.h:245-258), the initial
//    length and the partner slot; a particle's ends are in ascending link index, the
//    order LinkAccelSide::generateLinks sorts them into (LinkAccelSide.h:118-131).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "hidem_b200.h"

namespace hidem {

constexpr int kWarp = 32;
constexpr uint32_t kSideIsB = 0x80000000u;  // partner word: this side is link end B
constexpr uint32_t kSlotMask = 0x7fffffffu;

// Particle record. Field order is the same in both precisions; the mixed record is
// exactly 64 bytes (two 32-byte sectors), the fp64 record 128 bytes.
template <class LP>
struct alignas(16) PRec;

template <>
struct alignas(16) PRec<float> {
    double x, y, z;
    float d[6];  // xDiff yDiff zDiff uDiff vDiff wDiff
    float r;
    float th[3];  // xTheta yTheta zTheta
};
template <>
struct alignas(16) PRec<double> {
    double x, y, z;
    double d[6];
    double r;
    double th[3];
    double pad[3];
};
static_assert(sizeof(PRec<float>) == 64, "mixed particle record must be 64 bytes");
static_assert(sizeof(PRec<double>) == 128, "fp64 particle record must be 128 bytes");

// A regular 2-D map in the reference's Map2d form (PLiB/Geometry/Map2d.h:23-60): lp
// values, x fastest; the grid metrics in float as the Map2d constructor computes them.
struct Map2dView {
    const void *data;
    float xMin, yMin, xMax, yMax, xRes, yRes, invXMaxMin, invYMaxMin;
    int xPoints, yPoints;
};

// A collision mesh with its MeshAccel grid (PLiB/Geometry/MeshAccel.h:15-47,
// PLiB/MeshData.h:21-35): vertices and normals in lp, cell lists, face force sums.
template <class LP>
struct MeshView {
    const LP *vx, *vy, *vz;        // vertex j of triangle t at 3t + j
    const LP *nx, *ny, *nz;        // per triangle
    const int *starts, *sizes, *values;  // the reference's per-cell lists
    const int *qStarts, *qSizes, *qValues;  // the same lists without the triangles that
                                            // no particle of the cell can reach
    LP *fx, *fy, *fz;              // face forces, accumulated
    LP xLower, yLower, zLower, xUpper, yUpper, zUpper;
    LP xInv, yInv, zInv;           // 1 / cell size, as MeshAccel stores them
    LP force, drag;                // meshForce, meshDrag of the sample main
    int xCount, yCount, zCount;
};

// Constants of the default functors and of the sample integrate step, in lp
// precision, computed on the host exactly as the sample main computes them
// (HiDEM/MeshBlock/MainMeshBlock.cpp:106-156).
template <class LP>
struct Consts {
    // HiDEMDefNeighForceFunc
    LP invDt, attractDistance, attractScaleForce, damping, dampingRotation, scaleE;
    // HiDEMDefLinkForceFunc (its own invDt / damping / dampingRotation: a caller's main
    // may construct the two functors with different values)
    LP linkInvDt, linkDamping, linkDampingRotation, E, W2, W4, G;
    // HiDEMDefLinkBreakFunc
    LP bendBreak, maxLoad;
    // integrate (mainInvDt: the sample main's invDt, used by the velocity limit)
    LP mainInvDt, dt, invDt2, dtSqr, invDtSqr, g, lift, rhoIce, rhoWater, waterLevel;
    LP airDrag, waterDrag, bedDrag, bedFriction, bedHeight, bedInteract, bedStiffness, scale;
    LP maxVel, maxRot, breakTime;
    double lower[3], upper[3];
    int bmin[3], bmax[3];
    int useBed, useVel, useBnd, useFixed, useFront;
    // GlacierDem bed / friction maps and external force maps (x, y, z, u, v, w)
    Map2dView bedMap, fricMap, extMap[6];
    int useBedMap, useFricMap, useExtMaps;
    // collision mesh of the MeshConstrainedDem sample
    MeshView<LP> mesh;
    int useMesh;
};

// Grid of the last rebuild (NeighbourGrid members, PLiB/NeighbourGrid.h:25-52).
struct GridInfo {
    double xMin, yMin, zMin, h;
    int X, Y, Z;
    long long total;
    long long off[27];  // NeighbourGrid::dirOffsets (NeighbourGrid.cpp:100-108)
};

// Warp-blocked ELL addressing.
struct Ell {
    const long long *off;  // per block of 32 slots
    __host__ __device__ static inline long long at(const long long *off, int slot, int k) {
        return off[slot >> 5] + (long long)k * kWarp + (slot & 31);
    }
};

// Per-step launch arguments of the fused / split step kernels.
template <class LP>
struct StepArgs {
    const PRec<LP> *in;
    PRec<LP> *out;
    const uint8_t *type;
    const uint32_t *counts;   // (#contacts) | (#link ends << 16) per slot
    const long long *nOff;    // contact-list block offsets
    const int32_t *nbr;       // contact partner slots
    const long long *sOff;    // link-end block offsets
    const uint32_t *sPartner; // partner slot | kSideIsB
    LP *ct[6];                // CT0..CT5 per side
    uint8_t *sState;          // per-side state mirror
    uint8_t *linkState;       // per-link state mirror (input order), kept equal to sState
    const LP *sL0;            // initial length per side
    const int32_t *sLink;     // link index per side
    LP *force;                // [6][n] (split path only)
    int n;
    long long step;           // timestep whose forces are computed
    int breakPending;         // apply the previous step's link update first
    long long breakStep;      // the previous step (break events are tagged with it)
    int reduceDiff;           // fold max(0, new diffs) into diffMax
    unsigned long long *diffMax;  // 3 words (float or double bit patterns)
    int2 *events;             // (link, step) of links that broke
    unsigned long long *eventCount;
    long long eventCap;
    int *errorFlag;
    int maxContacts, maxEnds; // widest rows of this layout
    LP bendBreak, maxLoad;    // HiDEMDefLinkBreakFunc thresholds (per context in a batch)
    // halo send records written by the force pass itself (split path; null: none): the
    // slot's position in the send list or -1, and the packed buffer of 6 lp per position
    const int32_t *sendPos;
    LP *sendBuf;
};

}  // namespace hidem
