// Per-pair, per-side, per-link and per-particle arithmetic of the default HiDEM
// functors, written for the device. Every expression keeps the reference's operand
// order and association (HiDEM/Common/HiDEMDefaultFunctions.h) and the translation
// units are compiled with -fmad=false and IEEE division / square root, so results
// are bit-identical to the reference's IEEE CPU build for the same inputs.
#pragma once
#include "internal.h"

namespace hidem {

__device__ __forceinline__ float lsqrt(float v) { return sqrtf(v); }
__device__ __forceinline__ double lsqrt(double v) { return sqrt(v); }
__device__ __forceinline__ float labs_(float v) { return fabsf(v); }
__device__ __forceinline__ double labs_(double v) { return fabs(v); }

// Contact / damping between two particles: HiDEMDefNeighForceFunc::operator()
// (HiDEMDefaultFunctions.h:21-87). s = self (xDiff..wDiff), sr its radius, o / orr the
// other. contact_terms returns the six values the functor adds to the forces; adding
// them to F in component order is exactly the functor's update.
template <class LP>
__device__ __forceinline__ void contact_terms(const Consts<LP> &c, LP mask, LP xDist, LP yDist,
                                              LP zDist, const LP *s, LP sr, const LP *o, LP orr,
                                              LP *t) {
    LP xDist2 = xDist * xDist;
    LP yDist2 = yDist * yDist;
    LP zDist2 = zDist * zDist;
    LP particleDistance2 = xDist2 + yDist2 + zDist2;
    LP radSum = sr + orr;
    LP activeDist2 = (radSum + c.attractDistance) * (radSum + c.attractDistance);
    mask = (particleDistance2 >= activeDist2) ? LP(0) : mask;
    LP particleDistance = lsqrt(particleDistance2);
    LP invDist = LP(1) / particleDistance;
    LP xComp = xDist * invDist;
    LP yComp = yDist * invDist;
    LP zComp = zDist * invDist;
    LP Cnst = 0;
    LP dimDist = radSum - particleDistance;
    Cnst = (particleDistance < radSum) ? lsqrt(dimDist * dimDist * dimDist) : Cnst;
    Cnst = (particleDistance >= radSum && particleDistance < radSum + c.attractDistance)
               ? c.attractScaleForce * dimDist
               : Cnst;
    Cnst = Cnst * c.scaleE;
    t[0] = mask * ((-c.damping) * ((s[0] - o[0]) * c.invDt) + (Cnst * xComp));
    t[1] = mask * ((-c.damping) * ((s[1] - o[1]) * c.invDt) + (Cnst * yComp));
    t[2] = mask * ((-c.damping) * ((s[2] - o[2]) * c.invDt) + (Cnst * zComp));
    t[3] = mask * ((-c.dampingRotation) * ((s[3] - o[3]) * c.invDt));
    t[4] = mask * ((-c.dampingRotation) * ((s[4] - o[4]) * c.invDt));
    t[5] = mask * ((-c.dampingRotation) * ((s[5] - o[5]) * c.invDt));
}

// A pair beyond the active distance gets mask 0, and every term the functor adds is then
// 0 times a finite value (the distance is positive there): adding those signed zeros
// leaves each force component's value unchanged (a zero component at most changes its
// sign, which no later operation can observe), so such pairs skip the arithmetic. A NaN
// distance fails the comparison and takes the full path, as in the functor.
template <class LP>
__device__ __forceinline__ void contact_pair(const Consts<LP> &c, LP mask, LP xDist, LP yDist,
                                             LP zDist, const LP *s, LP sr, const LP *o, LP orr,
                                             LP *F) {
    {
        const LP particleDistance2 = xDist * xDist + yDist * yDist + zDist * zDist;
        const LP radSum = sr + orr;
        const LP activeDist2 = (radSum + c.attractDistance) * (radSum + c.attractDistance);
        if (particleDistance2 >= activeDist2) return;
    }
    LP t[6];
    contact_terms<LP>(c, mask, xDist, yDist, zDist, s, sr, o, orr, t);
#pragma unroll
    for (int k = 0; k < 6; ++k) F[k] = F[k] + t[k];
}

// Bonded beam on one link end: HiDEMDefLinkForceFunc::operator()
// (HiDEMDefaultFunctions.h:90-204). CT is this side's history state (in/out). The
// functor adds two values to each force component, first the damping term (dp), later
// the CT term (ct); beam_terms returns both, beam_side applies them in that order.
template <class LP>
__device__ __forceinline__ void beam_terms(const Consts<LP> &c, LP mask, LP xDist, LP yDist,
                                           LP zDist, const LP *s, const LP *o, LP *CT, LP *dp,
                                           LP *ct) {
    dp[0] = (-c.linkDamping * ((s[0] - o[0]) * c.linkInvDt)) * mask;
    dp[1] = (-c.linkDamping * ((s[1] - o[1]) * c.linkInvDt)) * mask;
    dp[2] = (-c.linkDamping * ((s[2] - o[2]) * c.linkInvDt)) * mask;
    dp[3] = (-c.linkDampingRotation * ((s[3] - o[3]) * c.linkInvDt)) * mask;
    dp[4] = (-c.linkDampingRotation * ((s[4] - o[4]) * c.linkInvDt)) * mask;
    dp[5] = (-c.linkDampingRotation * ((s[5] - o[5]) * c.linkInvDt)) * mask;

    LP xDist2 = xDist * xDist;
    LP yDist2 = yDist * yDist;
    if (xDist == LP(0) && yDist == LP(0)) {
        xDist2 = LP(1e-10);
        yDist2 = LP(1e-10);
    }
    LP zDist2 = zDist * zDist;
    LP distSum = xDist2 + yDist2 + zDist2;
    LP invLI = LP(1) / lsqrt(distSum);
    LP invLP = LP(1) / lsqrt(xDist2 + yDist2);
    LP invLILP = invLI * invLP;
    LP LI = invLI * distSum;

    LP T00 = xDist * invLI, T01 = yDist * invLI, T02 = zDist * invLI;
    LP T10 = -yDist * invLP, T11 = xDist * invLP;
    LP T20 = -(zDist * xDist) * invLILP;
    LP T21 = -(zDist * yDist) * invLILP;
    LP T22 = (xDist2 + yDist2) * invLILP;

    LP B0 = T00 * s[0] + T01 * s[1] + T02 * s[2];
    LP B1 = T10 * s[0] + T11 * s[1];
    LP B2 = T20 * s[0] + T21 * s[1] + T22 * s[2];
    LP B4 = T10 * s[3] + T11 * s[4];
    LP B5 = T20 * s[3] + T21 * s[4] + T22 * s[5];
    LP B6 = T00 * o[0] + T01 * o[1] + T02 * o[2];
    LP B7 = T10 * o[0] + T11 * o[1];
    LP B8 = T20 * o[0] + T21 * o[1] + T22 * o[2];
    LP B10 = T10 * o[3] + T11 * o[4];
    LP B11 = T20 * o[3] + T21 * o[4] + T22 * o[5];

    LP L2 = LI * LI;
    LP L3 = LI * LI * LI;
    LP LIDiv6 = (LP(1) / LP(6)) * invLI;
    LP K0 = c.E * c.W2 * invLI;
    LP K1 = c.E * c.W4 / L3;
    LP K5 = c.E * c.W4 / (LP(2) * L2);

    CT[0] = CT[0] + (K0 * B0 + (-K0) * B6);
    CT[1] = CT[1] + (K1 * B1 + K5 * B5 + (-K1) * B7 + K5 * B11);
    CT[2] = CT[2] + (K1 * B2 + (-K5) * B4 + (-K1) * B8 + (-K5) * B10);

    ct[0] = (-(T00 * CT[0] + T10 * CT[1] + T20 * CT[2])) * mask;
    ct[1] = (-(T01 * CT[0] + T11 * CT[1] + T21 * CT[2])) * mask;
    ct[2] = (-(T02 * CT[0] + T22 * CT[2])) * mask;

    LP K2 = c.G * c.W4 * LIDiv6;
    LP K3 = c.E * c.W4 * LIDiv6 * LP(2);
    LP K4 = c.E * c.W4 * LIDiv6;
    LP B3 = T00 * s[3] + T01 * s[4] + T02 * s[5];
    LP B9 = T00 * o[3] + T01 * o[4] + T02 * o[5];

    CT[3] = CT[3] + (K2 * B3 + (-K2) * B9);
    CT[4] = CT[4] + ((-K5) * B2 + K3 * B4 + K5 * B8 + K4 * B10);
    CT[5] = CT[5] + (K5 * B1 + K3 * B5 + (-K5) * B7 + K4 * B11);

    ct[3] = (-(T00 * CT[3] + T10 * CT[4] + T20 * CT[5])) * mask;
    ct[4] = (-(T01 * CT[3] + T11 * CT[4] + T21 * CT[5])) * mask;
    ct[5] = (-(T02 * CT[3] + T22 * CT[5])) * mask;
}

template <class LP>
__device__ __forceinline__ void beam_side(const Consts<LP> &c, LP mask, LP xDist, LP yDist,
                                          LP zDist, const LP *s, const LP *o, LP *CT, LP *F) {
    LP dp[6], ct[6];
    beam_terms<LP>(c, mask, xDist, yDist, zDist, s, o, CT, dp, ct);
#pragma unroll
    for (int k = 0; k < 6; ++k) F[k] = (F[k] + dp[k]) + ct[k];
}

// Link break test: HiDEMDefLinkBreakFunc::operator() (HiDEMDefaultFunctions.h:207-242)
// with end A as particle 1 and end B as particle 2 and the functor's two thresholds.
// Returns the new state.
template <class LP>
__device__ __forceinline__ uint8_t break_link(const LP bendBreak, const LP maxLoad,
                                              const PRec<LP> &a, const PRec<LP> &b,
                                              uint8_t state, LP initialLen) {
    if (state == 0) return 0;
    LP xDist = (LP)(a.x - b.x);
    LP yDist = (LP)(a.y - b.y);
    LP zDist = (LP)(a.z - b.z);
    LP stretchLength = lsqrt((xDist * xDist) + (yDist * yDist) + (zDist * zDist));
    LP ax = labs_(a.th[0] - b.th[0]);
    LP ay = labs_(a.th[1] - b.th[1]);
    LP az = labs_(a.th[2] - b.th[2]);
    LP myz = (ay < az) ? az : ay;  // std::max(ay, az)
    LP maxBend = (ax < myz) ? myz : ax;
    LP load = (stretchLength - initialLen) / initialLen + bendBreak * maxBend;
    return (load >= maxLoad) ? uint8_t(0) : state;
}
template <class LP>
__device__ __forceinline__ uint8_t break_link(const Consts<LP> &c, const PRec<LP> &a,
                                              const PRec<LP> &b, uint8_t state, LP initialLen) {
    return break_link<LP>(c.bendBreak, c.maxLoad, a, b, state, initialLen);
}

// Map2d::interp (PLiB/Geometry/Map2d.h:93-152, indices from getIndexes 93-111):
// bilinear interpolation on the map's grid in float arithmetic, the cell corner found by
// floor and clamped to the grid, the edge cases of a degenerate cell handled as there.
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
template <class LP>
__device__ __forceinline__ LP map_interp(const Map2dView &m, float x, float y) {
    const LP *d = static_cast<const LP *>(m.data);
    // (the float value is clamped before the integer conversion, which leaves every
    // in-range index as it is)
    float fx = floorf(((x - m.xMin) * m.invXMaxMin) * (float)(m.xPoints - 1));
    float fy = floorf(((y - m.yMin) * m.invYMaxMin) * (float)(m.yPoints - 1));
    fx = fminf(fmaxf(fx, -1.0f), (float)m.xPoints);
    fy = fminf(fmaxf(fy, -1.0f), (float)m.yPoints);
    const int xp = (int)fx, yp = (int)fy;
    const int xl = clampi(xp, 0, m.xPoints - 1), yl = clampi(yp, 0, m.yPoints - 1);
    const int xh = clampi(xp + 1, 0, m.xPoints - 1), yh = clampi(yp + 1, 0, m.yPoints - 1);
    if (xl == xh && yl == yh) return d[xl + yl * m.xPoints];
    const float v00 = (float)d[xl + yl * m.xPoints];
    const float v01 = (float)d[xl + yh * m.xPoints];
    const float v10 = (float)d[xh + yl * m.xPoints];
    const float v11 = (float)d[xh + yh * m.xPoints];
    const float x0 = x - m.xMin, y0 = y - m.yMin;
    const float x1 = (float)xl * m.xRes, x2 = (float)xh * m.xRes;
    const float y1 = (float)yl * m.yRes, y2 = (float)yh * m.yRes;
    const float invX21 = 1.0f / (x2 - x1);
    const float c1 = (x2 - x0) * invX21, c2 = (x0 - x1) * invX21;
    float fxy1 = (c1 * v00) + (c2 * v10);
    float fxy2 = (c1 * v01) + (c2 * v11);
    if (xl == xh) {
        fxy1 = v00;
        fxy2 = v01;
    } else if (yl == yh) {
        return (LP)fxy1;
    }
    const float invY21 = 1.0f / (y2 - y1);
    return (LP)((((y2 - y0) * invY21) * fxy1) + (((y0 - y1) * invY21) * fxy2));
}

// ------------------------------------------------------------------ collision mesh
// Real3f of the reference (PLiB/Util/Real3.h:142-258): float components; dot sums
// left to right, cross by components, no fused multiply-adds.
struct V3f {
    float x, y, z;
};
__device__ __forceinline__ V3f v3_sub(V3f a, V3f b) { return V3f{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3f v3_mul(V3f a, V3f b) { return V3f{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ float v3_dot(V3f a, V3f b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
__device__ __forceinline__ V3f v3_cross(V3f a, V3f b) {
    return V3f{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float sign_f(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

// squared distance of point p from an edge e = b - a with q = p - a: the edge term of
// MeshAccel::triSDF2, the projection parameter clamped to [0, 1] in lp (clamp3)
template <class LP>
__device__ __forceinline__ float tri_edge2(V3f e, V3f q) {
    const float t = v3_dot(e, q) / v3_dot(e, e);
    LP tl = (LP)t;
    tl = tl < LP(0) ? LP(0) : (tl > LP(1) ? LP(1) : tl);
    const float tc = (float)tl;
    const V3f d = v3_sub(v3_mul(e, V3f{tc, tc, tc}), q);
    return v3_dot(d, d);
}

// MeshAccel::triSDF2 (PLiB/Geometry/MeshAccel.h:329-372): squared distance of p from the
// triangle abc — the nearest edge when p projects outside it, else the plane distance.
template <class LP>
__device__ __forceinline__ LP tri_sdf2(V3f p, V3f a, V3f b, V3f c) {
    const V3f ba = v3_sub(b, a), pa = v3_sub(p, a);
    const V3f cb = v3_sub(c, b), pb = v3_sub(p, b);
    const V3f ac = v3_sub(a, c), pc = v3_sub(p, c);
    const V3f nor = v3_cross(ba, ac);
    const float s = sign_f(v3_dot(v3_cross(ba, nor), pa)) + sign_f(v3_dot(v3_cross(cb, nor), pb)) +
                    sign_f(v3_dot(v3_cross(ac, nor), pc));
    if (s < 2.0f) {
        const float e1 = tri_edge2<LP>(ba, pa), e2 = tri_edge2<LP>(cb, pb), e3 = tri_edge2<LP>(ac, pc);
        const float m12 = (e2 < e1) ? e2 : e1;  // std::min(e1, e2)
        return (LP)((e3 < m12) ? e3 : m12);
    }
    const float dn = v3_dot(nor, pa);
    return (LP)(dn * dn / v3_dot(nor, nor));
}

template <class LP>
__device__ __forceinline__ V3f mesh_vertex(const MeshView<LP> &m, int i) {
    return V3f{(float)m.vx[i], (float)m.vy[i], (float)m.vz[i]};
}

// MeshAccel::getCell of a point given as lp (getCellCord, MeshAccel.h:295-316): the
// point as Real3f, minus the lower corner, times the inverse cell size, truncated.
// -1 where the cell lies outside the grid (which the reference's bounding-box test
// admits only through rounding at the upper faces, and then reads past its arrays).
template <class LP>
__device__ __forceinline__ int mesh_cell(const MeshView<LP> &m, LP x, LP y, LP z) {
    const float cx = (float)((LP)(float)x - m.xLower);
    const float cy = (float)((LP)(float)y - m.yLower);
    const float cz = (float)((LP)(float)z - m.zLower);
    const int xc = (int)((LP)cx * m.xInv), yc = (int)((LP)cy * m.yInv), zc = (int)((LP)cz * m.zInv);
    if (xc < 0 || yc < 0 || zc < 0 || xc >= m.xCount || yc >= m.yCount || zc >= m.zCount) return -1;
    return (xc * m.yCount * m.zCount) + (yc * m.zCount) + zc;
}

// MeshAccel::getClosestTriAccel (MeshAccel.h:375-412): the closest triangle of the
// point's cell within interactDist (the first of equals), or -1; *dist2 its squared
// distance. The cell's list is the reference's with the triangles removed that lie
// farther from every point of the cell than any particle's interaction distance
// (k_mesh_prune): those never pass the distance test, so the closest triangle and its
// distance are the same, found with fewer distance evaluations.
template <class LP>
__device__ __forceinline__ int mesh_closest(const MeshView<LP> &m, LP x, LP y, LP z, LP interactDist,
                                            LP *dist2) {
    if (x > m.xUpper || y > m.yUpper || z > m.zUpper || x < m.xLower || y < m.yLower || z < m.zLower)
        return -1;
    const int cell = mesh_cell(m, x, y, z);
    if (cell < 0) return -1;
    const int start = m.qStarts[cell], size = m.qSizes[cell];
    if (size == 0) return -1;
    const V3f p{(float)x, (float)y, (float)z};
    const LP id2 = interactDist * interactDist;
    LP minDist = sizeof(LP) == 4 ? (LP)3.40282347e+38f : (LP)1.7976931348623157e+308;
    int closest = -1;
    for (int i = start; i < start + size; ++i) {
        const int tri = m.qValues[i];
        const LP cur = tri_sdf2<LP>(p, mesh_vertex(m, 3 * tri), mesh_vertex(m, 3 * tri + 1),
                                    mesh_vertex(m, 3 * tri + 2));
        if (id2 > cur && cur < minDist) {
            minDist = cur;
            closest = tri;
        }
    }
    *dist2 = minDist;
    return closest;
}

// The sample integrate step on one particle (HiDEM/MeshBlock/MainMeshBlock.cpp:182-261:
// gravity / buoyancy, air / water drag, HiDEMDefTimeIntegration
// HiDEMDefaultFunctions.h:318-370) plus the optional GlacierDem bed terms
// (HiDEM/GlacierDem/MainDem.cpp:176-207), HiDEMDefVelocityLimit (245-290),
// HiDEMDefBoundaryCondition (293-315) and the fixed-layer / front-pressure extensions.
// `p` is updated in place; F is the particle's accumulated force.
template <class LP>
__device__ __forceinline__ void integrate_particle(const Consts<LP> &c, PRec<LP> &p, uint8_t type,
                                                   LP *F) {
    if (c.useFixed && (type & HIDEM_TYPE_FIXED)) {
        for (int k = 0; k < 6; ++k) p.d[k] = LP(0);
        return;
    }
    double xCord = p.x, yCord = p.y, zCord = p.z;
    const LP xDiff = p.d[0], yDiff = p.d[1], zDiff = p.d[2];
    const LP uDiff = p.d[3], vDiff = p.d[4], wDiff = p.d[5];
    LP xTheta = p.th[0], yTheta = p.th[1], zTheta = p.th[2];
    const LP radius = p.r;
    const LP diameter = radius * LP(2);

    // bed height and friction under the particle: the GlacierDem maps
    // (InputBed::getHeight / getFric, PLiB/Geometry/InputGeometry.h:58-68) or constants
    LP bedHeight = c.bedHeight, bedFriction = c.bedFriction;
    if (c.useBed && c.useBedMap) bedHeight = map_interp<LP>(c.bedMap, (float)xCord, (float)yCord);
    LP dragCoeff;
    if (c.useBed && ((zCord + (double)radius) - (double)bedHeight < (double)c.bedInteract)) {
        if (c.useFricMap) bedFriction = map_interp<LP>(c.fricMap, (float)xCord, (float)yCord);
        LP a = c.bedDrag * bedFriction;
        LP b = LP(1e+5) * c.scale * c.scale;
        dragCoeff = (b < a) ? b : a;  // std::min(a, b)
    } else if (zCord > (double)c.waterLevel) {
        dragCoeff = c.airDrag;
    } else {
        dragCoeff = c.waterDrag;
    }
    LP xForce = F[0], yForce = F[1], zForce = F[2];
    LP uForce = F[3], vForce = F[4], wForce = F[5];
    const LP particleMass = c.rhoIce * diameter * diameter * diameter;
    const LP particleMomentInertia = particleMass * diameter * diameter / LP(6);

    if (zCord > (double)c.waterLevel) zForce = zForce + -c.g * particleMass;
    if (zCord <= (double)c.waterLevel) zForce = zForce + c.lift * particleMass;
    if (c.useBed && zCord + (double)radius < (double)bedHeight)
        zForce = (LP)((double)zForce +
                      (double)c.bedStiffness * ((double)bedHeight - (zCord + (double)radius)));
    // collision mesh (HiDEM/MeshConstrainedDem/MainMeshDem.cpp:220-235)
    if (c.useMesh) {
        LP dist2;
        const int tri = mesh_closest(c.mesh, (LP)xCord, (LP)yCord, (LP)zCord, c.bedInteract + radius, &dist2);
        if (tri >= 0) {
            const float maxDist = (float)(c.bedInteract + radius);
            const LP dist = lsqrt(dist2);
            dragCoeff = c.mesh.drag * ((LP)maxDist - dist);
            const LP fx = -c.mesh.nx[tri] * ((LP)maxDist - dist) * c.mesh.force;
            const LP fy = -c.mesh.ny[tri] * ((LP)maxDist - dist) * c.mesh.force;
            const LP fz = -c.mesh.nz[tri] * ((LP)maxDist - dist) * c.mesh.force;
            atomicAdd(&c.mesh.fx[tri], fx);
            atomicAdd(&c.mesh.fy[tri], fy);
            atomicAdd(&c.mesh.fz[tri], fz);
            xForce = xForce + fx;
            yForce = yForce + fy;
            zForce = zForce + fz;
        }
    }
    // external force maps (ExternalForces, PLiB/ExternalForces.h; MainDem.cpp:211-216)
    if (c.useExtMaps) {
        const float fx = (float)xCord, fy = (float)yCord;
        xForce = xForce + map_interp<LP>(c.extMap[0], fx, fy);
        yForce = yForce + map_interp<LP>(c.extMap[1], fx, fy);
        zForce = zForce + map_interp<LP>(c.extMap[2], fx, fy);
        uForce = uForce + map_interp<LP>(c.extMap[3], fx, fy);
        vForce = vForce + map_interp<LP>(c.extMap[4], fx, fy);
        wForce = wForce + map_interp<LP>(c.extMap[5], fx, fy);
    }
    if (c.useFront && (type & HIDEM_TYPE_FRONT) && zCord < (double)c.waterLevel) {
        LP depth = (LP)((double)c.waterLevel - zCord);
        xForce = xForce - c.rhoWater * c.g * depth * diameter * diameter;
    }

    const LP dragInvDt2 = dragCoeff * c.invDt2;
    const LP massDtSqr = particleMass * c.invDtSqr;
    const LP pMassDtSqr = particleMass / c.dtSqr;
    const LP pMemDtSqr = particleMomentInertia / c.dtSqr;
    const LP invC1 = LP(1) / (pMassDtSqr + dragCoeff * c.invDt2);
    const LP invC2 = LP(1) / (pMemDtSqr + dragCoeff * c.invDt2);
    const LP interDtSqr = particleMomentInertia * c.invDtSqr;
    const LP xDN = (xForce + massDtSqr * xDiff + dragInvDt2 * -xDiff) * invC1;
    const LP yDN = (yForce + massDtSqr * yDiff + dragInvDt2 * -yDiff) * invC1;
    const LP zDN = (zForce + massDtSqr * zDiff + dragInvDt2 * -zDiff) * invC1;
    const LP uDN = (uForce + interDtSqr * uDiff + dragInvDt2 * -uDiff) * invC2;
    const LP vDN = (vForce + interDtSqr * vDiff + dragInvDt2 * -vDiff) * invC2;
    const LP wDN = (wForce + interDtSqr * wDiff + dragInvDt2 * -wDiff) * invC2;

    const double xPrev = xCord, yPrev = yCord, zPrev = zCord;
    const LP xThPrev = xTheta, yThPrev = yTheta, zThPrev = zTheta;
    xCord = xCord + (double)xDN;
    yCord = yCord + (double)yDN;
    zCord = zCord + (double)zDN;
    xTheta = xTheta + uDN;
    yTheta = yTheta + vDN;
    zTheta = zTheta + wDN;

    if (c.useVel) {
        const LP xVel = xDN * c.mainInvDt, yVel = yDN * c.mainInvDt, zVel = zDN * c.mainInvDt;
        const LP xTV = (xTheta - xThPrev) * c.mainInvDt;
        const LP yTV = (yTheta - yThPrev) * c.mainInvDt;
        const LP zTV = (zTheta - zThPrev) * c.mainInvDt;
        if (xVel > c.maxVel) xCord = (double)(c.dt * c.maxVel) + xPrev;
        if (yVel > c.maxVel) yCord = (double)(c.dt * c.maxVel) + yPrev;
        if (zVel > c.maxVel) zCord = (double)(c.dt * c.maxVel) + zPrev;
        if (xTV > c.maxRot) xTheta = c.dt * c.maxRot + xThPrev;
        if (yTV > c.maxRot) yTheta = c.dt * c.maxRot + yThPrev;
        if (zTV > c.maxRot) zTheta = c.dt * c.maxRot + zThPrev;
        if (xVel < -c.maxVel) xCord = (double)(c.dt * -c.maxVel) + xPrev;
        if (yVel < -c.maxVel) yCord = (double)(c.dt * -c.maxVel) + yPrev;
        if (zVel < -c.maxVel) zCord = (double)(c.dt * -c.maxVel) + zPrev;
        if (xTV < -c.maxRot) xTheta = c.dt * -c.maxRot + xThPrev;
        if (yTV < -c.maxRot) yTheta = c.dt * -c.maxRot + yThPrev;
        if (zTV < -c.maxRot) zTheta = c.dt * -c.maxRot + zThPrev;
    }
    if (c.useBnd) {
        if (xCord + (double)radius < c.lower[0] && c.bmin[0]) xCord = xPrev;
        if (xCord - (double)radius > c.upper[0] && c.bmax[0]) xCord = xPrev;
        if (yCord + (double)radius < c.lower[1] && c.bmin[1]) yCord = yPrev;
        if (yCord - (double)radius > c.upper[1] && c.bmax[1]) yCord = yPrev;
        if (zCord + (double)radius < c.lower[2] && c.bmin[2]) zCord = zPrev;
        if (zCord - (double)radius > c.upper[2] && c.bmax[2]) zCord = zPrev;
    }
    p.x = xCord;
    p.y = yCord;
    p.z = zCord;
    p.th[0] = xTheta;
    p.th[1] = yTheta;
    p.th[2] = zTheta;
    p.d[0] = (LP)(xCord - xPrev);
    p.d[1] = (LP)(yCord - yPrev);
    p.d[2] = (LP)(zCord - zPrev);
    p.d[3] = xTheta - xThPrev;
    p.d[4] = yTheta - yThPrev;
    p.d[5] = zTheta - zThPrev;
}

}  // namespace hidem
