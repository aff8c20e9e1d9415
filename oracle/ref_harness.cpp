// Oracle harness around the reference's own CPU hot path — TEST INFRASTRUCTURE ONLY.
//
// This file is compiled against the unmodified reference headers where they lie
// (NeighbourGrid, NeighAccel, LinkAccelSide, CombinedAccel, LinkGenerator,
// HiDEMDefaultFunctions, the particle/link data handlers) by oracle/Makefile, with
// the project-written shims in oracle/refshim/ standing in for MPI, HDF5 and the
// CMake-generated Global.h. The outputs go to oracle/_ref/ and are used only by the
// tests, by __graft_entry__.smoke() and by bench.py's CPU reference arm. Nothing in
// the product links or loads it.
//
// What is project code here (because the reference has it only inside HiDEMLib.h,
// which needs toml11, or inside a sample main):
//   * the derived constants of the sample main (HiDEM/MeshBlock/MainMeshBlock.cpp:106-156),
//   * the integrate functor of the sample mains (MainMeshBlock.cpp:182-261 plus the
//     GlacierDem bed terms HiDEM/GlacierDem/MainDem.cpp:176-207 and the project's
//     fixed-layer / front-pressure extensions, identical in the product),
//   * the gridService rebuild policy (HiDEMLib/HiDEMLib.h:533-628, 424-474),
//   * the timestep loop order (MainMeshBlock.cpp:274-323).
// Redistribution (HiDEMLib/HiDEMDistribution.h:99-198) only permutes storage on one
// rank; the harness keeps the caller's order and performs the rebuild it triggers.
//
// Overload note: HiDEMDefaultFunctions.h calls unqualified sqrt() and abs() on lpReal_t.
// The harness is built with -include math.h -include stdlib.h so that these resolve to
// the float overloads (as in the reference's CUDA build, where device code sees CUDA's
// float overloads). Without them, a g++ translation unit that includes the functor
// header first (as MainMeshBlock.cpp does) binds abs(float) to int abs(int).

#include <cassert>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <chrono>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "Global.h"
#include "HiDEM/Common/HiDEMDefaultFunctions.h"
#include "NeighbourGrid.h"
#include "Accel/CombinedAccel.h"
#include "Geometry/Map.h"
#include "Geometry/Map2d.h"
#include "Geometry/MeshAccel.h"
#include <AtomicOps.h>
#include "Generators/LinkGenerator.h"
#include "HiDEMParticleData.h"
#include "HiDEMLinkData.h"
#include "ParticleDataHandler.h"
#include "LinkDataHandler.h"

#include "hidem_b200.h"

// maps of the next sessions (slot 0 bed height, 1 bed friction, 2..7 external forces)
static Map2d<lpReal_t> *g_maps[8] = {};

// collision mesh of the next sessions: the reference's MeshAccel over copies of the
// vertex / normal arrays (the MeshData layout, PLiB/MeshData.h:21-35), the sample main's
// meshForce / meshDrag, and the face force sums (CollisionMesh xFaceForce..zFaceForce)
static MeshAccel *g_accel = nullptr;
static std::vector<lpReal_t> g_mv[3], g_mn[3], g_face[3];
static lpReal_t g_meshForce = 0, g_meshDrag = 0;

using PData = ParticleDataHandler<HiDEMParticleData>;
using LData = LinkDataHandler<HiDEMLinkData>;

namespace {

struct Derived {
    // the sample main's locals, in its types (MainMeshBlock.cpp:69-156)
    lpReal_t breakTime, dt, scale, beamWidth, E, waterLevel, attractDistance, attractScaleForce;
    lpReal_t maxVel, maxRot, rhoWater, rhoIce, bedStiffness, bedInteract, waterDrag, airDrag, bedDrag;
    lpReal_t g, damping, dampingRotation, maxLoad, bendBreak;
    lpReal_t lift, invDt, invDt2, dtSqr, invDtSqr, G, W2, W4, scaleE;
    lpReal_t bedHeight, bedFriction;
    double searchDistance, interactDist;
};

Derived derive(const hidem_params &P) {
    Derived d;
    d.breakTime = P.breakTime;
    d.dt = P.dt;
    d.scale = P.scale;
    d.beamWidth = P.beamWidth;
    d.E = P.E;
    d.waterLevel = P.waterLevel;
    d.attractDistance = P.attractDistance;
    d.attractScaleForce = P.attractScaleForce;
    d.maxVel = P.maxVel;
    d.maxRot = P.maxRot;
    d.rhoWater = P.rhoWater;
    d.rhoIce = P.rhoIce;
    d.bedStiffness = P.bedStiffness;
    d.bedInteract = P.bedInteract;
    d.waterDrag = P.waterDrag;
    d.airDrag = P.airDrag;
    d.bedDrag = P.bedDrag;
    d.g = P.g;
    d.damping = P.damping;
    d.dampingRotation = P.dampingRotation;
    d.maxLoad = P.maxLoad;
    d.bendBreak = P.bendBreak;
    d.bedHeight = P.bedHeight;
    d.bedFriction = P.bedFriction;

    d.beamWidth *= d.scale;
    d.bedInteract *= d.scale;
    d.bedStiffness *= d.scale * d.scale;
    d.waterDrag *= d.scale * d.scale;
    d.airDrag *= d.scale * d.scale;
    d.bedDrag *= d.scale * d.scale;
    d.damping *= d.scale * d.scale;
    d.dampingRotation *= d.scale * d.scale;
    d.attractDistance *= d.scale;
    d.lift = (d.rhoWater - d.rhoIce) / d.rhoIce * d.g;
    d.invDt = 1.0 / d.dt;
    d.invDt2 = 1.0 / (2.0 * d.dt);
    d.dtSqr = pow(d.dt, 2.0);
    d.invDtSqr = 1.0 / pow(d.dt, 2.0);
    d.G = d.E / 2.0;
    d.W2 = d.beamWidth * d.beamWidth;
    d.W4 = d.beamWidth * d.beamWidth * d.beamWidth * d.beamWidth;
    d.scaleE = d.E * d.scale;

    lpReal_t maxRadius = P.maxRadius;
    lpReal_t maxParticleDist = maxRadius * 2.0;  // HiDEMLib.h:759
    d.searchDistance = P.searchDistanceScale * maxParticleDist;
    d.interactDist = d.searchDistance - maxParticleDist;
    return d;
}

template <class T>
void copy_in(ManVec<T> &dst, const void *src, int64_t n) {
    const T *s = static_cast<const T *>(src);
    for (int64_t i = 0; i < n; ++i) dst[i] = s[i];
}
template <class T>
void copy_out(void *dst, ManVec<T> &src, int64_t n) {
    if (!dst) return;
    T *d = static_cast<T *>(dst);
    for (int64_t i = 0; i < n; ++i) d[i] = src[i];
}

PData *make_particles(const hidem_particle_soa *p, int64_t n) {
    PData *pd = new PData();
    pd->resize(n);
    copy_in<hpReal_t>(pd->xCord, p->xCord, n);
    copy_in<hpReal_t>(pd->yCord, p->yCord, n);
    copy_in<hpReal_t>(pd->zCord, p->zCord, n);
    copy_in<lpReal_t>(pd->xTheta, p->xTheta, n);
    copy_in<lpReal_t>(pd->yTheta, p->yTheta, n);
    copy_in<lpReal_t>(pd->zTheta, p->zTheta, n);
    copy_in<lpReal_t>(pd->xDiff, p->xDiff, n);
    copy_in<lpReal_t>(pd->yDiff, p->yDiff, n);
    copy_in<lpReal_t>(pd->zDiff, p->zDiff, n);
    copy_in<lpReal_t>(pd->uDiff, p->uDiff, n);
    copy_in<lpReal_t>(pd->vDiff, p->vDiff, n);
    copy_in<lpReal_t>(pd->wDiff, p->wDiff, n);
    copy_in<lpReal_t>(pd->radius, p->radius, n);
    for (int64_t i = 0; i < n; ++i) {
        pd->owners[i] = 0;  // one rank owns everything
        pd->type[i] = p->type ? p->type[i] : 0;
        pd->globalKeys[i] = p->globalKeys ? p->globalKeys[i] : i;
        pd->xForce[i] = pd->yForce[i] = pd->zForce[i] = 0;
        pd->uForce[i] = pd->vForce[i] = pd->wForce[i] = 0;
    }
    pd->generateOnwedList();
    return pd;
}

}  // namespace

extern "C" {

int hidem_ref_precision(void) { return sizeof(lpReal_t) == 4 ? HIDEM_PREC_MIXED : HIDEM_PREC_FP64; }

int hidem_ref_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Cell (ix,iy,iz) of every particle: NeighbourGrid::generate with the run's search
// distance (PLiB/NeighbourGrid.cpp:48-161).
int hidem_ref_cells(const hidem_params *P, const hidem_particle_soa *p, int64_t n, int32_t *ix,
                    int32_t *iy, int32_t *iz, int64_t dims[3], double mins[3]) {
    Derived d = derive(*P);
    PData *pd = make_particles(p, n);
    NeighbourGrid *grid = new NeighbourGrid();
    grid->generate(*pd, d.searchDistance);
    for (int64_t i = 0; i < n; ++i) {
        auto [x, y, z] = grid->getCord((int)grid->colours[i]);
        ix[i] = x;
        iy[i] = y;
        iz[i] = z;
    }
    dims[0] = grid->xGridSize;
    dims[1] = grid->yGridSize;
    dims[2] = grid->zGridSize;
    mins[0] = grid->xMin;
    mins[1] = grid->yMin;
    mins[2] = grid->zMin;
    delete grid;
    delete pd;
    return 0;
}

// Contact list: NeighAccel::generateNeighbours (PLiB/Accel/NeighAccel.h:25-137), rows
// packed in the reference's per-particle order.
int hidem_ref_neighbours(const hidem_params *P, const hidem_particle_soa *p, int64_t n,
                         int32_t *counts, int32_t *list, int64_t cap, int64_t *total) {
    Derived d = derive(*P);
    PData *pd = make_particles(p, n);
    CombinedAccel *accel = new CombinedAccel();
    accel->grid.generate(*pd, d.searchDistance);
    accel->nList.generateNeighbours(accel->grid, *pd, d.searchDistance, d.interactDist);
    int64_t off = 0;
    for (int64_t i = 0; i < n; ++i) {
        int c = accel->nList.numNeighs[i];
        counts[i] = c;
        for (int k = 0; k < c; ++k) {
            if (list && off < cap) list[off] = accel->nList.getPartNeighId(k, (pInd_t)i);
            ++off;
        }
    }
    *total = off;
    delete accel;
    delete pd;
    return (list && off > cap) ? HIDEM_ERR_CAPACITY : 0;
}

// LinkGenerator::generateLinksDistance with the given distance scale
// (PLiB/Generators/LinkGenerator.h:30-37,60-181). Output order is the generator's
// (thread-dependent); compare as a set.
int hidem_ref_links(const hidem_particle_soa *p, int64_t n, double maxRadius, double scale,
                    int64_t *keyA, int64_t *keyB, void *initialLen, int64_t cap, int64_t *count) {
    PData *pd = make_particles(p, n);
    for (int64_t i = 0; i < n; ++i) pd->type[i] = 0;
    OffloadHashMap<gKey_t, pInd_t> mapper;
    pd->remap(mapper);
    LinkGenerator *gen = new LinkGenerator();
    gen->setDistScale(scale);
    ManVec<ElementaryLink> links = gen->generateLinksDistance(maxRadius, *pd);
    *count = links.size();
    for (size_t i = 0; i < links.size() && (int64_t)i < cap; ++i) {
        keyA[i] = links[i].globalKeyParticleA;
        keyB[i] = links[i].globalKeyParticleB;
        static_cast<lpReal_t *>(initialLen)[i] = links[i].initialLen;
    }
    delete gen;
    delete pd;
    return (int64_t)links.size() > cap ? HIDEM_ERR_CAPACITY : 0;
}

// A persistent run of the sample-main timestep loop: the reference's particle and link
// data, its CombinedAccel and the rebuild policy state, kept between calls so that
// steps can be timed without the setup.
struct RefSession {
    Derived d;
    hidem_params P;
    PData *pd = nullptr;
    LData *ld = nullptr;
    CombinedAccel *accel = nullptr;
    OffloadHashMap<gKey_t, pInd_t> *pMapper = nullptr;
    int64_t n = 0, L = 0, step = 0, start = 0;
    double accumulatedDist = 0;
    std::vector<uint8_t> before;
    std::vector<int64_t> evLink, evStep, regen;

    ~RefSession() {
        delete accel;
        delete ld;
        delete pd;
        delete pMapper;
    }

    void setup(const hidem_params *Pin, const hidem_particle_soa *p, int64_t nIn,
               const hidem_link_soa *l, int64_t LIn, int64_t startStep) {
        P = *Pin;
        d = derive(P);
        n = nIn;
        L = LIn;
        step = start = startStep;
        pd = make_particles(p, n);
        pMapper = new OffloadHashMap<gKey_t, pInd_t>();
        pd->remap(*pMapper);
        ld = new LData();
        {
            ManVec<ElementaryLink> links;
            links.resize(L);
            const lpReal_t *L0 = static_cast<const lpReal_t *>(l->initialLen);
            for (int64_t i = 0; i < L; ++i) {
                ElementaryLink e;
                e.globalKey = l->globalKeys ? l->globalKeys[i] : i;
                e.globalKeyParticleA = l->globalKeyEndA[i];
                e.globalKeyParticleB = l->globalKeyEndB[i];
                e.particleLinkNum = l->particleLinkNum ? l->particleLinkNum[i] : 0;
                e.owner = 0;
                e.initialLen = L0[i];
                e.state = l->state[i];
                links[i] = e;
            }
            ld->appendInitLinks(links);
        }
        if (l->CT[0]) {
            ManVec<ctReal_t> *ct[6] = {&ld->CT0_flat, &ld->CT1_flat, &ld->CT2_flat,
                                       &ld->CT3_flat, &ld->CT4_flat, &ld->CT5_flat};
            for (int k = 0; k < 6; ++k) copy_in<ctReal_t>(*ct[k], l->CT[k], 2 * L);
        }
        ld->makeLocalPartEnds(*pMapper);
        accel = new CombinedAccel();
        before.resize(L);
    }

    // gridService (HiDEMLib.h:533-628) on one rank; returns whether it rebuilt.
    bool gridService() {
        PData &pData = *pd;
        const int64_t t = step;
        bool rg = (t == start);
        if (P.gridRegenInterval != -1) {
            rg = (t % P.gridRegenInterval) == 0;
        } else if (t % 10 == 0) {
            // accumulateDist / getMaxDistOwned (HiDEMLib.h:424-474)
            double mx = 0.0, my = 0.0, mz = 0.0;
            for (int64_t i = 0; i < n; ++i) {
                double a = pData.xDiff[i], b = pData.yDiff[i], c = pData.zDiff[i];
                if (a > mx) mx = a;
                if (b > my) my = b;
                if (c > mz) mz = c;
            }
            lpReal_t xM = mx, yM = my, zM = mz;
            double currDist = 10 * std::sqrt((xM * xM) + (yM * yM) + (zM * zM));
            accumulatedDist += currDist;
            if (accumulatedDist >= d.interactDist / 2.0) rg = true;
        }
        if (t == P.firstBalanceTimestep) rg = true;
        if (rg) {
            accumulatedDist = 0;
            accel->generateNeighbours(pData, *ld, d.searchDistance, d.interactDist);
            accel->generateLinks(pData, *ld, d.searchDistance, d.interactDist);
            accel->lAccel.sortSideData(pData, *ld);
            accel->generateIndexes(pData, *ld, d.searchDistance, d.interactDist);
            regen.push_back(t);
        }
        return rg;
    }

    // computePartForce + applyForce + gated linkUpdate + finalizeTs (MainMeshBlock.cpp:295-320).
    // The bed / friction / external force maps, when set, are the reference's own Map2d
    // (PLiB/Geometry/Map2d.h), used as GlacierDem uses them (MainDem.cpp:176-216).
    void rest_of_step() {
        PData &pData = *pd;
        LData &lData = *ld;
        const Derived &dd = d;
        const Real3 lowerLimit(P.lowerLimit[0], P.lowerLimit[1], P.lowerLimit[2]);
        const Real3 upperLimit(P.upperLimit[0], P.upperLimit[1], P.upperLimit[2]);
        const bool useBed = P.useBed, useVel = P.useVelocityLimit, useBnd = P.useBoundary;
        const bool useFixed = P.useFixed, useFront = P.useFrontPressure;
        const bool bMinX = P.boundaryMin[0], bMinY = P.boundaryMin[1], bMinZ = P.boundaryMin[2];
        const bool bMaxX = P.boundaryMax[0], bMaxY = P.boundaryMax[1], bMaxZ = P.boundaryMax[2];
        // integrate functor: sample integrate lambda (MainMeshBlock.cpp:182-261) with the
        // GlacierDem bed terms (MainDem.cpp:176-207) and the fixed / front extensions.
        auto integrate = [=](pInd_t pInd, PData &p) {
            const uint8_t type = p.type[pInd];
            if (useFixed && (type & HIDEM_TYPE_FIXED)) {
                p.xDiff[pInd] = 0;
                p.yDiff[pInd] = 0;
                p.zDiff[pInd] = 0;
                p.uDiff[pInd] = 0;
                p.vDiff[pInd] = 0;
                p.wDiff[pInd] = 0;
                return;
            }
            hpReal_t xCord = p.xCord[pInd], yCord = p.yCord[pInd], zCord = p.zCord[pInd];
            hpReal_t xCordPrev = 0, yCordPrev = 0, zCordPrev = 0;
            lpReal_t xDiff = p.xDiff[pInd], yDiff = p.yDiff[pInd], zDiff = p.zDiff[pInd];
            lpReal_t xTheta = p.xTheta[pInd], yTheta = p.yTheta[pInd], zTheta = p.zTheta[pInd];
            lpReal_t xThetaPrev = 0, yThetaPrev = 0, zThetaPrev = 0;
            lpReal_t uDiff = p.uDiff[pInd], vDiff = p.vDiff[pInd], wDiff = p.wDiff[pInd];
            lpReal_t radius = p.radius[pInd];
            lpReal_t diameter = radius * lpReal_t(2.0);

            lpReal_t bedzCord = (useBed && g_maps[0]) ? g_maps[0]->interp(xCord, yCord) : dd.bedHeight;
            lpReal_t dragCoeff;
            if (useBed && (zCord + radius) - bedzCord < dd.bedInteract) {
                lpReal_t fric = g_maps[1] ? g_maps[1]->interp(xCord, yCord) : dd.bedFriction;
                dragCoeff = std::min(dd.bedDrag * fric, lpReal_t(1e+5) * dd.scale * dd.scale);
            } else if (zCord > dd.waterLevel) {
                dragCoeff = dd.airDrag;
            } else {
                dragCoeff = dd.waterDrag;
            }
            lpReal_t xForce = p.xForce[pInd], yForce = p.yForce[pInd], zForce = p.zForce[pInd];
            lpReal_t uForce = p.uForce[pInd], vForce = p.vForce[pInd], wForce = p.wForce[pInd];

            lpReal_t particleMass = dd.rhoIce * diameter * diameter * diameter;
            lpReal_t particleMomentInertia = particleMass * diameter * diameter / lpReal_t(6.0);

            if (zCord > dd.waterLevel) zForce += -dd.g * particleMass;
            if (zCord <= dd.waterLevel) zForce += dd.lift * particleMass;
            if (useBed && zCord + radius < bedzCord)
                zForce += dd.bedStiffness * (bedzCord - (zCord + radius));
            // collision mesh: Mesh::closestTriFun (PLiB/Geometry/Mesh.h:69-83) with the
            // sample's lambda (HiDEM/MeshConstrainedDem/MainMeshDem.cpp:220-235)
            if (g_accel) {
                auto [tri, dist, searched] = g_accel->getClosestTriAccel(
                    xCord, yCord, zCord, dd.bedInteract + radius, g_mv[0].data(), g_mv[1].data(), g_mv[2].data());
                if (tri >= 0) {
                    float maxDist = dd.bedInteract + radius;
                    dist = sqrt(dist);
                    dragCoeff = g_meshDrag * ((maxDist - dist));
                    lpReal_t xForceCol = -g_mn[0][tri] * (maxDist - dist) * g_meshForce;
                    lpReal_t yForceCol = -g_mn[1][tri] * (maxDist - dist) * g_meshForce;
                    lpReal_t zForceCol = -g_mn[2][tri] * (maxDist - dist) * g_meshForce;
                    Atomic::atomicAddVal(g_face[0][tri], xForceCol);
                    Atomic::atomicAddVal(g_face[1][tri], yForceCol);
                    Atomic::atomicAddVal(g_face[2][tri], zForceCol);
                    xForce += xForceCol;
                    yForce += yForceCol;
                    zForce += zForceCol;
                }
            }
            if (g_maps[2]) {
                xForce += g_maps[2]->interp(xCord, yCord);
                yForce += g_maps[3]->interp(xCord, yCord);
                zForce += g_maps[4]->interp(xCord, yCord);
                uForce += g_maps[5]->interp(xCord, yCord);
                vForce += g_maps[6]->interp(xCord, yCord);
                wForce += g_maps[7]->interp(xCord, yCord);
            }
            if (useFront && (type & HIDEM_TYPE_FRONT) && zCord < dd.waterLevel) {
                lpReal_t depth = (lpReal_t)(dd.waterLevel - zCord);
                xForce -= dd.rhoWater * dd.g * depth * diameter * diameter;
            }

            auto vel = HiDEMDefTimeIntegration(dragCoeff, dd.invDt2, particleMass, dd.invDtSqr, dd.dtSqr,
                                               particleMomentInertia, dd.invDt,
                                               xForce, xDiff, xCord, xCordPrev,
                                               yForce, yDiff, yCord, yCordPrev,
                                               zForce, zDiff, zCord, zCordPrev,
                                               uForce, uDiff, xTheta, xThetaPrev,
                                               vForce, vDiff, yTheta, yThetaPrev,
                                               wForce, wDiff, zTheta, zThetaPrev);
            if (useVel) {
                auto [xVel, yVel, zVel, xThetaVel, yThetaVel, zThetaVel] = vel;
                HiDEMDefVelocityLimit(dd.maxVel, dd.maxRot, dd.dt,
                                      xVel, xCord, xCordPrev, yVel, yCord, yCordPrev,
                                      zVel, zCord, zCordPrev,
                                      xThetaVel, xTheta, xThetaPrev, yThetaVel, yTheta, yThetaPrev,
                                      zThetaVel, zTheta, zThetaPrev);
            }
            if (useBnd) {
                HiDEMDefBoundaryCondition(radius, lowerLimit, upperLimit, bMinX, bMaxX, bMinY, bMaxY,
                                          bMinZ, bMaxZ, xCord, xCordPrev, yCord, yCordPrev, zCord,
                                          zCordPrev);
            }
            p.xCord[pInd] = xCord;
            p.yCord[pInd] = yCord;
            p.zCord[pInd] = zCord;
            p.xTheta[pInd] = xTheta;
            p.yTheta[pInd] = yTheta;
            p.zTheta[pInd] = zTheta;
            p.xDiff[pInd] = static_cast<lpReal_t>(xCord - xCordPrev);
            p.yDiff[pInd] = static_cast<lpReal_t>(yCord - yCordPrev);
            p.zDiff[pInd] = static_cast<lpReal_t>(zCord - zCordPrev);
            p.uDiff[pInd] = xTheta - xThetaPrev;
            p.vDiff[pInd] = yTheta - yThetaPrev;
            p.wDiff[pInd] = zTheta - zThetaPrev;
        };

        HiDEMDefNeighForceFunc nFunc(dd.invDt, dd.attractDistance, dd.attractScaleForce, dd.damping,
                                     dd.dampingRotation, dd.scaleE);
        HiDEMDefLinkForceFunc lFunc(dd.invDt, dd.damping, dd.dampingRotation, dd.E, dd.W2, dd.W4, dd.G);
        HiDEMDefLinkBreakFunc bFunc(dd.bendBreak, dd.maxLoad);

        // computePartForce (HiDEMLib.h:316-382) -> CombinedAccel::iterateCombined
        auto fullArgs = make4Pack(
            packVecPtrs(pData.xDiff, pData.yDiff, pData.zDiff, pData.uDiff, pData.vDiff,
                        pData.wDiff, pData.radius),
            packVecPtrs(),
            packVecPtrs(lData.CT0_flat, lData.CT1_flat, lData.CT2_flat, lData.CT3_flat,
                        lData.CT4_flat, lData.CT5_flat),
            packVecPtrs(pData.xForce, pData.yForce, pData.zForce, pData.uForce, pData.vForce,
                        pData.wForce));
        accel->iterateCombinedPre(OffloadExec(), pData, lData, nFunc, lFunc, fullArgs);
        Iterator::syncAll();

        // applyForce (HiDEMLib.h:303-314)
        pData.iterateAllParticles(OffloadExec(), integrate, pData);
        Iterator::syncAll();

        // linkUpdate, gated as in MainMeshBlock.cpp:312
        const int64_t t = step;
        if ((lpReal_t)(t * dd.dt) > dd.breakTime) {
            for (int64_t i = 0; i < L; ++i) before[i] = lData.state[i];
            accel->iterateLinks(OffloadExec(), pData, lData, bFunc,
                                make3Pack(packVecPtrs(pData.xCord, pData.yCord, pData.zCord,
                                                      pData.xTheta, pData.yTheta, pData.zTheta),
                                          packVecPtrs(), packVecPtrs(lData.state, lData.initialLen)));
            Iterator::syncAll();
            for (int64_t i = 0; i < L; ++i) {
                if (before[i] != 0 && lData.state[i] == 0) {
                    evLink.push_back(i);
                    evStep.push_back(t);
                }
            }
        }
        step = t + 1;  // finalizeTs
    }

    // Runs nsteps; `seconds` covers the loop except the rebuild of its first step.
    void advance(int32_t nsteps, double *seconds) {
        auto t0 = std::chrono::steady_clock::now();
        for (int32_t s = 0; s < nsteps; ++s) {
            gridService();
            if (s == 0) t0 = std::chrono::steady_clock::now();
            rest_of_step();
        }
        auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    }

    void read(hidem_particle_soa *p, hidem_link_soa *l, void *force_out[6]) {
        PData &pData = *pd;
        LData &lData = *ld;
        copy_out<hpReal_t>(p->xCord, pData.xCord, n);
        copy_out<hpReal_t>(p->yCord, pData.yCord, n);
        copy_out<hpReal_t>(p->zCord, pData.zCord, n);
        copy_out<lpReal_t>(p->xTheta, pData.xTheta, n);
        copy_out<lpReal_t>(p->yTheta, pData.yTheta, n);
        copy_out<lpReal_t>(p->zTheta, pData.zTheta, n);
        copy_out<lpReal_t>(p->xDiff, pData.xDiff, n);
        copy_out<lpReal_t>(p->yDiff, pData.yDiff, n);
        copy_out<lpReal_t>(p->zDiff, pData.zDiff, n);
        copy_out<lpReal_t>(p->uDiff, pData.uDiff, n);
        copy_out<lpReal_t>(p->vDiff, pData.vDiff, n);
        copy_out<lpReal_t>(p->wDiff, pData.wDiff, n);
        if (force_out) {
            copy_out<lpReal_t>(force_out[0], pData.xForce, n);
            copy_out<lpReal_t>(force_out[1], pData.yForce, n);
            copy_out<lpReal_t>(force_out[2], pData.zForce, n);
            copy_out<lpReal_t>(force_out[3], pData.uForce, n);
            copy_out<lpReal_t>(force_out[4], pData.vForce, n);
            copy_out<lpReal_t>(force_out[5], pData.wForce, n);
        }
        if (l->state)
            for (int64_t i = 0; i < L; ++i) l->state[i] = lData.state[i];
        if (l->CT[0]) {
            ManVec<ctReal_t> *ct[6] = {&lData.CT0_flat, &lData.CT1_flat, &lData.CT2_flat,
                                       &lData.CT3_flat, &lData.CT4_flat, &lData.CT5_flat};
            for (int k = 0; k < 6; ++k) {
                ctReal_t *dst = static_cast<ctReal_t *>(l->CT[k]);
                for (int64_t i = 0; i < L; ++i) {
                    dst[2 * i] = (*ct[k])[lData.sideIndEndA[i]];
                    dst[2 * i + 1] = (*ct[k])[lData.sideIndEndB[i]];
                }
            }
        }
    }
};

void *hidem_ref_open(const hidem_params *P, const hidem_particle_soa *p, int64_t n,
                     const hidem_link_soa *l, int64_t L, int64_t start_step) {
    RefSession *s = new RefSession();
    s->setup(P, p, n, l, L, start_step);
    return s;
}

int hidem_ref_advance(void *h, int32_t nsteps, double *seconds) {
    if (!h || nsteps < 0) return HIDEM_ERR_ARG;
    static_cast<RefSession *>(h)->advance(nsteps, seconds);
    return 0;
}

void hidem_ref_close(void *h) { delete static_cast<RefSession *>(h); }

// Bed / friction / external force maps of the next sessions (NULL: none), built as the
// reference's Map2d objects (grid points, then the values point by point).
void hidem_ref_set_maps(const hidem_map2d *bed, const hidem_map2d *friction, const hidem_map2d *ext) {
    for (auto &m : g_maps) {
        delete m;
        m = nullptr;
    }
    auto make = [](const hidem_map2d *src) {
        auto *m = new Map2d<lpReal_t>(src->x_points, src->y_points, src->x_min, src->y_min, src->x_max,
                                      src->y_max);
        const lpReal_t *v = static_cast<const lpReal_t *>(src->data);
        for (int y = 0; y < src->y_points; ++y)
            for (int x = 0; x < src->x_points; ++x) m->setPointInd(x, y, v[x + y * src->x_points]);
        return m;
    };
    if (bed) g_maps[0] = make(bed);
    if (friction) g_maps[1] = make(friction);
    if (ext)
        for (int k = 0; k < 6; ++k) g_maps[2 + k] = make(&ext[k]);
}

// Collision mesh of the next sessions (NULL: none): the reference's MeshAccel built by
// its own generateAccel as CollisionMesh::generateAccel calls it (CollisionMesh.h:31-38:
// cell size and search distance both the given size). Face forces start at zero.
void hidem_ref_set_mesh(const hidem_mesh *m) {
    delete g_accel;
    g_accel = nullptr;
    for (int k = 0; k < 3; ++k) {
        g_mv[k].clear();
        g_mn[k].clear();
        g_face[k].clear();
    }
    if (!m || m->triangles < 1) return;
    const void *v[3] = {m->x_vertex, m->y_vertex, m->z_vertex};
    const void *nrm[3] = {m->x_normal, m->y_normal, m->z_normal};
    for (int k = 0; k < 3; ++k) {
        const lpReal_t *src = static_cast<const lpReal_t *>(v[k]);
        g_mv[k].assign(src, src + 3 * (size_t)m->triangles);
        const lpReal_t *ns = static_cast<const lpReal_t *>(nrm[k]);
        g_mn[k].assign(ns, ns + (size_t)m->triangles);
        g_face[k].assign((size_t)m->triangles, lpReal_t(0));
    }
    g_meshForce = (lpReal_t)m->mesh_force;
    g_meshDrag = (lpReal_t)m->mesh_drag;
    g_accel = new MeshAccel();
    const lpReal_t cs = (lpReal_t)m->cell_size;
    g_accel->generateAccel(std::max(cs, cs), std::max(cs, cs), g_mv[0].data(), g_mv[1].data(), g_mv[2].data(),
                           m->triangles);
}

int hidem_ref_mesh_face_forces(void *x, void *y, void *z) {
    if (!g_accel) return HIDEM_ERR_STATE;
    void *out[3] = {x, y, z};
    for (int k = 0; k < 3; ++k)
        if (out[k]) std::memcpy(out[k], g_face[k].data(), sizeof(lpReal_t) * g_face[k].size());
    return 0;
}

int hidem_ref_mesh_accel(int32_t counts[3], double lower[3], double upper[3], int32_t *sizes,
                         int32_t *starts, int32_t *values, int64_t values_cap, int64_t *values_count) {
    if (!g_accel) return HIDEM_ERR_STATE;
    MeshAccel &a = *g_accel;
    const int c[3] = {a.xCount, a.yCount, a.zCount};
    const double lo[3] = {a.xLower, a.yLower, a.zLower}, hi[3] = {a.xUpper, a.yUpper, a.zUpper};
    for (int k = 0; k < 3; ++k) {
        if (counts) counts[k] = c[k];
        if (lower) lower[k] = lo[k];
        if (upper) upper[k] = hi[k];
    }
    const size_t cells = (size_t)a.xCount * a.yCount * a.zCount;
    for (size_t i = 0; i < cells; ++i) {
        if (sizes) sizes[i] = a.sizes[i];
        if (starts) starts[i] = a.starts[i];
    }
    const int64_t nv = (int64_t)a.values.size();
    if (values)
        for (int64_t i = 0; i < nv && i < values_cap; ++i) values[i] = a.values[i];
    if (values_count) *values_count = nv;
    return 0;
}

// One-shot form: setup, nsteps of the loop, write-back (particles in place; links: state
// and CT), forces of the last step, break events (link index, step), rebuild steps.
int hidem_ref_run(const hidem_params *P, hidem_particle_soa *p, int64_t n, hidem_link_soa *l,
                  int64_t L, int64_t start_step, int32_t nsteps, void *force_out[6],
                  int64_t *ev_link, int64_t *ev_step, int64_t ev_cap, int64_t *ev_count,
                  int64_t *regen_steps, int64_t regen_cap, int64_t *regen_count,
                  double *seconds) {
    RefSession s;
    s.setup(P, p, n, l, L, start_step);
    s.advance(nsteps, seconds);
    s.read(p, l, force_out);
    int64_t nev = (int64_t)s.evLink.size();
    for (int64_t i = 0; i < nev && i < ev_cap; ++i) {
        ev_link[i] = s.evLink[i];
        ev_step[i] = s.evStep[i];
    }
    if (ev_count) *ev_count = nev;
    int64_t nr = (int64_t)s.regen.size();
    for (int64_t i = 0; i < nr && i < regen_cap; ++i) regen_steps[i] = s.regen[i];
    if (regen_count) *regen_count = nr;
    return 0;
}

}  // extern "C"
