/*
 * Precision-generic body of the oracle (TEST INFRASTRUCTURE ONLY). Included twice
 * by hidem_oracle.c with
 *   LP      = float  | double   (lpReal_t = ctReal_t, PLiB/Global.h.in:47-52)
 *   LSQRT   = sqrtf  | sqrt     (the float overload is the one the reference's CUDA
 *                                build binds; see oracle/ref_harness.cpp)
 *   LABS    = fabsf  | fabs
 *   SFX(x)  = x##_mixed | x##_fp64
 * Every expression keeps the reference's operand order and association, since the
 * point of the oracle is bit-exact agreement with the reference's IEEE build.
 */

typedef struct SFX(derived) {
    /* locals of the sample main (HiDEM/MeshBlock/MainMeshBlock.cpp:69-156) */
    LP breakTime, dt, scale, beamWidth, E, waterLevel, attractDistance, attractScaleForce;
    LP maxVel, maxRot, rhoWater, rhoIce, bedStiffness, bedInteract, waterDrag, airDrag, bedDrag;
    LP g, damping, dampingRotation, maxLoad, bendBreak;
    LP lift, invDt, invDt2, dtSqr, invDtSqr, G, W2, W4, scaleE;
    LP bedHeight, bedFriction;
    double searchDistance, interactDist;
} SFX(derived);

/* MainMeshBlock.cpp:69-156 (raw values read as lpReal_t, then scaled) and
 * HiDEMLib/HiDEMLib.h:757-761 (search distances). */
static SFX(derived) SFX(derive)(const hidem_params *P) {
    SFX(derived) d;
    d.breakTime = (LP)P->breakTime;
    d.dt = (LP)P->dt;
    d.scale = (LP)P->scale;
    d.beamWidth = (LP)P->beamWidth;
    d.E = (LP)P->E;
    d.waterLevel = (LP)P->waterLevel;
    d.attractDistance = (LP)P->attractDistance;
    d.attractScaleForce = (LP)P->attractScaleForce;
    d.maxVel = (LP)P->maxVel;
    d.maxRot = (LP)P->maxRot;
    d.rhoWater = (LP)P->rhoWater;
    d.rhoIce = (LP)P->rhoIce;
    d.bedStiffness = (LP)P->bedStiffness;
    d.bedInteract = (LP)P->bedInteract;
    d.waterDrag = (LP)P->waterDrag;
    d.airDrag = (LP)P->airDrag;
    d.bedDrag = (LP)P->bedDrag;
    d.g = (LP)P->g;
    d.damping = (LP)P->damping;
    d.dampingRotation = (LP)P->dampingRotation;
    d.maxLoad = (LP)P->maxLoad;
    d.bendBreak = (LP)P->bendBreak;
    d.bedHeight = (LP)P->bedHeight;
    d.bedFriction = (LP)P->bedFriction;

    LP s2 = d.scale * d.scale;
    d.beamWidth = d.beamWidth * d.scale;
    d.bedInteract = d.bedInteract * d.scale;
    d.bedStiffness = d.bedStiffness * s2;
    d.waterDrag = d.waterDrag * s2;
    d.airDrag = d.airDrag * s2;
    d.bedDrag = d.bedDrag * s2;
    d.damping = d.damping * s2;
    d.dampingRotation = d.dampingRotation * s2;
    d.attractDistance = d.attractDistance * d.scale;
    d.lift = (d.rhoWater - d.rhoIce) / d.rhoIce * d.g;
    d.invDt = (LP)(1.0 / (double)d.dt);
    d.invDt2 = (LP)(1.0 / (2.0 * (double)d.dt));
    d.dtSqr = (LP)pow((double)d.dt, 2.0);
    d.invDtSqr = (LP)(1.0 / pow((double)d.dt, 2.0));
    d.G = (LP)((double)d.E / 2.0);
    d.W2 = d.beamWidth * d.beamWidth;
    d.W4 = d.beamWidth * d.beamWidth * d.beamWidth * d.beamWidth;
    d.scaleE = d.E * d.scale;

    LP maxRadius = (LP)P->maxRadius;
    LP maxParticleDist = (LP)((double)maxRadius * 2.0);
    d.searchDistance = P->searchDistanceScale * (double)maxParticleDist;
    d.interactDist = d.searchDistance - (double)maxParticleDist;
    return d;
}

/* ------------------------------------------------------------------ grid */

typedef struct SFX(grid) {
    double xMin, yMin, zMin, h;
    int X, Y, Z;
    int64_t total;
    int64_t *colour;     /* per particle */
    int32_t *order;      /* iteration order: sorted by (colour, index) */
    int32_t *cellStart;  /* per linear cell, -1 if empty */
    int32_t *cellCount;
    int64_t off[27];
} SFX(grid);

/* NeighbourGrid::generateNeighbourGrid + colourParticles + generateIterationList
 * (PLiB/NeighbourGrid.cpp:72-184; getLimits PLiB/ParticleData.h:47-59; getGridSize
 * NeighbourGrid.cpp:40-46; getGridId / getGridColor NeighbourGrid.cpp:25-33). The
 * colour->bucket hash map becomes a dense per-cell table with the same lookups. */
static void SFX(grid_build)(SFX(grid) *gd, const double *x, const double *y, const double *z,
                            int64_t n, double h) {
    double xMax = x[0], yMax = y[0], zMax = z[0];
    double xMin = x[0], yMin = y[0], zMin = z[0];
    for (int64_t i = 1; i < n; ++i) {
        if (x[i] < xMin) xMin = x[i];
        if (x[i] > xMax) xMax = x[i];
        if (y[i] < yMin) yMin = y[i];
        if (y[i] > yMax) yMax = y[i];
        if (z[i] < zMin) zMin = z[i];
        if (z[i] > zMax) zMax = z[i];
    }
    gd->xMin = xMin;
    gd->yMin = yMin;
    gd->zMin = zMin;
    gd->h = h;
    gd->X = 1 + (int)floor((xMax - xMin) / h);
    gd->Y = 1 + (int)floor((yMax - yMin) / h);
    gd->Z = 1 + (int)floor((zMax - zMin) / h);
    gd->total = (int64_t)gd->X * gd->Y * gd->Z;
    int k = 0;
    for (int zD = -1; zD < 2; ++zD)
        for (int yD = -1; yD < 2; ++yD)
            for (int xD = -1; xD < 2; ++xD)
                gd->off[k++] = (int64_t)xD + (int64_t)yD * gd->X + (int64_t)zD * gd->X * gd->Y;

    gd->colour = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    gd->order = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    gd->cellStart = (int32_t *)malloc(sizeof(int32_t) * (size_t)gd->total);
    gd->cellCount = (int32_t *)calloc((size_t)gd->total, sizeof(int32_t));
    for (int64_t i = 0; i < n; ++i) {
        int ix = (int)floor((x[i] - xMin) / h);
        int iy = (int)floor((y[i] - yMin) / h);
        int iz = (int)floor((z[i] - zMin) / h);
        int c = (int)((int64_t)ix + (int64_t)iy * gd->X + (int64_t)iz * gd->X * gd->Y);
        gd->colour[i] = c;
        gd->cellCount[c]++;
    }
    int32_t run = 0;
    for (int64_t c = 0; c < gd->total; ++c) {
        gd->cellStart[c] = gd->cellCount[c] ? run : -1;
        run += gd->cellCount[c];
    }
    /* stable placement in index order == sort by (colour, index) */
    int32_t *cursor = (int32_t *)calloc((size_t)gd->total, sizeof(int32_t));
    for (int64_t i = 0; i < n; ++i) {
        int64_t c = gd->colour[i];
        gd->order[gd->cellStart[c] + cursor[c]++] = (int32_t)i;
    }
    free(cursor);
}

static void SFX(grid_free)(SFX(grid) *gd) {
    free(gd->colour);
    free(gd->order);
    free(gd->cellStart);
    free(gd->cellCount);
}

/* NeighAccel::iterateBlocks filter (PLiB/Accel/NeighAccel.h:98-137) walked by
 * NeighbourGrid::iteratePossibleNeighbours (PLiB/NeighbourGrid.h:87-105). With
 * list == NULL only counts. */
static int SFX(neigh_row)(const SFX(grid) *gd, const double *x, const double *y,
                          const double *z, const LP *radius, int64_t p, double interactDist,
                          int32_t *row) {
    int count = 0;
    int colour = (int)gd->colour[p];
    double xc = x[p], yc = y[p], zc = z[p];
    for (int k = 0; k < 27; ++k) {
        int target = (int)(colour + gd->off[k]);
        if (target < 0 || (int64_t)target >= gd->total) continue;
        int32_t start = gd->cellStart[target];
        if (start < 0) continue;
        int32_t end = start + gd->cellCount[target];
        for (int32_t i = start; i < end; ++i) {
            int32_t q = gd->order[i];
            if (q == p) continue;
            LP xDist = (LP)(xc - x[q]);
            LP xDist2 = xDist * xDist;
            LP yDist = (LP)(yc - y[q]);
            LP yDist2 = yDist * yDist;
            LP zDist = (LP)(zc - z[q]);
            LP zDist2 = zDist * zDist;
            LP particleDistance2 = xDist2 + yDist2 + zDist2;
            LP particleDistance = LSQRT(particleDistance2);
            LP radSum = radius[p] + radius[q];
            LP dist = particleDistance - radSum;
            if ((double)dist < interactDist) {
                if (row) row[count] = q;
                ++count;
            }
        }
    }
    return count;
}

/* ------------------------------------------------------------- functors */

/* HiDEMDefNeighForceFunc::operator() (HiDEM/Common/HiDEMDefaultFunctions.h:21-87). */
static inline void SFX(contact)(const SFX(derived) *d, LP mask, LP xDist, LP yDist, LP zDist,
                                const LP *self, const LP *other, LP *F) {
    LP xDist2 = xDist * xDist;
    LP yDist2 = yDist * yDist;
    LP zDist2 = zDist * zDist;
    LP particleDistance2 = xDist2 + yDist2 + zDist2;
    LP radSum = self[6] + other[6];
    LP activeDist2 = (radSum + d->attractDistance) * (radSum + d->attractDistance);
    mask = (particleDistance2 >= activeDist2) ? (LP)0 : mask;
    LP particleDistance = LSQRT(particleDistance2);
    LP invDist = (LP)1 / particleDistance;
    LP xComp = xDist * invDist;
    LP yComp = yDist * invDist;
    LP zComp = zDist * invDist;
    LP Cnst = 0;
    LP dimDist = radSum - particleDistance;
    Cnst = (particleDistance < radSum) ? LSQRT(dimDist * dimDist * dimDist) : Cnst;
    Cnst = (particleDistance >= radSum && particleDistance < radSum + d->attractDistance)
               ? d->attractScaleForce * dimDist
               : Cnst;
    Cnst = Cnst * d->scaleE;
    F[0] = F[0] + mask * ((-d->damping) * ((self[0] - other[0]) * d->invDt) + (Cnst * xComp));
    F[1] = F[1] + mask * ((-d->damping) * ((self[1] - other[1]) * d->invDt) + (Cnst * yComp));
    F[2] = F[2] + mask * ((-d->damping) * ((self[2] - other[2]) * d->invDt) + (Cnst * zComp));
    F[3] = F[3] + mask * ((-d->dampingRotation) * ((self[3] - other[3]) * d->invDt));
    F[4] = F[4] + mask * ((-d->dampingRotation) * ((self[4] - other[4]) * d->invDt));
    F[5] = F[5] + mask * ((-d->dampingRotation) * ((self[5] - other[5]) * d->invDt));
}

/* HiDEMDefLinkForceFunc::operator() (HiDEMDefaultFunctions.h:90-204): damping,
 * link frame T, increments B, stiffness K, CT accumulation, force and moment. */
static inline void SFX(beam)(const SFX(derived) *d, LP mask, LP xDist, LP yDist, LP zDist,
                             const LP *s, const LP *o, LP *CT, LP *F) {
    F[0] = F[0] + (-d->damping * ((s[0] - o[0]) * d->invDt)) * mask;
    F[1] = F[1] + (-d->damping * ((s[1] - o[1]) * d->invDt)) * mask;
    F[2] = F[2] + (-d->damping * ((s[2] - o[2]) * d->invDt)) * mask;
    F[3] = F[3] + (-d->dampingRotation * ((s[3] - o[3]) * d->invDt)) * mask;
    F[4] = F[4] + (-d->dampingRotation * ((s[4] - o[4]) * d->invDt)) * mask;
    F[5] = F[5] + (-d->dampingRotation * ((s[5] - o[5]) * d->invDt)) * mask;

    LP xDist2 = xDist * xDist;
    LP yDist2 = yDist * yDist;
    if (xDist == 0 && yDist == 0) {
        xDist2 = (LP)1e-10;
        yDist2 = (LP)1e-10;
    }
    LP zDist2 = zDist * zDist;
    LP distSum = xDist2 + yDist2 + zDist2;
    LP invLI = (LP)1 / LSQRT(distSum);
    LP invLP = (LP)1 / LSQRT(xDist2 + yDist2);
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
    LP LIDiv6 = ((LP)1 / (LP)6) * invLI;
    LP K0 = d->E * d->W2 * invLI;
    LP K1 = d->E * d->W4 / L3;
    LP K5 = d->E * d->W4 / ((LP)2 * L2);

    CT[0] = CT[0] + (K0 * B0 + (-K0) * B6);
    CT[1] = CT[1] + (K1 * B1 + K5 * B5 + (-K1) * B7 + K5 * B11);
    CT[2] = CT[2] + (K1 * B2 + (-K5) * B4 + (-K1) * B8 + (-K5) * B10);

    F[0] = F[0] + (-(T00 * CT[0] + T10 * CT[1] + T20 * CT[2])) * mask;
    F[1] = F[1] + (-(T01 * CT[0] + T11 * CT[1] + T21 * CT[2])) * mask;
    F[2] = F[2] + (-(T02 * CT[0] + T22 * CT[2])) * mask;

    LP K2 = d->G * d->W4 * LIDiv6;
    LP K3 = d->E * d->W4 * LIDiv6 * (LP)2;
    LP K4 = d->E * d->W4 * LIDiv6;
    LP B3 = T00 * s[3] + T01 * s[4] + T02 * s[5];
    LP B9 = T00 * o[3] + T01 * o[4] + T02 * o[5];

    CT[3] = CT[3] + (K2 * B3 + (-K2) * B9);
    CT[4] = CT[4] + ((-K5) * B2 + K3 * B4 + K5 * B8 + K4 * B10);
    CT[5] = CT[5] + (K5 * B1 + K3 * B5 + (-K5) * B7 + K4 * B11);

    F[3] = F[3] + (-(T00 * CT[3] + T10 * CT[4] + T20 * CT[5])) * mask;
    F[4] = F[4] + (-(T01 * CT[3] + T11 * CT[4] + T21 * CT[5])) * mask;
    F[5] = F[5] + (-(T02 * CT[3] + T22 * CT[5])) * mask;
}

/* The IceBlock sample's own link functor (HiDEM/IceBlock/MainIceBlock.cpp:173-262), the
 * variant a caller passes through the templated computePartForce: no guard for exactly
 * vertical links, LI and LP as square roots, invLILP = 1 / (LI * LP), LIDiv6 =
 * 1 / (6 * LI); the rest as the default functor. */
static inline void SFX(beam_iceblock)(const SFX(derived) *d, LP mask, LP xDist, LP yDist, LP zDist,
                                      const LP *s, const LP *o, LP *CT, LP *F) {
    F[0] = F[0] + (-d->damping * ((s[0] - o[0]) * d->invDt)) * mask;
    F[1] = F[1] + (-d->damping * ((s[1] - o[1]) * d->invDt)) * mask;
    F[2] = F[2] + (-d->damping * ((s[2] - o[2]) * d->invDt)) * mask;
    F[3] = F[3] + (-d->dampingRotation * ((s[3] - o[3]) * d->invDt)) * mask;
    F[4] = F[4] + (-d->dampingRotation * ((s[4] - o[4]) * d->invDt)) * mask;
    F[5] = F[5] + (-d->dampingRotation * ((s[5] - o[5]) * d->invDt)) * mask;
    LP xDist2 = xDist * xDist;
    LP yDist2 = yDist * yDist;
    LP zDist2 = zDist * zDist;
    LP LI = LSQRT(xDist2 + yDist2 + zDist2);
    LP LPl = LSQRT(xDist2 + yDist2);
    LP invLI = (LP)1 / LI;
    LP invLP = (LP)1 / LPl;
    LP invLILP = (LP)1 / (LI * LPl);
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
    LP LIDiv6 = (LP)1 / ((LP)6 * LI);
    LP K0 = d->E * d->W2 * invLI;
    LP K1 = d->E * d->W4 / L3;
    LP K5 = d->E * d->W4 / ((LP)2 * L2);
    CT[0] = CT[0] + (K0 * B0 + (-K0) * B6);
    CT[1] = CT[1] + (K1 * B1 + K5 * B5 + (-K1) * B7 + K5 * B11);
    CT[2] = CT[2] + (K1 * B2 + (-K5) * B4 + (-K1) * B8 + (-K5) * B10);
    F[0] = F[0] + (-(T00 * CT[0] + T10 * CT[1] + T20 * CT[2])) * mask;
    F[1] = F[1] + (-(T01 * CT[0] + T11 * CT[1] + T21 * CT[2])) * mask;
    F[2] = F[2] + (-(T02 * CT[0] + T22 * CT[2])) * mask;
    LP K2 = d->G * d->W4 * LIDiv6;
    LP K3 = d->E * d->W4 * LIDiv6 * (LP)2;
    LP K4 = d->E * d->W4 * LIDiv6;
    LP B3 = T00 * s[3] + T01 * s[4] + T02 * s[5];
    LP B9 = T00 * o[3] + T01 * o[4] + T02 * o[5];
    CT[3] = CT[3] + (K2 * B3 + (-K2) * B9);
    CT[4] = CT[4] + ((-K5) * B2 + K3 * B4 + K5 * B8 + K4 * B10);
    CT[5] = CT[5] + (K5 * B1 + K3 * B5 + (-K5) * B7 + K4 * B11);
    F[3] = F[3] + (-(T00 * CT[3] + T10 * CT[4] + T20 * CT[5])) * mask;
    F[4] = F[4] + (-(T01 * CT[3] + T11 * CT[4] + T21 * CT[5])) * mask;
    F[5] = F[5] + (-(T02 * CT[3] + T22 * CT[5])) * mask;
}

/* HiDEMDefLinkBreakFunc::operator() (HiDEMDefaultFunctions.h:207-242). Returns the
 * new state. */
static inline uint8_t SFX(break_test)(const SFX(derived) *d, double x1, double y1, double z1,
                                      LP tx1, LP ty1, LP tz1, double x2, double y2, double z2,
                                      LP tx2, LP ty2, LP tz2, uint8_t state, LP initialLen) {
    if (state == 0) return 0;
    LP xDist = (LP)(x1 - x2);
    LP yDist = (LP)(y1 - y2);
    LP zDist = (LP)(z1 - z2);
    LP stretchLength = LSQRT((xDist * xDist) + (yDist * yDist) + (zDist * zDist));
    LP ax = LABS(tx1 - tx2), ay = LABS(ty1 - ty2), az = LABS(tz1 - tz2);
    LP myz = (ay < az) ? az : ay;   /* std::max(a, b) == (a < b) ? b : a */
    LP maxBend = (ax < myz) ? myz : ax;
    LP load = (stretchLength - initialLen) / initialLen + d->bendBreak * maxBend;
    if (load >= d->maxLoad) return 0;
    return state;
}

/* --------------------------------------------------------- public entries */

/* Map2d::interp (PLiB/Geometry/Map2d.h:113-152) with getIndexes (93-111) and the
 * constructor's float grid metrics (43-58): bilinear, float arithmetic, clamped. */
static LP SFX(map_interp)(const hidem_map2d *m, float x, float y) {
    const LP *d = (const LP *)m->data;
    const float xRes = (m->x_max - m->x_min) / (float)(m->x_points - 1);
    const float yRes = (m->y_max - m->y_min) / (float)(m->y_points - 1);
    const float invX = 1.0f / (m->x_max - m->x_min);
    const float invY = 1.0f / (m->y_max - m->y_min);
    float fx = floorf(((x - m->x_min) * invX) * (float)(m->x_points - 1));
    float fy = floorf(((y - m->y_min) * invY) * (float)(m->y_points - 1));
    fx = fminf(fmaxf(fx, -1.0f), (float)m->x_points);
    fy = fminf(fmaxf(fy, -1.0f), (float)m->y_points);
    int xp = (int)fx, yp = (int)fy;
    int xl = clampi_(xp, 0, m->x_points - 1), yl = clampi_(yp, 0, m->y_points - 1);
    int xh = clampi_(xp + 1, 0, m->x_points - 1), yh = clampi_(yp + 1, 0, m->y_points - 1);
    if (xl == xh && yl == yh) return d[xl + yl * m->x_points];
    float v00 = (float)d[xl + yl * m->x_points], v01 = (float)d[xl + yh * m->x_points];
    float v10 = (float)d[xh + yl * m->x_points], v11 = (float)d[xh + yh * m->x_points];
    float x0 = x - m->x_min, y0 = y - m->y_min;
    float x1 = (float)xl * xRes, x2 = (float)xh * xRes, y1 = (float)yl * yRes, y2 = (float)yh * yRes;
    float invX21 = 1.0f / (x2 - x1);
    float c1 = (x2 - x0) * invX21, c2 = (x0 - x1) * invX21;
    float fxy1 = (c1 * v00) + (c2 * v10), fxy2 = (c1 * v01) + (c2 * v11);
    if (xl == xh) {
        fxy1 = v00;
        fxy2 = v01;
    } else if (yl == yh) {
        return (LP)fxy1;
    }
    float invY21 = 1.0f / (y2 - y1);
    return (LP)((((y2 - y0) * invY21) * fxy1) + (((y0 - y1) * invY21) * fxy2));
}

static void SFX(get_particle_arrays)(const hidem_particle_soa *p, const LP **th, const LP **df,
                                     const LP **rad) {
    th[0] = (const LP *)p->xTheta;
    th[1] = (const LP *)p->yTheta;
    th[2] = (const LP *)p->zTheta;
    df[0] = (const LP *)p->xDiff;
    df[1] = (const LP *)p->yDiff;
    df[2] = (const LP *)p->zDiff;
    df[3] = (const LP *)p->uDiff;
    df[4] = (const LP *)p->vDiff;
    df[5] = (const LP *)p->wDiff;
    *rad = (const LP *)p->radius;
}

static int SFX(cells)(const hidem_params *P, const hidem_particle_soa *p, int64_t n, int32_t *ix,
                      int32_t *iy, int32_t *iz, int64_t dims[3], double mins[3]) {
    SFX(derived) d = SFX(derive)(P);
    SFX(grid) gd;
    SFX(grid_build)(&gd, p->xCord, p->yCord, p->zCord, n, d.searchDistance);
    for (int64_t i = 0; i < n; ++i) {
        int64_t c = gd.colour[i];
        ix[i] = (int32_t)(c % gd.X);
        iy[i] = (int32_t)((c / gd.X) % gd.Y);
        iz[i] = (int32_t)(c / ((int64_t)gd.X * gd.Y));
    }
    dims[0] = gd.X;
    dims[1] = gd.Y;
    dims[2] = gd.Z;
    mins[0] = gd.xMin;
    mins[1] = gd.yMin;
    mins[2] = gd.zMin;
    SFX(grid_free)(&gd);
    return 0;
}

static int SFX(neighbours)(const hidem_params *P, const hidem_particle_soa *p, int64_t n,
                           int32_t *counts, int32_t *list, int64_t cap, int64_t *total) {
    SFX(derived) d = SFX(derive)(P);
    SFX(grid) gd;
    SFX(grid_build)(&gd, p->xCord, p->yCord, p->zCord, n, d.searchDistance);
    const LP *rad = (const LP *)p->radius;
    int64_t off = 0;
    /* one row at a time; rows longer than the buffer are refused (a crowded cell of a few
       thousand particles still fits) */
    static _Thread_local int32_t row[16384];
    int rc = 0;
    for (int64_t i = 0; i < n; ++i) {
        int c = SFX(neigh_row)(&gd, p->xCord, p->yCord, p->zCord, rad, i, d.interactDist, NULL);
        counts[i] = c;
        if (list) {
            if (c > 16384) { rc = HIDEM_ERR_CAPACITY; break; }
            SFX(neigh_row)(&gd, p->xCord, p->yCord, p->zCord, rad, i, d.interactDist, row);
            for (int k = 0; k < c; ++k) {
                if (off + k < cap) list[off + k] = row[k];
            }
        }
        off += c;
    }
    *total = off;
    SFX(grid_free)(&gd);
    if (list && off > cap) rc = HIDEM_ERR_CAPACITY;
    return rc;
}

/* Link ends of one particle, in ascending link index: the result of
 * LinkAccelSide::generateLinks + generatePerParticleIndexes
 * (PLiB/Accel/LinkAccelSide.h:43-143): (link, other particle, side index). */
typedef struct SFX(adj) {
    int32_t *start;  /* n+1 */
    int32_t *link, *other, *side;
} SFX(adj);

static void SFX(adj_build)(SFX(adj) *a, const int32_t *pA, const int32_t *pB, int64_t n,
                           int64_t L) {
    a->start = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
    for (int64_t l = 0; l < L; ++l) {
        a->start[pA[l] + 1]++;
        a->start[pB[l] + 1]++;
    }
    for (int64_t i = 0; i < n; ++i) a->start[i + 1] += a->start[i];
    a->link = (int32_t *)malloc(sizeof(int32_t) * (size_t)(2 * L + 1));
    a->other = (int32_t *)malloc(sizeof(int32_t) * (size_t)(2 * L + 1));
    a->side = (int32_t *)malloc(sizeof(int32_t) * (size_t)(2 * L + 1));
    int32_t *cur = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    /* links visited in ascending index: each particle's ends come out sorted */
    for (int64_t l = 0; l < L; ++l) {
        int32_t a0 = pA[l], b0 = pB[l];
        int32_t ia = a->start[a0] + cur[a0]++;
        a->link[ia] = (int32_t)l;
        a->other[ia] = b0;
        a->side[ia] = (int32_t)(2 * l);
        int32_t ib = a->start[b0] + cur[b0]++;
        a->link[ib] = (int32_t)l;
        a->other[ib] = a0;
        a->side[ib] = (int32_t)(2 * l + 1);
    }
    free(cur);
}

static void SFX(adj_free)(SFX(adj) *a) {
    free(a->start);
    free(a->link);
    free(a->other);
    free(a->side);
}

/* ------------------------------------------------------------ collision mesh */

/* MeshAccel grid of a collision mesh (PLiB/Geometry/MeshAccel.h:15-47) */
typedef struct SFX(mesh_accel) {
    LP xLower, yLower, zLower, xUpper, yUpper, zUpper, xInv, yInv, zInv, cellSize, maxDist;
    int xCount, yCount, zCount;
    int64_t cells, nvalues;
    int32_t *sizes, *starts, *values;
} SFX(mesh_accel);

/* MeshAccel::triSDF2 (MeshAccel.h:329-372) in Real3f arithmetic (PLiB/Util/Real3.h:
 * 142-258): float components, dot summed left to right; the edge parameter clamped in
 * lp (clamp3 / clamp, PLiB/Util/Util.h:245-253); std::min(a, b) == (b < a) ? b : a. */
static float SFX(tri_edge2)(v3f e, v3f q) {
    float t = v3f_dot(e, q) / v3f_dot(e, e);
    LP tl = (LP)t;
    tl = tl < (LP)0 ? (LP)0 : (tl > (LP)1 ? (LP)1 : tl);
    float tc = (float)tl;
    v3f dd = v3f_sub(v3f_mul(e, (v3f){tc, tc, tc}), q);
    return v3f_dot(dd, dd);
}

static LP SFX(tri_sdf2)(v3f pt, v3f a, v3f b, v3f c) {
    v3f ba = v3f_sub(b, a), pa = v3f_sub(pt, a), cb = v3f_sub(c, b), pb = v3f_sub(pt, b);
    v3f ac = v3f_sub(a, c), pc = v3f_sub(pt, c);
    v3f nor = v3f_cross(ba, ac);
    float sg = sign_f(v3f_dot(v3f_cross(ba, nor), pa)) + sign_f(v3f_dot(v3f_cross(cb, nor), pb)) +
               sign_f(v3f_dot(v3f_cross(ac, nor), pc));
    if (sg < 2.0f) {
        float e1 = SFX(tri_edge2)(ba, pa), e2 = SFX(tri_edge2)(cb, pb), e3 = SFX(tri_edge2)(ac, pc);
        float m12 = (e2 < e1) ? e2 : e1;
        return (LP)((e3 < m12) ? e3 : m12);
    }
    float dn = v3f_dot(nor, pa);
    return (LP)(dn * dn / v3f_dot(nor, nor));
}

static v3f SFX(mesh_vtx)(const hidem_mesh *m, int64_t i) {
    const LP *vx = (const LP *)m->x_vertex, *vy = (const LP *)m->y_vertex, *vz = (const LP *)m->z_vertex;
    v3f r = {(float)vx[i], (float)vy[i], (float)vz[i]};
    return r;
}

/* MeshAccel::getCell / getCellCord (MeshAccel.h:295-316): the point as Real3f, the
 * lower corner subtracted in lp and stored back to float, times the inverse cell size in
 * lp, truncated; -1 outside the grid. */
static int SFX(mesh_cell)(const SFX(mesh_accel) *A, LP x, LP y, LP z) {
    float cx = (float)((LP)(float)x - A->xLower);
    float cy = (float)((LP)(float)y - A->yLower);
    float cz = (float)((LP)(float)z - A->zLower);
    int xc = (int)((LP)cx * A->xInv), yc = (int)((LP)cy * A->yInv), zc = (int)((LP)cz * A->zInv);
    if (xc < 0 || yc < 0 || zc < 0 || xc >= A->xCount || yc >= A->yCount || zc >= A->zCount) return -1;
    return (xc * A->yCount * A->zCount) + (yc * A->zCount) + zc;
}

/* MeshAccel::generateAccel (MeshAccel.h:57-165): bounding box of the vertices grown by one
 * cell, 1 + size / cellSize cells per axis (z fastest), and per cell the triangles whose
 * triSDF2 from the cell centre is below 3 cellSize^2 + cellSize, ascending. */
static void SFX(mesh_build)(const hidem_mesh *m, SFX(mesh_accel) *A) {
    const LP *vx = (const LP *)m->x_vertex, *vy = (const LP *)m->y_vertex, *vz = (const LP *)m->z_vertex;
    LP hi = sizeof(LP) == 4 ? (LP)FLT_MAX : (LP)DBL_MAX;
    LP xU = -hi, yU = -hi, zU = -hi, xL = hi, yL = hi, zL = hi;
    for (int64_t i = 0; i < 3 * (int64_t)m->triangles; ++i) {
        xU = (vx[i] < xU) ? xU : vx[i];
        xL = (xL < vx[i]) ? xL : vx[i];
        yU = (vy[i] < yU) ? yU : vy[i];
        yL = (yL < vy[i]) ? yL : vy[i];
        zU = (vz[i] < zU) ? zU : vz[i];
        zL = (zL < vz[i]) ? zL : vz[i];
    }
    LP cs = (LP)m->cell_size;
    A->xUpper = xU + cs;
    A->yUpper = yU + cs;
    A->zUpper = zU + cs;
    A->xLower = xL - cs;
    A->yLower = yL - cs;
    A->zLower = zL - cs;
    LP xSize = A->xUpper - A->xLower, ySize = A->yUpper - A->yLower, zSize = A->zUpper - A->zLower;
    A->cellSize = cs;
    A->xInv = (LP)1.0f / cs;
    A->yInv = (LP)1.0f / cs;
    A->zInv = (LP)1.0f / cs;
    A->xCount = (int)((LP)1 + xSize / cs);
    A->yCount = (int)((LP)1 + ySize / cs);
    A->zCount = (int)((LP)1 + zSize / cs);
    A->maxDist = (cs * cs) + (cs * cs) + (cs * cs) + cs;
    A->cells = (int64_t)A->xCount * A->yCount * A->zCount;
    A->sizes = (int32_t *)calloc((size_t)A->cells, sizeof(int32_t));
    A->starts = (int32_t *)calloc((size_t)A->cells, sizeof(int32_t));
    for (int pass = 0; pass < 2; ++pass) {
        for (int x = 0; x < A->xCount; ++x)
            for (int y = 0; y < A->yCount; ++y)
                for (int zz = 0; zz < A->zCount; ++zz) {
                    LP half = (LP)0.5f * cs;
                    LP xPos = ((LP)x * cs + half) + A->xLower;
                    LP yPos = ((LP)y * cs + half) + A->yLower;
                    LP zPos = ((LP)zz * cs + half) + A->zLower;
                    int cell = SFX(mesh_cell)(A, xPos, yPos, zPos);
                    if (cell < 0) continue;
                    v3f pt = {(float)xPos, (float)yPos, (float)zPos};
                    int found = 0;
                    for (int i = 0; i < m->triangles; ++i) {
                        LP dd = SFX(tri_sdf2)(pt, SFX(mesh_vtx)(m, 3 * (int64_t)i), SFX(mesh_vtx)(m, 3 * (int64_t)i + 1),
                                              SFX(mesh_vtx)(m, 3 * (int64_t)i + 2));
                        if (dd < A->maxDist) {
                            if (pass == 1) A->values[A->starts[cell] + found] = i;
                            ++found;
                        }
                    }
                    if (pass == 0) A->sizes[cell] = found;
                }
        if (pass == 0) {
            int64_t acc = 0;
            for (int64_t c = 0; c < A->cells; ++c) {
                A->starts[c] = (int32_t)acc;
                acc += A->sizes[c];
            }
            A->nvalues = acc;
            A->values = (int32_t *)malloc(sizeof(int32_t) * (size_t)(acc + 1));
        }
    }
}

static void SFX(mesh_free)(SFX(mesh_accel) *A) {
    free(A->sizes);
    free(A->starts);
    free(A->values);
}

/* MeshAccel::getClosestTriAccel (MeshAccel.h:375-412) as Mesh::closestTriFun calls it
 * (Mesh.h:69-83): the closest triangle of the point's cell within interactDist, or -1. */
static int SFX(mesh_closest)(const hidem_mesh *m, const SFX(mesh_accel) *A, LP x, LP y, LP z,
                             LP interactDist, LP *dist2) {
    if (x > A->xUpper || y > A->yUpper || z > A->zUpper || x < A->xLower || y < A->yLower || z < A->zLower)
        return -1;
    int cell = SFX(mesh_cell)(A, x, y, z);
    if (cell < 0) return -1;
    v3f pt = {(float)x, (float)y, (float)z};
    LP id2 = interactDist * interactDist;
    LP minDist = sizeof(LP) == 4 ? (LP)FLT_MAX : (LP)DBL_MAX;
    int closest = -1;
    for (int32_t i = A->starts[cell]; i < A->starts[cell] + A->sizes[cell]; ++i) {
        int tri = A->values[i];
        LP cur = SFX(tri_sdf2)(pt, SFX(mesh_vtx)(m, 3 * (int64_t)tri), SFX(mesh_vtx)(m, 3 * (int64_t)tri + 1),
                               SFX(mesh_vtx)(m, 3 * (int64_t)tri + 2));
        if (id2 > cur && cur < minDist) {
            minDist = cur;
            closest = tri;
        }
    }
    *dist2 = minDist;
    return closest;
}

static int SFX(run)(const hidem_params *P, hidem_particle_soa *p, int64_t n, hidem_link_soa *l,
                    int64_t L, int64_t start_step, int32_t nsteps, void *force_out[6],
                    int64_t *ev_link, int64_t *ev_step, int64_t ev_cap, int64_t *ev_count,
                    int64_t *regen_steps, int64_t regen_cap, int64_t *regen_count,
                    double *seconds) {
    const SFX(derived) d = SFX(derive)(P);
    double *x = p->xCord, *y = p->yCord, *z = p->zCord;
    LP *th[3] = {(LP *)p->xTheta, (LP *)p->yTheta, (LP *)p->zTheta};
    LP *df[6] = {(LP *)p->xDiff, (LP *)p->yDiff, (LP *)p->zDiff,
                 (LP *)p->uDiff, (LP *)p->vDiff, (LP *)p->wDiff};
    const LP *rad = (const LP *)p->radius;
    const uint8_t *type = p->type;
    LP *F = (LP *)calloc((size_t)(6 * n), sizeof(LP));
    uint8_t *state = l->state;
    const LP *L0 = (const LP *)l->initialLen;
    LP *CT = (LP *)calloc((size_t)(12 * L + 1), sizeof(LP)); /* side-major: CT[side*6 + k] */
    if (l->CT[0]) {
        for (int k = 0; k < 6; ++k) {
            const LP *src = (const LP *)l->CT[k];
            for (int64_t s = 0; s < 2 * L; ++s) CT[s * 6 + k] = src[s];
        }
    }

    /* link ends -> input particle indices by globalKey (LinkData::makeLocalPartEnds,
     * PLiB/LinkData.h:91-115) */
    int32_t *pA = (int32_t *)malloc(sizeof(int32_t) * (size_t)(L + 1));
    int32_t *pB = (int32_t *)malloc(sizeof(int32_t) * (size_t)(L + 1));
    {
        int64_t kmax = 0;
        for (int64_t i = 0; i < n; ++i)
            if (p->globalKeys[i] > kmax) kmax = p->globalKeys[i];
        int32_t *lookup = (int32_t *)malloc(sizeof(int32_t) * (size_t)(kmax + 1));
        for (int64_t k = 0; k <= kmax; ++k) lookup[k] = -1;
        for (int64_t i = 0; i < n; ++i) lookup[p->globalKeys[i]] = (int32_t)i;
        for (int64_t i = 0; i < L; ++i) {
            int64_t a = l->globalKeyEndA[i], b = l->globalKeyEndB[i];
            if (a < 0 || a > kmax || b < 0 || b > kmax || lookup[a] < 0 || lookup[b] < 0) {
                free(lookup);
                free(pA);
                free(pB);
                free(F);
                free(CT);
                return HIDEM_ERR_NOT_FOUND;
            }
            pA[i] = lookup[a];
            pB[i] = lookup[b];
        }
        free(lookup);
    }
    SFX(adj) adj;
    SFX(adj_build)(&adj, pA, pB, n, L);

    int32_t *ncount = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    int32_t *nstart = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
    int32_t *nlist = NULL;
    double accumulatedDist = 0;
    int64_t nev = 0, nregen = 0;
    const int useFixed = P->useFixed, useFront = P->useFrontPressure, useBed = P->useBed;
    const int useVel = P->useVelocityLimit, useBnd = P->useBoundary;
    /* collision mesh: MeshAccel grid, face force sums (of this run, in particle order) and
     * the per-particle contribution of the current step */
    SFX(mesh_accel) macc;
    memset(&macc, 0, sizeof macc);
    int32_t *mtri = NULL;
    LP *mcol = NULL, *mface = NULL;
    if (g_mesh_set) {
        SFX(mesh_build)(&g_mesh, &macc);
        mtri = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
        mcol = (LP *)malloc(sizeof(LP) * 3 * (size_t)n);
        mface = (LP *)calloc(3 * (size_t)g_mesh.triangles, sizeof(LP));
    }
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);

    for (int64_t t = start_step; t < start_step + nsteps; ++t) {
        /* ---- gridService (HiDEMLib/HiDEMLib.h:533-628) ---- */
        int regen = (t == start_step);
        if (P->gridRegenInterval != -1) {
            regen = (t % P->gridRegenInterval) == 0;
        } else if (t % 10 == 0) {
            /* accumulateDist / getMaxDistOwned (HiDEMLib.h:424-474) */
            double mx = 0.0, my = 0.0, mz = 0.0;
            for (int64_t i = 0; i < n; ++i) {
                double a = df[0][i], b = df[1][i], c = df[2][i];
                if (a > mx) mx = a;
                if (b > my) my = b;
                if (c > mz) mz = c;
            }
            LP xM = (LP)mx, yM = (LP)my, zM = (LP)mz;
            LP root = LSQRT((xM * xM) + (yM * yM) + (zM * zM));
            double currDist = (double)((LP)10 * root);
            accumulatedDist += currDist;
            if (accumulatedDist >= d.interactDist / 2.0) regen = 1;
        }
        if (t == P->firstBalanceTimestep) regen = 1;
        if (regen) {
            accumulatedDist = 0;
            SFX(grid) gd;
            SFX(grid_build)(&gd, x, y, z, n, d.searchDistance);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i)
                ncount[i] = SFX(neigh_row)(&gd, x, y, z, rad, i, d.interactDist, NULL);
            for (int64_t i = 0; i < n; ++i) nstart[i + 1] = nstart[i] + ncount[i];
            free(nlist);
            nlist = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nstart[n] + 1));
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i)
                SFX(neigh_row)(&gd, x, y, z, rad, i, d.interactDist, nlist + nstart[i]);
            SFX(grid_free)(&gd);
            if (regen_steps && nregen < regen_cap) regen_steps[nregen] = t;
            ++nregen;
        }
        if (t == start_step) clock_gettime(CLOCK_MONOTONIC, &t0); /* time excludes the first rebuild */

        /* ---- computePartForce: CombinedAccel::iterateCombined
         *      (PLiB/Accel/CombinedAccel.h:122-197) ---- */
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            LP f[6] = {0, 0, 0, 0, 0, 0};
            LP self[7], other[7];
            for (int k = 0; k < 6; ++k) self[k] = df[k][i];
            self[6] = rad[i];
            double xc = x[i], yc = y[i], zc = z[i];
            for (int32_t k = nstart[i]; k < nstart[i + 1]; ++k) {
                int32_t q = nlist[k];
                for (int c = 0; c < 6; ++c) other[c] = df[c][q];
                other[6] = rad[q];
                SFX(contact)(&d, (LP)1, (LP)(xc - x[q]), (LP)(yc - y[q]), (LP)(zc - z[q]), self,
                             other, f);
            }
            for (int32_t k = adj.start[i]; k < adj.start[i + 1]; ++k) {
                int32_t q = adj.other[k];
                for (int c = 0; c < 6; ++c) other[c] = df[c][q];
                other[6] = rad[q];
                LP mask = state[adj.link[k]] == 0 ? (LP)0 : (LP)1;
                if (g_link_variant == 1)
                    SFX(beam_iceblock)(&d, mask, (LP)(xc - x[q]), (LP)(yc - y[q]), (LP)(zc - z[q]), self,
                                       other, CT + (int64_t)adj.side[k] * 6, f);
                else
                    SFX(beam)(&d, mask, (LP)(xc - x[q]), (LP)(yc - y[q]), (LP)(zc - z[q]), self, other,
                              CT + (int64_t)adj.side[k] * 6, f);
            }
            for (int c = 0; c < 6; ++c) F[c * n + i] = f[c];
        }

        /* ---- applyForce: the sample integrate lambda (MainMeshBlock.cpp:182-261,
         *      bed terms MainDem.cpp:176-207, fixed / front extensions) ---- */
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            uint8_t ty = type ? type[i] : 0;
            if (mtri) mtri[i] = -1;
            if (useFixed && (ty & HIDEM_TYPE_FIXED)) {
                for (int c = 0; c < 6; ++c) df[c][i] = 0;
                continue;
            }
            double xCord = x[i], yCord = y[i], zCord = z[i];
            LP xDiff = df[0][i], yDiff = df[1][i], zDiff = df[2][i];
            LP uDiff = df[3][i], vDiff = df[4][i], wDiff = df[5][i];
            LP xTheta = th[0][i], yTheta = th[1][i], zTheta = th[2][i];
            LP radius = rad[i];
            LP diameter = radius * (LP)2;
            LP bedHeight = d.bedHeight, bedFriction = d.bedFriction;
            if (useBed && g_map_set[0]) bedHeight = SFX(map_interp)(&g_maps[0], (float)xCord, (float)yCord);
            LP dragCoeff;
            if (useBed && ((zCord + (double)radius) - (double)bedHeight < (double)d.bedInteract)) {
                if (g_map_set[1]) bedFriction = SFX(map_interp)(&g_maps[1], (float)xCord, (float)yCord);
                LP a = d.bedDrag * bedFriction;
                LP b = (LP)1e+5 * d.scale * d.scale;
                dragCoeff = (b < a) ? b : a; /* std::min(a, b) */
            } else if (zCord > (double)d.waterLevel) {
                dragCoeff = d.airDrag;
            } else {
                dragCoeff = d.waterDrag;
            }
            LP xForce = F[0 * n + i], yForce = F[1 * n + i], zForce = F[2 * n + i];
            LP uForce = F[3 * n + i], vForce = F[4 * n + i], wForce = F[5 * n + i];
            LP particleMass = d.rhoIce * diameter * diameter * diameter;
            LP particleMomentInertia = particleMass * diameter * diameter / (LP)6;
            if (zCord > (double)d.waterLevel) zForce = zForce + -d.g * particleMass;
            if (zCord <= (double)d.waterLevel) zForce = zForce + d.lift * particleMass;
            if (useBed && zCord + (double)radius < (double)bedHeight)
                zForce = (LP)((double)zForce +
                              (double)d.bedStiffness * ((double)bedHeight - (zCord + (double)radius)));
            /* collision mesh (HiDEM/MeshConstrainedDem/MainMeshDem.cpp:220-235) */
            if (g_mesh_set) {
                LP dist2 = 0;
                int tri = SFX(mesh_closest)(&g_mesh, &macc, (LP)xCord, (LP)yCord, (LP)zCord,
                                            d.bedInteract + radius, &dist2);
                mtri[i] = tri;
                if (tri >= 0) {
                    const LP *nx = (const LP *)g_mesh.x_normal, *ny = (const LP *)g_mesh.y_normal;
                    const LP *nz = (const LP *)g_mesh.z_normal;
                    float maxDist = (float)(d.bedInteract + radius);
                    LP dist = LSQRT(dist2);
                    LP mForce = (LP)g_mesh.mesh_force, mDrag = (LP)g_mesh.mesh_drag;
                    dragCoeff = mDrag * ((LP)maxDist - dist);
                    LP fx = -nx[tri] * ((LP)maxDist - dist) * mForce;
                    LP fy = -ny[tri] * ((LP)maxDist - dist) * mForce;
                    LP fz = -nz[tri] * ((LP)maxDist - dist) * mForce;
                    mcol[3 * i] = fx;
                    mcol[3 * i + 1] = fy;
                    mcol[3 * i + 2] = fz;
                    xForce = xForce + fx;
                    yForce = yForce + fy;
                    zForce = zForce + fz;
                }
            }
            /* external force maps (MainDem.cpp:211-216) */
            if (g_map_set[2]) {
                float fx = (float)xCord, fy = (float)yCord;
                xForce = xForce + SFX(map_interp)(&g_maps[2], fx, fy);
                yForce = yForce + SFX(map_interp)(&g_maps[3], fx, fy);
                zForce = zForce + SFX(map_interp)(&g_maps[4], fx, fy);
                uForce = uForce + SFX(map_interp)(&g_maps[5], fx, fy);
                vForce = vForce + SFX(map_interp)(&g_maps[6], fx, fy);
                wForce = wForce + SFX(map_interp)(&g_maps[7], fx, fy);
            }
            if (useFront && (ty & HIDEM_TYPE_FRONT) && zCord < (double)d.waterLevel) {
                LP depth = (LP)((double)d.waterLevel - zCord);
                xForce = xForce - d.rhoWater * d.g * depth * diameter * diameter;
            }
            /* HiDEMDefTimeIntegration (HiDEMDefaultFunctions.h:318-370) */
            LP dragInvDt2 = dragCoeff * d.invDt2;
            LP massDtSqr = particleMass * d.invDtSqr;
            LP pMassDtSqr = particleMass / d.dtSqr;
            LP pMemDtSqr = particleMomentInertia / d.dtSqr;
            LP invC1 = (LP)1 / (pMassDtSqr + dragCoeff * d.invDt2);
            LP invC2 = (LP)1 / (pMemDtSqr + dragCoeff * d.invDt2);
            LP interDtSqr = particleMomentInertia * d.invDtSqr;
            LP xDN = (xForce + massDtSqr * xDiff + dragInvDt2 * -xDiff) * invC1;
            LP yDN = (yForce + massDtSqr * yDiff + dragInvDt2 * -yDiff) * invC1;
            LP zDN = (zForce + massDtSqr * zDiff + dragInvDt2 * -zDiff) * invC1;
            LP uDN = (uForce + interDtSqr * uDiff + dragInvDt2 * -uDiff) * invC2;
            LP vDN = (vForce + interDtSqr * vDiff + dragInvDt2 * -vDiff) * invC2;
            LP wDN = (wForce + interDtSqr * wDiff + dragInvDt2 * -wDiff) * invC2;
            double xPrev = xCord, yPrev = yCord, zPrev = zCord;
            LP xThPrev = xTheta, yThPrev = yTheta, zThPrev = zTheta;
            xCord = xCord + (double)xDN;
            yCord = yCord + (double)yDN;
            zCord = zCord + (double)zDN;
            xTheta = xTheta + uDN;
            yTheta = yTheta + vDN;
            zTheta = zTheta + wDN;
            if (useVel) {
                /* HiDEMDefVelocityLimit (HiDEMDefaultFunctions.h:245-290) */
                LP xVel = xDN * d.invDt, yVel = yDN * d.invDt, zVel = zDN * d.invDt;
                LP xTV = (xTheta - xThPrev) * d.invDt, yTV = (yTheta - yThPrev) * d.invDt;
                LP zTV = (zTheta - zThPrev) * d.invDt;
                if (xVel > d.maxVel) xCord = (double)(d.dt * d.maxVel) + xPrev;
                if (yVel > d.maxVel) yCord = (double)(d.dt * d.maxVel) + yPrev;
                if (zVel > d.maxVel) zCord = (double)(d.dt * d.maxVel) + zPrev;
                if (xTV > d.maxRot) xTheta = d.dt * d.maxRot + xThPrev;
                if (yTV > d.maxRot) yTheta = d.dt * d.maxRot + yThPrev;
                if (zTV > d.maxRot) zTheta = d.dt * d.maxRot + zThPrev;
                if (xVel < -d.maxVel) xCord = (double)(d.dt * -d.maxVel) + xPrev;
                if (yVel < -d.maxVel) yCord = (double)(d.dt * -d.maxVel) + yPrev;
                if (zVel < -d.maxVel) zCord = (double)(d.dt * -d.maxVel) + zPrev;
                if (xTV < -d.maxRot) xTheta = d.dt * -d.maxRot + xThPrev;
                if (yTV < -d.maxRot) yTheta = d.dt * -d.maxRot + yThPrev;
                if (zTV < -d.maxRot) zTheta = d.dt * -d.maxRot + zThPrev;
            }
            if (useBnd) {
                /* HiDEMDefBoundaryCondition (HiDEMDefaultFunctions.h:293-315) */
                if (xCord + (double)radius < P->lowerLimit[0] && P->boundaryMin[0]) xCord = xPrev;
                if (xCord - (double)radius > P->upperLimit[0] && P->boundaryMax[0]) xCord = xPrev;
                if (yCord + (double)radius < P->lowerLimit[1] && P->boundaryMin[1]) yCord = yPrev;
                if (yCord - (double)radius > P->upperLimit[1] && P->boundaryMax[1]) yCord = yPrev;
                if (zCord + (double)radius < P->lowerLimit[2] && P->boundaryMin[2]) zCord = zPrev;
                if (zCord - (double)radius > P->upperLimit[2] && P->boundaryMax[2]) zCord = zPrev;
            }
            x[i] = xCord;
            y[i] = yCord;
            z[i] = zCord;
            th[0][i] = xTheta;
            th[1][i] = yTheta;
            th[2][i] = zTheta;
            df[0][i] = (LP)(xCord - xPrev);
            df[1][i] = (LP)(yCord - yPrev);
            df[2][i] = (LP)(zCord - zPrev);
            df[3][i] = xTheta - xThPrev;
            df[4][i] = yTheta - yThPrev;
            df[5][i] = zTheta - zThPrev;
        }

        /* face forces (CollisionMesh::addForceToFace, CollisionMesh.h:46-52), summed here in
         * particle order */
        if (mtri) {
            for (int64_t i = 0; i < n; ++i) {
                int tri = mtri[i];
                if (tri < 0) continue;
                for (int k = 0; k < 3; ++k) mface[3 * (int64_t)tri + k] = mface[3 * (int64_t)tri + k] + mcol[3 * i + k];
            }
        }

        /* ---- linkUpdate gated as MainMeshBlock.cpp:312; per link
         *      CombinedAccel::iterateLinks (CombinedAccel.h:200-235) ---- */
        if ((LP)((LP)t * d.dt) > d.breakTime) {
            for (int64_t li = 0; li < L; ++li) {
                uint8_t s0 = state[li];
                if (s0 == 0) continue;
                int32_t a = pA[li], b = pB[li];
                uint8_t s1 = SFX(break_test)(&d, x[a], y[a], z[a], th[0][a], th[1][a], th[2][a],
                                             x[b], y[b], z[b], th[0][b], th[1][b], th[2][b], s0,
                                             L0[li]);
                if (s1 == 0) {
                    state[li] = 0;
                    if (nev < ev_cap) {
                        ev_link[nev] = li;
                        ev_step[nev] = t;
                    }
                    ++nev;
                }
            }
        }
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (seconds) *seconds = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    if (ev_count) *ev_count = nev;
    if (regen_count) *regen_count = nregen;
    if (force_out) {
        for (int c = 0; c < 6; ++c)
            if (force_out[c]) memcpy(force_out[c], F + c * n, sizeof(LP) * (size_t)n);
    }
    if (l->CT[0]) {
        for (int k = 0; k < 6; ++k) {
            LP *dst = (LP *)l->CT[k];
            for (int64_t s = 0; s < 2 * L; ++s) dst[s] = CT[s * 6 + k];
        }
    }
    if (g_mesh_set) {
        free(g_mesh_face);
        g_mesh_face = mface;
        g_mesh_face_lp = (int)sizeof(LP);
        SFX(mesh_free)(&macc);
        free(mtri);
        free(mcol);
    }
    SFX(adj_free)(&adj);
    free(ncount);
    free(nstart);
    free(nlist);
    free(pA);
    free(pB);
    free(F);
    free(CT);
    return 0;
}
