// A sample main's own functors run through include/hidem_b200_iterate.cuh (TEST CODE): what
// a HiDEM user writes when passing lambdas to computePartForce / linkUpdate / applyForce.
// The contact and break functors restate the default ones (HiDEM/Common/HiDEMDefaultFunctions.h:
// 21-87, 207-242); the link functor is either the default one (90-204) or the IceBlock
// sample's own (HiDEM/IceBlock/MainIceBlock.cpp:173-262). Built by the test with nvcc
// -fmad=false -prec-div=true -prec-sqrt=true, as the library is.
#include <cmath>

#include "hidem_b200_iterate.cuh"

namespace {

template <class LP>
struct NeighF {
    LP invDt, attractDistance, attractScaleForce, damping, dampingRotation, scaleE;
    __device__ void operator()(LP mask, const LP &xDist, const LP &yDist, const LP &zDist, const LP &xDiff,
                               const LP &yDiff, const LP &zDiff, const LP &uDiff, const LP &vDiff,
                               const LP &wDiff, const LP &radius, const LP &xDiffOther,
                               const LP &yDiffOther, const LP &zDiffOther, const LP &uDiffOther,
                               const LP &vDiffOther, const LP &wDiffOther, const LP &radiusOther,
                               LP &xForce, LP &yForce, LP &zForce, LP &uForce, LP &vForce,
                               LP &wForce) const {
        LP d2 = xDist * xDist + yDist * yDist + zDist * zDist;
        LP rs = radius + radiusOther;
        LP act2 = (rs + attractDistance) * (rs + attractDistance);
        mask = d2 >= act2 ? LP(0) : mask;
        LP d = sqrt(d2);
        LP inv = LP(1) / d;
        LP dim = rs - d;
        LP C = 0;
        C = d < rs ? sqrt(dim * dim * dim) : C;
        C = (d >= rs && d < rs + attractDistance) ? attractScaleForce * dim : C;
        C = C * scaleE;
        xForce = xForce + mask * ((-damping) * ((xDiff - xDiffOther) * invDt) + (C * (xDist * inv)));
        yForce = yForce + mask * ((-damping) * ((yDiff - yDiffOther) * invDt) + (C * (yDist * inv)));
        zForce = zForce + mask * ((-damping) * ((zDiff - zDiffOther) * invDt) + (C * (zDist * inv)));
        uForce = uForce + mask * ((-dampingRotation) * ((uDiff - uDiffOther) * invDt));
        vForce = vForce + mask * ((-dampingRotation) * ((vDiff - vDiffOther) * invDt));
        wForce = wForce + mask * ((-dampingRotation) * ((wDiff - wDiffOther) * invDt));
    }
};

// VARIANT 0: the default link functor; 1: the IceBlock sample's
template <class LP, int VARIANT>
struct LinkF {
    LP invDt, damping, dampingRotation, E, W2, W4, G;
    __device__ void operator()(LP &mask, const LP &xDist, const LP &yDist, const LP &zDist, const LP &xDiff,
                               const LP &yDiff, const LP &zDiff, const LP &uDiff, const LP &vDiff,
                               const LP &wDiff, const LP &, const LP &xDiffOther, const LP &yDiffOther,
                               const LP &zDiffOther, const LP &uDiffOther, const LP &vDiffOther,
                               const LP &wDiffOther, const LP &, LP &CT0, LP &CT1, LP &CT2, LP &CT3,
                               LP &CT4, LP &CT5, LP &xForce, LP &yForce, LP &zForce, LP &uForce,
                               LP &vForce, LP &wForce) const {
        xForce = xForce + (-damping * ((xDiff - xDiffOther) * invDt)) * mask;
        yForce = yForce + (-damping * ((yDiff - yDiffOther) * invDt)) * mask;
        zForce = zForce + (-damping * ((zDiff - zDiffOther) * invDt)) * mask;
        uForce = uForce + (-dampingRotation * ((uDiff - uDiffOther) * invDt)) * mask;
        vForce = vForce + (-dampingRotation * ((vDiff - vDiffOther) * invDt)) * mask;
        wForce = wForce + (-dampingRotation * ((wDiff - wDiffOther) * invDt)) * mask;
        LP x2 = xDist * xDist, y2 = yDist * yDist, z2 = zDist * zDist;
        LP invLI, invLP, invLILP, LI, LIDiv6;
        if (VARIANT == 0) {
            if (xDist == LP(0) && yDist == LP(0)) {
                x2 = LP(1e-10);
                y2 = LP(1e-10);
            }
            const LP sum = x2 + y2 + z2;
            invLI = LP(1) / sqrt(sum);
            invLP = LP(1) / sqrt(x2 + y2);
            invLILP = invLI * invLP;
            LI = invLI * sum;
            LIDiv6 = (LP(1) / LP(6)) * invLI;
        } else {
            LI = sqrt(x2 + y2 + z2);
            const LP LPl = sqrt(x2 + y2);
            invLI = LP(1) / LI;
            invLP = LP(1) / LPl;
            invLILP = LP(1) / (LI * LPl);
            LIDiv6 = LP(1) / (LP(6) * LI);
        }
        const LP T00 = xDist * invLI, T01 = yDist * invLI, T02 = zDist * invLI;
        const LP T10 = -yDist * invLP, T11 = xDist * invLP;
        const LP T20 = -(zDist * xDist) * invLILP, T21 = -(zDist * yDist) * invLILP;
        const LP T22 = (x2 + y2) * invLILP;
        const LP B0 = T00 * xDiff + T01 * yDiff + T02 * zDiff;
        const LP B1 = T10 * xDiff + T11 * yDiff;
        const LP B2 = T20 * xDiff + T21 * yDiff + T22 * zDiff;
        const LP B4 = T10 * uDiff + T11 * vDiff;
        const LP B5 = T20 * uDiff + T21 * vDiff + T22 * wDiff;
        const LP B6 = T00 * xDiffOther + T01 * yDiffOther + T02 * zDiffOther;
        const LP B7 = T10 * xDiffOther + T11 * yDiffOther;
        const LP B8 = T20 * xDiffOther + T21 * yDiffOther + T22 * zDiffOther;
        const LP B10 = T10 * uDiffOther + T11 * vDiffOther;
        const LP B11 = T20 * uDiffOther + T21 * vDiffOther + T22 * wDiffOther;
        const LP L2 = LI * LI, L3 = LI * LI * LI;
        const LP K0 = E * W2 * invLI, K1 = E * W4 / L3, K5 = E * W4 / (LP(2) * L2);
        CT0 = CT0 + (K0 * B0 + (-K0) * B6);
        CT1 = CT1 + (K1 * B1 + K5 * B5 + (-K1) * B7 + K5 * B11);
        CT2 = CT2 + (K1 * B2 + (-K5) * B4 + (-K1) * B8 + (-K5) * B10);
        xForce = xForce + (-(T00 * CT0 + T10 * CT1 + T20 * CT2)) * mask;
        yForce = yForce + (-(T01 * CT0 + T11 * CT1 + T21 * CT2)) * mask;
        zForce = zForce + (-(T02 * CT0 + T22 * CT2)) * mask;
        const LP K2 = G * W4 * LIDiv6, K3 = E * W4 * LIDiv6 * LP(2), K4 = E * W4 * LIDiv6;
        const LP B3 = T00 * uDiff + T01 * vDiff + T02 * wDiff;
        const LP B9 = T00 * uDiffOther + T01 * vDiffOther + T02 * wDiffOther;
        CT3 = CT3 + (K2 * B3 + (-K2) * B9);
        CT4 = CT4 + ((-K5) * B2 + K3 * B4 + K5 * B8 + K4 * B10);
        CT5 = CT5 + (K5 * B1 + K3 * B5 + (-K5) * B7 + K4 * B11);
        uForce = uForce + (-(T00 * CT3 + T10 * CT4 + T20 * CT5)) * mask;
        vForce = vForce + (-(T01 * CT3 + T11 * CT4 + T21 * CT5)) * mask;
        wForce = wForce + (-(T02 * CT3 + T22 * CT5)) * mask;
    }
};

template <class LP>
struct BreakF {
    LP bendBreak, maxLoad;
    __device__ void operator()(const double &x1, const double &y1, const double &z1, const LP &tx1,
                               const LP &ty1, const LP &tz1, const double &x2, const double &y2,
                               const double &z2, const LP &tx2, const LP &ty2, const LP &tz2,
                               uint8_t &state, LP &initialLen) const {
        if (state == 0) return;
        const LP xd = (LP)(x1 - x2), yd = (LP)(y1 - y2), zd = (LP)(z1 - z2);
        const LP len = sqrt((xd * xd) + (yd * yd) + (zd * zd));
        const LP ax = fabs(tx1 - tx2), ay = fabs(ty1 - ty2), az = fabs(tz1 - tz2);
        const LP myz = ay < az ? az : ay;
        const LP bend = ax < myz ? myz : ax;
        const LP load = (len - initialLen) / initialLen + bendBreak * bend;
        if (load >= maxLoad) state = 0;
    }
};

// a caller's own integrate lambda: plain explicit update x += diff, the diffs scaled by
// the force (no counterpart in the samples; it checks the field plumbing of applyForce)
template <class LP>
struct Drift {
    LP scale;
    __device__ void operator()(long long p, hidem_iter::ParticleData<LP> &d) const {
        d.xDiff[p] = d.xDiff[p] + scale * d.xForce[p];
        d.yDiff[p] = d.yDiff[p] + scale * d.yForce[p];
        d.zDiff[p] = d.zDiff[p] + scale * d.zForce[p];
        d.xCord[p] = d.xCord[p] + (double)d.xDiff[p];
        d.yCord[p] = d.yCord[p] + (double)d.yDiff[p];
        d.zCord[p] = d.zCord[p] + (double)d.zDiff[p];
        d.zTheta[p] = d.zTheta[p] + scale * d.wForce[p];
    }
};

template <class LP>
int run_step(hidem_ctx *ctx, int variant, bool userBreak, bool breakOpen, const hidem_functor_params &f) {
    hidem_device_view v;
    if (hidem_get_device_view(ctx, &v) != HIDEM_OK) return 10;
    NeighF<LP> nf{(LP)f.neigh_invDt, (LP)f.neigh_attractDistance, (LP)f.neigh_attractScaleForce,
                  (LP)f.neigh_damping, (LP)f.neigh_dampingRotation, (LP)f.neigh_scaleE};
    cudaError_t e;
    if (variant == 0) {
        LinkF<LP, 0> lf{(LP)f.link_invDt, (LP)f.link_damping, (LP)f.link_dampingRotation, (LP)f.link_E,
                        (LP)f.link_W2, (LP)f.link_W4, (LP)f.link_G};
        e = hidem_iter::computePartForce<LP>(v, nf, lf);
    } else {
        LinkF<LP, 1> lf{(LP)f.link_invDt, (LP)f.link_damping, (LP)f.link_dampingRotation, (LP)f.link_E,
                        (LP)f.link_W2, (LP)f.link_W4, (LP)f.link_G};
        e = hidem_iter::computePartForce<LP>(v, nf, lf);
    }
    if (e != cudaSuccess) return 11;
    if (hidem_integrate(ctx) != HIDEM_OK) return 12;
    if (!breakOpen) return 0;
    if (userBreak) {
        if (hidem_get_device_view(ctx, &v) != HIDEM_OK) return 13;
        BreakF<LP> bf{(LP)f.break_bendBreak, (LP)f.break_maxLoad};
        if (hidem_iter::linkUpdate<LP>(v, bf) != cudaSuccess) return 14;
    } else if (hidem_link_update(ctx) != HIDEM_OK) {
        return 15;
    }
    return 0;
}

}  // namespace

// n timesteps of the sample loop (MainMeshBlock.cpp:274-323: gridService, computePartForce
// with the caller's functors, the library's integrate, linkUpdate with the caller's break
// functor or the library's when t dt > breakTime (in lp, as the sample main), finalizeTs)
extern "C" int harness_steps(hidem_ctx *ctx, int variant, int user_break, int nsteps, double dt,
                             double breakTime) {
    hidem_functor_params f;
    if (hidem_get_functor_params(ctx, &f) != HIDEM_OK) return 1;
    hidem_device_view v;
    for (int t = 0; t < nsteps; ++t) {
        if (hidem_grid_service(ctx) != HIDEM_OK) return 3;
        if (hidem_get_device_view(ctx, &v) != HIDEM_OK) return 4;
        const long long step = v.step;
        const bool mixed = v.precision == HIDEM_PREC_MIXED;
        const bool open = mixed ? (float)((float)step * (float)dt) > (float)breakTime
                                : (double)step * dt > breakTime;
        const int rc = mixed ? run_step<float>(ctx, variant, user_break != 0, open, f)
                             : run_step<double>(ctx, variant, user_break != 0, open, f);
        if (rc) return rc;
        if (hidem_finalize_ts(ctx) != HIDEM_OK) return 5;
    }
    return hidem_synchronize(ctx) == HIDEM_OK ? 0 : 6;
}

// forces of the caller's functors on the current state, no step taken
extern "C" int harness_forces(hidem_ctx *ctx, int variant) {
    hidem_functor_params f;
    if (hidem_get_functor_params(ctx, &f) != HIDEM_OK) return 1;
    hidem_device_view v;
    if (hidem_get_device_view(ctx, &v) != HIDEM_OK) return 4;
    cudaError_t e;
    if (v.precision == HIDEM_PREC_MIXED) {
        NeighF<float> nf{(float)f.neigh_invDt, (float)f.neigh_attractDistance, (float)f.neigh_attractScaleForce,
                         (float)f.neigh_damping, (float)f.neigh_dampingRotation, (float)f.neigh_scaleE};
        LinkF<float, 1> l1{(float)f.link_invDt, (float)f.link_damping, (float)f.link_dampingRotation,
                           (float)f.link_E, (float)f.link_W2, (float)f.link_W4, (float)f.link_G};
        LinkF<float, 0> l0{l1.invDt, l1.damping, l1.dampingRotation, l1.E, l1.W2, l1.W4, l1.G};
        e = variant ? hidem_iter::computePartForce<float>(v, nf, l1) : hidem_iter::computePartForce<float>(v, nf, l0);
    } else {
        NeighF<double> nf{f.neigh_invDt, f.neigh_attractDistance, f.neigh_attractScaleForce,
                          f.neigh_damping, f.neigh_dampingRotation, f.neigh_scaleE};
        LinkF<double, 1> l1{f.link_invDt, f.link_damping, f.link_dampingRotation, f.link_E, f.link_W2,
                            f.link_W4, f.link_G};
        LinkF<double, 0> l0{l1.invDt, l1.damping, l1.dampingRotation, l1.E, l1.W2, l1.W4, l1.G};
        e = variant ? hidem_iter::computePartForce<double>(v, nf, l1) : hidem_iter::computePartForce<double>(v, nf, l0);
    }
    if (e != cudaSuccess) return 11;
    return hidem_synchronize(ctx) == HIDEM_OK ? 0 : 6;
}

// applyForce with a caller's integrate lambda, and Iterator::iterate over the slots
extern "C" int harness_apply(hidem_ctx *ctx, double scale) {
    hidem_device_view v;
    if (hidem_get_device_view(ctx, &v) != HIDEM_OK) return 4;
    cudaError_t e = v.precision == HIDEM_PREC_MIXED
                        ? hidem_iter::applyForce<float>(v, Drift<float>{(float)scale})
                        : hidem_iter::applyForce<double>(v, Drift<double>{scale});
    if (e != cudaSuccess) return 11;
    return hidem_synchronize(ctx) == HIDEM_OK ? 0 : 6;
}

namespace {
struct CountContacts {
    __device__ void operator()(long long s, const uint32_t *counts, unsigned long long *out) const {
        atomicAdd(out, (unsigned long long)(counts[s] & 0xffffu));
    }
};
}  // namespace

extern "C" long long harness_iterate_count(hidem_ctx *ctx) {
    hidem_device_view v;
    if (hidem_get_device_view(ctx, &v) != HIDEM_OK) return -1;
    unsigned long long *d = nullptr, h = 0;
    if (cudaMalloc(&d, sizeof h) != cudaSuccess) return -2;
    cudaMemsetAsync(d, 0, sizeof h, static_cast<cudaStream_t>(v.stream));
    hidem_iter::OffloadExec pol(v);
    if (hidem_iter::Iterator::iterate(pol, CountContacts{}, (long long)v.n, v.counts, d) != cudaSuccess) return -3;
    hidem_iter::Iterator::syncAll(pol);
    cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return (long long)h;
}
