// C ABI of libhidem_b200: the context, the HiDEMLib-shaped step operations and the
// host side of the rebuild (HiDEMLib::gridService) policy.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "kernels.h"

using namespace hidem;

namespace hidem {

// NVTX range around a host call, named after the reference's phase (its xvtxRangePush
// ranges, Iterators/DevPortabilityLayer.h:298-332): visible in Nsight timelines, free
// when no profiler is attached (NVTX forwards to nothing then).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// Host-side work over large arrays (the per-particle fields kept on the host) split over a
// few threads, so that it keeps pace with the host-device copies it overlaps.
template <class F>
void host_parallel(long long n, F body) {
    const long long chunk = 1ll << 20;
    const int threads = (int)std::min<long long>(8, (n + chunk - 1) / chunk);
    if (threads <= 1) {
        body(0ll, n);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([=] { body(n * t / threads, n * (t + 1) / threads); });
    for (auto &th : pool) th.join();
}

inline void host_copy(void *dst, const void *src, size_t bytes) {
    host_parallel((long long)bytes, [=](long long a, long long b) {
        std::memcpy(static_cast<char *>(dst) + a, static_cast<const char *>(src) + a, (size_t)(b - a));
    });
}
// whether a caller's array lives in device memory (which the host cannot read directly)
inline bool on_device(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice;
}
// bytes between a caller's array (host or device memory) and host memory
inline cudaError_t from_caller(void *hostDst, const void *src, size_t bytes) {
    if (on_device(src)) return cudaMemcpy(hostDst, src, bytes, cudaMemcpyDeviceToHost);
    host_copy(hostDst, src, bytes);
    return cudaSuccess;
}
inline cudaError_t to_caller(void *dst, const void *hostSrc, size_t bytes) {
    if (on_device(dst)) return cudaMemcpy(dst, hostSrc, bytes, cudaMemcpyHostToDevice);
    host_copy(dst, hostSrc, bytes);
    return cudaSuccess;
}
// per-thread text of the last failure of a call that has no context
thread_local std::string g_nocontext_error;
}  // namespace hidem

namespace {

std::string &g_create_error = hidem::g_nocontext_error;

struct SideSet {
    uint32_t *partner = nullptr;
    void *ct[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    uint8_t *state = nullptr;
    void *L0 = nullptr;
    int32_t *link = nullptr;
    long long cap = 0;
};

}  // namespace

struct hidem_ctx {
    hidem_params P{};
    int mixed = 1;
    size_t lp = 4;  // bytes of lp / ct
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;

    Consts<float> cf{};
    Consts<double> cd{};
    double searchDistance = 0, interactDist = 0;

    long long n = 0, L = 0;
    long long step = 0, startStep = 0;
    bool haveParticles = false, haveLinks = false, built = false;

    // particles (slot order), double buffered
    void *rec[2] = {nullptr, nullptr};
    int cur = 0;  // record buffer holding the current state
    int ord = 0;  // which of type/orig/cellOf matches the current slot order
    uint8_t *type[2] = {nullptr, nullptr};
    int32_t *orig[2] = {nullptr, nullptr};
    int32_t *cellOf[2] = {nullptr, nullptr};
    int32_t *slotOf = nullptr;
    int32_t *perm = nullptr;
    int32_t *bigCells = nullptr;  // crowded cells of a rebuild's sort (n / 32 + 2 entries, count last)
    int32_t *haloSendPos = nullptr;  // per slot: position in the halo send list, or -1
    void *force = nullptr;

    // grid
    GridInfo grid{};
    int32_t *cellCount = nullptr, *cellStart = nullptr, *cursor = nullptr;
    long long cellCap = 0;
    int *scanSums32 = nullptr;
    long long *scanSums64 = nullptr;
    long long scanCap = 0;
    double *boundsPartial = nullptr, *boundsOut = nullptr;

    // contact list + per-slot counts
    uint32_t *counts = nullptr;
    int *blockWidth = nullptr;
    long long *nOff = nullptr, *sOff = nullptr, *offTotal = nullptr;
    int32_t *nbr = nullptr;
    long long nbrCap = 0;
    long long numPairs = 0, maxNeigh = 0, maxLinksPP = 0;

    // links (input order)
    int32_t *linkA = nullptr, *linkB = nullptr;
    void *L0link = nullptr;
    uint8_t *linkState = nullptr;  // per-link state, kept equal to the sides' states
    int32_t *linkSlotA = nullptr, *linkSlotB = nullptr;  // both ends' slots since the last rebuild
    int32_t *plStart = nullptr, *plLink = nullptr;
    uint8_t *plEnd = nullptr;
    int32_t *sideSlot[2] = {nullptr, nullptr};
    SideSet side[2];
    int curSide = 0;  // always 0: rebuild swaps the new layout into side[0]
    // the caller's link fields the step never reads, kept on the device for get_links
    int32_t *dLinkOwners = nullptr, *dLinkNum = nullptr;
    long long *dLinkKeys = nullptr, *dLinkKeyA = nullptr, *dLinkKeyB = nullptr;

    // particle metadata kept on the host (input order)
    std::vector<int32_t> owners;
    std::vector<int64_t> keys;

    // events and reductions
    int2 *events = nullptr;
    unsigned long long *eventCount = nullptr;
    long long eventCap = 0, eventsRead = 0;
    unsigned long long *diffMax = nullptr;
    int *errorFlag = nullptr;

    // optional CUDA-event timing of the fused step kernel (pairs recorded around launches)
    bool profile = false;
    std::vector<cudaEvent_t> evPool;
    size_t evUsed = 0;

    double accumulatedDist = 0;
    long long regenCount = 0, lastRegen = -1;
    long long prevTotalCells = 0, gridGrowthEvents = 0;  // NeighbourGrid.cpp:89-92 warning
    int32_t checks = 0;                                 // HIDEM_CHECK_* bits
    long long launches = 0;
    int smCount = 148;

    // step kernel: fixed by the caller, or timed on the first fused steps (AUTO)
    int stepKernel = HIDEM_STEP_KERNEL_AUTO;
    int tunedKernel = HIDEM_STEP_KERNEL_AUTO;
    int tuneStep = 0;
    cudaEvent_t tuneEv[2 * 16] = {};

    double *energyBuf = nullptr;  // kinetic-energy partials + result
    int energyBlocks = 0;

    // GlacierDem maps on the device: 0 bed height, 1 bed friction, 2..7 external forces
    void *mapData[8] = {};
    Map2dView mapView[8] = {};
    bool mapSet[8] = {};

    // collision mesh: vertices (x, y, z), normals, face forces, MeshAccel cell lists
    void *meshVtx[3] = {}, *meshNrm[3] = {}, *meshFace[3] = {};
    int *meshSizes = nullptr, *meshStarts = nullptr, *meshValues = nullptr;
    int *meshQSizes = nullptr, *meshQStarts = nullptr, *meshQValues = nullptr;  // query lists
    uint8_t *meshKeep = nullptr;  // triangles the query lists always keep
    long long meshCells = 0, meshValueCount = 0, meshQValueCount = 0;
    double meshCellSize = 0;
    double maxParticleRadius = 0;  // over the particles last set
    int meshTris = 0;
    bool meshSet = false;
    MeshView<float> meshF{};
    MeshView<double> meshD{};

    // slab decomposition: a grid box given for the next rebuild, and the halo force lists
    // (particle indices in input order)
    bool frameOnce = false;
    double frame[6] = {};
    int32_t *haloSend = nullptr, *haloRecv = nullptr;
    long long nHaloSend = 0, nHaloRecv = 0;
};

namespace {

hidem_status fail(hidem_ctx *c, hidem_status s, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return s;
}

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(ctx, HIDEM_ERR_CUDA, "%s failed: %s (%s:%d)", #call,                 \
                        cudaGetErrorString(e_), __FILE__, __LINE__);                         \
    } while (0)

#define TRY(expr)                            \
    do {                                     \
        hidem_status s_ = (expr);            \
        if (s_ != HIDEM_OK) return s_;       \
    } while (0)

template <class T>
hidem_status dalloc(hidem_ctx *ctx, T **p, long long count) {
    if (*p) {
        CK(cudaFreeAsync(*p, ctx->stream));
        *p = nullptr;
    }
    if (count <= 0) count = 1;
    CK(cudaMallocAsync((void **)p, sizeof(T) * (size_t)count, ctx->stream));
    return HIDEM_OK;
}
hidem_status dalloc_bytes(hidem_ctx *ctx, void **p, size_t bytes) {
    if (*p) {
        CK(cudaFreeAsync(*p, ctx->stream));
        *p = nullptr;
    }
    if (bytes == 0) bytes = 16;
    CK(cudaMallocAsync(p, bytes, ctx->stream));
    return HIDEM_OK;
}
template <class T>
void dfree(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}

// Derived constants of the sample main (HiDEM/MeshBlock/MainMeshBlock.cpp:69-156) in lp
// precision, and the search distances of HiDEMLib::setup (HiDEMLib.h:757-761).
template <class LP>
void derive(const hidem_params &P, Consts<LP> &c, double &searchDistance, double &interactDist) {
    LP scale = (LP)P.scale;
    LP s2 = scale * scale;
    LP dt = (LP)P.dt;
    LP E = (LP)P.E;
    LP beamWidth = (LP)P.beamWidth * scale;
    LP rhoWater = (LP)P.rhoWater, rhoIce = (LP)P.rhoIce, g = (LP)P.g;
    c.invDt = (LP)(1.0 / (double)dt);
    c.attractDistance = (LP)P.attractDistance * scale;
    c.attractScaleForce = (LP)P.attractScaleForce;
    c.damping = (LP)P.damping * s2;
    c.dampingRotation = (LP)P.dampingRotation * s2;
    c.scaleE = E * scale;
    c.E = E;
    c.W2 = beamWidth * beamWidth;
    c.W4 = beamWidth * beamWidth * beamWidth * beamWidth;
    c.G = (LP)((double)E / 2.0);
    c.bendBreak = (LP)P.bendBreak;
    c.maxLoad = (LP)P.maxLoad;
    c.linkInvDt = c.invDt;
    c.linkDamping = c.damping;
    c.linkDampingRotation = c.dampingRotation;
    c.mainInvDt = c.invDt;
    c.dt = dt;
    c.invDt2 = (LP)(1.0 / (2.0 * (double)dt));
    c.dtSqr = (LP)std::pow((double)dt, 2.0);
    c.invDtSqr = (LP)(1.0 / std::pow((double)dt, 2.0));
    c.g = g;
    c.lift = (rhoWater - rhoIce) / rhoIce * g;
    c.rhoIce = rhoIce;
    c.rhoWater = rhoWater;
    c.waterLevel = (LP)P.waterLevel;
    c.airDrag = (LP)P.airDrag * s2;
    c.waterDrag = (LP)P.waterDrag * s2;
    c.bedDrag = (LP)P.bedDrag * s2;
    c.bedFriction = (LP)P.bedFriction;
    c.bedHeight = (LP)P.bedHeight;
    c.bedInteract = (LP)P.bedInteract * scale;
    c.bedStiffness = (LP)P.bedStiffness * s2;
    c.scale = scale;
    c.maxVel = (LP)P.maxVel;
    c.maxRot = (LP)P.maxRot;
    c.breakTime = (LP)P.breakTime;
    for (int k = 0; k < 3; ++k) {
        c.lower[k] = P.lowerLimit[k];
        c.upper[k] = P.upperLimit[k];
        c.bmin[k] = P.boundaryMin[k] != 0;
        c.bmax[k] = P.boundaryMax[k] != 0;
    }
    c.useBed = P.useBed != 0;
    c.useVel = P.useVelocityLimit != 0;
    c.useBnd = P.useBoundary != 0;
    c.useFixed = P.useFixed != 0;
    c.useFront = P.useFrontPressure != 0;
    LP maxRadius = (LP)P.maxRadius;
    LP maxParticleDist = (LP)((double)maxRadius * 2.0);
    searchDistance = P.searchDistanceScale * (double)maxParticleDist;
    interactDist = searchDistance - (double)maxParticleDist;
}

hidem_status check_params(hidem_ctx *ctx, const hidem_params *p) {
    if (!p) return fail(ctx, HIDEM_ERR_ARG, "params is NULL");
    if (p->precision != HIDEM_PREC_FP64 && p->precision != HIDEM_PREC_MIXED)
        return fail(ctx, HIDEM_ERR_ARG, "unknown precision %d", p->precision);
    if (!(p->dt > 0)) return fail(ctx, HIDEM_ERR_ARG, "dt must be > 0");
    if (!(p->maxRadius > 0)) return fail(ctx, HIDEM_ERR_ARG, "maxRadius must be > 0");
    if (!(p->searchDistanceScale > 1))
        return fail(ctx, HIDEM_ERR_ARG, "searchDistanceScale must be > 1");
    return HIDEM_OK;
}

// The maps and the collision mesh set on the context, in both precisions' constants.
template <class LP>
void attach_maps_to(const hidem_ctx *ctx, Consts<LP> &c) {
    c.bedMap = ctx->mapView[0];
    c.fricMap = ctx->mapView[1];
    for (int k = 0; k < 6; ++k) c.extMap[k] = ctx->mapView[2 + k];
    c.useBedMap = ctx->mapSet[0] ? 1 : 0;
    c.useFricMap = ctx->mapSet[1] ? 1 : 0;
    c.useExtMaps = ctx->mapSet[2] ? 1 : 0;
    if constexpr (sizeof(LP) == 4)
        c.mesh = ctx->meshF;
    else
        c.mesh = ctx->meshD;
    c.useMesh = ctx->meshSet ? 1 : 0;
}
void attach_maps(hidem_ctx *ctx) {
    attach_maps_to<float>(ctx, ctx->cf);
    attach_maps_to<double>(ctx, ctx->cd);
}

hidem_status apply_params(hidem_ctx *ctx, const hidem_params *p) {
    TRY(check_params(ctx, p));
    ctx->P = *p;
    ctx->mixed = p->precision == HIDEM_PREC_MIXED;
    ctx->lp = ctx->mixed ? 4 : 8;
    double sd, id;
    derive<float>(*p, ctx->cf, sd, id);
    derive<double>(*p, ctx->cd, ctx->searchDistance, ctx->interactDist);
    attach_maps(ctx);
    if (ctx->mixed) {
        ctx->searchDistance = sd;
        ctx->interactDist = id;
    }
    return HIDEM_OK;
}

hidem_status check_device_error(hidem_ctx *ctx) {
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, ctx->errorFlag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (flag) {
        CK(cudaMemsetAsync(ctx->errorFlag, 0, sizeof(int), ctx->stream));
        const char *what = flag == 1   ? "particle outside the grid bounds"
                           : flag == 2 ? "more than 65535 contacts for one particle"
                           : flag == 3 ? "more than 65535 link ends for one particle"
                           : flag == 4 ? "shared-memory staging copies did not complete in time"
                           : flag == 5 ? "more than 4096 particles in one neighbour-grid cell"
                                       : "device check failed";
        return fail(ctx, flag == 5 ? HIDEM_ERR_CAPACITY : HIDEM_ERR_DEVICE, "device check %d: %s", flag, what);
    }
    return HIDEM_OK;
}

template <class LP>
PRec<LP> *recp(hidem_ctx *ctx, int b) {
    return static_cast<PRec<LP> *>(ctx->rec[b]);
}

template <class LP>
SideView<LP> side_view(SideSet &s) {
    SideView<LP> v;
    v.partner = s.partner;
    for (int k = 0; k < 6; ++k) v.ct[k] = static_cast<LP *>(s.ct[k]);
    v.state = s.state;
    v.L0 = static_cast<LP *>(s.L0);
    v.link = s.link;
    return v;
}

// grows a side set to at least `cap` link ends, with a quarter of headroom so that the
// two sets a rebuild alternates between stop reallocating (cudaFree synchronises the device)
hidem_status side_alloc(hidem_ctx *ctx, SideSet &s, long long cap) {
    if (s.cap >= cap && s.partner) return HIDEM_OK;
    if (cap <= 0) cap = 1;
    cap += cap / 4;
    TRY(dalloc(ctx, &s.partner, cap));
    for (int k = 0; k < 6; ++k) TRY(dalloc_bytes(ctx, &s.ct[k], ctx->lp * (size_t)cap));
    TRY(dalloc(ctx, &s.state, cap));
    TRY(dalloc_bytes(ctx, &s.L0, ctx->lp * (size_t)cap));
    TRY(dalloc(ctx, &s.link, cap));
    s.cap = cap;
    return HIDEM_OK;
}

void side_free(SideSet &s) {
    dfree(s.partner);
    for (int k = 0; k < 6; ++k) dfree(s.ct[k]);
    dfree(s.state);
    dfree(s.L0);
    dfree(s.link);
    s.cap = 0;
}

long long nblocks32(long long n) { return (n + 31) / 32; }

hidem_status ensure_scan(hidem_ctx *ctx, long long n) {
    long long need = (n + 1023) / 1024 + 1;
    if (ctx->scanCap >= need) return HIDEM_OK;
    TRY(dalloc(ctx, &ctx->scanSums32, need));
    TRY(dalloc(ctx, &ctx->scanSums64, need));
    ctx->scanCap = need;
    return HIDEM_OK;
}

// --------------------------------------------------------------- rebuild

// CombinedAccel::generateNeighbours + generateLinks (+ LinkAccelSide::sortSideData):
// bounds, cell colours, counting sort into cell order (inside a cell by input index),
// permutation of the particle records, contact list, link-end layout.
template <class LP>
hidem_status rebuild(hidem_ctx *ctx) {
    NvtxRange nvtx_range("generateNeighbourGrid + contact list + link ends");
    cudaStream_t st = ctx->stream;
    const int n = (int)ctx->n;
    const int cur = ctx->cur, nxt = 1 - cur;

    // 1. bounds (ParticleData::getLimits)
    const int nbB = std::min<long long>(std::max<long long>(1, (n + 255) / 256), 4 * ctx->smCount);
    launch_bounds<LP>(recp<LP>(ctx, cur), n, ctx->boundsPartial, nbB, ctx->boundsOut, st);
    ctx->launches += 2;
    double b[6];
    CK(cudaMemcpyAsync(b, ctx->boundsOut, sizeof b, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // the bounds carry a NaN of any coordinate; an infinite one shows as an infinite bound
    for (int k = 0; k < 6; ++k)
        if (!std::isfinite(b[k]))
            return fail(ctx, HIDEM_ERR_DEVICE, "non-finite particle coordinates (NaN or infinite %c)",
                        "xyz"[k % 3]);
    if (ctx->frameOnce) {
        // the box spanning every rank's particles (hidem_regenerate_frame)
        const double *f = ctx->frame;
        if (!(f[0] <= b[0] && f[1] <= b[1] && f[2] <= b[2] && b[3] <= f[3] && b[4] <= f[4] && b[5] <= f[5]))
            return fail(ctx, HIDEM_ERR_ARG, "particles outside the given grid box");
        std::memcpy(b, f, sizeof b);
    }

    // 2. grid (NeighbourGrid::generateNeighbourGrid, NeighbourGrid.cpp:72-114)
    GridInfo &g = ctx->grid;
    g.xMin = b[0];
    g.yMin = b[1];
    g.zMin = b[2];
    g.h = ctx->searchDistance;
    double ex = std::floor((b[3] - b[0]) / g.h), ey = std::floor((b[4] - b[1]) / g.h),
           ez = std::floor((b[5] - b[2]) / g.h);
    if (ex > 2e9 || ey > 2e9 || ez > 2e9)
        return fail(ctx, HIDEM_ERR_CAPACITY, "grid extent too large");
    g.X = 1 + (int)ex;
    g.Y = 1 + (int)ey;
    g.Z = 1 + (int)ez;
    g.total = (long long)g.X * g.Y * g.Z;
    if (g.total >= (1ll << 31))
        return fail(ctx, HIDEM_ERR_CAPACITY, "grid has %lld cells (limit 2^31)", g.total);
    // NeighbourGrid::generateNeighbourGrid's explosion warning (NeighbourGrid.cpp:89-92): a
    // grid more than 10x the last one's cells is counted; with HIDEM_CHECK_GRID_GROWTH the
    // rebuild is refused instead
    if (ctx->prevTotalCells != 0 && g.total / 10 > ctx->prevTotalCells) {
        ctx->gridGrowthEvents += 1;
        if (ctx->checks & HIDEM_CHECK_GRID_GROWTH)
            return fail(ctx, HIDEM_ERR_DEVICE,
                        "grid of %lld cells is more than 10x the last rebuild's %lld: did something explode?",
                        g.total, ctx->prevTotalCells);
    }
    ctx->prevTotalCells = g.total;
    int k = 0;
    for (int zD = -1; zD < 2; ++zD)
        for (int yD = -1; yD < 2; ++yD)
            for (int xD = -1; xD < 2; ++xD)
                g.off[k++] = (long long)xD + (long long)yD * g.X + (long long)zD * g.X * g.Y;
    if (ctx->cellCap < g.total) {
        long long cap = g.total + g.total / 4 + 1024;
        TRY(dalloc(ctx, &ctx->cellCount, cap));
        TRY(dalloc(ctx, &ctx->cellStart, cap));
        TRY(dalloc(ctx, &ctx->cursor, cap));
        ctx->cellCap = cap;
    }
    TRY(ensure_scan(ctx, std::max<long long>(g.total, nblocks32(n) + 1)));

    // 3. colours + counting sort (colourParticles / generateIterationList)
    CK(cudaMemsetAsync(ctx->cellCount, 0, sizeof(int) * (size_t)g.total, st));
    CK(cudaMemsetAsync(ctx->cursor, 0, sizeof(int) * (size_t)g.total, st));
    const int od = ctx->ord, nd = 1 - od;
    launch_cells<LP>(recp<LP>(ctx, cur), n, g, ctx->cellOf[od], ctx->cellCount, ctx->errorFlag, st);
    ctx->launches += 1;
    ctx->launches += launch_scan<int, int>(ctx->cellCount, g.total, 1, ctx->cellStart,
                                           ctx->scanSums32, nullptr, st);
    launch_scatter(ctx->cellOf[od], n, ctx->cellStart, ctx->cursor, ctx->perm, st);
    ctx->launches += launch_sort_cells(ctx->cellStart, ctx->cellCount, g.total, ctx->orig[od], ctx->perm,
                                       ctx->bigCells, ctx->bigCells + ctx->n / kSmallCell + 1,
                                       ctx->errorFlag, 5, ctx->smCount, st);
    launch_permute<LP>(ctx->perm, n, recp<LP>(ctx, cur), recp<LP>(ctx, nxt), ctx->type[od],
                       ctx->type[nd], ctx->orig[od], ctx->orig[nd], ctx->cellOf[od],
                       ctx->cellOf[nd], ctx->slotOf, st);
    ctx->launches += 3;
    if (ctx->L > 0) {
        launch_link_slots(ctx->linkA, ctx->linkB, ctx->slotOf, ctx->L, ctx->linkSlotA, ctx->linkSlotB, st);
        ctx->launches += 1;
    }
    if (ctx->nHaloSend > 0 && ctx->haloSendPos) {
        launch_send_pos(ctx->slotOf, ctx->haloSend, ctx->nHaloSend, n, ctx->haloSendPos, st);
        ctx->launches += 1;
    }
    ctx->cur = nxt;
    ctx->ord = nd;
    const int c = nd;   // slot-order arrays
    const int rc = nxt; // record buffer

    // 4. contact list (NeighAccel::generateNeighbours: count pass, widths, fill pass)
    const long long nb32 = nblocks32(n);
    CK(cudaMemsetAsync(ctx->blockWidth, 0, sizeof(int) * (size_t)(nb32 + 1), st));
    launch_nbr_count<LP>(recp<LP>(ctx, rc), n, ctx->cellOf[c], g, ctx->cellStart, ctx->cellCount,
                         ctx->interactDist, ctx->counts, ctx->blockWidth, ctx->errorFlag, st);
    ctx->launches += 1;
    ctx->launches += launch_scan<int, long long>(ctx->blockWidth, nb32 + 1, 32ll, ctx->nOff,
                                                 ctx->scanSums64, ctx->offTotal, st);
    long long nTotal = 0;
    CK(cudaMemcpyAsync(&nTotal, ctx->offTotal, sizeof nTotal, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    TRY(check_device_error(ctx));
    if (nTotal > ctx->nbrCap) {
        long long cap = nTotal + nTotal / 8 + 1024;
        TRY(dalloc(ctx, &ctx->nbr, cap));
        ctx->nbrCap = cap;
    }
    launch_nbr_fill<LP>(recp<LP>(ctx, rc), n, ctx->cellOf[c], g, ctx->cellStart, ctx->cellCount,
                        ctx->interactDist, ctx->nOff, ctx->nbr, st);
    ctx->launches += 1;

    // 5. link ends in the new slot order (LinkAccelSide::generateLinks + sortSideData)
    CK(cudaMemsetAsync(ctx->blockWidth, 0, sizeof(int) * (size_t)(nb32 + 1), st));
    launch_side_count(ctx->orig[c], n, ctx->plStart, ctx->counts, ctx->blockWidth, ctx->errorFlag, st);
    ctx->launches += 1;
    ctx->launches += launch_scan<int, long long>(ctx->blockWidth, nb32 + 1, 32ll, ctx->sOff,
                                                 ctx->scanSums64, ctx->offTotal, st);
    // the contact-list statistics travel with the link-end total
    launch_count_stats(ctx->counts, n, ctx->offTotal + 1, ctx->smCount, st);
    ctx->launches += 1;
    long long tot[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(tot, ctx->offTotal, sizeof tot, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    TRY(check_device_error(ctx));
    const long long sTotal = tot[0];
    if (sTotal >= (1ll << 31))
        return fail(ctx, HIDEM_ERR_CAPACITY, "%lld link-end slots (limit 2^31)", sTotal);
    // side[0] / sideSlot[0] hold the current layout; the new one is built in [1], then swapped
    TRY(side_alloc(ctx, ctx->side[1], std::max<long long>(sTotal, 2 * ctx->L)));
    if (ctx->L > 0) {
        launch_side_fill<LP>(ctx->orig[c], n, ctx->slotOf, ctx->plStart, ctx->plLink, ctx->plEnd,
                             ctx->linkA, ctx->linkB, static_cast<const LP *>(ctx->L0link),
                             ctx->sideSlot[0], side_view<LP>(ctx->side[0]), ctx->sOff,
                             side_view<LP>(ctx->side[1]), ctx->sideSlot[1], st);
        ctx->launches += 1;
    }
    std::swap(ctx->sideSlot[0], ctx->sideSlot[1]);
    std::swap(ctx->side[0], ctx->side[1]);

    ctx->numPairs = tot[1];
    ctx->maxNeigh = tot[2];
    ctx->maxLinksPP = tot[3];
    ctx->built = true;
    ctx->regenCount += 1;
    ctx->lastRegen = ctx->step;
    CK(cudaGetLastError());
    return HIDEM_OK;
}

hidem_status do_rebuild(hidem_ctx *ctx) {
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "no particles set");
    return ctx->mixed ? rebuild<float>(ctx) : rebuild<double>(ctx);
}

// max over particles of max(0, x/y/zDiff) -> accumulated displacement
// (HiDEMLib::accumulateDist, HiDEMLib.h:463-474), from three device words.
template <class LP>
void diff_words(const unsigned long long w[3], double out[3]) {
    for (int k = 0; k < 3; ++k) {
        if (sizeof(LP) == 4) {
            uint32_t u = (uint32_t)w[k];
            float f;
            std::memcpy(&f, &u, 4);
            out[k] = (double)f;
        } else {
            std::memcpy(&out[k], &w[k], 8);
        }
    }
}

// the maxima are lp values held in doubles (exactly)
template <class LP>
double curr_dist(const double mx[3]) {
    const LP m[3] = {(LP)mx[0], (LP)mx[1], (LP)mx[2]};
    LP root = std::sqrt((m[0] * m[0]) + (m[1] * m[1]) + (m[2] * m[2]));
    return (double)((LP)10 * root);
}

double curr_dist_of(const hidem_ctx *ctx, const double mx[3]) {
    return ctx->mixed ? curr_dist<float>(mx) : curr_dist<double>(mx);
}

hidem_status read_diff_words(hidem_ctx *ctx, double mx[3]) {
    unsigned long long w[3];
    CK(cudaMemcpyAsync(w, ctx->diffMax, sizeof w, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->mixed)
        diff_words<float>(w, mx);
    else
        diff_words<double>(w, mx);
    return HIDEM_OK;
}

hidem_status read_diff_max(hidem_ctx *ctx, double *currDist) {
    double mx[3];
    TRY(read_diff_words(ctx, mx));
    *currDist = curr_dist_of(ctx, mx);
    return HIDEM_OK;
}

hidem_status reduce_diff_now(hidem_ctx *ctx) {
    CK(cudaMemsetAsync(ctx->diffMax, 0, 3 * sizeof(unsigned long long), ctx->stream));
    int nb = std::min<long long>(std::max<long long>(1, (ctx->n + 255) / 256), 4 * ctx->smCount);
    if (ctx->mixed)
        launch_max_diff<float>(recp<float>(ctx, ctx->cur), (int)ctx->n, ctx->diffMax, nb, ctx->stream);
    else
        launch_max_diff<double>(recp<double>(ctx, ctx->cur), (int)ctx->n, ctx->diffMax, nb, ctx->stream);
    ctx->launches += 1;
    return HIDEM_OK;
}

// Whether gridService at the current step reads the diff maxima (HiDEMLib.h:563-575).
bool gs_wants_diff(const hidem_ctx *ctx) {
    return ctx->P.gridRegenInterval == -1 && ctx->step % 10 == 0;
}

// The rest of HiDEMLib::gridService (HiDEMLib.h:533-628) on one rank, once the
// accumulated-distance increment of this step (when gs_wants_diff) is known.
// gridService's decision (accumulated distance updated; reset when it rebuilds)
bool gs_decide(hidem_ctx *ctx, double currDist) {
    const long long t = ctx->step;
    bool regen = (t == ctx->startStep);
    if (ctx->P.gridRegenInterval != -1) {
        regen = ctx->P.gridRegenInterval > 0 && (t % ctx->P.gridRegenInterval) == 0;
    } else if (t % 10 == 0) {
        ctx->accumulatedDist += currDist;
        if (ctx->accumulatedDist >= ctx->interactDist / 2.0) regen = true;
    }
    if (t == ctx->P.firstBalanceTimestep) regen = true;
    if (!ctx->built) regen = true;
    if (regen) ctx->accumulatedDist = 0;
    return regen;
}

hidem_status gs_finish(hidem_ctx *ctx, double currDist) {
    if (gs_decide(ctx, currDist)) TRY(do_rebuild(ctx));
    return HIDEM_OK;
}

// HiDEMLib::gridService on one rank. `diffReady` says the device words already hold this
// step's maxima (computed by the previous fused step).
hidem_status grid_service(hidem_ctx *ctx, bool diffReady) {
    double cd = 0;
    if (gs_wants_diff(ctx)) {
        if (!diffReady) TRY(reduce_diff_now(ctx));
        TRY(read_diff_max(ctx, &cd));
    }
    return gs_finish(ctx, cd);
}

// Whether gridService can do anything at the current step, and the number of steps
// from the current one to the next step where it can.
bool gs_due(const hidem_ctx *ctx) {
    const long long t = ctx->step;
    const long long iv = ctx->P.gridRegenInterval;
    return !ctx->built || t == ctx->startStep || t == ctx->P.firstBalanceTimestep ||
           (iv == -1 && t % 10 == 0) || (iv > 0 && t % iv == 0);
}
long long gs_next_due(const hidem_ctx *ctx) {
    const long long t = ctx->step;
    const long long iv = ctx->P.gridRegenInterval;
    long long d = (long long)1 << 60;
    if (iv == -1) d = 10 - ((t % 10) + 10) % 10;
    else if (iv > 0) d = iv - ((t % iv) + iv) % iv;
    if (ctx->P.firstBalanceTimestep > t) d = std::min<long long>(d, ctx->P.firstBalanceTimestep - t);
    if (ctx->startStep > t) d = std::min<long long>(d, ctx->startStep - t);
    return d;
}

template <class LP>
const Consts<LP> &consts(hidem_ctx *ctx);
template <>
const Consts<float> &consts<float>(hidem_ctx *ctx) { return ctx->cf; }
template <>
const Consts<double> &consts<double>(hidem_ctx *ctx) { return ctx->cd; }

template <class LP>
StepArgs<LP> step_args(hidem_ctx *ctx) {
    StepArgs<LP> a{};
    a.in = recp<LP>(ctx, ctx->cur);
    a.out = recp<LP>(ctx, 1 - ctx->cur);
    a.type = ctx->type[ctx->ord];
    a.counts = ctx->counts;
    a.nOff = ctx->nOff;
    a.nbr = ctx->nbr;
    a.sOff = ctx->sOff;
    SideSet &s = ctx->side[ctx->curSide];
    a.sPartner = s.partner;
    for (int k = 0; k < 6; ++k) a.ct[k] = static_cast<LP *>(s.ct[k]);
    a.sState = s.state;
    a.linkState = ctx->linkState;
    a.sL0 = static_cast<const LP *>(s.L0);
    a.sLink = s.link;
    a.force = static_cast<LP *>(ctx->force);
    a.n = (int)ctx->n;
    a.step = ctx->step;
    a.bendBreak = consts<LP>(ctx).bendBreak;
    a.maxLoad = consts<LP>(ctx).maxLoad;
    a.diffMax = ctx->diffMax;
    a.events = ctx->events;
    a.eventCount = ctx->eventCount;
    a.eventCap = ctx->eventCap;
    a.errorFlag = ctx->errorFlag;
    return a;
}


// HiDEMDefLinkBreakFunc gate of the sample main: t * dt > breakTime, in lp
// (MainMeshBlock.cpp:312).
template <class LP>
bool break_active(hidem_ctx *ctx, long long t) {
    const Consts<LP> &c = consts<LP>(ctx);
    return (LP)((LP)t * c.dt) > c.breakTime;
}

template <class LP>
hidem_status link_update_now(hidem_ctx *ctx, long long tagStep) {
    SideSet &s = ctx->side[ctx->curSide];
    // the ends' slots are refreshed at every rebuild; before one, from the current slotOf
    if (!ctx->built && ctx->L > 0) {
        launch_link_slots(ctx->linkA, ctx->linkB, ctx->slotOf, ctx->L, ctx->linkSlotA, ctx->linkSlotB, ctx->stream);
        ctx->launches += 1;
    }
    launch_link_break<LP>(consts<LP>(ctx), recp<LP>(ctx, ctx->cur), ctx->linkSlotA, ctx->linkSlotB,
                          ctx->sideSlot[ctx->curSide], s.state, ctx->linkState,
                          static_cast<const LP *>(ctx->L0link), ctx->L, tagStep, ctx->events,
                          ctx->eventCount, ctx->eventCap, ctx->stream);
    if (ctx->L > 0) ctx->launches += 1;
    return HIDEM_OK;
}

hidem_status profile_pair(hidem_ctx *ctx, cudaEvent_t *e0, cudaEvent_t *e1) {
    while (ctx->evPool.size() < ctx->evUsed + 2) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        ctx->evPool.push_back(e);
    }
    *e0 = ctx->evPool[ctx->evUsed];
    *e1 = ctx->evPool[ctx->evUsed + 1];
    ctx->evUsed += 2;
    return HIDEM_OK;
}

// Step-kernel autotuner: the first kTuneRounds * 3 fused steps of a context cycle
// through the candidate kernels with an event pair around each launch; after the rounds
// have run, the fastest (summed over all but the first round) is kept.
constexpr int kTuneCandidates[] = {HIDEM_STEP_KERNEL_ITEMS, HIDEM_STEP_KERNEL_THREAD,
                                   HIDEM_STEP_KERNEL_THREAD_CAPPED, HIDEM_STEP_KERNEL_THREAD_ASYNC,
                                   HIDEM_STEP_KERNEL_TWO_PASS};
constexpr int kNumCandidates = (int)(sizeof(kTuneCandidates) / sizeof(int));
constexpr int kTuneRounds = 3;
static_assert(2 * kNumCandidates * kTuneRounds <= (int)(sizeof(hidem_ctx::tuneEv) / sizeof(cudaEvent_t)),
              "one event pair per tuning step");

// the force kernel of a step kernel choice (TWO_PASS: the register-capped one, unfused)
int force_kernel(int k) { return k == HIDEM_STEP_KERNEL_TWO_PASS ? HIDEM_STEP_KERNEL_THREAD_CAPPED : k; }

int step_kernel_now(hidem_ctx *ctx, cudaEvent_t *e0, cudaEvent_t *e1) {
    *e0 = *e1 = nullptr;
    if (ctx->stepKernel != HIDEM_STEP_KERNEL_AUTO) return ctx->stepKernel;
    if (ctx->tunedKernel != HIDEM_STEP_KERNEL_AUTO) return ctx->tunedKernel;
    if (ctx->tuneStep < kNumCandidates * kTuneRounds) {
        const int k = ctx->tuneStep++;
        for (int q = 0; q < 2; ++q)
            if (!ctx->tuneEv[2 * k + q] && cudaEventCreate(&ctx->tuneEv[2 * k + q]) != cudaSuccess)
                ctx->tuneEv[2 * k + q] = nullptr;
        *e0 = ctx->tuneEv[2 * k];
        *e1 = ctx->tuneEv[2 * k + 1];
        return kTuneCandidates[k % kNumCandidates];
    }
    return HIDEM_STEP_KERNEL_THREAD;  // rounds done, choice made at the next sync
}

// the kernel of a launch outside the tuning rounds
int step_kernel_settled(const hidem_ctx *ctx) {
    if (ctx->stepKernel != HIDEM_STEP_KERNEL_AUTO) return ctx->stepKernel;
    if (ctx->tunedKernel != HIDEM_STEP_KERNEL_AUTO) return ctx->tunedKernel;
    return HIDEM_STEP_KERNEL_THREAD;
}

// called after the stream has been synchronised
void step_kernel_resolve(hidem_ctx *ctx) {
    if (ctx->stepKernel != HIDEM_STEP_KERNEL_AUTO || ctx->tunedKernel != HIDEM_STEP_KERNEL_AUTO ||
        ctx->tuneStep < kNumCandidates * kTuneRounds)
        return;
    double t[kNumCandidates] = {};
    for (int k = kNumCandidates; k < kNumCandidates * kTuneRounds; ++k) {
        float ms = 0;
        if (!ctx->tuneEv[2 * k] || !ctx->tuneEv[2 * k + 1] ||
            cudaEventElapsedTime(&ms, ctx->tuneEv[2 * k], ctx->tuneEv[2 * k + 1]) != cudaSuccess) {
            cudaGetLastError();
            ctx->tunedKernel = HIDEM_STEP_KERNEL_THREAD;
            return;
        }
        t[k % kNumCandidates] += ms;
    }
    int best = 0;
    for (int q = 1; q < kNumCandidates; ++q)
        if (t[q] < t[best]) best = q;
    ctx->tunedKernel = kTuneCandidates[best];
}

// n whole timesteps, one fused kernel each (MainMeshBlock.cpp:274-323).
template <class LP>
hidem_status run_steps(hidem_ctx *ctx, int nsteps) {
    bool pending = false;      // link update of step-1 not applied yet
    long long pendingStep = 0;
    bool diffReady = false;
    for (int s = 0; s < nsteps; ++s) {
        const long long t = ctx->step;
        cudaEvent_t e0 = nullptr, e1 = nullptr, t0 = nullptr, t1 = nullptr;
        const int kern = step_kernel_now(ctx, &t0, &t1);
        if (kern == HIDEM_STEP_KERNEL_TWO_PASS && pending) {
            // the previous (fused) step's link update, where the reference runs it
            TRY(link_update_now<LP>(ctx, pendingStep));
            pending = false;
        }
        if (ctx->P.gridRegenInterval == -1 && t % 10 == 0) {
            // gridService reads the maxima of the diffs at the start of step t
            TRY(grid_service(ctx, diffReady));
        } else {
            TRY(grid_service(ctx, false));
        }
        diffReady = false;
        if (kern == HIDEM_STEP_KERNEL_TWO_PASS) {
            // force pass, integrate pass (in place), break pass (MainMeshBlock.cpp:295-320)
            if (ctx->profile) TRY(profile_pair(ctx, &e0, &e1));
            if (e0) CK(cudaEventRecord(e0, ctx->stream));
            if (t0) CK(cudaEventRecord(t0, ctx->stream));
            launch_step<LP>(consts<LP>(ctx), step_args<LP>(ctx), false, (int)ctx->maxNeigh,
                            (int)ctx->maxLinksPP, HIDEM_STEP_KERNEL_THREAD_CAPPED, ctx->stream);
            launch_integrate<LP>(consts<LP>(ctx), recp<LP>(ctx, ctx->cur), ctx->type[ctx->ord],
                                 static_cast<const LP *>(ctx->force), (int)ctx->n, ctx->stream);
            ctx->launches += 2;
            if (break_active<LP>(ctx, t)) TRY(link_update_now<LP>(ctx, t));
            if (t1) CK(cudaEventRecord(t1, ctx->stream));
            if (e1) CK(cudaEventRecord(e1, ctx->stream));
            ctx->step = t + 1;
            continue;
        }
        StepArgs<LP> a = step_args<LP>(ctx);
        a.breakPending = pending ? 1 : 0;
        a.breakStep = pendingStep;
        a.reduceDiff = (ctx->P.gridRegenInterval == -1 && (t + 1) % 10 == 0) ? 1 : 0;
        if (a.reduceDiff) {
            CK(cudaMemsetAsync(ctx->diffMax, 0, 3 * sizeof(unsigned long long), ctx->stream));
            diffReady = true;
        }
        if (ctx->profile) TRY(profile_pair(ctx, &e0, &e1));
        if (e0) CK(cudaEventRecord(e0, ctx->stream));
        if (t0) CK(cudaEventRecord(t0, ctx->stream));
        launch_step<LP>(consts<LP>(ctx), a, true, (int)ctx->maxNeigh, (int)ctx->maxLinksPP, kern,
                        ctx->stream);
        if (t1) CK(cudaEventRecord(t1, ctx->stream));
        if (e1) CK(cudaEventRecord(e1, ctx->stream));
        ctx->launches += 1;
        ctx->cur = 1 - ctx->cur;  // the slot order (type / orig / cellOf) is unchanged
        pending = break_active<LP>(ctx, t);
        pendingStep = t;
        ctx->step = t + 1;  // finalizeTs
    }
    if (pending) TRY(link_update_now<LP>(ctx, pendingStep));
    CK(cudaGetLastError());
    TRY(check_device_error(ctx));
    step_kernel_resolve(ctx);
    return HIDEM_OK;
}

template <class LP>
SoaIn<LP> soa_layout(void *base, long long n) {
    // caller-order particle fields as contiguous arrays inside one device buffer
    SoaIn<LP> s;
    char *b = static_cast<char *>(base);
    s.x = reinterpret_cast<const double *>(b);
    s.y = s.x + n;
    s.z = s.y + n;
    const LP *lp = reinterpret_cast<const LP *>(b + 24 * n);
    for (int k = 0; k < 6; ++k) s.d[k] = lp + k * n;
    s.r = lp + 6 * n;
    for (int k = 0; k < 3; ++k) s.th[k] = lp + (7 + k) * n;
    return s;
}

template <class LP>
hidem_status upload_particles(hidem_ctx *ctx, const hidem_particle_soa *p, long long n) {
    cudaStream_t st = ctx->stream;
    // stage the caller's arrays in the second record buffer, pack into the first
    SoaIn<LP> s = soa_layout<LP>(ctx->rec[1], n);
    CK(cudaMemcpyAsync((void *)s.x, p->xCord, 8 * (size_t)n, cudaMemcpyDefault, st));
    CK(cudaMemcpyAsync((void *)s.y, p->yCord, 8 * (size_t)n, cudaMemcpyDefault, st));
    CK(cudaMemcpyAsync((void *)s.z, p->zCord, 8 * (size_t)n, cudaMemcpyDefault, st));
    const void *d[6] = {p->xDiff, p->yDiff, p->zDiff, p->uDiff, p->vDiff, p->wDiff};
    const void *th[3] = {p->xTheta, p->yTheta, p->zTheta};
    for (int k = 0; k < 6; ++k) {
        if (d[k]) CK(cudaMemcpyAsync((void *)s.d[k], d[k], sizeof(LP) * (size_t)n, cudaMemcpyDefault, st));
        else s.d[k] = nullptr;
    }
    CK(cudaMemcpyAsync((void *)s.r, p->radius, sizeof(LP) * (size_t)n, cudaMemcpyDefault, st));
    for (int k = 0; k < 3; ++k) {
        if (th[k]) CK(cudaMemcpyAsync((void *)s.th[k], th[k], sizeof(LP) * (size_t)n, cudaMemcpyDefault, st));
        else s.th[k] = nullptr;
    }
    launch_pack_records<LP>(s, (int)n, static_cast<PRec<LP> *>(ctx->rec[0]), st);
    ctx->launches += 1;
    return HIDEM_OK;
}

}  // namespace

// Many contexts advanced together (no counterpart in the reference): one launch per
// timestep and group of contexts; runs of launches between two gridService points are
// replayed from CUDA graphs.
struct hidem_batch {
    std::vector<hidem_ctx *> ctxs;
    int mixed = 1;
    int device = 0;
    int flags = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    void *entries = nullptr;                 // device BatchEntry<LP>[nctx], then int[4 * nctx]:
                                             // the groups' particle CTA offsets, then their
                                             // link CTA offsets
    int *tbl = nullptr;                      // device: the entry of every CTA of each group's
    long long tblCap = 0;                    // particle launches, then of its link launch
    void *staging = nullptr;                 // pinned host copy of the entries
    unsigned long long *diff = nullptr;      // device diff maxima, 3 words per context
    unsigned long long *diffHost = nullptr;  // pinned
    cudaEvent_t uploaded = nullptr;
    bool uploadPending = false;
    std::map<int, cudaGraphExec_t> graphs;   // by run length, for one launch shape
    std::string shape;                       // the launch shape the graphs were captured for
    // contexts that share every constant but the break thresholds form a group: one launch
    // per group and step, the group's constants as kernel parameters
    struct Group {
        int first = 0, count = 0;             // entries [first, first + count)
        int fbOffset = 0;                     // its CTA offsets in the offset array
        long long blocks = 0;                 // CTAs of its particle launches
        long long linkBlocks = 0;             // CTAs of its break pass (at least 1)
        long long tblOffset = 0, ltblOffset = 0;  // its CTA-entry tables in tbl
        int maxC = 0, maxE = 0;
        std::vector<unsigned char> consts;    // Consts<LP> of the group
    };
    std::vector<Group> groups;
    std::vector<int> order;                  // context index of each entry
    long long launches = 0, graphLaunches = 0, uploads = 0;
};

namespace {

constexpr int kBatchMaxRun = 10;

hidem_status bfail(hidem_batch *b, hidem_status s, const char *fmt, ...) {
    char buf[640];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (b) b->err = buf;
    return s;
}

#define BCK(call)                                                                            \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return bfail(b, HIDEM_ERR_CUDA, "%s failed: %s (%s:%d)", #call,                  \
                         cudaGetErrorString(e_), __FILE__, __LINE__);                        \
    } while (0)

// a call on context `idx` failed: keep its text
#define BTRY(expr)                                                                           \
    do {                                                                                     \
        hidem_status s_ = (expr);                                                            \
        if (s_ != HIDEM_OK)                                                                  \
            return bfail(b, s_, "context %d: %s", idx, b->ctxs[idx]->err.c_str());           \
    } while (0)

void batch_clear_graphs(hidem_batch *b) {
    for (auto &g : b->graphs) cudaGraphExecDestroy(g.second);
    b->graphs.clear();
    b->shape.clear();
}

// For the length of one batch call every context queues its work on the batch's stream
// and folds its diff maxima into the batch's array; both are given back on exit (after
// the stream has drained, so the contexts' own streams see finished work).
struct BatchBind {
    hidem_batch *b;
    std::vector<cudaStream_t> streams;
    std::vector<unsigned long long *> diffs;
    explicit BatchBind(hidem_batch *bb) : b(bb) {
        for (size_t i = 0; i < b->ctxs.size(); ++i) {
            hidem_ctx *c = b->ctxs[i];
            streams.push_back(c->stream);
            diffs.push_back(c->diffMax);
            c->stream = b->stream;
            c->diffMax = b->diff + 3 * i;
        }
    }
    ~BatchBind() {
        cudaStreamSynchronize(b->stream);
        for (size_t i = 0; i < b->ctxs.size(); ++i) {
            b->ctxs[i]->stream = streams[i];
            b->ctxs[i]->diffMax = diffs[i];
        }
    }
};

// the kernel a batch run uses: the first context's fixed or tuned choice (the
// asynchronous-copy kernel has no batched form: its register-capped sibling stands in),
// else the register-capped one-thread-per-particle kernel
int batch_kernel(const hidem_batch *b) {
    const hidem_ctx *c = b->ctxs[0];
    // the two-pass step unless the first context names another kernel (measured on the
    // 256-block ensemble: 2.96 ms per step against 3.53 ms for the capped fused kernel)
    int k = HIDEM_STEP_KERNEL_TWO_PASS;
    if (c->stepKernel != HIDEM_STEP_KERNEL_AUTO) k = c->stepKernel;
    else if (c->tunedKernel != HIDEM_STEP_KERNEL_AUTO) k = c->tunedKernel;
    return k == HIDEM_STEP_KERNEL_THREAD_ASYNC ? HIDEM_STEP_KERNEL_THREAD_CAPPED : k;
}

// Groups of contexts with equal constants apart from the break thresholds (compared
// byte for byte; the constants are value-initialised and assigned field by field, so
// their padding compares equal), with their CTA counts and row widths for `kernel`.
template <class LP>
void batch_group(hidem_batch *b, int kernel) {
    const int nc = (int)b->ctxs.size();
    const int per = batch_particles_per_cta(kernel);
    std::vector<std::vector<unsigned char>> keys(nc);
    for (int idx = 0; idx < nc; ++idx) {
        Consts<LP> k;
        std::memcpy(&k, &consts<LP>(b->ctxs[idx]), sizeof k);
        k.bendBreak = LP(0);
        k.maxLoad = LP(0);
        const unsigned char *kb = reinterpret_cast<const unsigned char *>(&k);
        keys[idx].assign(kb, kb + sizeof k);
    }
    b->groups.clear();
    b->order.clear();
    std::vector<char> done(nc, 0);
    int fb = 0;
    for (int idx = 0; idx < nc; ++idx) {
        if (done[idx]) continue;
        hidem_batch::Group g;
        g.first = (int)b->order.size();
        g.fbOffset = fb;
        g.consts = keys[idx];
        for (int j = idx; j < nc; ++j) {
            if (done[j] || keys[j] != keys[idx]) continue;
            done[j] = 1;
            const hidem_ctx *c = b->ctxs[j];
            b->order.push_back(j);
            g.blocks += (c->n + per - 1) / per;
            g.linkBlocks += (c->L + kStepThreads - 1) / kStepThreads;
            g.maxC = std::max(g.maxC, (int)c->maxNeigh);
            g.maxE = std::max(g.maxE, (int)c->maxLinksPP);
        }
        g.count = (int)b->order.size() - g.first;
        // a group without links still launches one (idle) break CTA: a launch of no CTAs is
        // an error
        g.linkBlocks = std::max<long long>(g.linkBlocks, 1);
        fb += g.count + 1;
        b->groups.push_back(std::move(g));
    }
    long long t = 0;
    for (auto &g : b->groups) {
        g.tblOffset = t;
        t += g.blocks;
    }
    for (auto &g : b->groups) {
        g.ltblOffset = t;
        t += g.linkBlocks;
    }
}

// what identifies the launches of a run: graphs are re-captured when it changes
std::string batch_shape(const hidem_batch *b, int kernel) {
    std::string sh(reinterpret_cast<const char *>(&kernel), sizeof kernel);
    const long long tp = (long long)reinterpret_cast<uintptr_t>(b->tbl);
    sh.append(reinterpret_cast<const char *>(&tp), sizeof tp);
    for (const auto &g : b->groups) {
        const long long v[9] = {g.first, g.count, g.fbOffset, g.blocks, g.maxC, g.maxE,
                                g.linkBlocks, g.tblOffset, g.ltblOffset};
        sh.append(reinterpret_cast<const char *>(v), sizeof v);
        sh.append(g.consts.begin(), g.consts.end());
    }
    return sh;
}

template <class LP>
hidem_status batch_upload(hidem_batch *b, const std::vector<char> &pending, int kernel) {
    const int nc = (int)b->ctxs.size();
    if (b->uploadPending) BCK(cudaEventSynchronize(b->uploaded));
    BatchEntry<LP> *h = static_cast<BatchEntry<LP> *>(b->staging);
    int *fb = reinterpret_cast<int *>(h + nc);
    int *lfb = fb + 2 * nc;
    const int per = batch_particles_per_cta(kernel);
    for (const auto &g : b->groups) {
        int firstBlock = 0, firstLink = 0;
        for (int q = 0; q < g.count; ++q) {
            const int idx = b->order[g.first + q];
            hidem_ctx *c = b->ctxs[idx];
            BatchEntry<LP> e{};
            e.a = step_args<LP>(c);
            e.a.maxContacts = (int)c->maxNeigh;
            e.a.maxEnds = (int)c->maxLinksPP;
            e.rec[0] = recp<LP>(c, 0);
            e.rec[1] = recp<LP>(c, 1);
            e.step0 = c->step;
            e.cur0 = c->cur;
            e.pend0 = pending[idx] ? 1 : 0;
            e.reduceEvery10 = c->P.gridRegenInterval == -1 ? 1 : 0;
            e.slotA = c->linkSlotA;
            e.slotB = c->linkSlotB;
            e.sideSlot = c->sideSlot[c->curSide];
            e.L0link = static_cast<const LP *>(c->L0link);
            e.L = c->L;
            h[g.first + q] = e;
            fb[g.fbOffset + q] = firstBlock;
            firstBlock += (int)((c->n + per - 1) / per);
            lfb[g.fbOffset + q] = firstLink;
            firstLink += (int)((c->L + kStepThreads - 1) / kStepThreads);
        }
        fb[g.fbOffset + g.count] = firstBlock;
        lfb[g.fbOffset + g.count] = firstLink;
    }
    BCK(cudaMemcpyAsync(b->entries, h, sizeof(BatchEntry<LP>) * nc + sizeof(int) * 4 * nc,
                        cudaMemcpyHostToDevice, b->stream));
    BCK(cudaEventRecord(b->uploaded, b->stream));
    // the entry of every CTA: one table per group and launch grid, filled on the device from
    // the offsets just uploaded (a group without links keeps its one break CTA on entry 0)
    long long need = 0;
    for (const auto &g : b->groups) need = std::max(need, g.ltblOffset + g.linkBlocks);
    if (need > b->tblCap) {
        BCK(cudaStreamSynchronize(b->stream));
        if (b->tbl) BCK(cudaFree(b->tbl));
        b->tbl = nullptr;
        b->tblCap = 0;
        BCK(cudaMalloc((void **)&b->tbl, sizeof(int) * (size_t)need));
        b->tblCap = need;
    }
    BCK(cudaMemsetAsync(b->tbl, 0, sizeof(int) * (size_t)need, b->stream));
    const int *dfb = reinterpret_cast<const int *>(static_cast<const BatchEntry<LP> *>(b->entries) + nc);
    for (const auto &g : b->groups) {
        launch_block_table(dfb + g.fbOffset, g.count, b->tbl + g.tblOffset, b->stream);
        launch_block_table(dfb + 2 * nc + g.fbOffset, g.count, b->tbl + g.ltblOffset, b->stream);
        b->ctxs[0]->launches += 2;
    }
    BCK(cudaGetLastError());
    b->uploadPending = true;
    b->uploads += 1;
    return HIDEM_OK;
}

template <class LP>
void batch_enqueue_step(hidem_batch *b, int kernel, int run) {
    const int nc = (int)b->ctxs.size();
    const BatchEntry<LP> *ent = static_cast<const BatchEntry<LP> *>(b->entries);
    const int *fb = reinterpret_cast<const int *>(ent + nc);
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        const auto &g = b->groups[gi];
        if (g.blocks == 0) continue;
        Consts<LP> c;
        std::memcpy(&c, g.consts.data(), sizeof c);
        if (kernel == HIDEM_STEP_KERNEL_TWO_PASS)
            launch_two_pass_batch<LP>(c, ent + g.first, fb + g.fbOffset, b->tbl + g.tblOffset,
                                      fb + 2 * nc + g.fbOffset, b->tbl + g.ltblOffset, run,
                                      (int)g.blocks, (int)g.linkBlocks, b->stream);
        else
            launch_step_batch<LP>(c, ent + g.first, fb + g.fbOffset, b->tbl + g.tblOffset, run,
                                  (int)g.blocks, g.maxC, g.maxE, kernel, b->stream);
    }
}

// `run` timesteps of the batch (one launch per group each), from a cached graph when
// graphs are on
template <class LP>
hidem_status batch_launch_run(hidem_batch *b, int run, int kernel) {
    const std::string sh = batch_shape(b, kernel);
    if (sh != b->shape) {
        batch_clear_graphs(b);
        b->shape = sh;
    }
    if (!(b->flags & HIDEM_BATCH_GRAPHS)) {
        for (int j = 0; j < run; ++j) batch_enqueue_step<LP>(b, kernel, j);
        BCK(cudaGetLastError());
        return HIDEM_OK;
    }
    auto it = b->graphs.find(run);
    if (it == b->graphs.end()) {
        cudaGraph_t g = nullptr;
        BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        for (int j = 0; j < run; ++j) batch_enqueue_step<LP>(b, kernel, j);
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (le != cudaSuccess || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return bfail(b, HIDEM_ERR_CUDA, "capturing the batched step failed: %s",
                         cudaGetErrorString(le != cudaSuccess ? le : ce));
        }
        cudaGraphExec_t x = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&x, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess)
            return bfail(b, HIDEM_ERR_CUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(ie));
        it = b->graphs.emplace(run, x).first;
    }
    BCK(cudaGraphLaunch(it->second, b->stream));
    b->graphLaunches += 1;
    return HIDEM_OK;
}

// nsteps timesteps of every context: per step exactly the work hidem_step does for each
// context alone (gridService, the fused step, the pending link update), in one launch
// per group.
// The rebuilds of the contexts in `list`, each on its own stream (`own`, the streams the
// contexts had before the batch bound them to its stream), several at a time from a few
// host threads, so that their host round trips and small kernels overlap (buffers grow
// with stream-ordered allocations, which do not wait for the rest of the device). The
// batch's stream is drained first (the records come from its launches) and every
// rebuild has completed on return.
hidem_status batch_rebuild_set(hidem_batch *b, const std::vector<int> &list,
                               const std::vector<cudaStream_t> &own, int maxThreads) {
    const int nthreads = (int)std::min<size_t>(list.size(), (size_t)maxThreads);
    std::atomic<int> next{0};
    std::vector<hidem_status> st(list.size(), HIDEM_OK);
    int device = 0;
    BCK(cudaGetDevice(&device));
    auto work = [&]() {
        cudaSetDevice(device);
        for (int k; (k = next.fetch_add(1)) < (int)list.size();) {
            hidem_ctx *c = b->ctxs[list[k]];
            c->stream = own[list[k]];
            st[k] = do_rebuild(c);
            if (cudaStreamSynchronize(c->stream) != cudaSuccess && st[k] == HIDEM_OK)
                st[k] = fail(c, HIDEM_ERR_CUDA, "rebuild stream synchronisation failed");
            c->stream = b->stream;
        }
    };
    if (nthreads <= 1) {
        work();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t) pool.emplace_back(work);
        for (auto &t : pool) t.join();
    }
    for (size_t k = 0; k < list.size(); ++k)
        if (st[k] != HIDEM_OK)
            return bfail(b, st[k], "context %d: %s", list[k], b->ctxs[list[k]]->err.c_str());
    return HIDEM_OK;
}

hidem_status batch_rebuild(hidem_batch *b, const std::vector<int> &list,
                           const std::vector<cudaStream_t> &own) {
    BCK(cudaStreamSynchronize(b->stream));
    return batch_rebuild_set(b, list, own, 8);
}

template <class LP>
hidem_status batch_run(hidem_batch *b, int nsteps) {
    const int nc = (int)b->ctxs.size();
    for (int idx = 0; idx < nc; ++idx) BCK(cudaStreamSynchronize(b->ctxs[idx]->stream));
    BatchBind bind(b);
    BCK(cudaMemsetAsync(b->diff, 0, 3 * sizeof(unsigned long long) * nc, b->stream));
    std::vector<char> pending(nc, 0), diffReady(nc, 0);
    std::vector<long long> pendStep(nc, 0);
    bool dirty = true;
    int s = 0;
    while (s < nsteps) {
        // gridService of every context due at its current step; one copy of the maxima
        bool anyDue = false, anyRead = false;
        for (int idx = 0; idx < nc; ++idx) {
            hidem_ctx *c = b->ctxs[idx];
            if (!gs_due(c)) continue;
            anyDue = true;
            if (gs_wants_diff(c)) {
                anyRead = true;
                if (!diffReady[idx]) BTRY(reduce_diff_now(c));
            }
        }
        if (anyRead) {
            BCK(cudaMemcpyAsync(b->diffHost, b->diff, 3 * sizeof(unsigned long long) * nc,
                                cudaMemcpyDeviceToHost, b->stream));
            BCK(cudaStreamSynchronize(b->stream));
        }
        if (anyDue) {
            std::vector<int> regen;
            for (int idx = 0; idx < nc; ++idx) {
                hidem_ctx *c = b->ctxs[idx];
                if (!gs_due(c)) continue;
                double mx[3] = {0.0, 0.0, 0.0};
                if (gs_wants_diff(c)) diff_words<LP>(b->diffHost + 3 * idx, mx);
                const double cd = gs_wants_diff(c) ? curr_dist<LP>(mx) : 0.0;
                if (gs_decide(c, cd)) regen.push_back(idx);
            }
            if (!regen.empty()) TRY(batch_rebuild(b, regen, bind.streams));
            dirty = true;
        }
        long long run = nsteps - s;
        for (int idx = 0; idx < nc; ++idx) run = std::min(run, gs_next_due(b->ctxs[idx]));
        run = std::min<long long>(run, kBatchMaxRun);
        const int kernel = batch_kernel(b);
        bool oneLaunch = !(b->flags & HIDEM_BATCH_PER_CONTEXT);
        if (oneLaunch) {
            if (dirty || b->shape.compare(0, sizeof kernel, reinterpret_cast<const char *>(&kernel),
                                          sizeof kernel) != 0) {
                // layouts or the kernel changed: regroup and lay the entries out again
                batch_group<LP>(b, kernel);
                dirty = true;
            }
            for (const auto &g : b->groups) {
                if (g.blocks > 0x7fffffffLL)
                    return bfail(b, HIDEM_ERR_CAPACITY, "too many particles for one batched launch");
                if (g.linkBlocks > 0x7fffffffLL)
                    return bfail(b, HIDEM_ERR_CAPACITY, "too many links for one batched launch");
                if (kernel == HIDEM_STEP_KERNEL_ITEMS && !batch_fits<LP>(g.maxC, g.maxE))
                    oneLaunch = false;
            }
        }
        hidem_ctx *c0 = b->ctxs[0];
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (c0->profile) {
            const int idx = 0;
            BTRY(profile_pair(c0, &e0, &e1));
            BCK(cudaEventRecord(e0, b->stream));
        }
        const bool twoPass = oneLaunch && kernel == HIDEM_STEP_KERNEL_TWO_PASS;
        if (twoPass) {
            // a link update still owed by a fused run, before the two-pass steps
            for (int idx = 0; idx < nc; ++idx)
                if (pending[idx]) {
                    BTRY(link_update_now<LP>(b->ctxs[idx], pendStep[idx]));
                    pending[idx] = 0;
                }
        }
        if (oneLaunch) {
            // every run's launches take their steps as 0 .. run - 1 after the entries' first
            // step (parameters fixed in a captured run): each run starts from the host's step
            // state, laid out again
            TRY(batch_upload<LP>(b, pending, kernel));
            dirty = false;
            TRY(batch_launch_run<LP>(b, (int)run, kernel));
            const long long per = twoPass ? 3 : 1;
            b->launches += per * run * (long long)b->groups.size();
            c0->launches += per * run * (long long)b->groups.size();
        } else {
            // per-context launches asked for, or rows too wide for the item kernel: the
            // single-context launch sequence, context after context
            dirty = true;
            for (int j = 0; j < run; ++j) {
                for (int idx = 0; idx < nc; ++idx) {
                    hidem_ctx *c = b->ctxs[idx];
                    const long long t = c->step + j;
                    StepArgs<LP> a = step_args<LP>(c);
                    const int par = (c->cur + j) & 1;
                    a.in = recp<LP>(c, par);
                    a.out = recp<LP>(c, par ^ 1);
                    a.step = t;
                    a.breakStep = t - 1;
                    a.breakPending = j > 0 ? (break_active<LP>(c, t - 1) ? 1 : 0) : (pending[idx] ? 1 : 0);
                    a.reduceDiff = (c->P.gridRegenInterval == -1 && (t + 1) % 10 == 0) ? 1 : 0;
                    if (a.reduceDiff)
                        BCK(cudaMemsetAsync(c->diffMax, 0, 3 * sizeof(unsigned long long), b->stream));
                    launch_step<LP>(consts<LP>(c), a, true, (int)c->maxNeigh, (int)c->maxLinksPP,
                                    force_kernel(step_kernel_settled(c)), b->stream);
                    c->launches += 1;
                    b->launches += 1;
                }
            }
            BCK(cudaGetLastError());
        }
        if (e1) BCK(cudaEventRecord(e1, b->stream));
        // the host's copy of each context's step state (finalizeTs per step)
        for (int idx = 0; idx < nc; ++idx) {
            hidem_ctx *c = b->ctxs[idx];
            for (long long j = 0; j < run; ++j) {
                const long long t = c->step;
                // two-pass steps apply their link update in the step and integrate in place
                pending[idx] = (!twoPass && break_active<LP>(c, t)) ? 1 : 0;
                pendStep[idx] = t;
                diffReady[idx] = (c->P.gridRegenInterval == -1 && (t + 1) % 10 == 0) ? 1 : 0;
                if (!twoPass) c->cur = 1 - c->cur;
                c->step = t + 1;
            }
        }
        s += (int)run;
    }
    for (int idx = 0; idx < nc; ++idx)
        if (pending[idx]) BTRY(link_update_now<LP>(b->ctxs[idx], pendStep[idx]));
    BCK(cudaGetLastError());
    for (int idx = 0; idx < nc; ++idx) BTRY(check_device_error(b->ctxs[idx]));
    return HIDEM_OK;
}

}  // namespace

namespace hidem {
hidem_status ctx_fail(hidem_ctx *ctx, hidem_status s, const std::string &msg) {
    return fail(ctx, s, "%s", msg.c_str());
}
int ctx_precision(const hidem_ctx *ctx) { return ctx->P.precision; }
}  // namespace hidem

// =================================================================== C ABI

namespace {
// the collision mesh's query lists for the current particles and parameters
hidem_status prune_mesh(hidem_ctx *ctx);
}  // namespace

extern "C" {

int hidem_abi_version(void) { return HIDEM_B200_ABI_VERSION; }

const char *hidem_create_error(void) { return g_create_error.c_str(); }

void hidem_params_default(hidem_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->dt = 0.0001;
    p->scale = 1.0;
    p->E = 1e+09;
    p->beamWidth = 0.6;
    p->damping = 1000.0;
    p->dampingRotation = 1000.0;
    p->attractDistance = 0.0;
    p->attractScaleForce = 0.0;
    p->maxLoad = 0.35;
    p->bendBreak = 0.35;
    p->breakTime = 10.0;
    p->g = 9.81;
    p->rhoIce = 910.0;
    p->rhoWater = 1030.0;
    p->waterLevel = 0.0;
    p->airDrag = 1.0;
    p->waterDrag = 10.0;
    p->bedDrag = 1000.0;
    p->bedStiffness = 2e+08;
    p->bedInteract = 2.0;
    p->maxVel = 20.0;
    p->maxRot = 5.0;
    p->searchDistanceScale = 1.4;
    p->gridRegenInterval = -1;
    p->firstBalanceTimestep = 2000;
    p->maxRadius = 0.5;
    p->bedHeight = 0.0;
    p->bedFriction = 1.0;
    p->precision = HIDEM_PREC_MIXED;
}

hidem_status hidem_create(const hidem_params *params, int device, hidem_ctx **out) {
    g_create_error.clear();
    if (!out) {
        g_create_error = "out is NULL";
        return HIDEM_ERR_ARG;
    }
    *out = nullptr;
    hidem_ctx *ctx = new hidem_ctx();
    hidem_status s = apply_params(ctx, params);
    if (s != HIDEM_OK) {
        g_create_error = ctx->err;
        delete ctx;
        return s;
    }
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || device < 0 || device >= count) {
        g_create_error = std::string("no CUDA device ") + std::to_string(device) + ": " +
                         (e != cudaSuccess ? cudaGetErrorString(e) : "index out of range");
        delete ctx;
        return HIDEM_ERR_CUDA;
    }
    ctx->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->smCount, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) {
        // the contexts' buffers come from the device's default stream-ordered pool: keep up
        // to 8 GiB of freed blocks for reuse (later contexts, regrown buffers) instead of
        // returning them to the driver at every synchronisation
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = 8ull << 30;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (e != cudaSuccess) {
        g_create_error = std::string("CUDA setup failed: ") + cudaGetErrorString(e);
        delete ctx;
        return HIDEM_ERR_CUDA;
    }
    s = dalloc(ctx, &ctx->errorFlag, 1);
    if (s == HIDEM_OK) s = dalloc(ctx, &ctx->diffMax, 3);
    if (s == HIDEM_OK) s = dalloc(ctx, &ctx->eventCount, 1);
    if (s == HIDEM_OK) s = dalloc(ctx, &ctx->boundsPartial, 6 * 4 * ctx->smCount + 6);
    if (s == HIDEM_OK) s = dalloc(ctx, &ctx->boundsOut, 6);
    if (s == HIDEM_OK) s = dalloc(ctx, &ctx->offTotal, 4);  // a scan total + the count statistics
    if (s == HIDEM_OK) {
        cudaMemsetAsync(ctx->errorFlag, 0, sizeof(int), ctx->stream);
        cudaMemsetAsync(ctx->eventCount, 0, sizeof(unsigned long long), ctx->stream);
        e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) s = fail(ctx, HIDEM_ERR_CUDA, "%s", cudaGetErrorString(e));
    }
    if (s != HIDEM_OK) {
        g_create_error = ctx->err;
        hidem_destroy(ctx);
        return s;
    }
    *out = ctx;
    return HIDEM_OK;
}

void hidem_destroy(hidem_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int b = 0; b < 2; ++b) {
        dfree(ctx->rec[b]);
        dfree(ctx->type[b]);
        dfree(ctx->orig[b]);
        dfree(ctx->cellOf[b]);
        dfree(ctx->sideSlot[b]);
        side_free(ctx->side[b]);
    }
    dfree(ctx->slotOf);
    dfree(ctx->perm);
    dfree(ctx->bigCells);
    dfree(ctx->haloSendPos);
    dfree(ctx->force);
    dfree(ctx->cellCount);
    dfree(ctx->cellStart);
    dfree(ctx->cursor);
    dfree(ctx->scanSums32);
    dfree(ctx->scanSums64);
    dfree(ctx->boundsPartial);
    dfree(ctx->boundsOut);
    dfree(ctx->counts);
    dfree(ctx->blockWidth);
    dfree(ctx->nOff);
    dfree(ctx->sOff);
    dfree(ctx->offTotal);
    dfree(ctx->nbr);
    dfree(ctx->linkA);
    dfree(ctx->linkB);
    dfree(ctx->L0link);
    dfree(ctx->linkState);
    dfree(ctx->linkSlotA);
    dfree(ctx->linkSlotB);
    dfree(ctx->plStart);
    dfree(ctx->plLink);
    dfree(ctx->plEnd);
    dfree(ctx->events);
    dfree(ctx->eventCount);
    dfree(ctx->diffMax);
    dfree(ctx->errorFlag);
    for (cudaEvent_t e : ctx->evPool) cudaEventDestroy(e);
    dfree(ctx->dLinkOwners);
    dfree(ctx->dLinkNum);
    dfree(ctx->dLinkKeys);
    dfree(ctx->dLinkKeyA);
    dfree(ctx->dLinkKeyB);
    for (void *m : ctx->mapData)
        if (m) cudaFree(m);
    for (int k = 0; k < 3; ++k) {
        dfree(ctx->meshVtx[k]);
        dfree(ctx->meshNrm[k]);
        dfree(ctx->meshFace[k]);
    }
    dfree(ctx->meshSizes);
    dfree(ctx->meshStarts);
    dfree(ctx->meshValues);
    dfree(ctx->meshQSizes);
    dfree(ctx->meshQStarts);
    dfree(ctx->meshQValues);
    dfree(ctx->meshKeep);
    dfree(ctx->energyBuf);
    dfree(ctx->haloSend);
    dfree(ctx->haloRecv);
    for (cudaEvent_t e : ctx->tuneEv)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *hidem_last_error(const hidem_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

hidem_status hidem_set_params(hidem_ctx *ctx, const hidem_params *params) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (params && params->precision != ctx->P.precision)
        return fail(ctx, HIDEM_ERR_ARG, "precision cannot change after creation");
    TRY(apply_params(ctx, params));
    return prune_mesh(ctx);
}

hidem_status hidem_set_timestep(hidem_ctx *ctx, int64_t step) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (step < 0) return fail(ctx, HIDEM_ERR_ARG, "negative timestep");
    ctx->step = step;
    ctx->startStep = step;
    ctx->built = false;
    return HIDEM_OK;
}

hidem_status hidem_set_particles(hidem_ctx *ctx, const hidem_particle_soa *p, int64_t n) {
    NvtxRange nvtx_range("set_particles");
    if (!ctx) return HIDEM_ERR_ARG;
    if (!p || n <= 0) return fail(ctx, HIDEM_ERR_ARG, "need at least one particle");
    if (n >= (1ll << 31) - 64) return fail(ctx, HIDEM_ERR_CAPACITY, "n = %lld exceeds int32 indexing", (long long)n);
    if (!p->xCord || !p->yCord || !p->zCord || !p->radius)
        return fail(ctx, HIDEM_ERR_ARG, "xCord/yCord/zCord/radius are required");
    CK(cudaSetDevice(ctx->device));
    const size_t lp = ctx->lp;
    const size_t recBytes = ctx->mixed ? sizeof(PRec<float>) : sizeof(PRec<double>);
    for (int b = 0; b < 2; ++b) {
        TRY(dalloc_bytes(ctx, &ctx->rec[b], recBytes * (size_t)n));
        TRY(dalloc(ctx, &ctx->type[b], n));
        TRY(dalloc(ctx, &ctx->orig[b], n));
        TRY(dalloc(ctx, &ctx->cellOf[b], n));
    }
    TRY(dalloc(ctx, &ctx->slotOf, n));
    TRY(dalloc(ctx, &ctx->perm, n));
    TRY(dalloc(ctx, &ctx->bigCells, n / kSmallCell + 2));
    TRY(dalloc_bytes(ctx, &ctx->force, 6 * lp * (size_t)n));
    TRY(dalloc(ctx, &ctx->counts, n));
    const long long nb32 = nblocks32(n);
    TRY(dalloc(ctx, &ctx->blockWidth, nb32 + 1));
    TRY(dalloc(ctx, &ctx->nOff, nb32 + 1));
    TRY(dalloc(ctx, &ctx->sOff, nb32 + 1));
    ctx->cur = 0;
    ctx->ord = 0;
    TRY(ctx->mixed ? upload_particles<float>(ctx, p, n) : upload_particles<double>(ctx, p, n));
    if (p->type)
        CK(cudaMemcpyAsync(ctx->type[0], p->type, (size_t)n, cudaMemcpyDefault, ctx->stream));
    else
        CK(cudaMemsetAsync(ctx->type[0], 0, (size_t)n, ctx->stream));
    launch_iota32(ctx->orig[0], (int)n, ctx->stream);
    launch_iota32(ctx->slotOf, (int)n, ctx->stream);
    ctx->launches += 2;
    CK(cudaMemsetAsync(ctx->counts, 0, 4 * (size_t)n, ctx->stream));
    CK(cudaMemsetAsync(ctx->force, 0, 6 * lp * (size_t)n, ctx->stream));
    ctx->owners.assign((size_t)n, 0);
    if (p->owners) CK(from_caller(ctx->owners.data(), p->owners, 4 * (size_t)n));
    ctx->keys.resize((size_t)n);
    if (p->globalKeys) CK(from_caller(ctx->keys.data(), p->globalKeys, 8 * (size_t)n));
    else for (int64_t i = 0; i < n; ++i) ctx->keys[i] = i;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    ctx->n = n;
    ctx->haveParticles = true;
    ctx->built = false;
    ctx->maxParticleRadius = -1.0;  // found on the device when a collision mesh needs it
    TRY(prune_mesh(ctx));
    ctx->startStep = ctx->step;
    // halo lists refer to particle indices of the previous particle set
    ctx->nHaloSend = ctx->nHaloRecv = 0;
    // a link set refers to particle indices of the previous particle set
    ctx->haveLinks = false;
    ctx->L = 0;
    return HIDEM_OK;
}

hidem_status hidem_set_links(hidem_ctx *ctx, const hidem_link_soa *l, int64_t L) {
    NvtxRange nvtx_range("set_links");
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "set particles before links");
    if (L < 0 || (L > 0 && (!l || !l->globalKeyEndA || !l->globalKeyEndB || !l->initialLen || !l->state)))
        return fail(ctx, HIDEM_ERR_ARG, "link arrays globalKeyEndA/B, initialLen, state are required");
    if (2 * L >= (1ll << 31)) return fail(ctx, HIDEM_ERR_CAPACITY, "L = %lld exceeds int32 side indexing", (long long)L);
    CK(cudaSetDevice(ctx->device));
    const long long n = ctx->n;
    const size_t lp = ctx->lp;
    // globalKey -> input index (LinkData::makeLocalPartEnds, PLiB/LinkData.h:91-115):
    // on the device when the keys are 0..n-1 in order or strictly ascending (a binary
    // search of the key table), else through a sorted key table on the host
    bool identity = true, ascending = true;
    {
        std::atomic<bool> all(true), up(true);
        const int64_t *k = ctx->keys.data();
        host_parallel(n, [&all, &up, k](long long a, long long b) {
            for (long long i = a; i < b && (all.load(std::memory_order_relaxed) || up.load(std::memory_order_relaxed)); ++i) {
                if (k[i] != i) all.store(false, std::memory_order_relaxed);
                if (i > 0 && !(k[i - 1] < k[i])) up.store(false, std::memory_order_relaxed);
            }
        });
        identity = all.load();
        ascending = up.load();
    }
    cudaStream_t st = ctx->stream;
    TRY(dalloc(ctx, &ctx->linkA, L));
    TRY(dalloc(ctx, &ctx->linkB, L));
    TRY(dalloc(ctx, &ctx->dLinkKeyA, L));
    TRY(dalloc(ctx, &ctx->dLinkKeyB, L));
    if (L > 0) {
        CK(cudaMemcpyAsync(ctx->dLinkKeyA, l->globalKeyEndA, 8 * (size_t)L, cudaMemcpyDefault, st));
        CK(cudaMemcpyAsync(ctx->dLinkKeyB, l->globalKeyEndB, 8 * (size_t)L, cudaMemcpyDefault, st));
    }
    long long bad = -1, self = -1;
    if (identity || ascending) {
        unsigned long long *mins = nullptr;
        long long *dkeys = nullptr;
        TRY(dalloc(ctx, &mins, 2));
        CK(cudaMemsetAsync(mins, 0xff, 2 * sizeof(unsigned long long), st));
        if (identity) {
            launch_link_keys_identity(ctx->dLinkKeyA, ctx->dLinkKeyB, L, n, ctx->linkA, ctx->linkB, mins,
                                      mins + 1, st);
        } else {
            TRY(dalloc(ctx, &dkeys, n));
            CK(cudaMemcpyAsync(dkeys, ctx->keys.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, st));
            launch_link_keys_sorted(dkeys, n, ctx->dLinkKeyA, ctx->dLinkKeyB, L, ctx->linkA, ctx->linkB,
                                    mins, mins + 1, st);
        }
        ctx->launches += 1;
        unsigned long long h[2];
        CK(cudaMemcpyAsync(h, mins, sizeof h, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        dfree(mins);
        if (dkeys) dfree(dkeys);
        if (h[0] != ~0ull) bad = (long long)h[0];
        if (h[1] != ~0ull) self = (long long)h[1];
    } else {
        // the caller's keys, where the host can read them
        std::vector<int64_t> hostKeyA, hostKeyB;
        const int64_t *keyA = l->globalKeyEndA, *keyB = l->globalKeyEndB;
        if (L > 0 && on_device(keyA)) {
            hostKeyA.resize((size_t)L);
            CK(cudaMemcpy(hostKeyA.data(), keyA, 8 * (size_t)L, cudaMemcpyDeviceToHost));
            keyA = hostKeyA.data();
        }
        if (L > 0 && on_device(keyB)) {
            hostKeyB.resize((size_t)L);
            CK(cudaMemcpy(hostKeyB.data(), keyB, 8 * (size_t)L, cudaMemcpyDeviceToHost));
            keyB = hostKeyB.data();
        }
        std::vector<std::pair<int64_t, int32_t>> km((size_t)n);
        for (long long i = 0; i < n; ++i) km[i] = {ctx->keys[i], (int32_t)i};
        std::sort(km.begin(), km.end());
        auto find = [&](int64_t key) -> int32_t {
            auto it = std::lower_bound(km.begin(), km.end(), std::make_pair(key, (int32_t)-1));
            if (it == km.end() || it->first != key) return -1;
            return it->second;
        };
        std::unique_ptr<int32_t[]> A(new int32_t[(size_t)std::max<long long>(L, 1)]);
        std::unique_ptr<int32_t[]> B(new int32_t[(size_t)std::max<long long>(L, 1)]);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < L; ++i) {
            A[i] = find(keyA[i]);
            B[i] = find(keyB[i]);
            if (A[i] < 0 || B[i] < 0) {
#pragma omp critical
                if (bad < 0 || i < bad) bad = i;
            } else if (A[i] == B[i]) {
#pragma omp critical
                if (self < 0 || i < self) self = i;
            }
        }
        if (bad < 0 && self < 0 && L > 0) {
            CK(cudaMemcpyAsync(ctx->linkA, A.get(), 4 * (size_t)L, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(ctx->linkB, B.get(), 4 * (size_t)L, cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
    }
    if (bad >= 0) {
        int64_t ka = 0, kb = 0;
        CK(from_caller(&ka, l->globalKeyEndA + bad, 8));
        CK(from_caller(&kb, l->globalKeyEndB + bad, 8));
        return fail(ctx, HIDEM_ERR_NOT_FOUND, "link %lld: dangling end (keys %lld, %lld)", bad,
                    (long long)ka, (long long)kb);
    }
    if (self >= 0) return fail(ctx, HIDEM_ERR_ARG, "link %lld joins a particle to itself", self);

    TRY(dalloc_bytes(ctx, &ctx->L0link, lp * (size_t)std::max<long long>(L, 1)));
    TRY(dalloc(ctx, &ctx->plStart, n + 1));
    TRY(dalloc(ctx, &ctx->plLink, 2 * L));
    TRY(dalloc(ctx, &ctx->plEnd, 2 * L));
    for (int b = 0; b < 2; ++b) TRY(dalloc(ctx, &ctx->sideSlot[b], 2 * L));
    side_free(ctx->side[0]);
    side_free(ctx->side[1]);
    TRY(side_alloc(ctx, ctx->side[0], 2 * L));
    ctx->curSide = 0;
    TRY(dalloc(ctx, &ctx->events, std::max<long long>(L, 1)));
    ctx->eventCap = std::max<long long>(L, 1);
    ctx->eventsRead = 0;
    TRY(ensure_scan(ctx, n + 2));
    int *deg = nullptr, *cursor = nullptr;
    TRY(dalloc(ctx, &deg, n + 1));
    TRY(dalloc(ctx, &cursor, n + 1));
    TRY(dalloc(ctx, &ctx->linkState, std::max<long long>(L, 1)));
    TRY(dalloc(ctx, &ctx->linkSlotA, std::max<long long>(L, 1)));
    TRY(dalloc(ctx, &ctx->linkSlotB, std::max<long long>(L, 1)));
    uint8_t *lstate = ctx->linkState;
    CK(cudaMemsetAsync(deg, 0, 4 * (size_t)(n + 1), st));
    CK(cudaMemsetAsync(cursor, 0, 4 * (size_t)(n + 1), st));
    if (L > 0) {
        CK(cudaMemcpyAsync(ctx->L0link, l->initialLen, lp * (size_t)L, cudaMemcpyDefault, st));
        CK(cudaMemcpyAsync(lstate, l->state, (size_t)L, cudaMemcpyDefault, st));
        for (int k = 0; k < 6; ++k) {
            if (l->CT[k])
                CK(cudaMemcpyAsync(ctx->side[0].ct[k], l->CT[k], lp * (size_t)(2 * L), cudaMemcpyDefault, st));
            else
                CK(cudaMemsetAsync(ctx->side[0].ct[k], 0, lp * (size_t)(2 * L), st));
        }
    }
    // per-particle link ends in ascending link index (LinkAccelSide::generateLinks) and the
    // flat initial side layout (side 2l+e)
    launch_link_lists(ctx->linkA, ctx->linkB, L, (int)n, deg, ctx->plStart, cursor, ctx->scanSums32,
                      ctx->plLink, ctx->plEnd, st);
    launch_side_init(lstate, L, ctx->sideSlot[0], ctx->side[0].state, st);
    ctx->launches += 7;
    // the fields only get_links returns: copied as given, or their defaults
    TRY(dalloc(ctx, &ctx->dLinkOwners, L));
    TRY(dalloc(ctx, &ctx->dLinkNum, L));
    TRY(dalloc(ctx, &ctx->dLinkKeys, L));
    if (L > 0) {
        if (l->owners) CK(cudaMemcpyAsync(ctx->dLinkOwners, l->owners, 4 * (size_t)L, cudaMemcpyDefault, st));
        else CK(cudaMemsetAsync(ctx->dLinkOwners, 0, 4 * (size_t)L, st));
        if (l->particleLinkNum) CK(cudaMemcpyAsync(ctx->dLinkNum, l->particleLinkNum, 4 * (size_t)L, cudaMemcpyDefault, st));
        else CK(cudaMemsetAsync(ctx->dLinkNum, 0, 4 * (size_t)L, st));
        if (l->globalKeys) CK(cudaMemcpyAsync(ctx->dLinkKeys, l->globalKeys, 8 * (size_t)L, cudaMemcpyDefault, st));
        else launch_iota64(ctx->dLinkKeys, L, st);
    }
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    dfree(deg);
    dfree(cursor);
    ctx->L = L;
    ctx->haveLinks = true;
    ctx->built = false;
    return HIDEM_OK;
}

hidem_status hidem_grid_service(hidem_ctx *ctx) {
    NvtxRange nvtx_range("gridService");
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles || !ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "particles and links must be set");
    CK(cudaSetDevice(ctx->device));
    return grid_service(ctx, false);
}

hidem_status hidem_regenerate(hidem_ctx *ctx) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles || !ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "particles and links must be set");
    CK(cudaSetDevice(ctx->device));
    ctx->accumulatedDist = 0;
    return do_rebuild(ctx);
}

hidem_status halo_forces(hidem_ctx *ctx, void *buf, bool pack);

// the split force pass; with sendBuf, the halo send records come out of the same kernel
// where the force pass is the thread-per-particle one, else from the pack kernel after it
static hidem_status compute_forces_into(hidem_ctx *ctx, void *sendBuf) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles || !ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "particles and links must be set");
    CK(cudaSetDevice(ctx->device));
    if (!ctx->built) TRY(do_rebuild(ctx));
    const int kern = force_kernel(step_kernel_settled(ctx));
    const bool fusedPack = sendBuf && ctx->nHaloSend > 0 && ctx->haloSendPos &&
                           (kern == HIDEM_STEP_KERNEL_THREAD || kern == HIDEM_STEP_KERNEL_THREAD_CAPPED);
    if (ctx->mixed) {
        StepArgs<float> a = step_args<float>(ctx);
        if (fusedPack) {
            a.sendPos = ctx->haloSendPos;
            a.sendBuf = static_cast<float *>(sendBuf);
        }
        launch_step<float>(ctx->cf, a, false, (int)ctx->maxNeigh, (int)ctx->maxLinksPP, kern,
                           ctx->stream);
    } else {
        StepArgs<double> a = step_args<double>(ctx);
        if (fusedPack) {
            a.sendPos = ctx->haloSendPos;
            a.sendBuf = static_cast<double *>(sendBuf);
        }
        launch_step<double>(ctx->cd, a, false, (int)ctx->maxNeigh, (int)ctx->maxLinksPP, kern,
                            ctx->stream);
    }
    ctx->launches += 1;
    CK(cudaGetLastError());
    if (sendBuf && !fusedPack) TRY(halo_forces(ctx, sendBuf, true));
    return HIDEM_OK;
}

hidem_status hidem_compute_forces(hidem_ctx *ctx) {
    NvtxRange nvtx_range("computePartForce");
    return compute_forces_into(ctx, nullptr);
}

hidem_status hidem_compute_forces_packed(hidem_ctx *ctx, void *device_out) {
    NvtxRange nvtx_range("computePartForce + halo pack");
    if (!ctx) return HIDEM_ERR_ARG;
    if (ctx->nHaloSend > 0 && !device_out) return fail(ctx, HIDEM_ERR_ARG, "null halo buffer");
    return compute_forces_into(ctx, ctx->nHaloSend > 0 ? device_out : nullptr);
}

hidem_status hidem_integrate(hidem_ctx *ctx) {
    NvtxRange nvtx_range("applyForce");
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "no particles set");
    CK(cudaSetDevice(ctx->device));
    if (ctx->mixed)
        launch_integrate<float>(ctx->cf, recp<float>(ctx, ctx->cur), ctx->type[ctx->ord],
                                static_cast<const float *>(ctx->force), (int)ctx->n, ctx->stream);
    else
        launch_integrate<double>(ctx->cd, recp<double>(ctx, ctx->cur), ctx->type[ctx->ord],
                                 static_cast<const double *>(ctx->force), (int)ctx->n, ctx->stream);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return HIDEM_OK;
}

hidem_status hidem_link_update(hidem_ctx *ctx) {
    NvtxRange nvtx_range("linkUpdate");
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles || !ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "particles and links must be set");
    CK(cudaSetDevice(ctx->device));
    TRY(ctx->mixed ? link_update_now<float>(ctx, ctx->step) : link_update_now<double>(ctx, ctx->step));
    CK(cudaGetLastError());
    return HIDEM_OK;
}

hidem_status hidem_finalize_ts(hidem_ctx *ctx) {
    if (!ctx) return HIDEM_ERR_ARG;
    ctx->step += 1;
    return HIDEM_OK;
}

hidem_status hidem_grid_service_local(hidem_ctx *ctx, double diff_max[3], int32_t *needs_reduce) {
    if (!ctx || !diff_max || !needs_reduce) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles || !ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "particles and links must be set");
    CK(cudaSetDevice(ctx->device));
    diff_max[0] = diff_max[1] = diff_max[2] = 0.0;
    *needs_reduce = gs_wants_diff(ctx) ? 1 : 0;
    if (*needs_reduce) {
        TRY(reduce_diff_now(ctx));
        TRY(read_diff_words(ctx, diff_max));
    }
    return HIDEM_OK;
}

hidem_status hidem_grid_service_decide(hidem_ctx *ctx, const double diff_max[3], int32_t *regen) {
    if (!ctx || !diff_max || !regen) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles || !ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "particles and links must be set");
    for (int k = 0; k < 3; ++k)
        if (!(diff_max[k] >= 0.0) || std::isinf(diff_max[k]))
            return fail(ctx, HIDEM_ERR_ARG, "diff_max[%d] = %g is not a finite maximum of max(0, diff)", k, diff_max[k]);
    const double cd = gs_wants_diff(ctx) ? curr_dist_of(ctx, diff_max) : 0.0;
    *regen = gs_decide(ctx, cd) ? 1 : 0;
    return HIDEM_OK;
}

hidem_status hidem_local_bounds(hidem_ctx *ctx, double lower[3], double upper[3]) {
    if (!ctx || !lower || !upper) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "no particles set");
    CK(cudaSetDevice(ctx->device));
    const long long n = ctx->n;
    const int nbB = (int)std::min<long long>(std::max<long long>(1, (n + 255) / 256), 4 * ctx->smCount);
    if (ctx->mixed)
        launch_bounds<float>(recp<float>(ctx, ctx->cur), (int)n, ctx->boundsPartial, nbB, ctx->boundsOut, ctx->stream);
    else
        launch_bounds<double>(recp<double>(ctx, ctx->cur), (int)n, ctx->boundsPartial, nbB, ctx->boundsOut, ctx->stream);
    ctx->launches += 2;
    double b[6];
    CK(cudaMemcpyAsync(b, ctx->boundsOut, sizeof b, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 6; ++k)
        if (!std::isfinite(b[k]))
            return fail(ctx, HIDEM_ERR_DEVICE, "non-finite particle coordinates (NaN or infinite %c)",
                        "xyz"[k % 3]);
    for (int k = 0; k < 3; ++k) {
        lower[k] = b[k];
        upper[k] = b[3 + k];
    }
    return HIDEM_OK;
}

hidem_status hidem_regenerate_frame(hidem_ctx *ctx, const double lower[3], const double upper[3]) {
    if (!ctx || !lower || !upper) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles || !ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "particles and links must be set");
    for (int k = 0; k < 3; ++k)
        if (!(lower[k] <= upper[k]) || std::isinf(lower[k]) || std::isinf(upper[k]))
            return fail(ctx, HIDEM_ERR_ARG, "grid box axis %d is [%g, %g]", k, lower[k], upper[k]);
    CK(cudaSetDevice(ctx->device));
    for (int k = 0; k < 3; ++k) {
        ctx->frame[k] = lower[k];
        ctx->frame[3 + k] = upper[k];
    }
    ctx->accumulatedDist = 0;
    ctx->frameOnce = true;
    const hidem_status st = do_rebuild(ctx);
    ctx->frameOnce = false;
    return st;
}

hidem_status hidem_set_halo_exchange(hidem_ctx *ctx, const int32_t *send_index, int64_t n_send,
                                     const int32_t *recv_index, int64_t n_recv) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "no particles set");
    if (n_send < 0 || n_recv < 0 || (n_send > 0 && !send_index) || (n_recv > 0 && !recv_index))
        return fail(ctx, HIDEM_ERR_ARG, "halo lists need non-negative counts and arrays");
    const int32_t *lists[2] = {send_index, recv_index};
    const int64_t counts[2] = {n_send, n_recv};
    for (int w = 0; w < 2; ++w)
        for (int64_t k = 0; k < counts[w]; ++k)
            if (lists[w][k] < 0 || lists[w][k] >= ctx->n)
                return fail(ctx, HIDEM_ERR_ARG, "%s_index[%lld] = %d is not a particle index (n = %lld)",
                            w ? "recv" : "send", (long long)k, lists[w][k], ctx->n);
    CK(cudaSetDevice(ctx->device));
    ctx->nHaloSend = ctx->nHaloRecv = 0;
    if (n_send > 0) {
        TRY(dalloc(ctx, &ctx->haloSend, n_send));
        CK(cudaMemcpyAsync(ctx->haloSend, send_index, 4 * (size_t)n_send, cudaMemcpyHostToDevice, ctx->stream));
    }
    if (n_recv > 0) {
        TRY(dalloc(ctx, &ctx->haloRecv, n_recv));
        CK(cudaMemcpyAsync(ctx->haloRecv, recv_index, 4 * (size_t)n_recv, cudaMemcpyHostToDevice, ctx->stream));
    }
    if (n_send > 0) {
        TRY(dalloc(ctx, &ctx->haloSendPos, ctx->n));
        launch_send_pos(ctx->slotOf, ctx->haloSend, n_send, (int)ctx->n, ctx->haloSendPos, ctx->stream);
        ctx->launches += 1;
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->nHaloSend = n_send;
    ctx->nHaloRecv = n_recv;
    return HIDEM_OK;
}

hidem_status halo_forces(hidem_ctx *ctx, void *buf, bool pack) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "no particles set");
    const long long m = pack ? ctx->nHaloSend : ctx->nHaloRecv;
    if (m > 0 && !buf) return fail(ctx, HIDEM_ERR_ARG, "null halo buffer");
    CK(cudaSetDevice(ctx->device));
    const int *index = pack ? ctx->haloSend : ctx->haloRecv;
    if (ctx->mixed)
        launch_halo_forces<float>(static_cast<float *>(ctx->force), ctx->slotOf, index, m, (int)ctx->n,
                                  static_cast<float *>(buf), pack, ctx->stream);
    else
        launch_halo_forces<double>(static_cast<double *>(ctx->force), ctx->slotOf, index, m, (int)ctx->n,
                                   static_cast<double *>(buf), pack, ctx->stream);
    if (m > 0) ctx->launches += 1;
    CK(cudaGetLastError());
    return HIDEM_OK;
}

hidem_status hidem_pack_halo_forces(hidem_ctx *ctx, void *device_out) { return halo_forces(ctx, device_out, true); }

hidem_status hidem_unpack_halo_forces(hidem_ctx *ctx, const void *device_in) {
    return halo_forces(ctx, const_cast<void *>(device_in), false);
}

hidem_status hidem_step(hidem_ctx *ctx, int32_t nsteps) {
    NvtxRange nvtx_range("hidem_step");
    if (!ctx) return HIDEM_ERR_ARG;
    if (nsteps < 0) return fail(ctx, HIDEM_ERR_ARG, "negative step count");
    if (!ctx->haveParticles || !ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "particles and links must be set");
    CK(cudaSetDevice(ctx->device));
    return ctx->mixed ? run_steps<float>(ctx, nsteps) : run_steps<double>(ctx, nsteps);
}

hidem_status hidem_synchronize(hidem_ctx *ctx) {
    if (!ctx) return HIDEM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    return check_device_error(ctx);
}

void *hidem_get_stream(hidem_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

hidem_status hidem_profile(hidem_ctx *ctx, int32_t enable) {
    if (!ctx) return HIDEM_ERR_ARG;
    ctx->profile = enable != 0;
    ctx->evUsed = 0;
    return HIDEM_OK;
}

hidem_status hidem_profile_read(hidem_ctx *ctx, double *step_kernel_ms, int64_t *launches) {
    if (!ctx) return HIDEM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    double total = 0;
    for (size_t k = 0; k + 1 < ctx->evUsed; k += 2) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->evPool[k], ctx->evPool[k + 1]));
        total += ms;
    }
    if (step_kernel_ms) *step_kernel_ms = total;
    if (launches) *launches = (int64_t)(ctx->evUsed / 2);
    return HIDEM_OK;
}

hidem_status hidem_get_particles(hidem_ctx *ctx, hidem_particle_soa *out) {
    if (!ctx || !out) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "no particles set");
    CK(cudaSetDevice(ctx->device));
    const long long n = ctx->n;
    cudaStream_t st = ctx->stream;
    // unpack the slot-ordered records into caller order in the idle record buffer
    void *stage = ctx->rec[1 - ctx->cur];
    const size_t lp = ctx->lp;
    if (ctx->mixed) {
        SoaIn<float> s = soa_layout<float>(stage, n);
        launch_unpack_records<float>(recp<float>(ctx, ctx->cur), ctx->orig[ctx->ord], (int)n, s, st);
    } else {
        SoaIn<double> s = soa_layout<double>(stage, n);
        launch_unpack_records<double>(recp<double>(ctx, ctx->cur), ctx->orig[ctx->ord], (int)n, s, st);
    }
    ctx->launches += 1;
    const char *b = static_cast<const char *>(stage);
    double *xyz[3] = {out->xCord, out->yCord, out->zCord};
    for (int k = 0; k < 3; ++k)
        if (xyz[k]) CK(cudaMemcpyAsync(xyz[k], b + 8 * (size_t)n * k, 8 * (size_t)n, cudaMemcpyDefault, st));
    const char *lpb = b + 24 * (size_t)n;
    void *lpf[10] = {out->xDiff, out->yDiff, out->zDiff, out->uDiff, out->vDiff, out->wDiff,
                     out->radius, out->xTheta, out->yTheta, out->zTheta};
    for (int k = 0; k < 10; ++k)
        if (lpf[k]) CK(cudaMemcpyAsync(lpf[k], lpb + lp * (size_t)n * k, lp * (size_t)n, cudaMemcpyDefault, st));
    if (out->type) {
        // the type bytes in caller order, staged in the rebuild's permutation scratch
        uint8_t *tstage = reinterpret_cast<uint8_t *>(ctx->perm);
        launch_scatter_u8(ctx->type[ctx->ord], ctx->orig[ctx->ord], (int)n, tstage, st);
        ctx->launches += 1;
        CK(cudaMemcpyAsync(out->type, tstage, (size_t)n, cudaMemcpyDefault, st));
    }
    // the host-held fields while the copies run
    if (out->owners) CK(to_caller(out->owners, ctx->owners.data(), 4 * (size_t)n));
    if (out->globalKeys) CK(to_caller(out->globalKeys, ctx->keys.data(), 8 * (size_t)n));
    CK(cudaStreamSynchronize(st));
    return HIDEM_OK;
}

hidem_status hidem_get_links(hidem_ctx *ctx, hidem_link_soa *out) {
    if (!ctx || !out) return HIDEM_ERR_ARG;
    if (!ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "no links set");
    CK(cudaSetDevice(ctx->device));
    const long long L = ctx->L;
    if (L == 0) return HIDEM_OK;
    cudaStream_t st = ctx->stream;
    SideSet &s = ctx->side[ctx->curSide];
    const size_t lp = ctx->lp;
    void *stage = nullptr;
    uint8_t *lstate = nullptr;
    TRY(dalloc_bytes(ctx, &stage, lp * (size_t)(2 * L)));
    TRY(dalloc(ctx, &lstate, L));
    const int *slot = ctx->sideSlot[ctx->curSide];
    // side data and link state back in caller order
    for (int k = 0; k < 6; ++k) {
        if (!out->CT[k]) continue;
        if (ctx->mixed)
            launch_gather_sides<float>(slot, L, static_cast<const float *>(s.ct[k]), static_cast<float *>(stage), nullptr, nullptr, st);
        else
            launch_gather_sides<double>(slot, L, static_cast<const double *>(s.ct[k]), static_cast<double *>(stage), nullptr, nullptr, st);
        CK(cudaMemcpyAsync(out->CT[k], stage, lp * (size_t)(2 * L), cudaMemcpyDefault, st));
        ctx->launches += 1;
    }
    if (out->state) {
        if (ctx->mixed)
            launch_gather_sides<float>(slot, L, nullptr, nullptr, s.state, lstate, st);
        else
            launch_gather_sides<double>(slot, L, nullptr, nullptr, s.state, lstate, st);
        CK(cudaMemcpyAsync(out->state, lstate, (size_t)L, cudaMemcpyDefault, st));
        ctx->launches += 1;
    }
    if (out->initialLen) CK(cudaMemcpyAsync(out->initialLen, ctx->L0link, lp * (size_t)L, cudaMemcpyDefault, st));
    if (out->owners) CK(cudaMemcpyAsync(out->owners, ctx->dLinkOwners, 4 * (size_t)L, cudaMemcpyDefault, st));
    if (out->globalKeys) CK(cudaMemcpyAsync(out->globalKeys, ctx->dLinkKeys, 8 * (size_t)L, cudaMemcpyDefault, st));
    if (out->globalKeyEndA) CK(cudaMemcpyAsync(out->globalKeyEndA, ctx->dLinkKeyA, 8 * (size_t)L, cudaMemcpyDefault, st));
    if (out->globalKeyEndB) CK(cudaMemcpyAsync(out->globalKeyEndB, ctx->dLinkKeyB, 8 * (size_t)L, cudaMemcpyDefault, st));
    if (out->particleLinkNum) CK(cudaMemcpyAsync(out->particleLinkNum, ctx->dLinkNum, 4 * (size_t)L, cudaMemcpyDefault, st));
    CK(cudaStreamSynchronize(st));
    dfree(stage);
    dfree(lstate);
    return HIDEM_OK;
}

hidem_status hidem_get_device_view(hidem_ctx *ctx, hidem_device_view *o) {
    if (!ctx || !o) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles || !ctx->haveLinks) return fail(ctx, HIDEM_ERR_STATE, "particles and links must be set");
    CK(cudaSetDevice(ctx->device));
    if (!ctx->built) TRY(do_rebuild(ctx));
    std::memset(o, 0, sizeof *o);
    SideSet &s = ctx->side[ctx->curSide];
    o->precision = ctx->P.precision;
    o->record_bytes = ctx->mixed ? (int32_t)sizeof(PRec<float>) : (int32_t)sizeof(PRec<double>);
    o->n = ctx->n;
    o->L = ctx->L;
    o->step = ctx->step;
    o->records = ctx->rec[ctx->cur];
    o->force = ctx->force;
    o->type = ctx->type[ctx->ord];
    o->input_index = ctx->orig[ctx->ord];
    o->slot_of = ctx->slotOf;
    o->counts = ctx->counts;
    o->contact_offsets = reinterpret_cast<const int64_t *>(ctx->nOff);
    o->contacts = ctx->nbr;
    o->end_offsets = reinterpret_cast<const int64_t *>(ctx->sOff);
    o->end_partner = s.partner;
    for (int k = 0; k < 6; ++k) o->end_ct[k] = s.ct[k];
    o->end_state = s.state;
    o->end_initial_length = s.L0;
    o->end_link = s.link;
    o->link_state = ctx->linkState;
    o->link_slot_a = ctx->linkSlotA;
    o->link_slot_b = ctx->linkSlotB;
    o->link_initial_length = ctx->L0link;
    o->link_end_index = ctx->sideSlot[ctx->curSide];
    o->events = ctx->events;
    o->event_count = ctx->eventCount;
    o->event_capacity = ctx->eventCap;
    o->stream = ctx->stream;
    return HIDEM_OK;
}

hidem_status hidem_get_forces(hidem_ctx *ctx, void *force[6]) {
    if (!ctx || !force) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "no particles set");
    CK(cudaSetDevice(ctx->device));
    const long long n = ctx->n;
    const size_t lp = ctx->lp;
    cudaStream_t st = ctx->stream;
    void *stage = ctx->rec[1 - ctx->cur];
    if (ctx->mixed)
        launch_unpack_force<float>(static_cast<const float *>(ctx->force), ctx->orig[ctx->ord], (int)n, static_cast<float *>(stage), st);
    else
        launch_unpack_force<double>(static_cast<const double *>(ctx->force), ctx->orig[ctx->ord], (int)n, static_cast<double *>(stage), st);
    ctx->launches += 1;
    for (int k = 0; k < 6; ++k)
        if (force[k])
            CK(cudaMemcpyAsync(force[k], static_cast<const char *>(stage) + lp * (size_t)n * k, lp * (size_t)n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return HIDEM_OK;
}

hidem_status hidem_get_cells(hidem_ctx *ctx, int32_t *ix, int32_t *iy, int32_t *iz, int64_t dims[3],
                             double mins[3]) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->built) return fail(ctx, HIDEM_ERR_STATE, "no neighbour structure built yet");
    CK(cudaSetDevice(ctx->device));
    const long long n = ctx->n;
    const GridInfo &g = ctx->grid;
    std::vector<int32_t> cell((size_t)n), orig((size_t)n);
    // cellOf follows the slot order of the current record buffer
    CK(cudaMemcpyAsync(cell.data(), ctx->cellOf[ctx->ord], 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(orig.data(), ctx->orig[ctx->ord], 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (long long s = 0; s < n; ++s) {
        long long c = cell[s], i = orig[s];
        if (ix) ix[i] = (int32_t)(c % g.X);
        if (iy) iy[i] = (int32_t)((c / g.X) % g.Y);
        if (iz) iz[i] = (int32_t)(c / ((long long)g.X * g.Y));
    }
    if (dims) {
        dims[0] = g.X;
        dims[1] = g.Y;
        dims[2] = g.Z;
    }
    if (mins) {
        mins[0] = g.xMin;
        mins[1] = g.yMin;
        mins[2] = g.zMin;
    }
    return HIDEM_OK;
}

hidem_status hidem_get_neighbours(hidem_ctx *ctx, int32_t *counts, int32_t *list, int64_t cap,
                                  int64_t *total) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->built) return fail(ctx, HIDEM_ERR_STATE, "no neighbour structure built yet");
    CK(cudaSetDevice(ctx->device));
    const long long n = ctx->n;
    const long long nb32 = nblocks32(n);
    std::vector<uint32_t> cnt((size_t)n);
    std::vector<int32_t> orig((size_t)n);
    std::vector<long long> off((size_t)nb32);
    CK(cudaMemcpyAsync(cnt.data(), ctx->counts, 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(orig.data(), ctx->orig[ctx->ord], 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(off.data(), ctx->nOff, 8 * (size_t)nb32, cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<int32_t> nbr((size_t)std::max<long long>(ctx->nbrCap, 1));
    CK(cudaMemcpyAsync(nbr.data(), ctx->nbr, 4 * (size_t)ctx->nbrCap, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<int32_t> slotOf((size_t)n);
    for (long long s = 0; s < n; ++s) slotOf[orig[s]] = (int32_t)s;
    long long acc = 0;
    for (long long i = 0; i < n; ++i) {
        const long long s = slotOf[i];
        const int c = (int)(cnt[s] & 0xffffu);
        if (counts) counts[i] = c;
        if (list) {
            for (int k = 0; k < c; ++k) {
                if (acc + k < cap) list[acc + k] = orig[nbr[off[s >> 5] + 32ll * k + (s & 31)]];
            }
        }
        acc += c;
    }
    if (total) *total = acc;
    if (list && acc > cap) return fail(ctx, HIDEM_ERR_CAPACITY, "contact list has %lld entries, cap %lld", acc, (long long)cap);
    return HIDEM_OK;
}

hidem_status hidem_get_break_events(hidem_ctx *ctx, int64_t *link_index, int64_t *step, int64_t cap,
                                    int64_t *count) {
    if (!ctx) return HIDEM_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    unsigned long long total = 0;
    CK(cudaMemcpyAsync(&total, ctx->eventCount, sizeof total, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    long long avail = std::min<long long>((long long)total, ctx->eventCap) - ctx->eventsRead;
    if (avail < 0) avail = 0;
    long long take = std::min<long long>(avail, cap);
    if (take > 0) {
        std::vector<int2> ev((size_t)take);
        CK(cudaMemcpy(ev.data(), ctx->events + ctx->eventsRead, sizeof(int2) * (size_t)take, cudaMemcpyDeviceToHost));
        for (long long k = 0; k < take; ++k) {
            if (link_index) link_index[k] = ev[k].x;
            if (step) step[k] = ev[k].y;
        }
        ctx->eventsRead += take;
    }
    if (count) *count = take;
    return HIDEM_OK;
}

hidem_status hidem_set_checks(hidem_ctx *ctx, int32_t flags) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (flags & ~HIDEM_CHECK_GRID_GROWTH) return fail(ctx, HIDEM_ERR_ARG, "unknown check flags 0x%x", flags);
    ctx->checks = flags;
    return HIDEM_OK;
}

hidem_status hidem_get_stats(hidem_ctx *ctx, hidem_stats *o) {
    if (!ctx || !o) return HIDEM_ERR_ARG;
    std::memset(o, 0, sizeof *o);
    o->step = ctx->step;
    o->num_particles = ctx->n;
    o->num_links = ctx->L;
    o->num_neighbour_pairs = ctx->numPairs;
    o->max_neighbours = ctx->maxNeigh;
    o->max_links_per_particle = ctx->maxLinksPP;
    o->grid_dims[0] = ctx->grid.X;
    o->grid_dims[1] = ctx->grid.Y;
    o->grid_dims[2] = ctx->grid.Z;
    o->grid_min[0] = ctx->grid.xMin;
    o->grid_min[1] = ctx->grid.yMin;
    o->grid_min[2] = ctx->grid.zMin;
    o->regen_count = ctx->regenCount;
    o->last_regen_step = ctx->lastRegen;
    o->accumulated_dist = ctx->accumulatedDist;
    o->search_distance = ctx->searchDistance;
    o->interact_distance = ctx->interactDist;
    o->kernel_launches = ctx->launches;
    o->grid_growth_events = ctx->gridGrowthEvents;
    if (ctx->haveLinks && ctx->L > 0) {
        unsigned long long total = 0;
        CK(cudaMemcpyAsync(&total, ctx->eventCount, sizeof total, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        o->broken_links = (int64_t)total;
    }
    return HIDEM_OK;
}

hidem_status hidem_kinetic_energy(hidem_ctx *ctx, double *translational, double *rotational,
                                  double *max_speed) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "no particles set");
    CK(cudaSetDevice(ctx->device));
    const int nb = (int)std::max<long long>(1, std::min<long long>((ctx->n + 255) / 256, 4LL * ctx->smCount));
    if (ctx->energyBlocks < nb) {
        TRY(dalloc(ctx, &ctx->energyBuf, 6LL * nb + 6));
        ctx->energyBlocks = nb;
    }
    double *out = ctx->energyBuf + 6 * ctx->energyBlocks;
    if (ctx->mixed)
        launch_energy<float>(ctx->cf, recp<float>(ctx, ctx->cur), (int)ctx->n, ctx->energyBuf, nb, out, ctx->stream);
    else
        launch_energy<double>(ctx->cd, recp<double>(ctx, ctx->cur), (int)ctx->n, ctx->energyBuf, nb, out, ctx->stream);
    ctx->launches += 2;
    double h[3];
    CK(cudaMemcpyAsync(h, out, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (translational) *translational = h[0];
    if (rotational) *rotational = h[1];
    if (max_speed) *max_speed = std::sqrt(h[2]);
    return HIDEM_OK;
}

hidem_status hidem_set_functor_params(hidem_ctx *ctx, const hidem_functor_params *f) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!f) return fail(ctx, HIDEM_ERR_ARG, "functor parameters are NULL");
    auto set = [&](auto &c) {
        using LP = std::decay_t<decltype(c.invDt)>;
        c.invDt = (LP)f->neigh_invDt;
        c.attractDistance = (LP)f->neigh_attractDistance;
        c.attractScaleForce = (LP)f->neigh_attractScaleForce;
        c.damping = (LP)f->neigh_damping;
        c.dampingRotation = (LP)f->neigh_dampingRotation;
        c.scaleE = (LP)f->neigh_scaleE;
        c.linkInvDt = (LP)f->link_invDt;
        c.linkDamping = (LP)f->link_damping;
        c.linkDampingRotation = (LP)f->link_dampingRotation;
        c.E = (LP)f->link_E;
        c.W2 = (LP)f->link_W2;
        c.W4 = (LP)f->link_W4;
        c.G = (LP)f->link_G;
        c.bendBreak = (LP)f->break_bendBreak;
        c.maxLoad = (LP)f->break_maxLoad;
    };
    set(ctx->cf);
    set(ctx->cd);
    return HIDEM_OK;
}

hidem_status hidem_get_functor_params(hidem_ctx *ctx, hidem_functor_params *out) {
    if (!ctx || !out) return HIDEM_ERR_ARG;
    auto get = [&](const auto &c) {
        out->neigh_invDt = (double)c.invDt;
        out->neigh_attractDistance = (double)c.attractDistance;
        out->neigh_attractScaleForce = (double)c.attractScaleForce;
        out->neigh_damping = (double)c.damping;
        out->neigh_dampingRotation = (double)c.dampingRotation;
        out->neigh_scaleE = (double)c.scaleE;
        out->link_invDt = (double)c.linkInvDt;
        out->link_damping = (double)c.linkDamping;
        out->link_dampingRotation = (double)c.linkDampingRotation;
        out->link_E = (double)c.E;
        out->link_W2 = (double)c.W2;
        out->link_W4 = (double)c.W4;
        out->link_G = (double)c.G;
        out->break_bendBreak = (double)c.bendBreak;
        out->break_maxLoad = (double)c.maxLoad;
    };
    if (ctx->mixed)
        get(ctx->cf);
    else
        get(ctx->cd);
    return HIDEM_OK;
}

hidem_status hidem_momentum(hidem_ctx *ctx, double linear[3], double angular[3]) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->haveParticles) return fail(ctx, HIDEM_ERR_STATE, "no particles set");
    CK(cudaSetDevice(ctx->device));
    const int nb = (int)std::max<long long>(1, std::min<long long>((ctx->n + 255) / 256, 4LL * ctx->smCount));
    if (ctx->energyBlocks < nb) {
        TRY(dalloc(ctx, &ctx->energyBuf, 6LL * nb + 6));
        ctx->energyBlocks = nb;
    }
    double *out = ctx->energyBuf + 6 * ctx->energyBlocks;
    if (ctx->mixed)
        launch_momentum<float>(ctx->cf, recp<float>(ctx, ctx->cur), (int)ctx->n, ctx->energyBuf, nb, out, ctx->stream);
    else
        launch_momentum<double>(ctx->cd, recp<double>(ctx, ctx->cur), (int)ctx->n, ctx->energyBuf, nb, out,
                                ctx->stream);
    ctx->launches += 2;
    double h[6];
    CK(cudaMemcpyAsync(h, out, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 3; ++k) {
        if (linear) linear[k] = h[k];
        if (angular) angular[k] = h[3 + k];
    }
    return HIDEM_OK;
}

// one map to the device (slot), or the slot cleared (m == NULL)
static hidem_status set_map(hidem_ctx *ctx, int slot, const hidem_map2d *m) {
    if (ctx->mapData[slot]) {
        CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->mapData[slot]);
        ctx->mapData[slot] = nullptr;
    }
    ctx->mapSet[slot] = false;
    ctx->mapView[slot] = Map2dView{};
    if (!m) return HIDEM_OK;
    if (!m->data || m->x_points < 2 || m->y_points < 2 || !(m->x_max > m->x_min) || !(m->y_max > m->y_min))
        return fail(ctx, HIDEM_ERR_ARG, "map %d: needs data, at least 2 x 2 points and max > min", slot);
    const size_t bytes = ctx->lp * (size_t)m->x_points * (size_t)m->y_points;
    CK(cudaMalloc(&ctx->mapData[slot], bytes));
    CK(cudaMemcpyAsync(ctx->mapData[slot], m->data, bytes, cudaMemcpyHostToDevice, ctx->stream));
    Map2dView v{};
    v.data = ctx->mapData[slot];
    v.xPoints = m->x_points;
    v.yPoints = m->y_points;
    v.xMin = m->x_min;
    v.yMin = m->y_min;
    v.xMax = m->x_max;
    v.yMax = m->y_max;
    // grid metrics as the Map2d constructor computes them, in float (Map2d.h:43-58)
    v.xRes = (v.xMax - v.xMin) / (float)(v.xPoints - 1);
    v.yRes = (v.yMax - v.yMin) / (float)(v.yPoints - 1);
    v.invXMaxMin = 1.0f / (v.xMax - v.xMin);
    v.invYMaxMin = 1.0f / (v.yMax - v.yMin);
    ctx->mapView[slot] = v;
    ctx->mapSet[slot] = true;
    return HIDEM_OK;
}

hidem_status hidem_set_bed_maps(hidem_ctx *ctx, const hidem_map2d *bed, const hidem_map2d *friction) {
    if (!ctx) return HIDEM_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    TRY(set_map(ctx, 0, bed));
    TRY(set_map(ctx, 1, friction));
    attach_maps(ctx);
    CK(cudaStreamSynchronize(ctx->stream));
    return HIDEM_OK;
}

hidem_status hidem_set_external_force_maps(hidem_ctx *ctx, const hidem_map2d *maps) {
    if (!ctx) return HIDEM_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    for (int k = 0; k < 6; ++k) TRY(set_map(ctx, 2 + k, maps ? &maps[k] : nullptr));
    attach_maps(ctx);
    CK(cudaStreamSynchronize(ctx->stream));
    return HIDEM_OK;
}

// ------------------------------------------------------------------ collision mesh

}  // extern "C"

namespace {

void free_mesh(hidem_ctx *ctx) {
    for (int k = 0; k < 3; ++k) {
        dfree(ctx->meshVtx[k]);
        dfree(ctx->meshNrm[k]);
        dfree(ctx->meshFace[k]);
        ctx->meshVtx[k] = ctx->meshNrm[k] = ctx->meshFace[k] = nullptr;
    }
    dfree(ctx->meshSizes);
    dfree(ctx->meshStarts);
    dfree(ctx->meshValues);
    dfree(ctx->meshQSizes);
    dfree(ctx->meshQStarts);
    dfree(ctx->meshQValues);
    dfree(ctx->meshKeep);
    ctx->meshSizes = ctx->meshStarts = ctx->meshValues = nullptr;
    ctx->meshQSizes = ctx->meshQStarts = ctx->meshQValues = nullptr;
    ctx->meshKeep = nullptr;
    ctx->meshCells = ctx->meshValueCount = ctx->meshQValueCount = 0;
    ctx->meshTris = 0;
    ctx->meshSet = false;
    ctx->meshF = MeshView<float>{};
    ctx->meshD = MeshView<double>{};
}

// MeshAccel::generateAccel (PLiB/Geometry/MeshAccel.h:57-165): bounding box of the
// vertices in lp (std::max / std::min folds), grown by one cell; counts
// 1 + size / cellSize; the per-cell triangle lists built on the device.
template <class LP>
hidem_status build_mesh(hidem_ctx *ctx, const hidem_mesh *mesh, MeshView<LP> &m) {
    const int T = mesh->triangles;
    const LP *vx = static_cast<const LP *>(mesh->x_vertex);
    const LP *vy = static_cast<const LP *>(mesh->y_vertex);
    const LP *vz = static_cast<const LP *>(mesh->z_vertex);
    const LP lowest = std::numeric_limits<LP>::lowest(), highest = std::numeric_limits<LP>::max();
    LP xU = lowest, yU = lowest, zU = lowest, xL = highest, yL = highest, zL = highest;
    for (long long i = 0; i < 3LL * T; ++i) {
        xU = (vx[i] < xU) ? xU : vx[i];  // std::max(x, xUpper)
        xL = (xL < vx[i]) ? xL : vx[i];  // std::min(x, xLower)
        yU = (vy[i] < yU) ? yU : vy[i];
        yL = (yL < vy[i]) ? yL : vy[i];
        zU = (vz[i] < zU) ? zU : vz[i];
        zL = (zL < vz[i]) ? zL : vz[i];
    }
    const LP cs = (LP)mesh->cell_size;
    xU = xU + cs;
    yU = yU + cs;
    zU = zU + cs;
    xL = xL - cs;
    yL = yL - cs;
    zL = zL - cs;
    const LP xSize = xU - xL, ySize = yU - yL, zSize = zU - zL;
    const double counts[3] = {(double)(LP(1) + xSize / cs), (double)(LP(1) + ySize / cs),
                              (double)(LP(1) + zSize / cs)};
    if (!(counts[0] * counts[1] * counts[2] < 2.0e9))
        return fail(ctx, HIDEM_ERR_CAPACITY, "collision mesh grid of %.0f x %.0f x %.0f cells is too large",
                    counts[0], counts[1], counts[2]);
    m.xLower = xL;
    m.yLower = yL;
    m.zLower = zL;
    m.xUpper = xU;
    m.yUpper = yU;
    m.zUpper = zU;
    m.xInv = 1.f / cs;
    m.yInv = 1.f / cs;
    m.zInv = 1.f / cs;
    m.xCount = (int)(LP(1) + xSize / cs);
    m.yCount = (int)(LP(1) + ySize / cs);
    m.zCount = (int)(LP(1) + zSize / cs);
    m.force = (LP)mesh->mesh_force;
    m.drag = (LP)mesh->mesh_drag;
    const LP maxDist = (cs * cs) + (cs * cs) + (cs * cs) + cs;
    const long long cells = (long long)m.xCount * m.yCount * m.zCount;
    ctx->meshCells = cells;
    ctx->meshCellSize = (double)cs;
    // triangles whose float normal is ill-conditioned (area small against the edges, or
    // not finite): their float distances need not follow the geometry, so the query lists
    // keep them in every cell that lists them
    {
        std::vector<uint8_t> keep((size_t)T);
        for (int t = 0; t < T; ++t) {
            const float ax = (float)vx[3 * t], ay = (float)vy[3 * t], az = (float)vz[3 * t];
            const float bx = (float)vx[3 * t + 1], by = (float)vy[3 * t + 1], bz = (float)vz[3 * t + 1];
            const float cx = (float)vx[3 * t + 2], cy = (float)vy[3 * t + 2], cz = (float)vz[3 * t + 2];
            const float bax = bx - ax, bay = by - ay, baz = bz - az;
            const float acx = ax - cx, acy = ay - cy, acz = az - cz;
            const float cbx = cx - bx, cby = cy - by, cbz = cz - bz;
            const float nx = bay * acz - baz * acy, ny = baz * acx - bax * acz, nz = bax * acy - bay * acx;
            const float n2 = nx * nx + ny * ny + nz * nz;
            const float e = std::max(std::max(bax * bax + bay * bay + baz * baz, acx * acx + acy * acy + acz * acz),
                                     cbx * cbx + cby * cby + cbz * cbz);
            keep[t] = (n2 > 1e-6f * e * e && std::isfinite(n2)) ? 0 : 1;
        }
        CK(cudaMalloc(&ctx->meshKeep, (size_t)T));
        CK(cudaMemcpy(ctx->meshKeep, keep.data(), (size_t)T, cudaMemcpyHostToDevice));
    }
    ctx->meshTris = T;
    const size_t vb = sizeof(LP) * 3 * (size_t)T, nb = sizeof(LP) * (size_t)T;
    const void *vsrc[3] = {mesh->x_vertex, mesh->y_vertex, mesh->z_vertex};
    const void *nsrc[3] = {mesh->x_normal, mesh->y_normal, mesh->z_normal};
    for (int k = 0; k < 3; ++k) {
        CK(cudaMalloc(&ctx->meshVtx[k], vb));
        CK(cudaMalloc(&ctx->meshNrm[k], nb));
        CK(cudaMalloc(&ctx->meshFace[k], nb));
        CK(cudaMemcpyAsync(ctx->meshVtx[k], vsrc[k], vb, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->meshNrm[k], nsrc[k], nb, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemsetAsync(ctx->meshFace[k], 0, nb, ctx->stream));
    }
    m.vx = static_cast<const LP *>(ctx->meshVtx[0]);
    m.vy = static_cast<const LP *>(ctx->meshVtx[1]);
    m.vz = static_cast<const LP *>(ctx->meshVtx[2]);
    m.nx = static_cast<const LP *>(ctx->meshNrm[0]);
    m.ny = static_cast<const LP *>(ctx->meshNrm[1]);
    m.nz = static_cast<const LP *>(ctx->meshNrm[2]);
    m.fx = static_cast<LP *>(ctx->meshFace[0]);
    m.fy = static_cast<LP *>(ctx->meshFace[1]);
    m.fz = static_cast<LP *>(ctx->meshFace[2]);
    // count pass, exclusive scan (the total into the last element of the scratch), fill
    const long long sumsLen = cells / 1024 + 2;
    int *scratch = nullptr;
    CK(cudaMalloc(&ctx->meshSizes, sizeof(int) * cells));
    CK(cudaMalloc(&ctx->meshStarts, sizeof(int) * cells));
    CK(cudaMalloc(&scratch, sizeof(int) * (sumsLen + 1)));
    CK(cudaMemsetAsync(ctx->meshSizes, 0, sizeof(int) * cells, ctx->stream));
    launch_mesh_cells<LP>(m, T, cs, maxDist, ctx->meshSizes, nullptr, nullptr, false, ctx->stream);
    launch_scan<int, int>(ctx->meshSizes, cells, 1, ctx->meshStarts, scratch, scratch + sumsLen, ctx->stream);
    int total = 0;
    cudaError_t e = cudaMemcpyAsync(&total, scratch + sumsLen, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(scratch);
    CK(e);
    ctx->meshValueCount = total;
    CK(cudaMalloc(&ctx->meshValues, sizeof(int) * (size_t)std::max(total, 1)));
    m.starts = ctx->meshStarts;
    m.sizes = ctx->meshSizes;
    m.values = ctx->meshValues;
    launch_mesh_cells<LP>(m, T, cs, maxDist, ctx->meshSizes, ctx->meshStarts, ctx->meshValues, true,
                          ctx->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return HIDEM_OK;
}

// The query lists for the current particles and parameters: the reach of the largest
// interaction distance bedInteract + radius (lp, as the integrate step forms it), with a
// relative and an absolute allowance for the float rounding of the distance tests.
template <class LP>
hidem_status prune_mesh_t(hidem_ctx *ctx, MeshView<LP> &m, const Consts<LP> &c) {
    dfree(ctx->meshQSizes);
    dfree(ctx->meshQStarts);
    dfree(ctx->meshQValues);
    ctx->meshQSizes = ctx->meshQStarts = ctx->meshQValues = nullptr;
    if (ctx->haveParticles && ctx->maxParticleRadius < 0) {
        // the largest radius of the particles last set (their records hold it)
        launch_max_radius<LP>(recp<LP>(ctx, ctx->cur), (int)ctx->n, reinterpret_cast<unsigned long long *>(ctx->offTotal),
                              ctx->stream);
        ctx->launches += 1;
        unsigned long long bits = 0;
        CK(cudaMemcpyAsync(&bits, ctx->offTotal, sizeof bits, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        double r;
        std::memcpy(&r, &bits, sizeof r);
        ctx->maxParticleRadius = r;
    }
    const LP rmax = (LP)std::max(ctx->maxParticleRadius, ctx->P.maxRadius);
    const LP id = c.bedInteract + rmax;
    const double reach = (double)id * (1.0 + 1e-4) + 1e-3;
    const double cs = ctx->meshCellSize;
    const double margin = 1e-4 * cs + 1e-3;
    const long long cells = ctx->meshCells;
    const long long sumsLen = cells / 1024 + 2;
    int *scratch = nullptr;
    CK(cudaMalloc(&ctx->meshQSizes, sizeof(int) * cells));
    CK(cudaMalloc(&ctx->meshQStarts, sizeof(int) * cells));
    CK(cudaMalloc(&scratch, sizeof(int) * (sumsLen + 1)));
    launch_mesh_prune<LP>(m, cs, margin, reach, ctx->meshKeep, ctx->meshQSizes, nullptr, nullptr, false, ctx->stream);
    launch_scan<int, int>(ctx->meshQSizes, cells, 1, ctx->meshQStarts, scratch, scratch + sumsLen, ctx->stream);
    int total = 0;
    cudaError_t e = cudaMemcpyAsync(&total, scratch + sumsLen, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(scratch);
    CK(e);
    ctx->meshQValueCount = total;
    CK(cudaMalloc(&ctx->meshQValues, sizeof(int) * (size_t)std::max(total, 1)));
    launch_mesh_prune<LP>(m, cs, margin, reach, ctx->meshKeep, ctx->meshQSizes, ctx->meshQStarts, ctx->meshQValues,
                          true, ctx->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    m.qStarts = ctx->meshQStarts;
    m.qSizes = ctx->meshQSizes;
    m.qValues = ctx->meshQValues;
    return HIDEM_OK;
}

hidem_status prune_mesh(hidem_ctx *ctx) {
    if (!ctx->meshSet) return HIDEM_OK;
    TRY(ctx->mixed ? prune_mesh_t<float>(ctx, ctx->meshF, ctx->cf) : prune_mesh_t<double>(ctx, ctx->meshD, ctx->cd));
    attach_maps(ctx);
    return HIDEM_OK;
}

}  // namespace

extern "C" {

hidem_status hidem_set_collision_mesh(hidem_ctx *ctx, const hidem_mesh *mesh) {
    if (!ctx) return HIDEM_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    free_mesh(ctx);
    attach_maps(ctx);
    if (!mesh) return HIDEM_OK;
    if (mesh->triangles < 1 || !mesh->x_vertex || !mesh->y_vertex || !mesh->z_vertex || !mesh->x_normal ||
        !mesh->y_normal || !mesh->z_normal)
        return fail(ctx, HIDEM_ERR_ARG, "collision mesh: needs at least one triangle, vertices and normals");
    if (!(mesh->cell_size > 0) || !std::isfinite(mesh->cell_size))
        return fail(ctx, HIDEM_ERR_ARG, "collision mesh: cell_size must be positive");
    hidem_status st = ctx->mixed ? build_mesh<float>(ctx, mesh, ctx->meshF) : build_mesh<double>(ctx, mesh, ctx->meshD);
    if (st != HIDEM_OK) {
        free_mesh(ctx);
        attach_maps(ctx);
        return st;
    }
    ctx->meshSet = true;
    st = prune_mesh(ctx);
    if (st != HIDEM_OK) {
        free_mesh(ctx);
        attach_maps(ctx);
        return st;
    }
    return HIDEM_OK;
}

hidem_status hidem_get_mesh_face_forces(hidem_ctx *ctx, void *x, void *y, void *z) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->meshSet) return fail(ctx, HIDEM_ERR_STATE, "no collision mesh");
    CK(cudaSetDevice(ctx->device));
    void *out[3] = {x, y, z};
    for (int k = 0; k < 3; ++k)
        if (out[k])
            CK(cudaMemcpyAsync(out[k], ctx->meshFace[k], ctx->lp * (size_t)ctx->meshTris, cudaMemcpyDeviceToHost,
                               ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return HIDEM_OK;
}

hidem_status hidem_zero_mesh_face_forces(hidem_ctx *ctx) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->meshSet) return fail(ctx, HIDEM_ERR_STATE, "no collision mesh");
    CK(cudaSetDevice(ctx->device));
    for (int k = 0; k < 3; ++k)
        CK(cudaMemsetAsync(ctx->meshFace[k], 0, ctx->lp * (size_t)ctx->meshTris, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return HIDEM_OK;
}

hidem_status hidem_get_mesh_accel(hidem_ctx *ctx, int32_t counts[3], double lower[3], double upper[3],
                                  int32_t *sizes, int32_t *starts, int32_t *values, int64_t values_cap,
                                  int64_t *values_count) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (!ctx->meshSet) return fail(ctx, HIDEM_ERR_STATE, "no collision mesh");
    CK(cudaSetDevice(ctx->device));
    const int c[3] = {ctx->mixed ? ctx->meshF.xCount : ctx->meshD.xCount,
                      ctx->mixed ? ctx->meshF.yCount : ctx->meshD.yCount,
                      ctx->mixed ? ctx->meshF.zCount : ctx->meshD.zCount};
    const double lo[3] = {ctx->mixed ? (double)ctx->meshF.xLower : ctx->meshD.xLower,
                          ctx->mixed ? (double)ctx->meshF.yLower : ctx->meshD.yLower,
                          ctx->mixed ? (double)ctx->meshF.zLower : ctx->meshD.zLower};
    const double hi[3] = {ctx->mixed ? (double)ctx->meshF.xUpper : ctx->meshD.xUpper,
                          ctx->mixed ? (double)ctx->meshF.yUpper : ctx->meshD.yUpper,
                          ctx->mixed ? (double)ctx->meshF.zUpper : ctx->meshD.zUpper};
    for (int k = 0; k < 3; ++k) {
        if (counts) counts[k] = c[k];
        if (lower) lower[k] = lo[k];
        if (upper) upper[k] = hi[k];
    }
    if (sizes)
        CK(cudaMemcpyAsync(sizes, ctx->meshSizes, sizeof(int) * ctx->meshCells, cudaMemcpyDeviceToHost, ctx->stream));
    if (starts)
        CK(cudaMemcpyAsync(starts, ctx->meshStarts, sizeof(int) * ctx->meshCells, cudaMemcpyDeviceToHost,
                           ctx->stream));
    if (values && values_cap > 0)
        CK(cudaMemcpyAsync(values, ctx->meshValues, sizeof(int) * std::min<long long>(values_cap, ctx->meshValueCount),
                           cudaMemcpyDeviceToHost, ctx->stream));
    if (values_count) *values_count = ctx->meshValueCount;
    CK(cudaStreamSynchronize(ctx->stream));
    return HIDEM_OK;
}

hidem_status hidem_set_step_kernel(hidem_ctx *ctx, int32_t kernel) {
    if (!ctx) return HIDEM_ERR_ARG;
    if (kernel < HIDEM_STEP_KERNEL_AUTO || kernel > HIDEM_STEP_KERNEL_TWO_PASS)
        return fail(ctx, HIDEM_ERR_ARG, "unknown step kernel %d", (int)kernel);
    ctx->stepKernel = kernel;
    return HIDEM_OK;
}

int32_t hidem_get_step_kernel(const hidem_ctx *ctx) {
    if (!ctx) return -1;
    return ctx->stepKernel != HIDEM_STEP_KERNEL_AUTO ? ctx->stepKernel : ctx->tunedKernel;
}

hidem_status hidem_batch_create(hidem_ctx *const *ctxs, int32_t nctx, int32_t flags,
                                hidem_batch **out) {
    g_create_error.clear();
    if (!out) {
        g_create_error = "out is NULL";
        return HIDEM_ERR_ARG;
    }
    *out = nullptr;
    if (!ctxs || nctx <= 0) {
        g_create_error = "no contexts";
        return HIDEM_ERR_ARG;
    }
    if (flags & ~(HIDEM_BATCH_GRAPHS | HIDEM_BATCH_PER_CONTEXT)) {
        g_create_error = "unknown batch flags";
        return HIDEM_ERR_ARG;
    }
    for (int i = 0; i < nctx; ++i) {
        if (!ctxs[i]) {
            g_create_error = "context " + std::to_string(i) + " is NULL";
            return HIDEM_ERR_ARG;
        }
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == ctxs[i]) {
                g_create_error = "context " + std::to_string(i) + " appears twice";
                return HIDEM_ERR_ARG;
            }
        if (ctxs[i]->device != ctxs[0]->device || ctxs[i]->mixed != ctxs[0]->mixed) {
            g_create_error = "contexts of one batch must share the device and the precision";
            return HIDEM_ERR_ARG;
        }
    }
    hidem_batch *b = new hidem_batch();
    b->ctxs.assign(ctxs, ctxs + nctx);
    b->mixed = ctxs[0]->mixed;
    b->device = ctxs[0]->device;
    b->flags = flags;
    const size_t eb = (b->mixed ? sizeof(BatchEntry<float>) : sizeof(BatchEntry<double>)) * (size_t)nctx +
                      sizeof(int) * 4 * (size_t)nctx;
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->entries, eb);
    if (e == cudaSuccess) e = cudaMallocHost(&b->staging, eb);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->diff, 3 * sizeof(unsigned long long) * (size_t)nctx);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&b->diffHost, 3 * sizeof(unsigned long long) * (size_t)nctx);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->uploaded, cudaEventDisableTiming);
    if (e == cudaSuccess) {
        if (b->mixed) prepare_step_batch<float>();
        else prepare_step_batch<double>();
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        g_create_error = std::string("batch setup failed: ") + cudaGetErrorString(e);
        hidem_batch_destroy(b);
        return HIDEM_ERR_CUDA;
    }
    *out = b;
    return HIDEM_OK;
}

void hidem_batch_destroy(hidem_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_clear_graphs(b);
    if (b->uploaded) cudaEventDestroy(b->uploaded);
    if (b->entries) cudaFree(b->entries);
    if (b->tbl) cudaFree(b->tbl);
    if (b->staging) cudaFreeHost(b->staging);
    if (b->diff) cudaFree(b->diff);
    if (b->diffHost) cudaFreeHost(b->diffHost);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char *hidem_batch_last_error(const hidem_batch *b) { return b ? b->err.c_str() : "null batch"; }

void *hidem_batch_get_stream(hidem_batch *b) { return b ? (void *)b->stream : nullptr; }

hidem_status hidem_batch_step(hidem_batch *b, int32_t nsteps) {
    NvtxRange nvtx_range("hidem_batch_step");
    if (!b) return HIDEM_ERR_ARG;
    b->err.clear();
    if (nsteps < 0) return bfail(b, HIDEM_ERR_ARG, "negative step count");
    for (size_t i = 0; i < b->ctxs.size(); ++i)
        if (!b->ctxs[i]->haveParticles || !b->ctxs[i]->haveLinks)
            return bfail(b, HIDEM_ERR_STATE, "context %d: particles and links must be set", (int)i);
    BCK(cudaSetDevice(b->device));
    return b->mixed ? batch_run<float>(b, nsteps) : batch_run<double>(b, nsteps);
}

hidem_status hidem_batch_counts(const hidem_batch *b, int64_t *launches, int64_t *graph_launches,
                                int64_t *uploads) {
    if (!b) return HIDEM_ERR_ARG;
    if (launches) *launches = b->launches;
    if (graph_launches) *graph_launches = b->graphLaunches;
    if (uploads) *uploads = b->uploads;
    return HIDEM_OK;
}

}  // extern "C"
