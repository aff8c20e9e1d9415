/*
 * hidem_b200_iterate.cuh — the reference's templated operator surface over the library's
 * device data, for code that brings its own functors (a sample main's lambdas), compiled
 * by the caller's nvcc for sm_100a:
 *
 *   ExecutionPolicy / SerialExec / ParallelExec / OffloadExec   (Iterators/ExecutionPolicy.h:36-76)
 *   Iterator::iterate / iterateIndirect / iterateBlocked / syncAll (Iterators/Iterator.h:391-616)
 *   ParticleData<LP>: the HiDEMParticleData fields a functor indexes with pInd
 *                     (HiDEMLib/HiDEMParticleData.h:17-66, PLiB/ParticleData.h:22-41)
 *   computePartForce(view, neighF, linkF)  (HiDEMLib.h:316-382, CombinedAccel::iterateCombined,
 *                                           PLiB/Accel/CombinedAccel.h:122-197)
 *   linkUpdate(view, breakF)               (HiDEMLib.h:256-269, CombinedAccel.h:200-235)
 *   applyForce(view, integrateF)           (HiDEMLib.h:303-314)
 *
 * The functors keep the reference's positional signatures (HiDEM/Docs/UsingHiDEMLib.md:326-604):
 *   contact (mask, xDist, yDist, zDist, self xDiff..wDiff radius, other xDiff..wDiff radius,
 *            xForce..wForce&)
 *   link    (mask&, xDist, yDist, zDist, self 7, other 7, CT0..CT5&, xForce..wForce&)
 *   break   (xCord1, yCord1, zCord1, xTheta1, yTheta1, zTheta1, xCord2, ..., zTheta2,
 *            state&, initialLen&)
 *   integrate (pInd, ParticleData<LP>&)
 * called in the reference's order — per particle the contacts in list order, then the link
 * ends in ascending link index, force components accumulated in that order — so functors
 * that restate the default ones give the library's own results bit for bit when compiled,
 * like the library, with -fmad=false -prec-div=true -prec-sqrt=true.
 *
 * The data comes from hidem_get_device_view (hidem_b200.h): particles in storage order,
 * which is the order the reference's pInd follows after its own reorder; take the view
 * again after any call that rebuilds or steps. Device work runs on the view's stream;
 * Iterator::syncAll waits for it. Lambdas passed to the Offload overloads need nvcc's
 * --extended-lambda; functor structs with __device__ call operators need nothing.
 */
#ifndef HIDEM_B200_ITERATE_CUH
#define HIDEM_B200_ITERATE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <type_traits>
#include <utility>

#include "hidem_b200.h"

namespace hidem_iter {

// ---------------------------------------------------------------- execution policies

class ExecutionPolicy {
public:
    enum ExecType { Serial, Parallel, Offload };
    ExecType type = Serial;
    int blockSize = 256;
};

class SerialExec : public ExecutionPolicy {
public:
    SerialExec() { type = Serial; }
};

class ParallelExec : public ExecutionPolicy {
public:
    ParallelExec() { type = Parallel; }
};

// device execution on a stream (the view's stream for the library's data)
class OffloadExec : public ExecutionPolicy {
public:
    cudaStream_t stream = 0;
    OffloadExec() { type = Offload; }
    explicit OffloadExec(cudaStream_t s) : stream(s) { type = Offload; }
    explicit OffloadExec(const hidem_device_view &v) : stream(static_cast<cudaStream_t>(v.stream)) {
        type = Offload;
    }
};

namespace detail {

template <class Tind, class F, class... Args>
__global__ void k_iterate(F fun, Tind max, Args... args) {
    for (Tind i = (Tind)(blockIdx.x * (long long)blockDim.x + threadIdx.x); i < max;
         i += (Tind)(gridDim.x * (long long)blockDim.x))
        fun(i, args...);
}

template <class Tind, class F, class... Args>
__global__ void k_iterate_indirect(F fun, const Tind *indexes, long long count, Args... args) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < count;
         k += gridDim.x * (long long)blockDim.x)
        fun(indexes[k], args...);
}

template <class Tind, class F, class... Args>
__global__ void k_iterate_blocked(F fun, Tind blockSize, Tind max, Args... args) {
    // one CTA per reference block; its threads cover the block's entries
    const Tind b = (Tind)blockIdx.x;
    for (Tind i = (Tind)threadIdx.x; i < blockSize; i += (Tind)blockDim.x)
        if (b * blockSize + i < max) fun(b, i, args...);
}

inline int grid_for(long long n, int threads) {
    long long g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;  // grid-stride beyond 32 CTAs per SM of a B200
    return (int)g;
}

inline cudaError_t check_launch() { return cudaGetLastError(); }

}  // namespace detail

// The reference's Iterator: host policies run the loop on the calling thread (Parallel with
// OpenMP when compiled with it), Offload runs one device thread per index on the stream.
struct Iterator {
    template <class Tind, class F, class... Args>
    static void iterate(SerialExec, F fun, Tind max, Args &...args) {
        for (Tind i = 0; i < max; ++i) fun(i, args...);
    }
    template <class Tind, class F, class... Args>
    static void iterate(ParallelExec, F fun, Tind max, Args &...args) {
#pragma omp parallel for
        for (long long i = 0; i < (long long)max; ++i) fun((Tind)i, args...);
    }
    template <class Tind, class F, class... Args>
    static cudaError_t iterate(OffloadExec pol, F fun, Tind max, Args... args) {
        if (max <= 0) return cudaSuccess;
        detail::k_iterate<Tind, F, Args...>
            <<<detail::grid_for((long long)max, pol.blockSize), pol.blockSize, 0, pol.stream>>>(fun, max, args...);
        return detail::check_launch();
    }

    template <class Tind, class F, class... Args>
    static void iterateIndirect(SerialExec, F fun, const Tind *indexes, size_t count, Args &...args) {
        for (size_t k = 0; k < count; ++k) fun(indexes[k], args...);
    }
    template <class Tind, class F, class... Args>
    static void iterateIndirect(ParallelExec, F fun, const Tind *indexes, size_t count, Args &...args) {
#pragma omp parallel for
        for (long long k = 0; k < (long long)count; ++k) fun(indexes[k], args...);
    }
    // `indexes` in device memory
    template <class Tind, class F, class... Args>
    static cudaError_t iterateIndirect(OffloadExec pol, F fun, const Tind *indexes, size_t count, Args... args) {
        if (count == 0) return cudaSuccess;
        detail::k_iterate_indirect<Tind, F, Args...>
            <<<detail::grid_for((long long)count, pol.blockSize), pol.blockSize, 0, pol.stream>>>(
                fun, indexes, (long long)count, args...);
        return detail::check_launch();
    }

    template <class Tind, class F, class... Args>
    static void iterateBlocked(SerialExec, F fun, Tind blockSize, Tind max, Args &...args) {
        const Tind blocks = (max + blockSize - 1) / blockSize;
        for (Tind b = 0; b < blocks; ++b)
            for (Tind i = 0; i < blockSize; ++i)
                if (b * blockSize + i < max) fun(b, i, args...);
    }
    template <class Tind, class F, class... Args>
    static cudaError_t iterateBlocked(OffloadExec pol, F fun, Tind blockSize, Tind max, Args... args) {
        const Tind blocks = (max + blockSize - 1) / blockSize;
        if (blocks <= 0) return cudaSuccess;
        const int threads = blockSize < 1024 ? (int)blockSize : 1024;
        detail::k_iterate_blocked<Tind, F, Args...><<<(unsigned)blocks, threads, 0, pol.stream>>>(fun, blockSize, max, args...);
        return detail::check_launch();
    }

    static cudaError_t syncAll(OffloadExec pol) { return cudaStreamSynchronize(pol.stream); }
    static cudaError_t syncAll() { return cudaDeviceSynchronize(); }
};

// ---------------------------------------------------------------- particle fields

// One field of the particle records (or of the force arrays), indexed like the reference's
// ManVec arrays: field[pInd].
template <class T>
struct Field {
    char *base = nullptr;
    long long stride = 0;
    __host__ __device__ T &operator[](long long i) const {
        return *reinterpret_cast<T *>(base + i * stride);
    }
};

// The HiDEMParticleData fields of the library's records (HiDEMLib/HiDEMParticleData.h:45-51,
// PLiB/ParticleData.h:22-41) plus the force arrays, for functors written against them.
template <class LP>
struct ParticleData {
    Field<double> xCord, yCord, zCord;
    Field<LP> xDiff, yDiff, zDiff, uDiff, vDiff, wDiff, radius, xTheta, yTheta, zTheta;
    Field<LP> xForce, yForce, zForce, uForce, vForce, wForce;
    Field<uint8_t> type;
    long long numLocal = 0;

    static ParticleData from(const hidem_device_view &v) {
        ParticleData d;
        char *r = static_cast<char *>(v.records);
        const long long s = v.record_bytes;
        const long long l = (long long)sizeof(LP);
        auto rf = [&](long long off) { Field<LP> f; f.base = r + off; f.stride = s; return f; };
        d.xCord.base = r; d.xCord.stride = s;
        d.yCord.base = r + 8; d.yCord.stride = s;
        d.zCord.base = r + 16; d.zCord.stride = s;
        d.xDiff = rf(24); d.yDiff = rf(24 + l); d.zDiff = rf(24 + 2 * l);
        d.uDiff = rf(24 + 3 * l); d.vDiff = rf(24 + 4 * l); d.wDiff = rf(24 + 5 * l);
        d.radius = rf(24 + 6 * l);
        d.xTheta = rf(24 + 7 * l); d.yTheta = rf(24 + 8 * l); d.zTheta = rf(24 + 9 * l);
        char *f = static_cast<char *>(v.force);
        Field<LP> *F[6] = {&d.xForce, &d.yForce, &d.zForce, &d.uForce, &d.vForce, &d.wForce};
        for (int k = 0; k < 6; ++k) {
            F[k]->base = f + (long long)k * v.n * l;
            F[k]->stride = l;
        }
        d.type.base = reinterpret_cast<char *>(v.type);
        d.type.stride = 1;
        d.numLocal = v.n;
        return d;
    }
};

// ---------------------------------------------------------------- the force loop

namespace detail {

template <class LP>
struct Rec {
    double x, y, z;
    LP d[6];
    LP r;
    LP th[3];
};

template <class LP>
__device__ __forceinline__ Rec<LP> rec_at(const char *records, long long recordBytes, long long slot) {
    const char *p = records + slot * recordBytes;
    Rec<LP> q;
    q.x = *reinterpret_cast<const double *>(p);
    q.y = *reinterpret_cast<const double *>(p + 8);
    q.z = *reinterpret_cast<const double *>(p + 16);
    const LP *l = reinterpret_cast<const LP *>(p + 24);
#pragma unroll
    for (int k = 0; k < 6; ++k) q.d[k] = l[k];
    q.r = l[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) q.th[k] = l[7 + k];
    return q;
}

// CombinedAccel::iterateCombined (CombinedAccel.h:122-197) for one particle slot.
template <class LP, class NF, class LF>
__global__ void k_part_force(hidem_device_view v, NF nf, LF lf) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= v.n) return;
    const char *rec = static_cast<const char *>(v.records);
    const long long rb = v.record_bytes;
    const Rec<LP> me = rec_at<LP>(rec, rb, i);
    const uint32_t cnt = v.counts[i];
    const int nn = (int)(cnt & 0xffffu), ns = (int)(cnt >> 16);
    LP F[6] = {LP(0), LP(0), LP(0), LP(0), LP(0), LP(0)};
    const long long nbase = v.contact_offsets[i >> 5] + (i & 31);
    for (int k = 0; k < nn; ++k) {
        const Rec<LP> o = rec_at<LP>(rec, rb, v.contacts[nbase + 32ll * k]);
        LP mask = LP(1);
        const LP xDist = (LP)(me.x - o.x), yDist = (LP)(me.y - o.y), zDist = (LP)(me.z - o.z);
        nf(mask, xDist, yDist, zDist, me.d[0], me.d[1], me.d[2], me.d[3], me.d[4], me.d[5], me.r,
           o.d[0], o.d[1], o.d[2], o.d[3], o.d[4], o.d[5], o.r, F[0], F[1], F[2], F[3], F[4], F[5]);
    }
    const long long sbase = v.end_offsets[i >> 5] + (i & 31);
    LP *ct[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) ct[q] = static_cast<LP *>(v.end_ct[q]);
    for (int k = 0; k < ns; ++k) {
        const long long e = sbase + 32ll * k;
        const Rec<LP> o = rec_at<LP>(rec, rb, (long long)(v.end_partner[e] & 0x7fffffffu));
        LP mask = v.end_state[e] == 0 ? LP(0) : LP(1);
        const LP xDist = (LP)(me.x - o.x), yDist = (LP)(me.y - o.y), zDist = (LP)(me.z - o.z);
        LP CT[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) CT[q] = ct[q][e];
        lf(mask, xDist, yDist, zDist, me.d[0], me.d[1], me.d[2], me.d[3], me.d[4], me.d[5], me.r,
           o.d[0], o.d[1], o.d[2], o.d[3], o.d[4], o.d[5], o.r, CT[0], CT[1], CT[2], CT[3], CT[4],
           CT[5], F[0], F[1], F[2], F[3], F[4], F[5]);
#pragma unroll
        for (int q = 0; q < 6; ++q) ct[q][e] = CT[q];
    }
    LP *force = static_cast<LP *>(v.force);
#pragma unroll
    for (int q = 0; q < 6; ++q) force[(long long)q * v.n + i] = F[q];
}

// CombinedAccel::iterateLinks / LinkData::iterateAllLinks (CombinedAccel.h:200-235,
// PLiB/LinkData.h:55-62): the break functor on every link with end A as particle 1; a
// changed state goes to the link and to both ends' copies, a link that breaks is recorded.
template <class LP, class BF>
__global__ void k_link_update(hidem_device_view v, BF bf, long long tagStep) {
    const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool broke = false;
    if (l < v.L) {
        const char *rec = static_cast<const char *>(v.records);
        const Rec<LP> a = rec_at<LP>(rec, v.record_bytes, v.link_slot_a[l]);
        const Rec<LP> b = rec_at<LP>(rec, v.record_bytes, v.link_slot_b[l]);
        uint8_t st = v.link_state[l];
        LP *L0 = static_cast<LP *>(v.link_initial_length);
        LP len = L0[l];
        const uint8_t st0 = st;
        const LP len0 = len;
        bf(a.x, a.y, a.z, a.th[0], a.th[1], a.th[2], b.x, b.y, b.z, b.th[0], b.th[1], b.th[2], st, len);
        const int ea = v.link_end_index[2 * l], eb = v.link_end_index[2 * l + 1];
        if (st != st0) {
            v.link_state[l] = st;
            v.end_state[ea] = st;
            v.end_state[eb] = st;
            broke = (st == 0);
        }
        if (!(len == len0)) {
            L0[l] = len;
            static_cast<LP *>(v.end_initial_length)[ea] = len;
            static_cast<LP *>(v.end_initial_length)[eb] = len;
        }
    }
    if (broke) {
        const unsigned long long slot = atomicAdd(v.event_count, 1ull);
        if ((long long)slot < v.event_capacity)
            static_cast<int2 *>(v.events)[slot] = make_int2((int)l, (int)tagStep);
    }
}

template <class LP, class IF>
__global__ void k_apply_force(ParticleData<LP> pd, IF fun) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < pd.numLocal) fun(i, pd);
}

template <class LP>
inline bool view_is(const hidem_device_view &v) {
    return (sizeof(LP) == 4) == (v.precision == HIDEM_PREC_MIXED);
}

}  // namespace detail

// HiDEMLib::computePartForce (HiDEMLib.h:316-382) with the caller's contact and link
// functors: the six force arrays of the view are written (read them through
// ParticleData<LP>::xForce.. or let hidem_integrate / applyForce use them) and every link
// end's CT is advanced. LP must be the view's lp type.
template <class LP, class NF, class LF>
cudaError_t computePartForce(const hidem_device_view &v, NF neighF, LF linkF) {
    if (!detail::view_is<LP>(v)) return cudaErrorInvalidValue;
    if (v.n <= 0) return cudaSuccess;
    detail::k_part_force<LP, NF, LF><<<(unsigned)((v.n + 127) / 128), 128, 0, static_cast<cudaStream_t>(v.stream)>>>(
        v, neighF, linkF);
    return cudaGetLastError();
}

// HiDEMLib::linkUpdate (HiDEMLib.h:256-269) with the caller's break functor. Break events
// are tagged with `tagStep` (the timestep being finished; the view's step field).
template <class LP, class BF>
cudaError_t linkUpdate(const hidem_device_view &v, BF breakF, long long tagStep) {
    if (!detail::view_is<LP>(v)) return cudaErrorInvalidValue;
    if (v.L <= 0) return cudaSuccess;
    detail::k_link_update<LP, BF><<<(unsigned)((v.L + 255) / 256), 256, 0, static_cast<cudaStream_t>(v.stream)>>>(
        v, breakF, tagStep);
    return cudaGetLastError();
}
template <class LP, class BF>
cudaError_t linkUpdate(const hidem_device_view &v, BF breakF) {
    return linkUpdate<LP, BF>(v, breakF, (long long)v.step);
}

// HiDEMLib::applyForce (HiDEMLib.h:303-314): fun(pInd, ParticleData<LP>&) for every
// particle, the sample main's integrate lambda.
template <class LP, class IF>
cudaError_t applyForce(const hidem_device_view &v, IF fun) {
    if (!detail::view_is<LP>(v)) return cudaErrorInvalidValue;
    if (v.n <= 0) return cudaSuccess;
    ParticleData<LP> pd = ParticleData<LP>::from(v);
    detail::k_apply_force<LP, IF><<<(unsigned)((v.n + 255) / 256), 256, 0, static_cast<cudaStream_t>(v.stream)>>>(pd, fun);
    return cudaGetLastError();
}

}  // namespace hidem_iter

#endif  // HIDEM_B200_ITERATE_CUH
