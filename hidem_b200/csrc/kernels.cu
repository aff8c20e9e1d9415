// CUDA kernels of the hot path (sm_100a). Built with -fmad=false and IEEE
// division / square root: see physics.cuh.
//
//   binning      k_bounds, k_bounds_final, k_cells, scan_*, k_scatter, k_sort_cells,
//                k_permute                         (NeighbourGrid::generate, NeighbourGrid.cpp:48-184)
//   contacts     k_nbr_count, k_nbr_fill           (NeighAccel::generateNeighbours, NeighAccel.h:25-137)
//   link ends    k_side_count, k_side_fill         (LinkAccelSide::generateLinks/sortSideData,
//                                                   LinkAccelSide.h:92-143,160-417)
//   timestep     k_step<FUSED>                     (CombinedAccel::iterateCombined + applyForce +
//                                                   linkUpdate, CombinedAccel.h:122-235)
//                k_integrate, k_link_break, k_max_diff
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "kernels.h"
#include "physics.cuh"

namespace hidem {

// ------------------------------------------------------------------ helpers

template <class LP>
__device__ __forceinline__ PRec<LP> load_rec(const PRec<LP> *p) {
    PRec<LP> r;
    const int4 *src = reinterpret_cast<const int4 *>(p);
    int4 *dst = reinterpret_cast<int4 *>(&r);
#pragma unroll
    for (int k = 0; k < (int)(sizeof(PRec<LP>) / 16); ++k) dst[k] = __ldg(src + k);
    return r;
}

template <class LP>
__device__ __forceinline__ void store_rec(PRec<LP> *p, const PRec<LP> &r) {
    int4 *dst = reinterpret_cast<int4 *>(p);
    const int4 *src = reinterpret_cast<const int4 *>(&r);
#pragma unroll
    for (int k = 0; k < (int)(sizeof(PRec<LP>) / 16); ++k) dst[k] = src[k];
}

__device__ __forceinline__ unsigned long long max_bits(float v) {
    return (unsigned long long)__float_as_uint(v);
}
__device__ __forceinline__ unsigned long long max_bits(double v) {
    return (unsigned long long)__double_as_longlong(v);
}

__device__ __forceinline__ void set_error(int *flag, int code) {
    if (flag) atomicCAS(flag, 0, code);
}

// ------------------------------------------------------------------ binning

// min / max that keep a NaN: fmin / fmax drop NaN operands, so one particle with a NaN
// coordinate would vanish from the bounds and then be binned from floor(NaN). With these
// a NaN anywhere reaches the result and the host refuses the rebuild. Equal to fmin /
// fmax for numbers.
__device__ __forceinline__ double nan_min(double a, double b) {
    return (a != a) ? a : ((b != b) ? b : fmin(a, b));
}
__device__ __forceinline__ double nan_max(double a, double b) {
    return (a != a) ? a : ((b != b) ? b : fmax(a, b));
}

// Per-block min / max of the three coordinates over all particles
// (ParticleData::getLimits, PLiB/ParticleData.h:47-59).
template <class LP>
__global__ void k_bounds(const PRec<LP> *__restrict__ rec, int n, double *__restrict__ partial) {
    double mn[3] = {INFINITY, INFINITY, INFINITY};
    double mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double *p = reinterpret_cast<const double *>(rec + i);
        double v[3] = {__ldg(p), __ldg(p + 1), __ldg(p + 2)};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = nan_min(mn[k], v[k]);
            mx[k] = nan_max(mx[k], v[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = nan_min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = nan_max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    __shared__ double sm[32][6];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        for (int k = 0; k < 3; ++k) {
            sm[w][k] = mn[k];
            sm[w][3 + k] = mx[k];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int nw = blockDim.x >> 5;
        for (int k = 0; k < 3; ++k) {
            double a = sm[0][k], b = sm[0][3 + k];
            for (int j = 1; j < nw; ++j) {
                a = nan_min(a, sm[j][k]);
                b = nan_max(b, sm[j][3 + k]);
            }
            partial[blockIdx.x * 6 + k] = a;
            partial[blockIdx.x * 6 + 3 + k] = b;
        }
    }
}

// min / max are exact and idempotent, so the block's fold order (each thread starts from
// one partial, repeated ones counting twice) gives the serial fold's result
constexpr int kBoundsFinalThreads = 256;
__global__ void k_bounds_final(const double *__restrict__ partial, int nb, double *__restrict__ out) {
    __shared__ double red[6][kBoundsFinalThreads];
    const int t = threadIdx.x;
    double v[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) v[k] = partial[(t % nb) * 6 + k];
    for (int b = t + kBoundsFinalThreads; b < nb; b += kBoundsFinalThreads)
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const double u = partial[b * 6 + k];
            v[k] = (k < 3) ? nan_min(v[k], u) : nan_max(v[k], u);
        }
#pragma unroll
    for (int k = 0; k < 6; ++k) red[k][t] = v[k];
    __syncthreads();
    for (int w = kBoundsFinalThreads / 2; w > 0; w >>= 1) {
        if (t < w)
#pragma unroll
            for (int k = 0; k < 6; ++k)
                red[k][t] = (k < 3) ? nan_min(red[k][t], red[k][t + w]) : nan_max(red[k][t], red[k][t + w]);
        __syncthreads();
    }
    if (t < 6) out[t] = red[t][0];
}

// Cell colour of every slot and the per-cell counts (NeighbourGrid::getGridId /
// getGridColor / colourParticles, NeighbourGrid.cpp:25-33,116-161).
template <class LP>
__global__ void k_cells(const PRec<LP> *__restrict__ rec, int n, GridInfo g,
                        int *__restrict__ cellOf, int *__restrict__ cellCount, int *errorFlag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const PRec<LP> *p = rec + i;
    int ix = (int)floor((p->x - g.xMin) / g.h);
    int iy = (int)floor((p->y - g.yMin) / g.h);
    int iz = (int)floor((p->z - g.zMin) / g.h);
    long long c = (long long)ix + (long long)iy * g.X + (long long)iz * g.X * g.Y;
    if (c < 0 || c >= g.total) {
        set_error(errorFlag, 1);
        c = 0;
    }
    cellOf[i] = (int)c;
    atomicAdd(cellCount + c, 1);
}

// Exclusive prefix sum in three passes (block sums, scan of block sums, add).
constexpr int kScanBlock = 1024;  // elements per block (256 threads x 4)

template <class TI, class TO>
__global__ void k_scan_blocks(const TI *__restrict__ in, long long n, TO scaleBy,
                              TO *__restrict__ out, TO *__restrict__ blockSums) {
    __shared__ TO sh[kScanBlock];
    long long base = (long long)blockIdx.x * kScanBlock;
    for (int k = threadIdx.x; k < kScanBlock; k += blockDim.x) {
        long long i = base + k;
        sh[k] = (i < n) ? (TO)in[i] * scaleBy : (TO)0;
    }
    __syncthreads();
    // Hillis-Steele would cost log steps x 1024; a simple two-level scan instead:
    // each thread scans 4 consecutive elements, then a warp-level scan of thread totals.
    int t = threadIdx.x;
    TO local[4];
    TO run = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        local[k] = run;
        run += sh[t * 4 + k];
    }
    // inclusive scan of `run` over 256 threads
    TO v = run;
    int lane = t & 31, w = t >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        TO u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    __shared__ TO wsum[8];
    if (lane == 31) wsum[w] = v;
    __syncthreads();
    if (t == 0) {
        TO acc = 0;
        for (int j = 0; j < 8; ++j) {
            TO s = wsum[j];
            wsum[j] = acc;
            acc += s;
        }
    }
    __syncthreads();
    TO excl = v - run + wsum[w];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        long long i = base + t * 4 + k;
        if (i < n) out[i] = excl + local[k];
    }
    if (t == blockDim.x - 1) blockSums[blockIdx.x] = excl + run;
}

template <class TO>
__global__ void k_scan_sums(TO *__restrict__ sums, long long nb, TO *__restrict__ total) {
    // one block: sequential over chunks of 1024 with the same two-level scheme
    __shared__ TO carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < nb; base += blockDim.x) {
        long long i = base + threadIdx.x;
        TO v = (i < nb) ? sums[i] : (TO)0;
        TO orig = v;
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            TO u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        __shared__ TO wsum[32];
        if (lane == 31) wsum[w] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            TO acc = 0;
            int nw = blockDim.x >> 5;
            for (int j = 0; j < nw; ++j) {
                TO s = wsum[j];
                wsum[j] = acc;
                acc += s;
            }
        }
        __syncthreads();
        TO excl = v - orig + wsum[w] + carry;
        if (i < nb) sums[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + orig;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <class TO>
__global__ void k_scan_add(TO *__restrict__ out, long long n, const TO *__restrict__ sums) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / kScanBlock];
}

// Counting-sort placement, unstable inside a cell (fixed by k_sort_cells).
__global__ void k_scatter(const int *__restrict__ cellOf, int n, const int *__restrict__ cellStart,
                          int *__restrict__ cursor, int *__restrict__ perm) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cellOf[i];
    int pos = cellStart[c] + atomicAdd(cursor + c, 1);
    perm[pos] = i;
}

// Orders each cell's members by input index: the (colour, index) order of
// NeighbourGrid::generateIterationList (NeighbourGrid.cpp:163-184). One thread per cell
// sorts a cell of at most kSmallCell members by insertion (a lattice cell holds a few);
// a larger cell goes to a list that k_sort_big_cells sorts with one CTA per cell, so that
// no thread's work grows with the square of a crowded cell's population.
__global__ void k_sort_cells(const int *__restrict__ cellStart, const int *__restrict__ cellCount,
                             long long total, const int *__restrict__ origOld, int *__restrict__ perm,
                             int *__restrict__ bigList, int *__restrict__ bigCount) {
    long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= total) return;
    int cnt = cellCount[c];
    if (cnt < 2) return;
    if (cnt > kSmallCell) {
        bigList[atomicAdd(bigCount, 1)] = (int)c;
        return;
    }
    int s = cellStart[c];
    for (int a = 1; a < cnt; ++a) {
        int v = perm[s + a];
        int key = origOld ? origOld[v] : v;
        int b = a - 1;
        while (b >= 0 && (origOld ? origOld[perm[s + b]] : perm[s + b]) > key) {
            perm[s + b + 1] = perm[s + b];
            --b;
        }
        perm[s + b + 1] = v;
    }
}

// One CTA per listed cell (grid-stride over the list): the (key, member) pairs of the cell
// in shared memory, a bitonic sort over the next power of two, the members written back in
// key order. Keys are input indices (non-negative, distinct), so the order is the one the
// insertion sort gives. A cell of more than kBigCellCap members is left unsorted and sets
// `errorCode` in the error flag: the caller refuses the result.
__global__ void __launch_bounds__(kBigCellThreads)
    k_sort_big_cells(const int *__restrict__ cellStart, const int *__restrict__ cellCount,
                     const int *__restrict__ origOld, int *__restrict__ perm,
                     const int *__restrict__ bigList, const int *__restrict__ bigCount,
                     int *errorFlag, int errorCode) {
    __shared__ unsigned long long sk[kBigCellCap];
    const int nbig = *bigCount;
    for (int b = blockIdx.x; b < nbig; b += gridDim.x) {
        const int c = bigList[b];
        const int cnt = cellCount[c];
        const int s = cellStart[c];
        if (cnt > kBigCellCap) {
            if (threadIdx.x == 0) set_error(errorFlag, errorCode);
            continue;
        }
        int m = kSmallCell;
        while (m < cnt) m <<= 1;
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            if (i < cnt) {
                const int v = perm[s + i];
                const unsigned key = (unsigned)(origOld ? origOld[v] : v);
                sk[i] = ((unsigned long long)key << 32) | (unsigned)v;
            } else {
                sk[i] = ~0ull;
            }
        }
        __syncthreads();
        for (int k = 2; k <= m; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < m; i += blockDim.x) {
                    const int p = i ^ j;
                    if (p > i) {
                        const unsigned long long x = sk[i], y = sk[p];
                        const bool up = (i & k) == 0;
                        if (up ? (x > y) : (x < y)) {
                            sk[i] = y;
                            sk[p] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) perm[s + i] = (int)(unsigned)(sk[i] & 0xffffffffull);
        __syncthreads();
    }
}

template <class LP>
__global__ void k_permute(const int *__restrict__ perm, int n, const PRec<LP> *__restrict__ recOld,
                          PRec<LP> *__restrict__ recNew, const uint8_t *__restrict__ typeOld,
                          uint8_t *__restrict__ typeNew, const int *__restrict__ origOld,
                          int *__restrict__ origNew, const int *__restrict__ cellOld,
                          int *__restrict__ cellNew, int *__restrict__ slotOf) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int o = perm[k];
    store_rec(recNew + k, load_rec(recOld + o));
    typeNew[k] = typeOld[o];
    int g = origOld[o];
    origNew[k] = g;
    cellNew[k] = cellOld[o];
    slotOf[g] = k;
}

// ------------------------------------------------------------------ contacts

// Walk of NeighbourGrid::iteratePossibleNeighbours (PLiB/NeighbourGrid.h:87-105) with
// the filter of NeighAccel::iterateBlocks (PLiB/Accel/NeighAccel.h:98-137). FILL=false
// counts, FILL=true writes the row.
template <class LP, bool FILL>
__device__ __forceinline__ int walk_cells(const PRec<LP> *__restrict__ rec, int i, int colour,
                                          const GridInfo &g, const int *__restrict__ cellStart,
                                          const int *__restrict__ cellCount, double interactDist,
                                          int32_t *__restrict__ row, long long rowBase) {
    const double xc = rec[i].x, yc = rec[i].y, zc = rec[i].z;
    const LP ri = rec[i].r;
    int count = 0;
    for (int k = 0; k < 27; ++k) {
        int target = (int)((long long)colour + g.off[k]);
        if (target < 0 || (long long)target >= g.total) continue;
        int cnt = cellCount[target];
        if (cnt == 0) continue;
        int start = cellStart[target];
        for (int j = start; j < start + cnt; ++j) {
            if (j == i) continue;
            const PRec<LP> *q = rec + j;
            LP xDist = (LP)(xc - q->x);
            LP xDist2 = xDist * xDist;
            LP yDist = (LP)(yc - q->y);
            LP yDist2 = yDist * yDist;
            LP zDist = (LP)(zc - q->z);
            LP zDist2 = zDist * zDist;
            LP particleDistance2 = xDist2 + yDist2 + zDist2;
            LP radSum = ri + q->r;
            // candidates farther than the interaction distance by a relative 1e-5 (far above
            // the rounding of the square root and the subtraction below) fail the test
            // whatever the rounding: skip the IEEE square root for them
            const double reach = interactDist + (double)radSum;
            if ((double)particleDistance2 > reach * reach * (1.0 + 1e-5) && reach > 0.0) continue;
            LP particleDistance = lsqrt(particleDistance2);
            LP dist = particleDistance - radSum;
            if ((double)dist < interactDist) {
                if (FILL) row[rowBase + (long long)count * kWarp] = j;
                ++count;
            }
        }
    }
    return count;
}

template <class LP>
__global__ void k_nbr_count(const PRec<LP> *__restrict__ rec, int n, const int *__restrict__ cellOf,
                            GridInfo g, const int *__restrict__ cellStart,
                            const int *__restrict__ cellCount, double interactDist,
                            uint32_t *__restrict__ counts, int *__restrict__ blockWidth,
                            int *errorFlag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int c = 0;
    // a failed check earlier in the rebuild (a particle outside the grid, a cell too crowded
    // to sort) ends the rebuild at the next host check: skip the walk, whose cost grows with
    // the square of a crowded cell's population
    const bool failed = *reinterpret_cast<volatile int *>(errorFlag) != 0;
    if (i < n) {
        if (!failed)
            c = walk_cells<LP, false>(rec, i, cellOf[i], g, cellStart, cellCount, interactDist, nullptr, 0);
        if (c > 0xffff) {
            set_error(errorFlag, 2);
            c = 0xffff;
        }
        counts[i] = (uint32_t)c;
    }
    int m = c;
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && (i >> 5) * kWarp < n) blockWidth[i >> 5] = m;
}

template <class LP>
__global__ void k_nbr_fill(const PRec<LP> *__restrict__ rec, int n, const int *__restrict__ cellOf,
                           GridInfo g, const int *__restrict__ cellStart,
                           const int *__restrict__ cellCount, double interactDist,
                           const long long *__restrict__ nOff, int32_t *__restrict__ nbr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    walk_cells<LP, true>(rec, i, cellOf[i], g, cellStart, cellCount, interactDist, nbr,
                         nOff[i >> 5] + (i & 31));
}

// Contact-list statistics of a rebuild from the per-slot counts (low 16 bits: contacts,
// high 16 bits: link ends): out[0] total contacts, out[1] the largest contact count,
// out[2] the largest link-end count (integer sums and maxima: order-independent).
__global__ void k_count_stats(const uint32_t *__restrict__ counts, int n, long long *__restrict__ out) {
    long long pairs = 0, mn = 0, ml = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t c = counts[i];
        const long long a = c & 0xffffu, e = c >> 16;
        pairs += a;
        mn = a > mn ? a : mn;
        ml = e > ml ? e : ml;
    }
    for (int o = 16; o > 0; o >>= 1) {
        pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
        const long long a = __shfl_xor_sync(0xffffffffu, mn, o), e = __shfl_xor_sync(0xffffffffu, ml, o);
        mn = a > mn ? a : mn;
        ml = e > ml ? e : ml;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(reinterpret_cast<unsigned long long *>(out), (unsigned long long)pairs);
        atomicMax(out + 1, mn);
        atomicMax(out + 2, ml);
    }
}

// ------------------------------------------------------------------ link ends

__global__ void k_side_count(const int *__restrict__ orig, int n, const int *__restrict__ plStart,
                             uint32_t *__restrict__ counts, int *__restrict__ blockWidth,
                             int *errorFlag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int c = 0;
    if (i < n) {
        int o = orig[i];
        c = plStart[o + 1] - plStart[o];
        if (c > 0xffff) {
            set_error(errorFlag, 3);
            c = 0xffff;
        }
        counts[i] = (counts[i] & 0xffffu) | ((uint32_t)c << 16);
    }
    int m = c;
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && (i >> 5) * kWarp < n) blockWidth[i >> 5] = m;
}

template <class LP>
__global__ void k_side_fill(const int *__restrict__ orig, int n, const int *__restrict__ slotOf,
                            const int *__restrict__ plStart, const int *__restrict__ plLink,
                            const uint8_t *__restrict__ plEnd, const int *__restrict__ linkA,
                            const int *__restrict__ linkB, const LP *__restrict__ L0link,
                            const int *__restrict__ sideSlotOld, SideView<LP> oldS,
                            const long long *__restrict__ sOff, SideView<LP> newS,
                            int *__restrict__ sideSlotNew) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int o = orig[i];
    int ps = plStart[o], pe = plStart[o + 1];
    long long base = sOff[i >> 5] + (i & 31);
    for (int k = 0; k < pe - ps; ++k) {
        int l = plLink[ps + k];
        int e = plEnd[ps + k];
        int other = e ? linkA[l] : linkB[l];
        long long dst = base + (long long)k * kWarp;
        int src = sideSlotOld[2 * l + e];
        newS.partner[dst] = (uint32_t)slotOf[other] | (e ? kSideIsB : 0u);
        newS.state[dst] = oldS.state[src];
#pragma unroll
        for (int c = 0; c < 6; ++c) newS.ct[c][dst] = oldS.ct[c][src];
        newS.L0[dst] = L0link[l];
        newS.link[dst] = l;
        sideSlotNew[2 * l + e] = (int)dst;
    }
}

// ------------------------------------------------------------------ timestep

// The first CHUNKS 16-byte chunks of a record (the fields a functor reads); the rest of
// the returned record is left unset and must not be read.
template <class LP, int CHUNKS>
__device__ __forceinline__ PRec<LP> load_rec_head(const PRec<LP> *p) {
    PRec<LP> r;
    const int4 *src = reinterpret_cast<const int4 *>(p);
    int4 *dst = reinterpret_cast<int4 *>(&r);
#pragma unroll
    for (int k = 0; k < CHUNKS; ++k) dst[k] = __ldg(src + k);
    return r;
}
// Hint the L2 to fetch a line that a later iteration will load (no register, no wait).
__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// chunks holding x, y, z, d[6], r
template <class LP>
constexpr int kContactChunks = (int)((3 * sizeof(double) + 7 * sizeof(LP) + 15) / 16);

// One particle per thread. FUSED: previous step's link update (if pending), contacts,
// link ends, integrate, write the record to the other buffer. Split (FUSED=false):
// contacts and link ends only, forces to a.force (HiDEMLib::computePartForce).
// Both item loops are software-pipelined: while item k is evaluated, the partner record
// (and for link ends the CT state, link state and initial length) of item k + 1 and the
// index of item k + 2 are already in flight, and the first link end's loads go out behind
// the last contact, so each thread keeps its dependent loads outstanding behind its
// arithmetic. The functors still run in the reference's order per particle.
template <class LP, bool FUSED>
__device__ __forceinline__ void step_thread_particle(const Consts<LP> &c, const StepArgs<LP> &a,
                                                     const int i) {
    const bool live = i < a.n;
    LP dmax[3] = {LP(0), LP(0), LP(0)};
    if (live) {
        PRec<LP> me = load_rec(a.in + i);
        const uint32_t cnt = __ldg(a.counts + i);
        const uint8_t ty = FUSED ? __ldg(a.type + i) : uint8_t(0);
        const int nn = (int)(cnt & 0xffffu), ns = (int)(cnt >> 16);
        LP F[6] = {0, 0, 0, 0, 0, 0};
        constexpr int HC = kContactChunks<LP>;

        const int32_t *nb = a.nbr + __ldg(a.nOff + (i >> 5)) + (i & 31);
        const long long sbase = __ldg(a.sOff + (i >> 5)) + (i & 31);
        PRec<LP> o;
        int jn = 0;
        if (nn > 0) o = load_rec_head<LP, HC>(a.in + __ldg(nb));
        if (nn > 1) jn = __ldg(nb + kWarp);
        // first link end's partner word while the contacts run
        uint32_t pwn = (ns > 0) ? __ldg(a.sPartner + sbase) : 0u;
        PRec<LP> o2;
        uint8_t stn = 0;
        LP ctn[6] = {0, 0, 0, 0, 0, 0};
        LP l0n = LP(0);
        uint32_t pwnn = 0;
        const bool brk = FUSED && a.breakPending;
        // the first link end's partner record, state and CT go out behind the last contact
        auto first_side = [&]() {
            if (ns > 0) {
                o2 = load_rec(a.in + (pwn & kSlotMask));
                stn = a.sState[sbase];
#pragma unroll
                for (int q = 0; q < 6; ++q) ctn[q] = a.ct[q][sbase];
                if (brk) l0n = __ldg(a.sL0 + sbase);
                if (ns > 1) pwnn = __ldg(a.sPartner + sbase + kWarp);
            }
        };
        if (nn == 0) first_side();
        for (int k = 0; k < nn; ++k) {
            const PRec<LP> cur = o;
            if (k + 1 < nn) {
                o = load_rec_head<LP, HC>(a.in + jn);
                if (k + 2 < nn) {
                    jn = __ldg(nb + (k + 2) * kWarp);
                    if (k + 3 < nn) prefetch_l2(nb + (k + 3) * kWarp);
                }
            } else {
                first_side();
            }
            contact_pair<LP>(c, LP(1), (LP)(me.x - cur.x), (LP)(me.y - cur.y), (LP)(me.z - cur.z),
                             me.d, me.r, cur.d, cur.r, F);
        }

        for (int k = 0; k < ns; ++k) {
            const long long si = sbase + (long long)k * kWarp;
            const PRec<LP> cur = o2;
            const uint32_t pw = pwn;
            uint8_t st = stn;
            const LP L0 = l0n;
            LP CT[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) CT[q] = ctn[q];
            if (k + 1 < ns) {
                pwn = pwnn;
                o2 = load_rec(a.in + (pwn & kSlotMask));
                stn = a.sState[si + kWarp];
#pragma unroll
                for (int q = 0; q < 6; ++q) ctn[q] = a.ct[q][si + kWarp];
                if (brk) l0n = __ldg(a.sL0 + si + kWarp);
                if (k + 2 < ns) {
                    pwnn = __ldg(a.sPartner + si + 2 * kWarp);
                    // the CT and state lines of item k + 2 start their way to L2
#pragma unroll
                    for (int q = 0; q < 6; ++q) prefetch_l2(a.ct[q] + si + 2 * kWarp);
                    prefetch_l2(a.sState + si + 2 * kWarp);
                }
            }
            if (brk && st != 0) {
                const uint8_t nst =
                    (pw & kSideIsB) ? break_link<LP>(a.bendBreak, a.maxLoad, cur, me, st, L0)
                                    : break_link<LP>(a.bendBreak, a.maxLoad, me, cur, st, L0);
                if (nst != st) {
                    a.sState[si] = nst;
                    a.linkState[__ldg(a.sLink + si)] = nst;  // both sides write the same value
                    if (nst == 0 && !(pw & kSideIsB)) {
                        unsigned long long slot = atomicAdd(a.eventCount, 1ull);
                        if ((long long)slot < a.eventCap)
                            a.events[slot] = make_int2(__ldg(a.sLink + si), (int)a.breakStep);
                    }
                    st = nst;
                }
            }
            const LP mask = (st == 0) ? LP(0) : LP(1);
            beam_side<LP>(c, mask, (LP)(me.x - cur.x), (LP)(me.y - cur.y), (LP)(me.z - cur.z),
                          me.d, cur.d, CT, F);
#pragma unroll
            for (int q = 0; q < 6; ++q) a.ct[q][si] = CT[q];
        }

        if (FUSED) {
            integrate_particle<LP>(c, me, ty, F);
            store_rec(a.out + i, me);
            dmax[0] = me.d[0] > LP(0) ? me.d[0] : LP(0);
            dmax[1] = me.d[1] > LP(0) ? me.d[1] : LP(0);
            dmax[2] = me.d[2] > LP(0) ? me.d[2] : LP(0);
        } else {
#pragma unroll
            for (int q = 0; q < 6; ++q) a.force[(long long)q * a.n + i] = F[q];
            // a particle another rank integrates: its record of the halo send buffer too
            if (a.sendPos) {
                const int sp = __ldg(a.sendPos + i);
                if (sp >= 0) {
#pragma unroll
                    for (int q = 0; q < 6; ++q) a.sendBuf[6ll * sp + q] = F[q];
                }
            }
        }
    }
    if (FUSED && a.reduceDiff) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            LP v = dmax[q];
            for (int o = 16; o > 0; o >>= 1) {
                LP u = __shfl_xor_sync(0xffffffffu, v, o);
                v = (u > v) ? u : v;
            }
            if ((threadIdx.x & 31) == 0 && v > LP(0)) atomicMax(a.diffMax + q, max_bits(v));
        }
    }
}

// CTAs per SM the register-capped variant asks the compiler for: 5 (96 registers) in the
// mixed build, 3 (168 registers) in fp64 — each the tightest cap that spills little.
template <class LP>
constexpr int kCapBlocks = sizeof(LP) == 4 ? 5 : 3;
// and the plain variant: 4 CTAs (128 registers) in the mixed build, no cap in fp64
template <class LP>
constexpr int kThreadBlocks = sizeof(LP) == 4 ? 4 : 1;
// and the asynchronous-copy variant (its partner data lives in shared memory)
template <class LP>
constexpr int kAsyncBlocks = sizeof(LP) == 4 ? 5 : 3;
// the register-capped force pass without the integrate tail (two-pass steps)
template <class LP>
constexpr int kCapBlocksForces = sizeof(LP) == 4 ? 5 : 3;

template <class LP, bool FUSED, int MINB>
__global__ void __launch_bounds__(kStepThreads, MINB)
    k_step(const Consts<LP> c, const StepArgs<LP> a) {
    step_thread_particle<LP, FUSED>(c, a, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---- shared-memory staging with bulk copies (cp.async.bulk + mbarrier) ----

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// ---- one thread per particle, partner data staged by asynchronous copies ----
//
// The same per-particle evaluation as step_thread_particle, but the next items' partner
// records (and, for link ends, CT0..CT5) travel with cp.async into this thread's own
// shared-memory slots instead of registers: two items are in flight behind the one being
// evaluated, and the registers that held the prefetched record are free (more CTAs per
// SM). Slot layout per CTA, chunk-major so that a warp's 16-byte reads are conflict-free:
// rec[slot][chunk][thread] (16 B), ct[slot][q][thread] (lp).
__device__ __forceinline__ void cp_async(void *smem, const void *gmem, int bytes16_4_8) {
    if (bytes16_4_8 == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
    else if (bytes16_4_8 == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most one group of this thread is still in flight
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <class LP>
constexpr int kRecChunks = (int)(sizeof(PRec<LP>) / 16);
template <class LP>
constexpr size_t async_smem_bytes() {
    return (size_t)2 * kStepThreads * (sizeof(PRec<LP>) + 6 * sizeof(LP));
}

template <class LP, bool FUSED>
__device__ __forceinline__ void step_thread_async(const Consts<LP> &c, const StepArgs<LP> &a,
                                                  const int i, unsigned char *smem) {
    constexpr int NC = kRecChunks<LP>;
    constexpr int HC = kContactChunks<LP>;
    const int t = threadIdx.x;
    int4 *srec = reinterpret_cast<int4 *>(smem);                                  // [2][NC][128]
    LP *sct = reinterpret_cast<LP *>(smem + (size_t)2 * NC * kStepThreads * 16);   // [2][6][128]
    auto rec_slot = [&](int s, int ch) { return srec + (s * NC + ch) * kStepThreads + t; };
    auto ct_slot = [&](int s, int q) { return sct + (s * 6 + q) * kStepThreads + t; };
    auto read_rec = [&](int s, int chunks) {
        PRec<LP> r;
        int4 *dst = reinterpret_cast<int4 *>(&r);
#pragma unroll
        for (int ch = 0; ch < NC; ++ch)
            if (ch < chunks) dst[ch] = *rec_slot(s, ch);
        return r;
    };

    const bool live = i < a.n;
    LP dmax[3] = {LP(0), LP(0), LP(0)};
    if (live) {
        PRec<LP> me = load_rec(a.in + i);
        const uint32_t cnt = __ldg(a.counts + i);
        const uint8_t ty = FUSED ? __ldg(a.type + i) : uint8_t(0);
        const int nn = (int)(cnt & 0xffffu), ns = (int)(cnt >> 16);
        LP F[6] = {0, 0, 0, 0, 0, 0};
        const int32_t *nb = a.nbr + __ldg(a.nOff + (i >> 5)) + (i & 31);
        const long long sbase = __ldg(a.sOff + (i >> 5)) + (i & 31);

        // contacts: item k's record in slot k & 1; items k + 1 and k + 2 in flight
        auto issue_contact = [&](int s, int j) {
            const int4 *src = reinterpret_cast<const int4 *>(a.in + j);
#pragma unroll
            for (int ch = 0; ch < HC; ++ch) cp_async(rec_slot(s, ch), src + ch, 16);
        };
        int j2 = 0;
        if (nn > 0) issue_contact(0, __ldg(nb));
        cp_async_commit();
        if (nn > 1) issue_contact(1, __ldg(nb + kWarp));
        cp_async_commit();
        if (nn > 2) j2 = __ldg(nb + 2 * kWarp);
        for (int k = 0; k < nn; ++k) {
            cp_async_wait1();
            const PRec<LP> cur = read_rec(k & 1, HC);
            if (k + 2 < nn) {
                issue_contact(k & 1, j2);
                if (k + 3 < nn) j2 = __ldg(nb + (k + 3) * kWarp);
            }
            cp_async_commit();
            contact_pair<LP>(c, LP(1), (LP)(me.x - cur.x), (LP)(me.y - cur.y), (LP)(me.z - cur.z),
                             me.d, me.r, cur.d, cur.r, F);
        }
        cp_async_wait0();

        // link ends: record and CT of item k in slot k & 1; state and initial length one
        // item ahead in registers
        const bool brk = FUSED && a.breakPending;
        auto issue_side = [&](int s, long long si, uint32_t pw) {
            const int4 *src = reinterpret_cast<const int4 *>(a.in + (pw & kSlotMask));
#pragma unroll
            for (int ch = 0; ch < NC; ++ch) cp_async(rec_slot(s, ch), src + ch, 16);
#pragma unroll
            for (int q = 0; q < 6; ++q) cp_async(ct_slot(s, q), a.ct[q] + si, (int)sizeof(LP));
        };
        uint32_t pw0 = 0, pw1 = 0, pw2 = 0;
        uint8_t stn = 0;
        LP l0n = LP(0);
        if (ns > 0) {
            pw0 = __ldg(a.sPartner + sbase);
            issue_side(0, sbase, pw0);
            stn = a.sState[sbase];
            if (brk) l0n = __ldg(a.sL0 + sbase);
        }
        cp_async_commit();
        if (ns > 1) {
            pw1 = __ldg(a.sPartner + sbase + kWarp);
            issue_side(1, sbase + kWarp, pw1);
        }
        cp_async_commit();
        if (ns > 2) pw2 = __ldg(a.sPartner + sbase + 2 * kWarp);
        for (int k = 0; k < ns; ++k) {
            const long long si = sbase + (long long)k * kWarp;
            const uint32_t pw = pw0;
            uint8_t st = stn;
            const LP L0 = l0n;
            cp_async_wait1();
            const PRec<LP> cur = read_rec(k & 1, NC);
            LP CT[6];
#pragma unroll
            for (int q = 0; q < 6; ++q) CT[q] = *ct_slot(k & 1, q);
            pw0 = pw1;
            pw1 = pw2;
            if (k + 1 < ns) {
                stn = a.sState[si + kWarp];
                if (brk) l0n = __ldg(a.sL0 + si + kWarp);
            }
            if (k + 2 < ns) {
                issue_side(k & 1, si + 2 * kWarp, pw1);
                if (k + 3 < ns) pw2 = __ldg(a.sPartner + si + 3 * kWarp);
            }
            cp_async_commit();
            if (brk && st != 0) {
                const uint8_t nst =
                    (pw & kSideIsB) ? break_link<LP>(a.bendBreak, a.maxLoad, cur, me, st, L0)
                                    : break_link<LP>(a.bendBreak, a.maxLoad, me, cur, st, L0);
                if (nst != st) {
                    a.sState[si] = nst;
                    a.linkState[__ldg(a.sLink + si)] = nst;  // both sides write the same value
                    if (nst == 0 && !(pw & kSideIsB)) {
                        unsigned long long slot = atomicAdd(a.eventCount, 1ull);
                        if ((long long)slot < a.eventCap)
                            a.events[slot] = make_int2(__ldg(a.sLink + si), (int)a.breakStep);
                    }
                    st = nst;
                }
            }
            const LP mask = (st == 0) ? LP(0) : LP(1);
            beam_side<LP>(c, mask, (LP)(me.x - cur.x), (LP)(me.y - cur.y), (LP)(me.z - cur.z),
                          me.d, cur.d, CT, F);
#pragma unroll
            for (int q = 0; q < 6; ++q) a.ct[q][si] = CT[q];
        }
        cp_async_wait0();

        if (FUSED) {
            integrate_particle<LP>(c, me, ty, F);
            store_rec(a.out + i, me);
            dmax[0] = me.d[0] > LP(0) ? me.d[0] : LP(0);
            dmax[1] = me.d[1] > LP(0) ? me.d[1] : LP(0);
            dmax[2] = me.d[2] > LP(0) ? me.d[2] : LP(0);
        } else {
#pragma unroll
            for (int q = 0; q < 6; ++q) a.force[(long long)q * a.n + i] = F[q];
        }
    }
    if (FUSED && a.reduceDiff) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            LP v = dmax[q];
            for (int o = 16; o > 0; o >>= 1) {
                LP u = __shfl_xor_sync(0xffffffffu, v, o);
                v = (u > v) ? u : v;
            }
            if ((threadIdx.x & 31) == 0 && v > LP(0)) atomicMax(a.diffMax + q, max_bits(v));
        }
    }
}

template <class LP, bool FUSED, int MINB>
__global__ void __launch_bounds__(kStepThreads, MINB)
    k_step_async(const Consts<LP> c, const StepArgs<LP> a) {
    extern __shared__ __align__(16) unsigned char smem[];
    step_thread_async<LP, FUSED>(c, a, blockIdx.x * blockDim.x + threadIdx.x, smem);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// 1-D bulk copy global -> shared; both addresses 16-byte aligned, size a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: gives up after kMbarSpins polls (each poll may suspend briefly)
constexpr int kMbarSpins = 1 << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    for (int it = 0; it < kMbarSpins; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Item-parallel step: one CTA per 32-slot ELL block. The CTA first stages, with bulk
// copies (cp.async.bulk + mbarrier), everything of its block that is contiguous in HBM:
// its 32 own records, its contact indices, and its link ends' partner words, CT0..CT5,
// states and initial lengths. Every (particle, contact) and (particle, link end) item is
// then evaluated by its own thread — one dependent global load per item, the partner
// record, served by L1 / L2 — and writes the values its functor adds to the forces into
// shared memory; one warp adds them in the reference's order (contacts in list order, then
// per link end the damping term and the CT term) and integrates, so the result is
// bit-identical to k_step.
template <class LP, bool FUSED>
__device__ __forceinline__ void step_items_block(const Consts<LP> &c, const StepArgs<LP> &a,
                                                 const int w, unsigned char *smem) {
    const StageLayout L = stage_layout(sizeof(PRec<LP>), sizeof(LP), a.maxContacts, a.maxEnds);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    PRec<LP> *own = reinterpret_cast<PRec<LP> *>(smem + L.own);
    double *ox = reinterpret_cast<double *>(smem + L.soa);  // own x, y, z: [3][32]
    LP *od = reinterpret_cast<LP *>(ox + 96);               // own d[6], r, th[3]: [10][32]
    int *cn = reinterpret_cast<int *>(od + 320);
    int *cs = cn + 32;
    const int *nb = reinterpret_cast<const int *>(smem + L.nbr);
    const uint32_t *spw = reinterpret_cast<const uint32_t *>(smem + L.spw);
    LP *sct = reinterpret_cast<LP *>(smem + L.sct);          // [6][maxEnds * 32]
    const uint8_t *sst = smem + L.sst;
    const LP *sl0 = reinterpret_cast<const LP *>(smem + L.sl0);
    LP *terms = reinterpret_cast<LP *>(smem + L.terms);
    const int ctStride = a.maxEnds * 32;

    const int base = w * 32;
    const int t = threadIdx.x;
    const int nown = min(32, a.n - base);
    const long long nOff0 = __ldg(a.nOff + w), sOff0 = __ldg(a.sOff + w);
    const int Wn = (int)((__ldg(a.nOff + w + 1) - nOff0) >> 5);
    const int Ws = (int)((__ldg(a.sOff + w + 1) - sOff0) >> 5);
    const bool wantL0 = FUSED && a.breakPending;
    LP *tc = terms;                  // [Wn][6][32]
    LP *ts = terms + Wn * 6 * 32;    // [Ws][12][32]

    if (t == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (t == 0) {
        const uint32_t ends = (uint32_t)(Ws * 32);
        uint32_t bytes = (uint32_t)(nown * sizeof(PRec<LP>)) + (uint32_t)(Wn * 32 * 4);
        if (ends)
            bytes += ends * (4u + 6u * (uint32_t)sizeof(LP) + 1u) +
                     (wantL0 ? ends * (uint32_t)sizeof(LP) : 0u);
        mbar_expect_tx(bar, bytes);
        bulk_g2s(own, a.in + base, (uint32_t)(nown * sizeof(PRec<LP>)), bar);
        if (Wn) bulk_g2s((void *)nb, a.nbr + nOff0, (uint32_t)(Wn * 32 * 4), bar);
        if (ends) {
            bulk_g2s((void *)spw, a.sPartner + sOff0, ends * 4u, bar);
            for (int u = 0; u < 6; ++u)
                bulk_g2s(sct + u * ctStride, a.ct[u] + sOff0, ends * (uint32_t)sizeof(LP), bar);
            bulk_g2s((void *)sst, a.sState + sOff0, ends, bar);
            if (wantL0) bulk_g2s((void *)sl0, a.sL0 + sOff0, ends * (uint32_t)sizeof(LP), bar);
        }
    }
    if (t < 32) {
        const int i = base + t;
        const uint32_t cnt = (i < a.n) ? __ldg(a.counts + i) : 0u;
        cn[t] = (int)(cnt & 0xffffu);
        cs[t] = (int)(cnt >> 16);
    }
    const bool ok = mbar_wait_bounded(bar, 0);
    if (__syncthreads_or(!ok)) {
        // the copies did not complete in time: flag it, give in-flight copies a bounded
        // chance to land in this CTA's shared memory, and leave without computing
        if (t == 0) set_error(a.errorFlag, 4);
        if (!ok) mbar_wait_bounded(bar, 0);
        __syncthreads();
        return;
    }
    // own records to structure-of-arrays (conflict-free lane-indexed reads below)
    if (t < nown) {
        const PRec<LP> r = own[t];
        ox[t] = r.x;
        ox[32 + t] = r.y;
        ox[64 + t] = r.z;
#pragma unroll
        for (int q = 0; q < 6; ++q) od[q * 32 + t] = r.d[q];
        od[6 * 32 + t] = r.r;
#pragma unroll
        for (int q = 0; q < 3; ++q) od[(7 + q) * 32 + t] = r.th[q];
    }
    __syncthreads();

    for (int q = t; q < Wn * 32; q += blockDim.x) {
        const int k = q >> 5, lane = q & 31;
        if (k < cn[lane]) {
            const PRec<LP> o = load_rec(a.in + nb[q]);
            LP s[6];
#pragma unroll
            for (int u = 0; u < 6; ++u) s[u] = od[u * 32 + lane];
            LP tt[6];
            contact_terms<LP>(c, LP(1), (LP)(ox[lane] - o.x), (LP)(ox[32 + lane] - o.y),
                              (LP)(ox[64 + lane] - o.z), s, od[6 * 32 + lane], o.d, o.r, tt);
#pragma unroll
            for (int u = 0; u < 6; ++u) tc[(k * 6 + u) * 32 + lane] = tt[u];
        }
    }

    for (int q = t; q < Ws * 32; q += blockDim.x) {
        const int k = q >> 5, lane = q & 31;
        if (k < cs[lane]) {
            const long long si = sOff0 + q;
            const uint32_t pw = spw[q];
            const PRec<LP> o = load_rec(a.in + (pw & kSlotMask));
            uint8_t st = sst[q];
            if (FUSED && a.breakPending && st != 0) {
                PRec<LP> me;
                me.x = ox[lane];
                me.y = ox[32 + lane];
                me.z = ox[64 + lane];
#pragma unroll
                for (int u = 0; u < 3; ++u) me.th[u] = od[(7 + u) * 32 + lane];
                const LP L0 = sl0[q];
                const uint8_t nst =
                    (pw & kSideIsB) ? break_link<LP>(a.bendBreak, a.maxLoad, o, me, st, L0)
                                    : break_link<LP>(a.bendBreak, a.maxLoad, me, o, st, L0);
                if (nst != st) {
                    a.sState[si] = nst;
                    a.linkState[__ldg(a.sLink + si)] = nst;  // both sides write the same value
                    if (nst == 0 && !(pw & kSideIsB)) {
                        unsigned long long slot = atomicAdd(a.eventCount, 1ull);
                        if ((long long)slot < a.eventCap)
                            a.events[slot] = make_int2(__ldg(a.sLink + si), (int)a.breakStep);
                    }
                    st = nst;
                }
            }
            const LP mask = (st == 0) ? LP(0) : LP(1);
            LP CT[6];
#pragma unroll
            for (int u = 0; u < 6; ++u) CT[u] = sct[u * ctStride + q];
            LP s[6];
#pragma unroll
            for (int u = 0; u < 6; ++u) s[u] = od[u * 32 + lane];
            LP dp[6], ctt[6];
            beam_terms<LP>(c, mask, (LP)(ox[lane] - o.x), (LP)(ox[32 + lane] - o.y),
                           (LP)(ox[64 + lane] - o.z), s, o.d, CT, dp, ctt);
#pragma unroll
            for (int u = 0; u < 6; ++u) a.ct[u][si] = CT[u];
#pragma unroll
            for (int u = 0; u < 6; ++u) {
                ts[(k * 12 + u) * 32 + lane] = dp[u];
                ts[(k * 12 + 6 + u) * 32 + lane] = ctt[u];
            }
        }
    }
    __syncthreads();

    if (t < 32) {
        const int i = base + t;
        LP dmax[3] = {LP(0), LP(0), LP(0)};
        if (i < a.n) {
            LP F[6] = {0, 0, 0, 0, 0, 0};
            const int nn = cn[t], ns = cs[t];
            for (int k = 0; k < nn; ++k) {
#pragma unroll
                for (int u = 0; u < 6; ++u) F[u] = F[u] + tc[(k * 6 + u) * 32 + t];
            }
            for (int k = 0; k < ns; ++k) {
#pragma unroll
                for (int u = 0; u < 6; ++u) {
                    F[u] = F[u] + ts[(k * 12 + u) * 32 + t];
                    F[u] = F[u] + ts[(k * 12 + 6 + u) * 32 + t];
                }
            }
            if (FUSED) {
                PRec<LP> me = own[t];
                integrate_particle<LP>(c, me, __ldg(a.type + i), F);
                store_rec(a.out + i, me);
                dmax[0] = me.d[0] > LP(0) ? me.d[0] : LP(0);
                dmax[1] = me.d[1] > LP(0) ? me.d[1] : LP(0);
                dmax[2] = me.d[2] > LP(0) ? me.d[2] : LP(0);
            } else {
#pragma unroll
                for (int u = 0; u < 6; ++u) a.force[(long long)u * a.n + i] = F[u];
            }
        }
        if (FUSED && a.reduceDiff) {
#pragma unroll
            for (int u = 0; u < 3; ++u) {
                LP v = dmax[u];
                for (int o = 16; o > 0; o >>= 1) {
                    LP x = __shfl_xor_sync(0xffffffffu, v, o);
                    v = (x > v) ? x : v;
                }
                if (t == 0 && v > LP(0)) atomicMax(a.diffMax + u, max_bits(v));
            }
        }
    }
}

template <class LP, bool FUSED>
__global__ void __launch_bounds__(kItemThreads)
    k_step_items(const Consts<LP> c, const StepArgs<LP> a) {
    extern __shared__ __align__(128) unsigned char smem[];
    step_items_block<LP, FUSED>(c, a, blockIdx.x, smem);
}

// One fused step of many independent contexts in one launch. CTA b belongs to the entry
// blockEntry[b], whose CTA range is [firstBlocks[e], firstBlocks[e + 1]); all entries share the
// launch's constants except the break thresholds (in each entry's arguments), and each
// entry's per-step arguments are derived from the launch's step s within the run (a
// parameter of the launch, fixed in a captured run) the way the single-context
// host loop sets them: records alternate between the two buffers, the link update of the
// previous step is applied first once the break gate t * dt > breakTime was open at that
// step (MainMeshBlock.cpp:312), the diff maxima are folded on steps t with
// (t + 1) % 10 == 0 and cleared on steps with t % 10 == 0 (after the host has read them
// at the start of that step). KIND selects the per-CTA body: the item kernel (32
// particles per CTA, dynamic shared memory for the widest entry) or one thread per
// particle (kStepThreads particles per CTA, registers capped or not).
template <class LP, int KIND>
__global__ void __launch_bounds__(KIND == HIDEM_STEP_KERNEL_ITEMS ? kItemThreads : kStepThreads,
                                  KIND == HIDEM_STEP_KERNEL_THREAD_CAPPED ? kCapBlocks<LP>
                                  : KIND == HIDEM_STEP_KERNEL_THREAD      ? kThreadBlocks<LP>
                                                                          : 1)
    k_step_batch(const Consts<LP> c, const BatchEntry<LP> *__restrict__ entries,
                 const int *__restrict__ firstBlocks, const int *__restrict__ blockEntry, int s) {
    extern __shared__ __align__(128) unsigned char smem[];
    // the context's arguments in shared memory (read as the loops go, not held in registers)
    __shared__ StepArgs<LP> sa;
    const int b = blockIdx.x;
    const int ei = __ldg(blockEntry + b);
    const BatchEntry<LP> &e = entries[ei];
    const int lb = b - __ldg(firstBlocks + ei);
    if (threadIdx.x == 0) {
        StepArgs<LP> a = e.a;
        const int par = (e.cur0 + s) & 1;
        a.in = e.rec[par];
        a.out = e.rec[par ^ 1];
        a.step = e.step0 + s;
        a.breakStep = a.step - 1;
        a.breakPending = (s > 0) ? ((LP)((LP)a.breakStep * c.dt) > c.breakTime ? 1 : 0) : e.pend0;
        a.reduceDiff = (e.reduceEvery10 && (a.step + 1) % 10 == 0) ? 1 : 0;
        sa = a;
    }
    __syncthreads();
    if (e.reduceEvery10 && sa.step % 10 == 0 && lb == 0 && threadIdx.x < 3)
        sa.diffMax[threadIdx.x] = 0ull;
    if (KIND == HIDEM_STEP_KERNEL_ITEMS)
        step_items_block<LP, true>(c, sa, lb, smem);
    else
        step_thread_particle<LP, true>(c, sa, lb * kStepThreads + threadIdx.x);
}

// ---- the two-pass step over a batch (three launches per step and group) ----

// The entry whose CTA range holds this CTA: a table of one entry index per CTA, filled when
// the batch's entries are uploaded (one load, where a search over the offsets took several
// dependent ones at the start of every CTA).
__device__ __forceinline__ int batch_entry(const int *blockEntry) { return __ldg(blockEntry + blockIdx.x); }

// tbl[offs[e] .. offs[e + 1]) = e for each of the `count` entries (one CTA per entry)
__global__ void k_block_table(const int *__restrict__ offs, int *__restrict__ tbl) {
    const int e = blockIdx.x;
    const int a = __ldg(offs + e), b = __ldg(offs + e + 1);
    for (int i = a + threadIdx.x; i < b; i += blockDim.x) tbl[i] = e;
}

template <class LP>
__global__ void __launch_bounds__(kStepThreads, kCapBlocksForces<LP>)
    k_force_batch(const Consts<LP> c, const BatchEntry<LP> *__restrict__ entries,
                  const int *__restrict__ firstBlocks, const int *__restrict__ blockEntry, int s) {
    // the context's arguments in shared memory, where the per-particle loop reads them as
    // it goes (as it reads a single context's from the parameter bank), rather than in
    // registers held across the loop
    __shared__ StepArgs<LP> sa;
    const int ei = batch_entry(blockEntry);
    const BatchEntry<LP> &e = entries[ei];
    if (threadIdx.x == 0) {
        StepArgs<LP> a = e.a;
        a.in = e.rec[e.cur0];
        a.out = e.rec[e.cur0];
        a.step = e.step0 + s;
        a.breakPending = 0;
        a.reduceDiff = 0;
        sa = a;
    }
    __syncthreads();
    const int lb = (int)blockIdx.x - __ldg(firstBlocks + ei);
    step_thread_particle<LP, false>(c, sa, lb * kStepThreads + threadIdx.x);
}

template <class LP>
__global__ void __launch_bounds__(kStepThreads)
    k_integrate_batch(const Consts<LP> c, const BatchEntry<LP> *__restrict__ entries,
                      const int *__restrict__ firstBlocks, const int *__restrict__ blockEntry, int s) {
    const int ei = batch_entry(blockEntry);
    const BatchEntry<LP> &e = entries[ei];
    const long long step = e.step0 + s;
    const int lb = (int)blockIdx.x - __ldg(firstBlocks + ei);
    const int i = lb * kStepThreads + threadIdx.x;
    const int n = e.a.n;
    PRec<LP> *rec = e.rec[e.cur0];
    if (e.reduceEvery10 && step % 10 == 0 && lb == 0 && threadIdx.x < 3) e.a.diffMax[threadIdx.x] = 0ull;
    LP dmax[3] = {LP(0), LP(0), LP(0)};
    if (i < n) {
        PRec<LP> me = load_rec(rec + i);
        LP F[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) F[q] = e.a.force[(long long)q * n + i];
        integrate_particle<LP>(c, me, e.a.type[i], F);
        store_rec(rec + i, me);
#pragma unroll
        for (int q = 0; q < 3; ++q) dmax[q] = me.d[q] > LP(0) ? me.d[q] : LP(0);
    }
    if (e.reduceEvery10 && (step + 1) % 10 == 0) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            LP m = dmax[q];
            for (int o = 16; o > 0; o >>= 1) {
                LP u = __shfl_xor_sync(0xffffffffu, m, o);
                m = (u > m) ? u : m;
            }
            if ((threadIdx.x & 31) == 0 && m > LP(0)) atomicMax(e.a.diffMax + q, max_bits(m));
        }
    }
}

// The break pass of the batch: one thread per link over a grid of its own (the links of
// entry e take CTAs [linkFirst[e], linkFirst[e + 1]), linkEntry maps a CTA to its entry),
// so that each thread's two record gathers are in flight beside every other thread's, as
// in the single-context pass.
template <class LP>
__global__ void __launch_bounds__(kStepThreads)
    k_break_batch(const Consts<LP> c, const BatchEntry<LP> *__restrict__ entries,
                  const int *__restrict__ linkFirst, const int *__restrict__ linkEntry, int s) {
    const int ei = batch_entry(linkEntry);
    const BatchEntry<LP> &e = entries[ei];
    const long long step = e.step0 + s;
    const long long l = (long long)((int)blockIdx.x - __ldg(linkFirst + ei)) * kStepThreads + threadIdx.x;
    // the sample main's gate t dt > breakTime (MainMeshBlock.cpp:312), in lp
    if ((LP)((LP)step * c.dt) > c.breakTime && l < e.L) {
        const uint8_t st = e.a.linkState[l];
        if (st != 0) {
            const PRec<LP> *rec = e.rec[e.cur0];
            const PRec<LP> pa = load_rec(rec + __ldg(e.slotA + l));
            const PRec<LP> pb = load_rec(rec + __ldg(e.slotB + l));
            const uint8_t nst = break_link<LP>(e.a.bendBreak, e.a.maxLoad, pa, pb, st, __ldg(e.L0link + l));
            if (nst != st) {
                e.a.linkState[l] = nst;
                e.a.sState[e.sideSlot[2 * l]] = nst;
                e.a.sState[e.sideSlot[2 * l + 1]] = nst;
                if (nst == 0) {
                    const unsigned long long slot = atomicAdd(e.a.eventCount, 1ull);
                    if ((long long)slot < e.a.eventCap) e.a.events[slot] = make_int2((int)l, (int)step);
                }
            }
        }
    }
}

// HiDEMLib::applyForce with the integrate step, in place (split path).
template <class LP>
__global__ void k_integrate(const Consts<LP> c, PRec<LP> *__restrict__ rec,
                            const uint8_t *__restrict__ type, const LP *__restrict__ force, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    PRec<LP> me = load_rec(rec + i);
    LP F[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) F[q] = force[(long long)q * n + i];
    integrate_particle<LP>(c, me, type[i], F);
    store_rec(rec + i, me);
}

// HiDEMLib::linkUpdate: the break functor over every link
// (CombinedAccel::iterateLinks, CombinedAccel.h:200-235), with a warp-compacted
// flag-and-select append of the links that broke.
template <class LP>
__global__ void k_link_break(const Consts<LP> c, const PRec<LP> *__restrict__ rec,
                             const int *__restrict__ endA, const int *__restrict__ endB,
                             const int *__restrict__ sideSlot,
                             uint8_t *__restrict__ sState, uint8_t *__restrict__ linkState,
                             const LP *__restrict__ L0link, long long L, long long step,
                             int2 *__restrict__ events, unsigned long long *__restrict__ eventCount,
                             long long eventCap) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool broke = false;
    if (l < L) {
        // state and initial length in link order (coalesced); the side copies only on a change
        uint8_t st = linkState[l];
        if (st != 0) {
            const PRec<LP> pa = load_rec(rec + __ldg(endA + l));
            const PRec<LP> pb = load_rec(rec + __ldg(endB + l));
            uint8_t nst = break_link<LP>(c, pa, pb, st, __ldg(L0link + l));
            if (nst != st) {
                linkState[l] = nst;
                sState[sideSlot[2 * l]] = nst;
                sState[sideSlot[2 * l + 1]] = nst;
                broke = (nst == 0);
            }
        }
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, broke);
    if (ballot) {
        const int lane = threadIdx.x & 31;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(eventCount, (unsigned long long)__popc(ballot));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (broke) {
            unsigned long long slot = base + __popc(ballot & ((1u << lane) - 1u));
            if ((long long)slot < eventCap) events[slot] = make_int2((int)l, (int)step);
        }
    }
}

// max(0, xDiff), max(0, yDiff), max(0, zDiff) over all particles
// (HiDEMLib::getMaxDistOwned, HiDEMLib.h:424-461).
template <class LP>
__global__ void k_max_diff(const PRec<LP> *__restrict__ rec, int n,
                           unsigned long long *__restrict__ out) {
    LP v[3] = {LP(0), LP(0), LP(0)};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const PRec<LP> &p = rec[i];
#pragma unroll
        for (int q = 0; q < 3; ++q) v[q] = (p.d[q] > v[q]) ? p.d[q] : v[q];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        LP m = v[q];
        for (int o = 16; o > 0; o >>= 1) {
            LP u = __shfl_xor_sync(0xffffffffu, m, o);
            m = (u > m) ? u : m;
        }
        if ((threadIdx.x & 31) == 0 && m > LP(0)) atomicMax(out + q, max_bits(m));
    }
}

// ------------------------------------------------------------------ launchers

static inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

template <class LP>
void launch_bounds(const PRec<LP> *rec, int n, double *partial, int nb, double *out, cudaStream_t s) {
    k_bounds<LP><<<nb, 256, 0, s>>>(rec, n, partial);
    k_bounds_final<<<1, kBoundsFinalThreads, 0, s>>>(partial, nb, out);
}

template <class LP>
void launch_cells(const PRec<LP> *rec, int n, const GridInfo &g, int *cellOf, int *cellCount,
                  int *errorFlag, cudaStream_t s) {
    k_cells<LP><<<nblk(n, 256), 256, 0, s>>>(rec, n, g, cellOf, cellCount, errorFlag);
}

template <class TI, class TO>
int launch_scan(const TI *in, long long n, TO scaleBy, TO *out, TO *sums, TO *total, cudaStream_t s) {
    long long nb = (n + kScanBlock - 1) / kScanBlock;
    if (nb == 0) nb = 1;
    k_scan_blocks<TI, TO><<<(unsigned)nb, 256, 0, s>>>(in, n, scaleBy, out, sums);
    k_scan_sums<TO><<<1, 1024, 0, s>>>(sums, nb, total);
    k_scan_add<TO><<<nblk(n > 0 ? n : 1, 256), 256, 0, s>>>(out, n, sums);
    return 3;
}
template int launch_scan<int, int>(const int *, long long, int, int *, int *, int *, cudaStream_t);
template int launch_scan<int, long long>(const int *, long long, long long, long long *, long long *,
                                         long long *, cudaStream_t);

// position of each slot in the halo send list (-1: not sent): pos[slotOf[index[k]]] = k
__global__ void k_send_pos(const int *__restrict__ slotOf, const int *__restrict__ index, long long m,
                           int *__restrict__ pos) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) pos[slotOf[index[k]]] = (int)k;
}

void launch_send_pos(const int *slotOf, const int *index, long long m, int n, int *pos, cudaStream_t s) {
    cudaMemsetAsync(pos, 0xff, sizeof(int) * (size_t)n, s);
    if (m > 0) k_send_pos<<<nblk(m, 256), 256, 0, s>>>(slotOf, index, m, pos);
}

__global__ void k_scatter_u8(const uint8_t *__restrict__ in, const int *__restrict__ to, int n,
                             uint8_t *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[to[i]] = in[i];
}

void launch_scatter_u8(const uint8_t *in, const int *to, int n, uint8_t *out, cudaStream_t s) {
    if (n > 0) k_scatter_u8<<<nblk(n, 256), 256, 0, s>>>(in, to, n, out);
}

void launch_scatter(const int *cellOf, int n, const int *cellStart, int *cursor, int *perm,
                    cudaStream_t s) {
    k_scatter<<<nblk(n, 256), 256, 0, s>>>(cellOf, n, cellStart, cursor, perm);
}

int launch_sort_cells(const int *cellStart, const int *cellCount, long long total,
                      const int *origOld, int *perm, int *bigList, int *bigCount, int *errorFlag,
                      int errorCode, int smCount, cudaStream_t s) {
    cudaMemsetAsync(bigCount, 0, sizeof(int), s);
    k_sort_cells<<<nblk(total, 256), 256, 0, s>>>(cellStart, cellCount, total, origOld, perm,
                                                  bigList, bigCount);
    k_sort_big_cells<<<2 * smCount, kBigCellThreads, 0, s>>>(cellStart, cellCount, origOld, perm,
                                                             bigList, bigCount, errorFlag, errorCode);
    return 2;
}

template <class LP>
void launch_permute(const int *perm, int n, const PRec<LP> *recOld, PRec<LP> *recNew,
                    const uint8_t *typeOld, uint8_t *typeNew, const int *origOld, int *origNew,
                    const int *cellOld, int *cellNew, int *slotOf, cudaStream_t s) {
    k_permute<LP><<<nblk(n, 256), 256, 0, s>>>(perm, n, recOld, recNew, typeOld, typeNew, origOld,
                                               origNew, cellOld, cellNew, slotOf);
}

template <class LP>
void launch_nbr_count(const PRec<LP> *rec, int n, const int *cellOf, const GridInfo &g,
                      const int *cellStart, const int *cellCount, double interactDist,
                      uint32_t *counts, int *blockWidth, int *errorFlag, cudaStream_t s) {
    k_nbr_count<LP><<<nblk(n, 128), 128, 0, s>>>(rec, n, cellOf, g, cellStart, cellCount,
                                                 interactDist, counts, blockWidth, errorFlag);
}

template <class LP>
void launch_nbr_fill(const PRec<LP> *rec, int n, const int *cellOf, const GridInfo &g,
                     const int *cellStart, const int *cellCount, double interactDist,
                     const long long *nOff, int32_t *nbr, cudaStream_t s) {
    k_nbr_fill<LP><<<nblk(n, 128), 128, 0, s>>>(rec, n, cellOf, g, cellStart, cellCount,
                                                interactDist, nOff, nbr);
}

void launch_count_stats(const uint32_t *counts, int n, long long *out, int smCount, cudaStream_t s) {
    cudaMemsetAsync(out, 0, 3 * sizeof(long long), s);
    const int blocks = std::max(1, std::min(nblk(n, 256), 4 * smCount));
    k_count_stats<<<blocks, 256, 0, s>>>(counts, n, out);
}

void launch_side_count(const int *orig, int n, const int *plStart, uint32_t *counts,
                       int *blockWidth, int *errorFlag, cudaStream_t s) {
    k_side_count<<<nblk(n, 256), 256, 0, s>>>(orig, n, plStart, counts, blockWidth, errorFlag);
}

template <class LP>
void launch_side_fill(const int *orig, int n, const int *slotOf, const int *plStart,
                      const int *plLink, const uint8_t *plEnd, const int *linkA, const int *linkB,
                      const LP *L0link, const int *sideSlotOld, const SideView<LP> &oldS,
                      const long long *sOff, const SideView<LP> &newS, int *sideSlotNew,
                      cudaStream_t s) {
    k_side_fill<LP><<<nblk(n, 256), 256, 0, s>>>(orig, n, slotOf, plStart, plLink, plEnd, linkA,
                                                 linkB, L0link, sideSlotOld, oldS, sOff, newS,
                                                 sideSlotNew);
}

template <class LP>
void launch_step(const Consts<LP> &c, const StepArgs<LP> &a0, bool fused, int maxContacts,
                 int maxEnds, int kernel, cudaStream_t s) {
    StepArgs<LP> a = a0;
    a.maxContacts = maxContacts;
    a.maxEnds = maxEnds;
    const StageLayout L = stage_layout(sizeof(PRec<LP>), sizeof(LP), maxContacts, maxEnds);
    if (kernel == HIDEM_STEP_KERNEL_ITEMS && L.total <= kItemSmemLimit) {
        // the shared-memory limit is a per-device attribute: set it once on each device
        // (setting it twice, as racing threads may, is harmless)
        static std::atomic<unsigned long long> configured[2];
        int dev = 0;
        cudaGetDevice(&dev);
        const unsigned long long bit = 1ull << (dev & 63);
        if (!(configured[fused ? 1 : 0].load() & bit)) {
            if (fused)
                cudaFuncSetAttribute(k_step_items<LP, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kItemSmemLimit);
            else
                cudaFuncSetAttribute(k_step_items<LP, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kItemSmemLimit);
            configured[fused ? 1 : 0].fetch_or(bit);
        }
        const int nb = nblk(a.n, 32);
        if (fused)
            k_step_items<LP, true><<<nb, kItemThreads, L.total, s>>>(c, a);
        else
            k_step_items<LP, false><<<nb, kItemThreads, L.total, s>>>(c, a);
        return;
    }
    // one thread per particle (also for rows too wide for the item kernel's buffers)
    const int nb = nblk(a.n, kStepThreads);
    if (kernel == HIDEM_STEP_KERNEL_THREAD_ASYNC) {
        const size_t sm = async_smem_bytes<LP>();
        if (fused)
            k_step_async<LP, true, kAsyncBlocks<LP>><<<nb, kStepThreads, sm, s>>>(c, a);
        else
            k_step_async<LP, false, kAsyncBlocks<LP>><<<nb, kStepThreads, sm, s>>>(c, a);
    } else if (kernel == HIDEM_STEP_KERNEL_THREAD_CAPPED) {
        if (fused)
            k_step<LP, true, kCapBlocks<LP>><<<nb, kStepThreads, 0, s>>>(c, a);
        else
            k_step<LP, false, kCapBlocksForces<LP>><<<nb, kStepThreads, 0, s>>>(c, a);
    } else {
        if (fused)
            k_step<LP, true, kThreadBlocks<LP>><<<nb, kStepThreads, 0, s>>>(c, a);
        else
            k_step<LP, false, kThreadBlocks<LP>><<<nb, kStepThreads, 0, s>>>(c, a);
    }
}

template <class LP>
bool batch_fits(int maxContacts, int maxEnds) {
    return stage_layout(sizeof(PRec<LP>), sizeof(LP), maxContacts, maxEnds).total <= kItemSmemLimit;
}

template <class LP>
void prepare_step_batch() {
    cudaFuncSetAttribute(k_step_batch<LP, HIDEM_STEP_KERNEL_ITEMS>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kItemSmemLimit);
}

int batch_particles_per_cta(int kernel) {
    return kernel == HIDEM_STEP_KERNEL_ITEMS ? 32 : kStepThreads;
}

void launch_block_table(const int *offs, int count, int *tbl, cudaStream_t s) {
    if (count > 0) k_block_table<<<count, 256, 0, s>>>(offs, tbl);
}

template <class LP>
void launch_step_batch(const Consts<LP> &c, const BatchEntry<LP> *entries, const int *firstBlocks,
                       const int *blockEntry, int run, int totalBlocks, int maxContacts, int maxEnds,
                       int kernel, cudaStream_t s) {
    if (kernel == HIDEM_STEP_KERNEL_ITEMS) {
        const StageLayout L = stage_layout(sizeof(PRec<LP>), sizeof(LP), maxContacts, maxEnds);
        k_step_batch<LP, HIDEM_STEP_KERNEL_ITEMS><<<totalBlocks, kItemThreads, L.total, s>>>(
            c, entries, firstBlocks, blockEntry, run);
    } else if (kernel == HIDEM_STEP_KERNEL_THREAD_CAPPED) {
        k_step_batch<LP, HIDEM_STEP_KERNEL_THREAD_CAPPED><<<totalBlocks, kStepThreads, 0, s>>>(
            c, entries, firstBlocks, blockEntry, run);
    } else {
        k_step_batch<LP, HIDEM_STEP_KERNEL_THREAD><<<totalBlocks, kStepThreads, 0, s>>>(
            c, entries, firstBlocks, blockEntry, run);
    }
}

template <class LP>
void launch_two_pass_batch(const Consts<LP> &c, const BatchEntry<LP> *entries, const int *firstBlocks,
                           const int *blockEntry, const int *linkFirst, const int *linkEntry, int run,
                           int totalBlocks, int totalLinkBlocks, cudaStream_t s) {
    k_force_batch<LP><<<totalBlocks, kStepThreads, 0, s>>>(c, entries, firstBlocks, blockEntry, run);
    k_integrate_batch<LP><<<totalBlocks, kStepThreads, 0, s>>>(c, entries, firstBlocks, blockEntry, run);
    k_break_batch<LP><<<totalLinkBlocks, kStepThreads, 0, s>>>(c, entries, linkFirst, linkEntry, run);
}

template <class LP>
void launch_integrate(const Consts<LP> &c, PRec<LP> *rec, const uint8_t *type, const LP *force,
                      int n, cudaStream_t s) {
    k_integrate<LP><<<nblk(n, 256), 256, 0, s>>>(c, rec, type, force, n);
}

template <class LP>
void launch_link_break(const Consts<LP> &c, const PRec<LP> *rec, const int *endA, const int *endB,
                       const int *sideSlot, uint8_t *sState, uint8_t *linkState, const LP *L0link,
                       long long L, long long step, int2 *events, unsigned long long *eventCount,
                       long long eventCap, cudaStream_t s) {
    if (L <= 0) return;
    k_link_break<LP><<<nblk(L, 256), 256, 0, s>>>(c, rec, endA, endB, sideSlot, sState,
                                                  linkState, L0link, L, step, events, eventCount,
                                                  eventCap);
}

// Kinetic energy with the integrate step's mass and moment of inertia (m = rho d^3,
// I = m d^2 / 6, MainMeshBlock.cpp:228-229) and velocities diff / dt; per-block sums in
// a fixed tree order, then one block over the partials, so the result is deterministic.
template <class LP>
__global__ void k_energy(const Consts<LP> c, const PRec<LP> *__restrict__ rec, int n,
                         double *__restrict__ partial) {
    __shared__ double red[3][256];
    double kt = 0, kr = 0, vmax = 0;
    const double dt = (double)c.dt, rho = (double)c.rhoIce;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const PRec<LP> p = load_rec(rec + i);
        const double d = 2.0 * (double)p.r;
        const double m = rho * d * d * d, I = m * d * d / 6.0;
        const double vx = p.d[0] / dt, vy = p.d[1] / dt, vz = p.d[2] / dt;
        const double wx = p.d[3] / dt, wy = p.d[4] / dt, wz = p.d[5] / dt;
        const double v2 = vx * vx + vy * vy + vz * vz;
        kt += 0.5 * m * v2;
        kr += 0.5 * I * (wx * wx + wy * wy + wz * wz);
        vmax = v2 > vmax ? v2 : vmax;
    }
    red[0][threadIdx.x] = kt;
    red[1][threadIdx.x] = kr;
    red[2][threadIdx.x] = vmax;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] = fmax(red[2][threadIdx.x], red[2][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; ++q) partial[q * gridDim.x + blockIdx.x] = red[q][0];
}

__global__ void k_energy_final(const double *__restrict__ partial, int nb, double *__restrict__ out) {
    __shared__ double red[3][256];
    double a = 0, b = 0, m = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        a += partial[i];
        b += partial[nb + i];
        m = fmax(m, partial[2 * nb + i]);
    }
    red[0][threadIdx.x] = a;
    red[1][threadIdx.x] = b;
    red[2][threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] = fmax(red[2][threadIdx.x], red[2][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; ++q) out[q] = red[q][0];
}

template <class LP>
void launch_energy(const Consts<LP> &c, const PRec<LP> *rec, int n, double *partial, int nb,
                   double *out, cudaStream_t s) {
    k_energy<LP><<<nb, 256, 0, s>>>(c, rec, n, partial);
    k_energy_final<<<1, 256, 0, s>>>(partial, nb, out);
}

// Linear momentum sum m v and angular momentum about the origin sum x (x) m v + I w, in
// double precision: per-block partials [6][gridDim.x] (tree sums in a fixed order), then
// one block folding them, so the result does not depend on scheduling.
template <class LP>
__global__ void k_momentum(const Consts<LP> c, const PRec<LP> *__restrict__ rec, int n,
                           double *__restrict__ partial) {
    __shared__ double red[6][256];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const double dt = (double)c.dt, rho = (double)c.rhoIce;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const PRec<LP> p = load_rec(rec + i);
        const double d = 2.0 * (double)p.r;
        const double m = rho * d * d * d, I = m * d * d / 6.0;
        const double px = m * (p.d[0] / dt), py = m * (p.d[1] / dt), pz = m * (p.d[2] / dt);
        acc[0] += px;
        acc[1] += py;
        acc[2] += pz;
        acc[3] += (p.y * pz - p.z * py) + I * (p.d[3] / dt);
        acc[4] += (p.z * px - p.x * pz) + I * (p.d[4] / dt);
        acc[5] += (p.x * py - p.y * px) + I * (p.d[5] / dt);
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) red[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
#pragma unroll
            for (int q = 0; q < 6; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) partial[q * gridDim.x + blockIdx.x] = red[q][0];
}

__global__ void k_momentum_final(const double *__restrict__ partial, int nb, double *__restrict__ out) {
    __shared__ double red[6][256];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
#pragma unroll
        for (int q = 0; q < 6; ++q) acc[q] += partial[q * nb + i];
#pragma unroll
    for (int q = 0; q < 6; ++q) red[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
#pragma unroll
            for (int q = 0; q < 6; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 6) out[threadIdx.x] = red[threadIdx.x][0];
}

template <class LP>
void launch_momentum(const Consts<LP> &c, const PRec<LP> *rec, int n, double *partial, int nb,
                     double *out, cudaStream_t s) {
    k_momentum<LP><<<nb, 256, 0, s>>>(c, rec, n, partial);
    k_momentum_final<<<1, 256, 0, s>>>(partial, nb, out);
}

template <class LP>
void launch_max_diff(const PRec<LP> *rec, int n, unsigned long long *out, int nb, cudaStream_t s) {
    k_max_diff<LP><<<nb, 256, 0, s>>>(rec, n, out);
}

#define HIDEM_INSTANTIATE(LP)                                                                      \
    template void launch_bounds<LP>(const PRec<LP> *, int, double *, int, double *, cudaStream_t); \
    template void launch_cells<LP>(const PRec<LP> *, int, const GridInfo &, int *, int *, int *,   \
                                   cudaStream_t);                                                  \
    template void launch_permute<LP>(const int *, int, const PRec<LP> *, PRec<LP> *,               \
                                     const uint8_t *, uint8_t *, const int *, int *, const int *,  \
                                     int *, int *, cudaStream_t);                                  \
    template void launch_nbr_count<LP>(const PRec<LP> *, int, const int *, const GridInfo &,       \
                                       const int *, const int *, double, uint32_t *, int *, int *, \
                                       cudaStream_t);                                              \
    template void launch_nbr_fill<LP>(const PRec<LP> *, int, const int *, const GridInfo &,        \
                                      const int *, const int *, double, const long long *,         \
                                      int32_t *, cudaStream_t);                                    \
    template void launch_side_fill<LP>(const int *, int, const int *, const int *, const int *,    \
                                       const uint8_t *, const int *, const int *, const LP *,      \
                                       const int *, const SideView<LP> &, const long long *,       \
                                       const SideView<LP> &, int *, cudaStream_t);                 \
    template void launch_step<LP>(const Consts<LP> &, const StepArgs<LP> &, bool, int, int, int,     \
                                  cudaStream_t);                                                   \
    template bool batch_fits<LP>(int, int);                                                        \
    template void prepare_step_batch<LP>();                                                        \
    template void launch_step_batch<LP>(const Consts<LP> &, const BatchEntry<LP> *, const int *,     \
                                        const int *, int, int, int, int, int, cudaStream_t);       \
    template void launch_two_pass_batch<LP>(const Consts<LP> &, const BatchEntry<LP> *, const int *, \
                                            const int *, const int *, const int *, int, int, int,  \
                                            cudaStream_t);                                         \
    template void launch_integrate<LP>(const Consts<LP> &, PRec<LP> *, const uint8_t *,            \
                                       const LP *, int, cudaStream_t);                             \
    template void launch_link_break<LP>(const Consts<LP> &, const PRec<LP> *, const int *,         \
                                        const int *, const int *, uint8_t *, uint8_t *,            \
                                        const LP *, long long, long long, int2 *,                  \
                                        unsigned long long *, long long, cudaStream_t);            \
    template void launch_max_diff<LP>(const PRec<LP> *, int, unsigned long long *, int,            \
                                      cudaStream_t);                                               \
    template void launch_momentum<LP>(const Consts<LP> &, const PRec<LP> *, int, double *, int,     \
                                      double *, cudaStream_t);                                     \
    template void launch_energy<LP>(const Consts<LP> &, const PRec<LP> *, int, double *, int,       \
                                    double *, cudaStream_t);

HIDEM_INSTANTIATE(float)
HIDEM_INSTANTIATE(double)

}  // namespace hidem

// ------------------------------------------------------------------ setup / readback
// Packing between the caller's SoA arrays (input order) and the slot-ordered records,
// and the per-particle link-end lists, done on the device so that setup and readback
// cost one copy of each array.

namespace hidem {

template <class LP>
__global__ void k_pack_records(SoaIn<LP> s, int n, PRec<LP> *__restrict__ rec) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    PRec<LP> r;
    r.x = s.x[i];
    r.y = s.y[i];
    r.z = s.z[i];
#pragma unroll
    for (int k = 0; k < 6; ++k) r.d[k] = s.d[k] ? s.d[k][i] : LP(0);
    r.r = s.r[i];
#pragma unroll
    for (int k = 0; k < 3; ++k) r.th[k] = s.th[k] ? s.th[k][i] : LP(0);
    if (sizeof(PRec<LP>) == 128) {
        double *pad = reinterpret_cast<double *>(&r) + 13;
        pad[0] = pad[1] = pad[2] = 0.0;
    }
    store_rec(rec + i, r);
}

template <class LP>
__global__ void k_unpack_records(const PRec<LP> *__restrict__ rec, const int *__restrict__ orig,
                                 int n, SoaIn<LP> s) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const PRec<LP> r = load_rec(rec + k);
    const int i = orig[k];
    const_cast<double *>(s.x)[i] = r.x;
    const_cast<double *>(s.y)[i] = r.y;
    const_cast<double *>(s.z)[i] = r.z;
#pragma unroll
    for (int q = 0; q < 6; ++q) const_cast<LP *>(s.d[q])[i] = r.d[q];
    const_cast<LP *>(s.r)[i] = r.r;
#pragma unroll
    for (int q = 0; q < 3; ++q) const_cast<LP *>(s.th[q])[i] = r.th[q];
}

template <class LP>
__global__ void k_unpack_force(const LP *__restrict__ force, const int *__restrict__ orig, int n,
                               LP *__restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = orig[k];
#pragma unroll
    for (int q = 0; q < 6; ++q) out[(long long)q * n + i] = force[(long long)q * n + k];
}

// Halo force exchange of a slab decomposition (CommunicatorPacked::packAllCommData /
// unpackAllCommData, HiDEMLib.h:337-372): one thread per (listed particle, component); the
// buffer holds 6 values per particle so that each peer's records are one contiguous run.
template <class LP>
__global__ void k_pack_halo(const LP *__restrict__ force, const int *__restrict__ slotOf,
                            const int *__restrict__ index, long long m, int n, LP *__restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6 * m) return;
    const long long k = t / 6;
    const int q = (int)(t - 6 * k);
    out[t] = force[(long long)q * n + slotOf[index[k]]];
}

template <class LP>
__global__ void k_unpack_halo(const LP *__restrict__ in, const int *__restrict__ slotOf,
                              const int *__restrict__ index, long long m, int n, LP *__restrict__ force) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6 * m) return;
    const long long k = t / 6;
    const int q = (int)(t - 6 * k);
    force[(long long)q * n + slotOf[index[k]]] = in[t];
}

// per-particle number of link ends
__global__ void k_link_degree(const int *__restrict__ A, const int *__restrict__ B, long long L,
                              int *__restrict__ deg) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= L) return;
    atomicAdd(deg + A[l], 1);
    atomicAdd(deg + B[l], 1);
}

__global__ void k_link_fill(const int *__restrict__ A, const int *__restrict__ B, long long L,
                            const int *__restrict__ start, int *__restrict__ cursor,
                            int *__restrict__ plLink, uint8_t *__restrict__ plEnd) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= L) return;
    int a = start[A[l]] + atomicAdd(cursor + A[l], 1);
    plLink[a] = (int)l;
    plEnd[a] = 0;
    int b = start[B[l]] + atomicAdd(cursor + B[l], 1);
    plLink[b] = (int)l;
    plEnd[b] = 1;
}

// a particle's ends in ascending link index (LinkAccelSide::generateLinks, LinkAccelSide.h:118-131)
__global__ void k_link_sort_ends(const int *__restrict__ start, int n, int *__restrict__ plLink,
                                 uint8_t *__restrict__ plEnd) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = start[i], e = start[i + 1];
    for (int a = s + 1; a < e; ++a) {
        const int v = plLink[a];
        const uint8_t ve = plEnd[a];
        int b = a - 1;
        while (b >= s && plLink[b] > v) {
            plLink[b + 1] = plLink[b];
            plEnd[b + 1] = plEnd[b];
            --b;
        }
        plLink[b + 1] = v;
        plEnd[b + 1] = ve;
    }
}

// flat initial side layout: side 2l+e, state copied from the link
__global__ void k_side_init(const uint8_t *__restrict__ linkState, long long L,
                            int *__restrict__ sideSlot, uint8_t *__restrict__ sideState) {
    long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 2 * L) return;
    sideSlot[s] = (int)s;
    sideState[s] = linkState[s >> 1];
}

// side data back in the caller's order: CT[k][2l+e] and the link state
template <class LP>
__global__ void k_gather_sides(const int *__restrict__ sideSlot, long long L,
                               const LP *__restrict__ ct, LP *__restrict__ out,
                               const uint8_t *__restrict__ sState, uint8_t *__restrict__ linkState) {
    long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 2 * L) return;
    const int src = sideSlot[s];
    if (ct) out[s] = ct[src];
    if (linkState && (s & 1) == 0) linkState[s >> 1] = sState[src];
}

__global__ void k_link_keys_identity(const long long *__restrict__ ka, const long long *__restrict__ kb,
                                     long long L, long long n, int *__restrict__ A, int *__restrict__ B,
                                     unsigned long long *badMin, unsigned long long *selfMin) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L;
         i += (long long)gridDim.x * blockDim.x) {
        const long long a = ka[i], b = kb[i];
        if (a < 0 || a >= n || b < 0 || b >= n) {
            atomicMin(badMin, (unsigned long long)i);
            A[i] = 0;
            B[i] = 0;
            continue;
        }
        A[i] = (int)a;
        B[i] = (int)b;
        if (a == b) atomicMin(selfMin, (unsigned long long)i);
    }
}

// link ends from particle keys in strictly ascending order (not 0..n-1): each end's index
// by a binary search of the key table
__device__ __forceinline__ int find_key(const long long *__restrict__ keys, long long n, long long k) {
    long long lo = 0, hi = n;  // first position with keys[pos] >= k
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (__ldg(keys + mid) < k) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && __ldg(keys + lo) == k) ? (int)lo : -1;
}

__global__ void k_link_keys_sorted(const long long *__restrict__ keys, long long n,
                                   const long long *__restrict__ ka, const long long *__restrict__ kb,
                                   long long L, int *__restrict__ A, int *__restrict__ B,
                                   unsigned long long *badMin, unsigned long long *selfMin) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L;
         i += (long long)gridDim.x * blockDim.x) {
        const int a = find_key(keys, n, ka[i]), b = find_key(keys, n, kb[i]);
        if (a < 0 || b < 0) {
            atomicMin(badMin, (unsigned long long)i);
            A[i] = 0;
            B[i] = 0;
            continue;
        }
        A[i] = a;
        B[i] = b;
        if (a == b) atomicMin(selfMin, (unsigned long long)i);
    }
}

void launch_link_keys_sorted(const long long *keys, long long n, const long long *keyA,
                             const long long *keyB, long long L, int *A, int *B,
                             unsigned long long *badMin, unsigned long long *selfMin, cudaStream_t st) {
    if (L <= 0) return;
    const int nb = (int)std::min<long long>((L + 255) / 256, 148LL * 32);
    k_link_keys_sorted<<<nb, 256, 0, st>>>(keys, n, keyA, keyB, L, A, B, badMin, selfMin);
}

__global__ void k_iota64(long long *out, long long count) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = i;
}

void launch_link_keys_identity(const long long *keyA, const long long *keyB, long long L,
                               long long n, int *A, int *B, unsigned long long *badMin,
                               unsigned long long *selfMin, cudaStream_t st) {
    if (L <= 0) return;
    const int nb = (int)std::min<long long>((L + 255) / 256, 148LL * 32);
    k_link_keys_identity<<<nb, 256, 0, st>>>(keyA, keyB, L, n, A, B, badMin, selfMin);
}

__global__ void k_iota32(int *out, int count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) out[i] = i;
}

// slots of both ends of every link in the current storage order (after a rebuild's permute)
__global__ void k_link_slots(const int *__restrict__ linkA, const int *__restrict__ linkB,
                             const int *__restrict__ slotOf, long long L, int *__restrict__ slotA,
                             int *__restrict__ slotB) {
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < L;
         l += (long long)gridDim.x * blockDim.x) {
        slotA[l] = slotOf[linkA[l]];
        slotB[l] = slotOf[linkB[l]];
    }
}

void launch_link_slots(const int *linkA, const int *linkB, const int *slotOf, long long L, int *slotA,
                       int *slotB, cudaStream_t st) {
    if (L <= 0) return;
    const int nb = (int)std::min<long long>((L + 255LL) / 256, 148LL * 32);
    k_link_slots<<<nb, 256, 0, st>>>(linkA, linkB, slotOf, L, slotA, slotB);
}

void launch_iota32(int *out, int count, cudaStream_t st) {
    if (count <= 0) return;
    const int nb = (int)std::min<long long>((count + 255LL) / 256, 148LL * 32);
    k_iota32<<<nb, 256, 0, st>>>(out, count);
}

// largest particle radius (radii are positive, so their IEEE bits order like the values)
template <class LP>
__global__ void k_max_radius(const PRec<LP> *__restrict__ rec, int n, unsigned long long *__restrict__ out) {
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = fmax(m, (double)rec[i].r);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

template <class LP>
void launch_max_radius(const PRec<LP> *rec, int n, unsigned long long *out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
    const int nb = (int)std::max<long long>(1, std::min<long long>((n + 255LL) / 256, 148LL * 4));
    k_max_radius<LP><<<nb, 256, 0, st>>>(rec, n, out);
}
template void launch_max_radius<float>(const PRec<float> *, int, unsigned long long *, cudaStream_t);
template void launch_max_radius<double>(const PRec<double> *, int, unsigned long long *, cudaStream_t);

void launch_iota64(long long *out, long long count, cudaStream_t st) {
    if (count <= 0) return;
    const int nb = (int)std::min<long long>((count + 255) / 256, 148LL * 32);
    k_iota64<<<nb, 256, 0, st>>>(out, count);
}

template <class LP>
void launch_pack_records(const SoaIn<LP> &s, int n, PRec<LP> *rec, cudaStream_t st) {
    k_pack_records<LP><<<nblk(n, 256), 256, 0, st>>>(s, n, rec);
}
template <class LP>
void launch_unpack_records(const PRec<LP> *rec, const int *orig, int n, const SoaIn<LP> &s,
                           cudaStream_t st) {
    k_unpack_records<LP><<<nblk(n, 256), 256, 0, st>>>(rec, orig, n, s);
}
template <class LP>
void launch_unpack_force(const LP *force, const int *orig, int n, LP *out, cudaStream_t st) {
    k_unpack_force<LP><<<nblk(n, 256), 256, 0, st>>>(force, orig, n, out);
}
template <class LP>
void launch_halo_forces(LP *force, const int *slotOf, const int *index, long long m, int n, LP *buf,
                        bool pack, cudaStream_t st) {
    if (m <= 0) return;
    if (pack)
        k_pack_halo<LP><<<nblk(6 * m, 256), 256, 0, st>>>(force, slotOf, index, m, n, buf);
    else
        k_unpack_halo<LP><<<nblk(6 * m, 256), 256, 0, st>>>(buf, slotOf, index, m, n, force);
}
void launch_link_lists(const int *A, const int *B, long long L, int n, int *deg, int *start,
                       int *cursor, int *sums, int *plLink, uint8_t *plEnd, cudaStream_t st) {
    if (L > 0) k_link_degree<<<nblk(L, 256), 256, 0, st>>>(A, B, L, deg);
    // start[0..n] = exclusive scan of deg[0..n] with deg[n] = 0
    launch_scan<int, int>(deg, (long long)n + 1, 1, start, sums, nullptr, st);
    if (L > 0) k_link_fill<<<nblk(L, 256), 256, 0, st>>>(A, B, L, start, cursor, plLink, plEnd);
    k_link_sort_ends<<<nblk(n, 256), 256, 0, st>>>(start, n, plLink, plEnd);
}
void launch_side_init(const uint8_t *linkState, long long L, int *sideSlot, uint8_t *sideState,
                      cudaStream_t st) {
    if (L > 0) k_side_init<<<nblk(2 * L, 256), 256, 0, st>>>(linkState, L, sideSlot, sideState);
}
template <class LP>
void launch_gather_sides(const int *sideSlot, long long L, const LP *ct, LP *out,
                         const uint8_t *sState, uint8_t *linkState, cudaStream_t st) {
    if (L > 0) k_gather_sides<LP><<<nblk(2 * L, 256), 256, 0, st>>>(sideSlot, L, ct, out, sState, linkState);
}

#define HIDEM_INSTANTIATE_IO(LP)                                                                   \
    template void launch_pack_records<LP>(const SoaIn<LP> &, int, PRec<LP> *, cudaStream_t);       \
    template void launch_unpack_records<LP>(const PRec<LP> *, const int *, int, const SoaIn<LP> &,  \
                                            cudaStream_t);                                         \
    template void launch_unpack_force<LP>(const LP *, const int *, int, LP *, cudaStream_t);       \
    template void launch_halo_forces<LP>(LP *, const int *, const int *, long long, int, LP *, bool, \
                                         cudaStream_t);                                            \
    template void launch_gather_sides<LP>(const int *, long long, const LP *, LP *,                \
                                          const uint8_t *, uint8_t *, cudaStream_t);
HIDEM_INSTANTIATE_IO(float)
HIDEM_INSTANTIATE_IO(double)

}  // namespace hidem
