// hidem_bin_cells_noalloc: the neighbour-grid binning of the rebuild (bounds, cell
// colour per particle, counting sort into the (cell, index) iteration order) for callers
// that cannot allocate device memory. Its scratch — per-block bounds partials, per-cell
// counters and cursors, the per-cell start offsets and the scan's block sums — lives in
// one file-scope __device__ array of fixed size, so the call itself never allocates.
//
// Every GPU that loads this library holds that array (about 4.1 MB) until the process
// exits. All calls on a device share it and it keeps the last call's contents, so the
// entry point clears what must start at zero on every call, and calls that overlap on
// the GPU (two streams, two host threads) race on it.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>

#include "kernels.h"

namespace hidem {
extern thread_local std::string g_nocontext_error;
}

namespace {

constexpr long long kNoAllocMaxCells = 262144;  // HIDEM_NOALLOC_MAX_CELLS
constexpr int kNoAllocBoundsBlocks = 512;
constexpr int kNoAllocScanBlock = 1024;
constexpr long long kNoAllocSums = kNoAllocMaxCells / kNoAllocScanBlock + 2;

struct NoAllocScratch {
    double partial[kNoAllocBoundsBlocks * 6];
    double bounds[8];
    int count[kNoAllocMaxCells];
    int cursor[kNoAllocMaxCells];
    int start[kNoAllocMaxCells];
    int big[kNoAllocMaxCells];  // cells of more than 32 members, sorted one CTA each
    int sums[kNoAllocSums];
    int total[4];
    int bigCount[4];
    int status[4];              // status[0]: nonzero when a cell held too many members to sort
};

// The only storage the entry point uses besides the caller's buffers.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// min / max that keep a NaN (fmin / fmax drop one), so that a single NaN coordinate reaches
// the bounds and the call refuses the input; equal to fmin / fmax for numbers
__device__ __forceinline__ double na_min(double a, double b) {
    return (a != a) ? a : ((b != b) ? b : fmin(a, b));
}
__device__ __forceinline__ double na_max(double a, double b) {
    return (a != a) ? a : ((b != b) ? b : fmax(a, b));
}

__global__ void k_na_bounds(const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, int n, double *__restrict__ partial) {
    double mn[3] = {INFINITY, INFINITY, INFINITY};
    double mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v[3] = {x[i], y[i], z[i]};
        for (int k = 0; k < 3; ++k) {
            mn[k] = na_min(mn[k], v[k]);
            mx[k] = na_max(mx[k], v[k]);
        }
    }
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = na_min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = na_max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    __shared__ double sm[32][6];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 3; ++k) {
            sm[w][k] = mn[k];
            sm[w][3 + k] = mx[k];
        }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) {
            double a = sm[0][k], b = sm[0][3 + k];
            for (int j = 1; j < (int)(blockDim.x >> 5); ++j) {
                a = na_min(a, sm[j][k]);
                b = na_max(b, sm[j][3 + k]);
            }
            partial[blockIdx.x * 6 + k] = a;
            partial[blockIdx.x * 6 + 3 + k] = b;
        }
    }
}

__global__ void k_na_bounds_final(const double *__restrict__ partial, int nb, double *__restrict__ out) {
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        double v = partial[k];
        for (int b = 1; b < nb; ++b) {
            double u = partial[b * 6 + k];
            v = (k < 3) ? na_min(v, u) : na_max(v, u);
        }
        out[k] = v;
    }
}

// colour = ix + iy*X + iz*X*Y with ix = floor((x - xMin) / h) (PLiB/NeighbourGrid.cpp:25-33)
__global__ void k_na_cells(const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, int n, double xMin, double yMin,
                           double zMin, double h, int X, int Y, long long total,
                           int *__restrict__ cellOf, int *__restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int ix = (int)floor((x[i] - xMin) / h);
    const int iy = (int)floor((y[i] - yMin) / h);
    const int iz = (int)floor((z[i] - zMin) / h);
    long long c = (long long)ix + (long long)iy * X + (long long)iz * X * Y;
    c = c < 0 ? 0 : (c >= total ? total - 1 : c);  // in range by construction of the bounds
    cellOf[i] = (int)c;
    atomicAdd(count + c, 1);
}

__global__ void k_na_scatter(const int *__restrict__ cellOf, int n, const int *__restrict__ start,
                             int *__restrict__ cursor, int *__restrict__ order) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = cellOf[i];
    order[start[c] + atomicAdd(cursor + c, 1)] = i;
}

hidem_status na_fail(hidem_status s, const std::string &msg) {
    hidem::g_nocontext_error = msg;
    return s;
}

}  // namespace

extern "C" hidem_status hidem_bin_cells_noalloc(const double *x, const double *y, const double *z,
                                                int64_t n, double cell_size, int32_t *cell_of,
                                                int32_t *order, int64_t dims[3], double mins[3],
                                                void *stream) {
    hidem::g_nocontext_error.clear();
    if (!x || !y || !z || !cell_of || !order || !dims || !mins)
        return na_fail(HIDEM_ERR_ARG, "hidem_bin_cells_noalloc: null pointer argument");
    if (n <= 0 || n >= (1ll << 31))
        return na_fail(HIDEM_ERR_ARG, "hidem_bin_cells_noalloc: n must be in [1, 2^31)");
    if (!(cell_size > 0) || !std::isfinite(cell_size))
        return na_fail(HIDEM_ERR_ARG, "hidem_bin_cells_noalloc: cell_size must be > 0");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64)
        return na_fail(HIDEM_ERR_CUDA, std::string("hidem_bin_cells_noalloc: no current device: ") +
                                           cudaGetErrorString(e));
    // The array's name is a host-side stand-in in this code; its device address comes from
    // the runtime with the device current. It is looked up on every call (it allocates
    // nothing), so that it is valid again after the caller resets the device.
    NoAllocScratch *S = nullptr;
    {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return na_fail(HIDEM_ERR_CUDA, std::string("hidem_bin_cells_noalloc: "
                                                       "cudaGetSymbolAddress failed: ") +
                                               cudaGetErrorString(e));
        S = static_cast<NoAllocScratch *>(p);
    }
    int smCount = 148;
    if (cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || smCount < 1)
        smCount = 148;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int ni = (int)n;

    // 1. bounds (ParticleData::getLimits, PLiB/ParticleData.h:47-59)
    int nb = (int)std::min<long long>((n + 255) / 256, kNoAllocBoundsBlocks);
    k_na_bounds<<<nb, 256, 0, st>>>(x, y, z, ni, S->partial);
    k_na_bounds_final<<<1, 32, 0, st>>>(S->partial, nb, S->bounds);
    double b[6];
    e = cudaMemcpyAsync(b, S->bounds, sizeof b, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return na_fail(HIDEM_ERR_CUDA, std::string("hidem_bin_cells_noalloc: ") + cudaGetErrorString(e));
    // the bounds carry a NaN of any coordinate; an infinite one shows as an infinite bound
    for (int k = 0; k < 6; ++k)
        if (!std::isfinite(b[k]))
            return na_fail(HIDEM_ERR_ARG, "hidem_bin_cells_noalloc: non-finite coordinates (NaN or infinite)");

    // 2. grid dims (NeighbourGrid::getGridSize, PLiB/NeighbourGrid.cpp:40-46)
    const double ex = std::floor((b[3] - b[0]) / cell_size);
    const double ey = std::floor((b[4] - b[1]) / cell_size);
    const double ez = std::floor((b[5] - b[2]) / cell_size);
    const double totalD = (1.0 + ex) * (1.0 + ey) * (1.0 + ez);
    if (totalD > (double)kNoAllocMaxCells) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "hidem_bin_cells_noalloc: the grid has %.0f cells, more than the fixed scratch "
                 "holds (HIDEM_NOALLOC_MAX_CELLS = %lld); use hidem_regenerate instead",
                 totalD, kNoAllocMaxCells);
        return na_fail(HIDEM_ERR_CAPACITY, msg);
    }
    const int X = 1 + (int)ex, Y = 1 + (int)ey, Z = 1 + (int)ez;
    const long long total = (long long)X * Y * Z;
    dims[0] = X;
    dims[1] = Y;
    dims[2] = Z;
    mins[0] = b[0];
    mins[1] = b[1];
    mins[2] = b[2];

    // 3. counters start at zero on every call: the array keeps the previous call's values
    e = cudaMemsetAsync(S->count, 0, sizeof(int) * (size_t)total, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->cursor, 0, sizeof(int) * (size_t)total, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->status, 0, sizeof S->status, st);
    if (e != cudaSuccess)
        return na_fail(HIDEM_ERR_CUDA, std::string("hidem_bin_cells_noalloc: ") + cudaGetErrorString(e));

    // 4. colours, per-cell counts, exclusive scan, placement, order inside cells
    k_na_cells<<<(ni + 255) / 256, 256, 0, st>>>(x, y, z, ni, b[0], b[1], b[2], cell_size, X, Y,
                                                 total, cell_of, S->count);
    hidem::launch_scan<int, int>(S->count, total, 1, S->start, S->sums, S->total, st);
    k_na_scatter<<<(ni + 255) / 256, 256, 0, st>>>(cell_of, ni, S->start, S->cursor, order);
    // inside each cell ascending input index, the order of NeighbourGrid::generateIterationList
    // (PLiB/NeighbourGrid.cpp:163-184); cells of more than 4096 members are refused
    hidem::launch_sort_cells(S->start, S->count, total, nullptr, order, S->big, S->bigCount, S->status,
                             1, smCount, st);
    e = cudaGetLastError();
    int status = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, S->status, sizeof status, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return na_fail(HIDEM_ERR_CUDA, std::string("hidem_bin_cells_noalloc: ") + cudaGetErrorString(e));
    if (status != 0)
        return na_fail(HIDEM_ERR_CAPACITY, "hidem_bin_cells_noalloc: a cell holds more than 4096 "
                                           "particles; use a smaller cell_size");
    return HIDEM_OK;
}
