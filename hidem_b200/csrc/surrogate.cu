// Learned warm start: the coordinate MLP that predicts the gravity/buoyancy-settled
// displacement of a particle from its position and the local ice geometry, trained and
// evaluated by this library's own kernels. No counterpart in the reference (HiDEM settles
// every geometry from rest). The hidden layers are BF16 GEMMs on the 5th-generation tensor
// cores: tiles staged by TMA (cp.async.bulk.tensor, 128-byte swizzle) through a 4-stage
// mbarrier ring, tcgen05.mma issued by one thread with the FP32 accumulator in tensor
// memory, and an epilogue (bias + SiLU, or the SiLU derivative) that reads the
// accumulator back with tcgen05.ld. The 3-wide output layer, the loss, the reductions
// and Adam run on the CUDA cores.
//
// Network: features(u) -> [Linear(K_l -> W) + SiLU] x L -> Linear(W -> 3), with
// u = the row's normalised inputs (the caller's: coordinates, local geometry, lattice
// neighbourhood) and Fourier features u_i, sin(2^f pi u_i), cos(2^f pi u_i) for f < F,
// zero-padded to K_0, a multiple of 128.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hidem_b200.h"

namespace hidem {
extern thread_local std::string g_nocontext_error;
}

namespace {

typedef __nv_bfloat16 bf16;

// ------------------------------------------------------------------ PTX helpers

__device__ __forceinline__ uint32_t su32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mb_init(uint64_t *b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mb_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mb_expect_tx(uint64_t *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mb_try(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// every wait is bounded: after kSpins polls the caller records an error and gives up
constexpr int kSpins = 1 << 22;
__device__ __forceinline__ bool mb_wait(uint64_t *b, uint32_t parity) {
    for (int i = 0; i < kSpins; ++i)
        if (mb_try(b, parity)) return true;
    return false;
}
// 2-D tiled TMA load of box {64 elements, rows} at (c0 = element column, c1 = row)
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(su32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(su32(bar)), "r"(c0), "r"(c1)
        : "memory");
}
__device__ __forceinline__ void tm_alloc(uint32_t *slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(slot)),
                 "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tm_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, both K-major, kind::f16 (BF16 in, FP32 accumulate)
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
// arrive on `bar` once every MMA issued so far by this thread has completed
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     su32(bar))
                 : "memory");
}
// 16 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tm_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// 32 consecutive FP32 columns of this thread's tensor-memory lane, one load and one wait
__device__ __forceinline__ void tm_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
        "%30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with the 128-byte
// swizzle: rows of 64 BF16 (128 B), 8-row atoms 1024 B apart (stride byte offset),
// descriptor version 1, layout type 2 (128-byte swizzle). Moving 16 elements along K
// inside the atom adds 32 B to the start address.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void set_err(int *flag, int code) {
    if (flag) atomicCAS(flag, 0, code);
}

// The derivative of SiLU with the fast exponential and division (the network trains in
// BF16; these need no IEEE rounding)
__device__ __forceinline__ float silu_grad(float z) {
    const float s = __fdividef(1.0f, 1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

}  // namespace

namespace {

// ------------------------------------------------------------------ tensor-core GEMM

// the backward pass's epilogues (the forward pass is k_mlp_fwd)
enum Epi { EPI_F32 = 0, EPI_SILU_GRAD = 2 };

struct GemmArgs {
    int M, N, K;             // C[M][N] = A[M][K] * B[N][K]^T
    int kTiles;              // 64-wide K tiles per CTA (split-K: gridDim.y splits)
    float *outF;             // EPI_F32: [split][M][ldo] (+ bias when given)
    long long splitStride;   // elements between split partials of outF
    bf16 *outH;              // EPI_SILU_GRAD: acc * SiLU'(zIn)
    const float *zIn;        // EPI_SILU_GRAD: pre-activation [M][ldo]
    const float *bias;       // [N] or null
    int ldo;
    int *err;
};

constexpr int kGemmStages = 4;
constexpr int kGemmThreads = 256;

template <int BN>
constexpr size_t gemm_smem_bytes() {
    return (size_t)kGemmStages * (128 * 128 + BN * 128) + 1024 + 256;
}

// One CTA: rows [128 * blockIdx.x, +128) x all BN columns, K tiles
// [kTiles * blockIdx.y, +kTiles). Thread 0 streams A / B tiles with TMA and issues the
// MMAs (4 of K = 16 per 64-wide tile); the eight warps then read the accumulator (warp w:
// lanes / rows 32 (w % 4) .. +31, column half w / 4) and apply the epilogue.
// EPI_SILU_GRAD: the CTA's 128 x BN pre-activation tile comes into shared memory by TMA
// (FP32 boxes of 64 columns x 128 rows, no swizzle) once the MMAs have released the
// pipeline stages, behind the eight warps' transpose buffers
constexpr uint32_t kZOff = 36864;

template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    k_umma_gemm(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
                const __grid_constant__ CUtensorMap tz, const GemmArgs g) {
    constexpr int S = kGemmStages;
    constexpr uint32_t ABYTES = 128 * 128, BBYTES = BN * 128, STAGE = ABYTES + BBYTES;
    constexpr uint32_t COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
    extern __shared__ unsigned char dyn[];
    unsigned char *sm =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + S * STAGE);
    uint64_t *empty = full + S;
    uint64_t *done = empty + S;
    uint64_t *zbar = done + 1;
    uint32_t *slot = reinterpret_cast<uint32_t *>(zbar + 1);
    static_assert(kZOff + 128u * BN * 4u <= (uint32_t)S * STAGE, "pre-activation tile exceeds the stages");
    __shared__ int sFail;
    const int tid = threadIdx.x, warp = tid >> 5;

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mb_init(full + s, 1);
            mb_init(empty + s, 1);
        }
        mb_init(done, 1);
        mb_init(zbar, 1);
        sFail = 0;
        mb_fence_init();
    }
    if (warp == 0) {
        tm_alloc(slot, COLS);
        tm_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    const int m0 = blockIdx.x * 128;
    const int kt0 = blockIdx.y * g.kTiles;
    const int nk = g.kTiles;

    if (tid == 0) {
        // kind::f16 descriptor: D FP32, A and B BF16, both K-major, N = BN, M = 128
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(128 >> 4) << 24);
        int issued = 0;
        auto load = [&](int i) {
            const int s = i % S;
            unsigned char *a = sm + s * STAGE;
            mb_expect_tx(full + s, STAGE);
            tma_load_2d(a, &ta, (kt0 + i) * 64, m0, full + s);
            tma_load_2d(a + ABYTES, &tb, (kt0 + i) * 64, 0, full + s);
        };
        for (; issued < nk && issued < S; ++issued) load(issued);
        bool ok = true;
        int i = 0;
        for (; i < nk; ++i) {
            const int s = i % S;
            const uint32_t par = (uint32_t)((i / S) & 1);
            if (!mb_wait(full + s, par)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t a0 = su32(sm + s * STAGE), b0 = a0 + ABYTES;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                tc_mma(tmem, sw128_desc(a0 + 32u * kk), sw128_desc(b0 + 32u * kk), idesc,
                       (i > 0 || kk > 0) ? 1u : 0u);
            tc_commit(empty + s);
            if (issued < nk) {
                if (!mb_wait(empty + s, par)) {
                    ok = false;
                    ++i;
                    break;
                }
                load(issued);
                ++issued;
            }
        }
        tc_commit(done);
        if (!ok) {
            sFail = 1;
            set_err(g.err, 1);
            // copies still in flight land in this CTA's shared memory: give them a
            // bounded chance to complete before the CTA exits
            for (int j = i; j < issued; ++j) mb_wait(full + (j % S), (uint32_t)((j / S) & 1));
        }
    }
    // the producer's own warp waits for it here rather than polling the accumulator
    // barrier beside it: polling lanes of a diverged warp delay the lane that issues
    if (warp == 0) __syncwarp();
    const bool accReady = mb_wait(done, 0);
    tc_fence_after();
    __syncthreads();
    // the MMAs have completed: their stages take the pre-activation tile
    bool zReady = true, zIssued = false;
    if (EPI == EPI_SILU_GRAD && accReady && !sFail) {
        zIssued = true;
        if (tid == 0) {
            mb_expect_tx(zbar, 128u * BN * 4u);
#pragma unroll
            for (int c = 0; c < BN / 64; ++c)
                tma_load_2d(sm + kZOff + c * (128 * 64 * 4), &tz, c * 64, m0, zbar);
        }
        zReady = mb_wait(zbar, 0);
        if (!zReady && tid == 0) set_err(g.err, 3);
    }
    if (accReady && !sFail && zReady) {
        // The accumulator lane of a thread is one row; stores are made coalesced by
        // passing each 32 x 32 block through shared memory (the pipeline stages are free
        // now): lane j then writes column c0 + j of 32 consecutive rows.
        float *stage = reinterpret_cast<float *>(sm) + warp * 32 * 33;
        const int lane = tid & 31;
        const int quarter = warp & 3;
        const int rowBase = m0 + quarter * 32;
        const uint32_t tlane = (uint32_t)(quarter * 32) << 16;
#pragma unroll 1
        for (int c0 = (warp >> 2) * (BN / 2); c0 < ((warp >> 2) + 1) * (BN / 2); c0 += 32) {
            float v[32];
            tm_ld16(tmem + tlane + (uint32_t)c0, v);
            tm_ld16(tmem + tlane + (uint32_t)(c0 + 16), v + 16);
#pragma unroll
            for (int j = 0; j < 32; ++j) stage[lane * 33 + j] = v[j];
            __syncwarp();
            const int col = c0 + lane;
            const float bias = g.bias ? g.bias[col] : 0.f;
            if (EPI == EPI_F32) {
#pragma unroll 4
                for (int r = 0; r < 32; ++r) {
                    const long long o = (long long)(rowBase + r) * g.ldo + col;
                    g.outF[blockIdx.y * g.splitStride + o] = stage[r * 33 + lane] + bias;
                }
            } else {
                // the 32 rows' pre-activations all in flight at once: each load is a
                // coalesced 128-byte row segment, and the warp's latency is paid once
                const float *zt = reinterpret_cast<const float *>(sm + kZOff + (col >> 6) * (128 * 64 * 4)) +
                                  quarter * 32 * 64 + (col & 63);
#pragma unroll 4
                for (int r = 0; r < 32; ++r) {
                    const long long o = (long long)(rowBase + r) * g.ldo + col;
                    g.outH[o] = __float2bfloat16_rn(stage[r * 33 + lane] * silu_grad(zt[r * 64]));
                }
            }
            __syncwarp();
        }
    } else if (tid == 0 && !accReady) {
        set_err(g.err, 2);
    }
    // a pre-activation copy that did not complete in time still lands in this CTA's
    // shared memory: a second bounded wait before the CTA exits
    if (zIssued && !zReady && tid == 0) mb_wait(zbar, 0);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tm_dealloc(tmem, COLS);
}

// ------------------------------------------------------------------ fused forward pass

constexpr int kMlpMaxLayers = 8;
constexpr int kMlpStages = 3;
constexpr int kOutCols = 3;
constexpr int kMlpThreads = 512;  // 16 warps: 4 lane quarters x 4 column quarters

// SiLU for the forward pass from the hardware tanh: z * (1 + tanh(z / 2)) / 2 (the result is
// rounded to BF16, far coarser than the approximation)
__device__ __forceinline__ float silu_fast(float z) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
    return 0.5f * z * (1.0f + t);
}

struct MlpMaps {
    CUtensorMap x;                  // features [rows][K0], boxes of 64 x 128
    CUtensorMap w[kMlpMaxLayers];   // hidden weights [W][K_l], boxes of 64 x W
};

struct MlpArgs {
    int layers, k0;                 // hidden layers, first layer's K
    const float *bias[kMlpMaxLayers];
    const float *wo, *bo;           // output layer [3][W], [3]
    float *y;                       // [rows][3]
    float *z[kMlpMaxLayers];        // pre-activations [rows][W] (null: not kept)
    bf16 *h[kMlpMaxLayers];         // activations [rows][W] (null: not kept)
    int *err;
};

template <int BN>
constexpr size_t mlp_smem_bytes() {
    return (size_t)kMlpStages * (128 * 128 + BN * 128) + (size_t)128 * BN * 2 + 1024 + 256;
}

// One CTA per 128-row block runs the whole network: features and weights stream through a
// 3-stage TMA ring; each hidden layer's accumulator (128 x BN FP32) sits in tensor memory;
// its epilogue (bias + SiLU, BF16) writes the activations back into shared memory in the
// 128-byte-swizzled K-major layout TMA would have written, so they are the next layer's A
// operand without a round trip through global memory (the pre-activations and activations
// go to global memory only when the training pass keeps them). The 3-wide output layer
// runs on the CUDA cores from the last activations: per row, a sequential FP32 sum over k.
// Thread 0 issues the copies and the MMAs (and prefetches the next layer's weights while
// the epilogue runs); the sixteen warps share the epilogues (warp w: accumulator lanes
// 32 (w % 4) .. +31, i.e. those rows, and the column quarter w / 4).
template <int BN>
__global__ void __launch_bounds__(kMlpThreads, 1)
    k_mlp_fwd(const __grid_constant__ MlpMaps maps, const MlpArgs g) {
    constexpr int S = kMlpStages;
    constexpr uint32_t ABYTES = 128 * 128, BBYTES = BN * 128, STAGE = ABYTES + BBYTES;
    constexpr uint32_t ACT_BLOCK = 128 * 128;   // 128 rows x 64 BF16 columns
    constexpr uint32_t COLS = BN;
    extern __shared__ unsigned char dyn[];
    unsigned char *sm =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
    unsigned char *act = sm + S * STAGE;
    uint64_t *full = reinterpret_cast<uint64_t *>(act + (size_t)128 * BN * 2);
    uint64_t *empty = full + S;
    uint64_t *done = empty + S;
    uint32_t *slot = reinterpret_cast<uint32_t *>(done + 1);
    __shared__ int sFail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int L = g.layers;
    const int nk0 = g.k0 / 64, nkw = BN / 64;
    const int nload = nk0 + (L - 1) * nkw;

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mb_init(full + s, 1);
            mb_init(empty + s, 1);
        }
        mb_init(done, 1);
        sFail = 0;
        mb_fence_init();
    }
    if (warp == 0) {
        tm_alloc(slot, COLS);
        tm_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    const int m0 = blockIdx.x * 128;

    // load i of the stream: k-tile kt of layer l (layer 0: features and weights)
    auto load = [&](int i) {
        const int s = i % S;
        unsigned char *a = sm + s * STAGE;
        if (i < nk0) {
            mb_expect_tx(full + s, STAGE);
            tma_load_2d(a, &maps.x, i * 64, m0, full + s);
            tma_load_2d(a + ABYTES, &maps.w[0], i * 64, 0, full + s);
        } else {
            const int l = 1 + (i - nk0) / nkw, kt = (i - nk0) % nkw;
            mb_expect_tx(full + s, BBYTES);
            tma_load_2d(a + ABYTES, &maps.w[l], kt * 64, 0, full + s);
        }
    };
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(128 >> 4) << 24);
    // i: next k-tile to consume; issued: k-tiles loaded; freed: k-tiles whose ring slot
    // has been handed to a later load (issued == freed + S until the stream is exhausted)
    int issued = 0, i = 0, freed = 0;
    if (tid == 0)
        for (; issued < nload && issued < S; ++issued) load(issued);
    // reload the slots of k-tiles up to j once their MMAs have completed
    auto refill_upto = [&](int j) -> bool {
        while (freed <= j && issued < nload) {
            if (!mb_wait(empty + (freed % S), (uint32_t)((freed / S) & 1))) return false;
            load(issued++);
            ++freed;
        }
        return true;
    };

    const int quarter = warp & 3, row = quarter * 32 + lane;
    const uint32_t tlane = (uint32_t)(quarter * 32) << 16;
    for (int l = 0; l < L; ++l) {
        const int nk = l == 0 ? nk0 : nkw;
        if (tid == 0 && !sFail) {
            for (int kt = 0; kt < nk; ++kt, ++i) {
                const int s = i % S;
                if (!mb_wait(full + s, (uint32_t)((i / S) & 1))) {
                    sFail = 1;
                    set_err(g.err, 1);
                    break;
                }
                tc_fence_after();
                const uint32_t a0 = l == 0 ? su32(sm + s * STAGE) : su32(act + kt * ACT_BLOCK);
                const uint32_t b0 = su32(sm + s * STAGE) + ABYTES;
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                    tc_mma(tmem, sw128_desc(a0 + 32u * kk), sw128_desc(b0 + 32u * kk), idesc,
                           (kt > 0 || kk > 0) ? 1u : 0u);
                tc_commit(empty + s);
                // refill the slot of the previous k-tile (its MMAs are the oldest in flight)
                if (!refill_upto(i - 1)) {
                    sFail = 1;
                    set_err(g.err, 1);
                    ++i;
                    break;
                }
            }
            tc_commit(done);
        }
        __syncthreads();
        const bool ok = !sFail && mb_wait(done, (uint32_t)(l & 1));
        tc_fence_after();
        if (!ok && tid == 0) set_err(g.err, 2);
        if (ok) {
            // the ring slot of the last k-tile of this layer is free now: refill it
            if (tid == 0 && !refill_upto(i - 1)) {
                sFail = 1;
                set_err(g.err, 1);
            }
            const float *bias = g.bias[l];
            float *zo = g.z[l];
            bf16 *ho = g.h[l];
            const long long grow = (long long)(m0 + row) * BN;
#pragma unroll 1
            for (int c0 = (warp >> 2) * (BN / 4); c0 < ((warp >> 2) + 1) * (BN / 4); c0 += 32) {
                float v[32];
                tm_ld16(tmem + tlane + (uint32_t)c0, v);
                tm_ld16(tmem + tlane + (uint32_t)(c0 + 16), v + 16);
                uint32_t hp[16];
#pragma unroll
                for (int j = 0; j < 32; j += 2) {
                    const float z0 = v[j] + bias[c0 + j], z1 = v[j + 1] + bias[c0 + j + 1];
                    v[j] = z0;
                    v[j + 1] = z1;
                    const __nv_bfloat162 h2 = __floats2bfloat162_rn(silu_fast(z0), silu_fast(z1));
                    hp[j >> 1] = *reinterpret_cast<const uint32_t *>(&h2);
                }
                if (zo) {
                    float4 *zp = reinterpret_cast<float4 *>(zo + grow + c0);
#pragma unroll
                    for (int q = 0; q < 8; ++q) zp[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                }
                if (ho) {
                    uint4 *hq = reinterpret_cast<uint4 *>(ho + grow + c0);
#pragma unroll
                    for (int q = 0; q < 4; ++q) hq[q] = make_uint4(hp[4 * q], hp[4 * q + 1], hp[4 * q + 2], hp[4 * q + 3]);
                }
                // 16-byte chunks of 8 columns into the swizzled K-major activation tile
                const int kb = c0 >> 6;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int ch = ((c0 & 63) >> 3) + q;
                    uint4 *dst = reinterpret_cast<uint4 *>(act + kb * ACT_BLOCK + row * 128 + ((ch ^ (row & 7)) << 4));
                    *dst = make_uint4(hp[4 * q], hp[4 * q + 1], hp[4 * q + 2], hp[4 * q + 3]);
                }
            }
        }
        // the activations are the tensor cores' next operand: generic-proxy writes made
        // visible to the async proxy, and the accumulator reads ordered before the next MMAs
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    // output layer: one thread per row, a sequential FP32 sum over k
    if (tid < 128 && !sFail) {
        float acc[kOutCols] = {0.f, 0.f, 0.f};
        const unsigned char *rowp = act + tid * 128;
        for (int k = 0; k < BN; ++k) {
            const int kb = k >> 6, ch = (k & 63) >> 3;
            const bf16 hv = *reinterpret_cast<const bf16 *>(rowp + kb * ACT_BLOCK + ((ch ^ (tid & 7)) << 4) + ((k & 7) << 1));
            const float h = __bfloat162float(hv);
#pragma unroll
            for (int j = 0; j < kOutCols; ++j) acc[j] += h * g.wo[j * BN + k];
        }
#pragma unroll
        for (int j = 0; j < kOutCols; ++j) g.y[(long long)(m0 + tid) * kOutCols + j] = acc[j] + g.bo[j];
    }
    if (tid == 0 && sFail) {
        // copies still in flight land in this CTA's shared memory: a bounded wait for them
        for (int j = i; j < issued; ++j) mb_wait(full + (j % S), (uint32_t)((j / S) & 1));
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tm_dealloc(tmem, COLS);
}

// ------------------------------------------------------------------ persistent ping-pong forward pass

constexpr int kPPStages = 3;
constexpr int kPPEpiWarps = 16;
constexpr int kPPThreads = 32 * (2 + kPPEpiWarps);  // warp 0: copies, warp 1: MMAs, 2-17: epilogues

// both blocks' activation tiles (128 x 256 BF16), the weight ring, barriers and alignment
constexpr size_t pp_smem_bytes() {
    return (size_t)2 * 128 * 256 * 2 + (size_t)kPPStages * 256 * 128 + 1024 + 256;
}

__device__ __forceinline__ void mb_arrive(uint64_t *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
// a bounded wait that also gives up once another role of the CTA has recorded a failure
__device__ __forceinline__ bool mb_wait_or_fail(uint64_t *b, uint32_t parity, const volatile int *fail) {
    for (int i = 0; i < kSpins; ++i) {
        if (mb_try(b, parity)) return true;
        if ((i & 255) == 255 && *fail) return false;
    }
    return false;
}

// One epilogue thread's share of a unit of k_mlp_pp: its row's 64 columns starting at
// c0s, 32 at a time, from tensor memory (taddr: the row's lane, the block's accumulator):
// bias + SiLU -> BF16. KEEP (training): pre-activations and activations to global memory.
// LAST: the output layer's partial sums over these columns, in k order, into o; otherwise
// the activations into the next layer's swizzled K-major A tile. The two flags are template
// parameters so that neither path costs the other instructions.
template <int BN, bool LAST, bool KEEP>
__device__ __forceinline__ void pp_epilogue(uint32_t taddr, int c0s, int row, long long grow, bool live,
                                            const float *__restrict__ bias, float *zo, bf16 *ho,
                                            const float *__restrict__ wo, unsigned char *ab, float *o) {
    constexpr uint32_t ACT_BLOCK = 128 * 128;
#pragma unroll 1
    for (int c0 = c0s; c0 < c0s + BN / 4; c0 += 16) {
        float v[16];
        tm_ld16(taddr + (uint32_t)c0, v);
        uint32_t hp[8];
        const float4 *b4 = reinterpret_cast<const float4 *>(bias + c0);
#pragma unroll
        for (int j = 0; j < 16; j += 4) {
            const float4 bb = __ldg(b4 + (j >> 2));
            const float z0 = v[j] + bb.x, z1 = v[j + 1] + bb.y, z2 = v[j + 2] + bb.z, z3 = v[j + 3] + bb.w;
            if (KEEP && live)
                reinterpret_cast<float4 *>(zo + grow * BN + c0)[j >> 2] = make_float4(z0, z1, z2, z3);
            const __nv_bfloat162 h01 = __floats2bfloat162_rn(silu_fast(z0), silu_fast(z1));
            const __nv_bfloat162 h23 = __floats2bfloat162_rn(silu_fast(z2), silu_fast(z3));
            hp[j >> 1] = *reinterpret_cast<const uint32_t *>(&h01);
            hp[(j >> 1) + 1] = *reinterpret_cast<const uint32_t *>(&h23);
            if (LAST) {
                const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
#pragma unroll
                for (int jj = 0; jj < kOutCols; ++jj) {
                    const float4 w = __ldg(reinterpret_cast<const float4 *>(wo + jj * BN + c0 + j));
                    o[jj] += f01.x * w.x;
                    o[jj] += f01.y * w.y;
                    o[jj] += f23.x * w.z;
                    o[jj] += f23.y * w.w;
                }
            }
        }
        if (KEEP && live) {
            uint4 *hq = reinterpret_cast<uint4 *>(ho + grow * BN + c0);
#pragma unroll
            for (int u = 0; u < 2; ++u) hq[u] = make_uint4(hp[4 * u], hp[4 * u + 1], hp[4 * u + 2], hp[4 * u + 3]);
        }
        if (!LAST) {
            // 16-byte chunks of 8 columns into the swizzled K-major tile
            const int kb = c0 >> 6;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int ch = ((c0 & 63) >> 3) + u;
                uint4 *dst = reinterpret_cast<uint4 *>(ab + kb * ACT_BLOCK + row * 128 + ((ch ^ (row & 7)) << 4));
                *dst = make_uint4(hp[4 * u], hp[4 * u + 1], hp[4 * u + 2], hp[4 * u + 3]);
            }
        }
    }
}

// The forward pass of a 256-wide network as a persistent kernel. Each CTA takes pairs of
// 128-row blocks and runs the two blocks through the layers in ping-pong, so that one
// block's epilogue (tensor memory -> bias + SiLU -> BF16 activations in shared memory)
// runs while the tensor cores compute the other block's layer. Tensor memory holds both
// blocks' accumulators (2 x 256 FP32 columns); shared memory holds both blocks'
// activation tiles (128 x 256 BF16, 128-byte-swizzled K-major: the next layer's A
// operand) and a 3-stage ring of weight k-tiles (256 x 64 BF16). The first layer's A
// operand, the block's feature tile 64 columns at a time, comes by TMA straight into the
// block's activation tile, cycling through its four 64-column slots. Roles:
//   warp 0 (one lane)  the TMA copies;
//   warp 1 (one lane)  tcgen05.mma and the commits;
//   warps 2-17         the epilogues: warp w reads accumulator lanes 32 (w % 4) .. +31
//                      (its rows) and the 64 columns 64 ((w - 2) / 4) .. +63.
// Unit (l, b) is layer l of block b, in the order (0, 0), (0, 1), (1, 0), ... of each pair.
// Its MMAs wait until the block's previous epilogue has released the accumulator and the
// activation tile (accFree[b]); its epilogue waits for its MMAs (accFull[b]). The 3-wide
// output layer runs in the last layer's epilogue: each warp sums its 64 columns in k order
// per row, and the four partial sums of a row are added in column order. The hidden layers'
// arithmetic is that of k_mlp_fwd (same MMAs in the same order, same epilogue).
template <int BN>
__global__ void __launch_bounds__(kPPThreads, 1)
    k_mlp_pp(const __grid_constant__ MlpMaps maps, const MlpArgs g, int rows) {
    static_assert(BN == 256, "the ping-pong forward pass is built for 256-wide layers");
    constexpr int S = kPPStages;
    constexpr uint32_t ACT_BLOCK = 128 * 128;  // 128 rows x 64 BF16 columns
    constexpr uint32_t ACT = 128 * BN * 2;     // one block's activation tile
    constexpr uint32_t BBYTES = BN * 128;      // one 64-wide weight k-tile
    constexpr int NA = BN / 64;                // feature slots of an activation tile
    // a feature slot is reused NA loads later; the copy into it starts only after the
    // producer has seen the MMAs of the load S earlier complete
    static_assert(NA >= S, "feature slots must not be reused before their MMAs complete");
    constexpr uint32_t EPI = 32 * kPPEpiWarps;
    extern __shared__ unsigned char dyn[];
    unsigned char *sm =
        reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(dyn) + 1023) & ~(uintptr_t)1023);
    unsigned char *act = sm;
    unsigned char *ring = sm + 2 * ACT;
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + S * BBYTES);
    uint64_t *empty = full + S;
    uint64_t *accFull = empty + S;
    uint64_t *accFree = accFull + 2;
    uint64_t *outBar = accFree + 2;
    uint64_t *fin = outBar + 2;
    uint32_t *slot = reinterpret_cast<uint32_t *>(fin + 1);
    __shared__ int sFail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int L = g.layers;
    const int nk0 = g.k0 / 64, nkw = BN / 64;
    const int nPairs = (rows / 128 + 1) / 2;

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mb_init(full + s, 1);
            mb_init(empty + s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mb_init(accFull + b, 1);
            mb_init(accFree + b, EPI);
            mb_init(outBar + b, EPI);
        }
        mb_init(fin, 1);
        sFail = 0;
        mb_fence_init();
    }
    if (warp == 0) {
        tm_alloc(slot, 2 * BN);
        tm_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    volatile int *fail = &sFail;

    if (warp == 0 && lane == 0) {
        // ---- copies: k counts the loads, n[b] the units of block b
        uint32_t k = 0, n[2] = {0, 0};
        bool ok = true;
        for (int p = blockIdx.x; ok && p < nPairs; p += gridDim.x) {
            for (int l = 0; ok && l < L; ++l) {
                for (int b = 0; ok && b < 2; ++b) {
                    const int m0 = (2 * p + b) * 128;
                    unsigned char *ab = act + b * ACT;
                    // the feature tiles overwrite the block's activation tile: wait for the
                    // epilogue of the block's previous unit to release it
                    if (l == 0 && n[b] > 0 && !mb_wait_or_fail(accFree + b, (n[b] - 1) & 1, fail)) {
                        ok = false;
                        break;
                    }
                    const int nk = l == 0 ? nk0 : nkw;
                    for (int kt = 0; kt < nk; ++kt) {
                        const int s = (int)(k % S);
                        const uint32_t r = k / S;
                        if (r > 0 && !mb_wait_or_fail(empty + s, (r - 1) & 1, fail)) {
                            ok = false;
                            break;
                        }
                        unsigned char *bt = ring + s * BBYTES;
                        if (l == 0) {
                            mb_expect_tx(full + s, ACT_BLOCK + BBYTES);
                            tma_load_2d(ab + (kt % NA) * ACT_BLOCK, &maps.x, kt * 64, m0, full + s);
                            tma_load_2d(bt, &maps.w[0], kt * 64, 0, full + s);
                        } else {
                            mb_expect_tx(full + s, BBYTES);
                            tma_load_2d(bt, &maps.w[l], kt * 64, 0, full + s);
                        }
                        ++k;
                    }
                    ++n[b];
                }
            }
        }
        if (!ok) {
            *fail = 1;
            set_err(g.err, 1);
            // copies still in flight land in this CTA's shared memory: a bounded wait for the
            // last S loads (each earlier one was consumed before its stage was reused)
            for (uint32_t j = k > (uint32_t)S ? k - S : 0u; j < k; ++j) mb_wait(full + j % S, (j / S) & 1);
        }
    } else if (warp == 1 && lane == 0) {
        // ---- MMAs: kind::f16, D FP32, A and B BF16 K-major, N = BN, M = 128
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(128 >> 4) << 24);
        uint32_t k = 0, n[2] = {0, 0};
        bool ok = true;
        for (int p = blockIdx.x; ok && p < nPairs; p += gridDim.x) {
            for (int l = 0; ok && l < L; ++l) {
                for (int b = 0; ok && b < 2; ++b) {
                    if (n[b] > 0 && !mb_wait_or_fail(accFree + b, (n[b] - 1) & 1, fail)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem + (uint32_t)(b * BN);
                    const unsigned char *ab = act + b * ACT;
                    const int nk = l == 0 ? nk0 : nkw;
                    for (int kt = 0; kt < nk; ++kt) {
                        const int s = (int)(k % S);
                        if (!mb_wait_or_fail(full + s, (k / S) & 1, fail)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t a0 = su32(ab + (l == 0 ? kt % NA : kt) * ACT_BLOCK);
                        const uint32_t b0 = su32(ring + s * BBYTES);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk)
                            tc_mma(d, sw128_desc(a0 + 32u * kk), sw128_desc(b0 + 32u * kk), idesc,
                                   (kt > 0 || kk > 0) ? 1u : 0u);
                        tc_commit(empty + s);
                        ++k;
                    }
                    if (!ok) break;
                    tc_commit(accFull + b);
                    ++n[b];
                }
            }
        }
        if (!ok) {
            *fail = 1;
            set_err(g.err, 1);
        }
        // every MMA issued has completed before the CTA releases tensor memory
        tc_commit(fin);
        mb_wait(fin, 0);
    } else if (warp >= 2) {
        // ---- epilogues
        const int q = warp & 3, cg = (warp - 2) >> 2;
        const int row = q * 32 + lane;
        const uint32_t tl = (uint32_t)(q * 32) << 16;
        uint32_t n[2] = {0, 0}, no[2] = {0, 0};
        bool ok = true;
        for (int p = blockIdx.x; ok && p < nPairs; p += gridDim.x) {
            for (int l = 0; ok && l < L; ++l) {
                for (int b = 0; ok && b < 2; ++b) {
                    if (!mb_wait_or_fail(accFull + b, n[b] & 1, fail)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const long long grow = (long long)(2 * p + b) * 128 + row;
                    const bool live = grow < rows;
                    const bool last = l == L - 1;
                    unsigned char *ab = act + b * ACT;
                    const float *bias = g.bias[l];
                    float *zo = g.z[l];
                    bf16 *ho = g.h[l];
                    float o[kOutCols] = {0.f, 0.f, 0.f};
                    const uint32_t taddr = tmem + tl + (uint32_t)(b * BN);
                    const int c0s = cg * (BN / 4);
                    if (zo) {
                        if (last)
                            pp_epilogue<BN, true, true>(taddr, c0s, row, grow, live, bias, zo, ho, g.wo, ab, o);
                        else
                            pp_epilogue<BN, false, true>(taddr, c0s, row, grow, live, bias, zo, ho, g.wo, ab, o);
                    } else {
                        if (last)
                            pp_epilogue<BN, true, false>(taddr, c0s, row, grow, live, bias, zo, ho, g.wo, ab, o);
                        else
                            pp_epilogue<BN, false, false>(taddr, c0s, row, grow, live, bias, zo, ho, g.wo, ab, o);
                    }
                    if (last) {
                        // the layer's MMAs have completed, so the activation tile is free: it
                        // carries the partial sums of column groups 1-3 to group 0's threads
                        float4 *part = reinterpret_cast<float4 *>(ab);
                        if (cg > 0) part[cg * 128 + row] = make_float4(o[0], o[1], o[2], 0.f);
                        mb_arrive(outBar + b);
                        if (cg == 0) {
                            if (!mb_wait_or_fail(outBar + b, no[b] & 1, fail)) {
                                ok = false;
                            } else if (live) {
#pragma unroll
                                for (int c = 1; c < 4; ++c) {
                                    const float4 pv = part[c * 128 + row];
                                    o[0] += pv.x;
                                    o[1] += pv.y;
                                    o[2] += pv.z;
                                }
#pragma unroll
                                for (int jj = 0; jj < kOutCols; ++jj) g.y[grow * kOutCols + jj] = o[jj] + g.bo[jj];
                            }
                        }
                        ++no[b];
                    }
                    // the activation writes (and reads) before the tensor cores' and the
                    // copies' next use of the tile, the accumulator reads before the next MMAs
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    tc_fence_before();
                    mb_arrive(accFree + b);
                    ++n[b];
                }
            }
        }
        if (!ok) {
            *fail = 1;
            set_err(g.err, 2);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tm_dealloc(tmem, 2 * BN);
    }
}

}  // namespace

namespace {

// ------------------------------------------------------------------ CUDA-core kernels

constexpr int kMaxIn = 128;  // normalised inputs per row, at most
constexpr int kOut = 3;      // displacement components

// first layer's input width: inputs * (1 + 2 bands) rounded up to a multiple of 128
int feature_width(int nin, int bands) {
    const int f = nin * (1 + 2 * bands);
    return std::max(128, (f + 127) / 128 * 128);
}

// Fourier features of the rows idx[b] (or b when idx is null) of `in` [n][nin]:
// u_i, then sin(2^f pi u_i), cos(2^f pi u_i) for f < bands (f-major), zero padding to K0.
// One warp per row: lane j takes inputs j, j + 32, ..., and for each of them its bands,
// one hardware sine / cosine pair per band (the features are rounded to BF16, far coarser
// than the approximation); for a fixed band the lanes' (sin, cos) pairs are consecutive
// 4-byte words of the row. Then the padding.
__global__ void k_features(const float *__restrict__ in, const int *__restrict__ idx, int rows,
                           int nin, int bands, int K0, bf16 *__restrict__ X) {
    const int b = blockIdx.x * blockDim.y + threadIdx.y;
    if (b >= rows) return;
    const int src = idx ? idx[b] : b;
    bf16 *x = X + (long long)b * K0;
    const bool pairs = (nin & 1) == 0;  // (sin, cos) pairs start on 4-byte boundaries
    for (int i = threadIdx.x; i < nin; i += blockDim.x) {
        const float v = in[(long long)src * nin + i];
        x[i] = __float2bfloat16_rn(v);
        for (int f = 0; f < bands; ++f) {
            float sv, cv;
            __sincosf((float)(1 << f) * 3.14159265358979f * v, &sv, &cv);
            const int c = nin + 2 * (nin * f + i);
            if (pairs) {
                *reinterpret_cast<__nv_bfloat162 *>(x + c) = __floats2bfloat162_rn(sv, cv);
            } else {
                x[c] = __float2bfloat16_rn(sv);
                x[c + 1] = __float2bfloat16_rn(cv);
            }
        }
    }
    for (int c = nin * (1 + 2 * bands) + threadIdx.x; c < K0; c += blockDim.x) x[c] = __float2bfloat16_rn(0.f);
}

// out[c][r] = in[r][c] for a [R][C] BF16 matrix: 64 x 64 tiles through shared memory, 256
// threads; rows are read and written as BF16 pairs (4-byte words, 128 bytes per warp), and the
// tile's row pitch of 65 elements keeps both the pair writes and the column reads free of
// bank conflicts. Odd R or C fall back to single elements at the edges they affect.
constexpr int kTrTile = 64, kTrPitch = kTrTile + 1;
__global__ void __launch_bounds__(256) k_transpose(const bf16 *__restrict__ in, int R, int C,
                                                   bf16 *__restrict__ out) {
    __shared__ bf16 t[kTrTile * kTrPitch];
    const int c0 = blockIdx.x * kTrTile, r0 = blockIdx.y * kTrTile;
    const bool evenC = (C & 1) == 0, evenR = (R & 1) == 0;
    for (int k = threadIdx.x; k < kTrTile * (kTrTile / 2); k += blockDim.x) {
        const int r = k >> 5, w = k & 31;
        const int gr = r0 + r, gc = c0 + 2 * w;
        bf16 a = __float2bfloat16_rn(0.f), b = a;
        if (gr < R) {
            const bf16 *src = in + (long long)gr * C + gc;
            if (evenC && gc + 1 < C) {
                const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162 *>(src);
                a = v.x;
                b = v.y;
            } else {
                if (gc < C) a = src[0];
                if (gc + 1 < C) b = src[1];
            }
        }
        t[r * kTrPitch + 2 * w] = a;
        t[r * kTrPitch + 2 * w + 1] = b;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kTrTile * (kTrTile / 2); k += blockDim.x) {
        const int c = k >> 5, w = k & 31;
        const int orow = c0 + c, ocol = r0 + 2 * w;
        if (orow >= C || ocol >= R) continue;
        __nv_bfloat162 v;
        v.x = t[(2 * w) * kTrPitch + c];
        v.y = t[(2 * w + 1) * kTrPitch + c];
        bf16 *dst = out + (long long)orow * R + ocol;
        if (evenR && ocol + 1 < R) {
            *reinterpret_cast<__nv_bfloat162 *>(dst) = v;
        } else {
            dst[0] = v.x;
            if (ocol + 1 < R) dst[1] = v.y;
        }
    }
}

// out[e] = sum over s of part[s * count + e]: a block of 32 x 8 threads per 32 elements, the
// 8 thread rows summing every 8th split (their loads of 32 consecutive elements coalesced),
// then the 8 partial sums added in order
__global__ void __launch_bounds__(256) k_sum_splits(const float *__restrict__ part, int splits,
                                                    long long count, float *__restrict__ out) {
    __shared__ float red[8][33];
    const long long e = (long long)blockIdx.x * 32 + threadIdx.x;
    float acc = 0.f;
    if (e < count) {
#pragma unroll 4
        for (int s = threadIdx.y; s < splits; s += 8) acc += part[s * count + e];
    }
    red[threadIdx.y][threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.y == 0 && e < count) {
        float t = 0.f;
#pragma unroll
        for (int j = 0; j < 8; ++j) t += red[j][threadIdx.x];
        out[e] = t;
    }
}
inline dim3 sum_splits_grid(long long count) { return dim3((unsigned)((count + 31) / 32)); }

// Column sums of a BF16 [rows][N] matrix (N even) over row chunks of kChunk: part[chunk][N].
// A block of 32 x 8 threads per 64 columns: each thread takes a column pair (one 4-byte load
// per row, 128 bytes per warp) and every 8th row of the chunk; the 8 partial sums are added
// in order.
constexpr int kChunk = 256;
__global__ void __launch_bounds__(256) k_colsum_bf16(const bf16 *__restrict__ A, int rows, int N,
                                                     float *__restrict__ part) {
    __shared__ float red[8][65];
    const int c = blockIdx.x * 64 + 2 * threadIdx.x;
    const int r0 = blockIdx.y * kChunk, r1 = min(rows, r0 + kChunk);
    float a0 = 0.f, a1 = 0.f;
    if (c < N) {
#pragma unroll 4
        for (int r = r0 + threadIdx.y; r < r1; r += 8) {
            const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(A + (long long)r * N + c));
            a0 += v.x;
            a1 += v.y;
        }
    }
    red[threadIdx.y][2 * threadIdx.x] = a0;
    red[threadIdx.y][2 * threadIdx.x + 1] = a1;
    __syncthreads();
    for (int q = threadIdx.y * 32 + threadIdx.x; q < 64; q += 256) {
        if (blockIdx.x * 64 + q >= N) continue;
        float t = 0.f;
#pragma unroll
        for (int j = 0; j < 8; ++j) t += red[j][q];
        part[(long long)blockIdx.y * N + blockIdx.x * 64 + q] = t;
    }
}

// MSE over the batch: dY = 2 (Y - T) / (rows * 3); per-block partial losses
__global__ void k_loss(const float *__restrict__ Y, const float *__restrict__ targets,
                       const int *__restrict__ idx, int rows, float *__restrict__ dY,
                       float *__restrict__ lossPart) {
    __shared__ float red[256];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (b < rows) {
        const int src = idx ? idx[b] : b;
        const float inv = 2.0f / (float)(rows * kOut);
#pragma unroll
        for (int j = 0; j < kOut; ++j) {
            const float d = Y[(long long)b * kOut + j] - targets[(long long)src * kOut + j];
            dY[(long long)b * kOut + j] = d * inv;
            l += d * d;
        }
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) lossPart[blockIdx.x] = red[0];
}

// Output layer backward into the last hidden layer:
// dZ[b][k] = (sum_j dY[b][j] Wo[j][k]) * SiLU'(Z[b][k]), stored BF16
__global__ void k_out_bwd(const float *__restrict__ dY, const float *__restrict__ Wo,
                          const float *__restrict__ Z, int rows, int W, bf16 *__restrict__ dZ) {
    // one CTA row per batch row (blockIdx.x), its columns over blockIdx.y
    const int b = blockIdx.x, k = blockIdx.y * blockDim.x + threadIdx.x;
    if (b >= rows || k >= W) return;
    const long long e = (long long)b * W + k;
    float g = 0.f;
#pragma unroll
    for (int j = 0; j < kOut; ++j) g += dY[(long long)b * kOut + j] * Wo[j * W + k];
    dZ[e] = __float2bfloat16_rn(g * silu_grad(Z[e]));
}

// Output layer weight / bias gradients over row chunks of kChunk:
// part[chunk][j][W + 1]: column k < W holds sum dY[b][j] H[b][k], column W sum dY[b][j].
// A block of 32 x 8 threads per 32 columns: each thread takes every 8th row of the chunk for
// its column; the 8 partial sums are added in order.
__global__ void __launch_bounds__(256) k_out_grad(const float *__restrict__ dY, const bf16 *__restrict__ H,
                                                  int rows, int W, float *__restrict__ part) {
    __shared__ float red[kOut][8][33];
    const int k = blockIdx.x * 32 + threadIdx.x;  // 0..W (W = bias)
    const int r0 = blockIdx.y * kChunk, r1 = min(rows, r0 + kChunk);
    float acc[kOut] = {0.f, 0.f, 0.f};
    if (k <= W) {
#pragma unroll 4
        for (int b = r0 + threadIdx.y; b < r1; b += 8) {
            const float h = (k < W) ? __bfloat162float(H[(long long)b * W + k]) : 1.f;
#pragma unroll
            for (int j = 0; j < kOut; ++j) acc[j] += dY[(long long)b * kOut + j] * h;
        }
    }
#pragma unroll
    for (int j = 0; j < kOut; ++j) red[j][threadIdx.y][threadIdx.x] = acc[j];
    __syncthreads();
    if (threadIdx.y < kOut && k <= W) {
        const int j = threadIdx.y;
        float t = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) t += red[j][q][threadIdx.x];
        part[((long long)blockIdx.y * kOut + j) * (W + 1) + k] = t;
    }
}

// Adam on a flat FP32 parameter array (t = step count after this update)
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, long long n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float gr = g[e];
    const float mm = b1 * m[e] + (1.f - b1) * gr;
    const float vv = b2 * v[e] + (1.f - b2) * gr * gr;
    m[e] = mm;
    v[e] = vv;
    p[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

// BF16 copies of a [R][C] FP32 weight: as is and transposed
__global__ void k_weight_bf16(const float *__restrict__ w, int R, int C, bf16 *__restrict__ wb,
                              bf16 *__restrict__ wbT) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)R * C) return;
    const int r = (int)(e / C), c = (int)(e % C);
    const bf16 h = __float2bfloat16_rn(w[e]);
    wb[e] = h;
    wbT[(long long)c * R + r] = h;
}

// Batch rows drawn uniformly (with replacement) from n samples: a splitmix64 hash of
// (seed, step, row)
__global__ void k_sample(unsigned long long seed, unsigned long long step, int rows, long long n,
                         int *__restrict__ idx) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= rows) return;
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (step * 0x100000001B3ull + (unsigned long long)b + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    idx[b] = (int)(z % (unsigned long long)n);
}

}  // namespace

// ------------------------------------------------------------------ host side

struct hidem_surrogate {
    hidem_surrogate_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int *dErr = nullptr;
    int L = 4, W = 256, B = 16384, splits = 64;
    int nin = 5, K0 = 128;                       // inputs per row, first layer's K
    long long np = 0;                            // parameter count
    std::vector<long long> offW, offB;           // hidden layer weight / bias offsets in P
    long long offWo = 0, offBo = 0;
    std::vector<int> Kl;                         // input width of hidden layer l
    float *P = nullptr, *G = nullptr, *Mm = nullptr, *Vv = nullptr;
    std::vector<bf16 *> Wb, WbT;                 // BF16 weights [W][K_l] and [K_l][W]
    bf16 *X0 = nullptr;                          // [B][K0]
    std::vector<float *> Z;                      // [B][W] pre-activations
    std::vector<bf16 *> H;                       // [B][W] activations
    float *Y = nullptr, *dY = nullptr;           // [B][3]
    bf16 *dZa = nullptr, *dZb = nullptr;         // [B][W]
    bf16 *dZT = nullptr, *inT = nullptr;         // [W][B], [max K][B]
    float *part = nullptr;                       // split / chunk partials
    long long partCap = 0;
    float *lossPart = nullptr, *lossHost = nullptr;
    int *idx = nullptr;
    float *dataIn = nullptr, *dataT = nullptr;   // training set [n][nin], [n][3]
    long long nData = 0;
    float *scratchIn = nullptr, *scratchT = nullptr;  // caller rows for predict / gradients
    int PB = 0;                                   // rows per predict chunk
    float *predIn = nullptr, *predY = nullptr;    // predict chunk: inputs [PB][nin], outputs [PB][3]
    bf16 *predX = nullptr;                        // predict chunk features [PB][K0]
    long long steps = 0;
    int smCount = 0;                              // SMs of the device (persistent grids)
    int forwardKind = HIDEM_SURROGATE_FORWARD_AUTO;
};

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// BF16 [rows][cols] row-major, boxes of 64 columns x boxRows rows, 128-byte swizzle
bool make_map(CUtensorMap *m, const void *base, long long rows, long long cols, int boxRows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * sizeof(bf16)};
    cuuint32_t box[2] = {64u, (cuuint32_t)boxRows};
    cuuint32_t es[2] = {1u, 1u};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// FP32 [rows][cols] row-major, boxes of 64 columns x boxRows rows, no swizzle
bool make_map_f32(CUtensorMap *m, const void *base, long long rows, long long cols, int boxRows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * sizeof(float)};
    cuuint32_t box[2] = {64u, (cuuint32_t)boxRows};
    cuuint32_t es[2] = {1u, 1u};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

hidem_status sfail(hidem_surrogate *s, hidem_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (s) s->err = buf;
    return st;
}

#define SCK(call)                                                                            \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return sfail(s, HIDEM_ERR_CUDA, "%s failed: %s (%s:%d)", #call,                  \
                         cudaGetErrorString(e_), __FILE__, __LINE__);                        \
    } while (0)
#define STRY(expr)                           \
    do {                                     \
        hidem_status s_ = (expr);            \
        if (s_ != HIDEM_OK) return s_;       \
    } while (0)

template <int BN, int EPI>
hidem_status gemm(hidem_surrogate *s, const bf16 *A, int M, int K, const bf16 *Bm, int splits,
                  GemmArgs g) {
    // per-device attribute, set once on each device (a repeated set is harmless)
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load() & bit)) {
        cudaFuncSetAttribute(k_umma_gemm<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gemm_smem_bytes<BN>());
        configured.fetch_or(bit);
    }
    if (M % 128 || K % 64 || (K / 64) % splits)
        return sfail(s, HIDEM_ERR_ARG, "GEMM shape %d x %d x %d (splits %d) is not tile-aligned", M, BN, K, splits);
    CUtensorMap ta, tb, tz;
    if (!make_map(&ta, A, M, K, 128) || !make_map(&tb, Bm, BN, K, BN))
        return sfail(s, HIDEM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    if (EPI == EPI_SILU_GRAD) {
        if (g.ldo != BN || !make_map_f32(&tz, g.zIn, M, BN, 128))
            return sfail(s, HIDEM_ERR_CUDA, "cuTensorMapEncodeTiled failed (pre-activations)");
    } else {
        tz = ta;  // not read
    }
    g.M = M;
    g.N = BN;
    g.K = K;
    g.kTiles = K / 64 / splits;
    g.err = s->dErr;
    k_umma_gemm<BN, EPI><<<dim3(M / 128, splits), kGemmThreads, gemm_smem_bytes<BN>(), s->stream>>>(ta, tb, tz, g);
    SCK(cudaGetLastError());
    return HIDEM_OK;
}

template <int EPI>
hidem_status gemm_n(hidem_surrogate *s, int N, const bf16 *A, int M, int K, const bf16 *Bm,
                    int splits, const GemmArgs &g) {
    if (N == 256) return gemm<256, EPI>(s, A, M, K, Bm, splits, g);
    if (N == 128) return gemm<128, EPI>(s, A, M, K, Bm, splits, g);
    return sfail(s, HIDEM_ERR_ARG, "GEMM width %d (128 or 256)", N);
}

// the partial buffer is sized at creation for the largest batch; a call that would need
// more is a bug, reported rather than reallocating under queued work
hidem_status ensure_part(hidem_surrogate *s, long long count) {
    if (s->partCap >= count) return HIDEM_OK;
    return sfail(s, HIDEM_ERR_CAPACITY, "partial buffer too small (%lld < %lld)", s->partCap, count);
}

hidem_status refresh_bf16(hidem_surrogate *s) {
    for (int l = 0; l < s->L; ++l) {
        const long long n = (long long)s->W * s->Kl[l];
        k_weight_bf16<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(s->P + s->offW[l], s->W, s->Kl[l], s->Wb[l], s->WbT[l]);
    }
    SCK(cudaGetLastError());
    return HIDEM_OK;
}

// forward over `rows` rows whose features are in X0 (keepZ: store pre-activations)
// The whole forward pass over `rows` rows of features X (a multiple of 128) in one fused
// launch (k_mlp_fwd); keepZ: the training pass, which keeps every layer's pre-activations
// and activations for the backward pass.
template <int BN>
hidem_status mlp_forward_t(hidem_surrogate *s, const bf16 *X, int rows, float *Y, bool keepZ) {
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load() & bit)) {
        cudaFuncSetAttribute(k_mlp_fwd<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_smem_bytes<BN>());
        configured.fetch_or(bit);
    }
    if (rows % 128) return sfail(s, HIDEM_ERR_ARG, "forward rows %d not a multiple of 128", rows);
    MlpMaps maps;
    std::memset(&maps, 0, sizeof maps);
    if (!make_map(&maps.x, X, rows, s->K0, 128)) return sfail(s, HIDEM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    MlpArgs a{};
    a.layers = s->L;
    a.k0 = s->K0;
    for (int l = 0; l < s->L; ++l) {
        if (!make_map(&maps.w[l], s->Wb[l], BN, s->Kl[l], BN))
            return sfail(s, HIDEM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
        a.bias[l] = s->P + s->offB[l];
        a.z[l] = keepZ ? s->Z[l] : nullptr;
        a.h[l] = keepZ ? s->H[l] : nullptr;
    }
    a.wo = s->P + s->offWo;
    a.bo = s->P + s->offBo;
    a.y = Y;
    a.err = s->dErr;
    k_mlp_fwd<BN><<<rows / 128, kMlpThreads, mlp_smem_bytes<BN>(), s->stream>>>(maps, a);
    SCK(cudaGetLastError());
    return HIDEM_OK;
}

// The same pass as the persistent ping-pong kernel (k_mlp_pp, 256-wide networks): one CTA
// per SM at most, each taking pairs of 128-row blocks.
hidem_status mlp_forward_pp(hidem_surrogate *s, const bf16 *X, int rows, float *Y, bool keepZ) {
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load() & bit)) {
        cudaFuncSetAttribute(k_mlp_pp<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pp_smem_bytes());
        configured.fetch_or(bit);
    }
    if (rows % 128) return sfail(s, HIDEM_ERR_ARG, "forward rows %d not a multiple of 128", rows);
    if (rows == 0) return HIDEM_OK;
    MlpMaps maps;
    std::memset(&maps, 0, sizeof maps);
    if (!make_map(&maps.x, X, rows, s->K0, 128)) return sfail(s, HIDEM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    MlpArgs a{};
    a.layers = s->L;
    a.k0 = s->K0;
    for (int l = 0; l < s->L; ++l) {
        if (!make_map(&maps.w[l], s->Wb[l], 256, s->Kl[l], 256))
            return sfail(s, HIDEM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
        a.bias[l] = s->P + s->offB[l];
        a.z[l] = keepZ ? s->Z[l] : nullptr;
        a.h[l] = keepZ ? s->H[l] : nullptr;
    }
    a.wo = s->P + s->offWo;
    a.bo = s->P + s->offBo;
    a.y = Y;
    a.err = s->dErr;
    const int pairs = (rows / 128 + 1) / 2;
    const int grid = std::min(pairs, std::max(1, s->smCount));
    k_mlp_pp<256><<<grid, kPPThreads, pp_smem_bytes(), s->stream>>>(maps, a, rows);
    SCK(cudaGetLastError());
    return HIDEM_OK;
}

hidem_status mlp_forward(hidem_surrogate *s, const bf16 *X, int rows, float *Y, bool keepZ) {
    if (s->W == 256 && s->forwardKind != HIDEM_SURROGATE_FORWARD_BLOCK)
        return mlp_forward_pp(s, X, rows, Y, keepZ);
    return s->W == 256 ? mlp_forward_t<256>(s, X, rows, Y, keepZ) : mlp_forward_t<128>(s, X, rows, Y, keepZ);
}

hidem_status forward(hidem_surrogate *s, int rows, bool keepZ) {
    return mlp_forward(s, s->X0, rows, s->Y, keepZ);
}

// loss and all gradients into G for the rows of X0 (targets[idx[b]] or targets[b])
hidem_status backward(hidem_surrogate *s, int rows, const float *targets, const int *idx) {
    const int W = s->W, L = s->L;
    const int nb = (rows + 255) / 256;
    k_loss<<<nb, 256, 0, s->stream>>>(s->Y, targets, idx, rows, s->dY, s->lossPart);
    // output layer
    const int chunks = (rows + kChunk - 1) / kChunk;
    STRY(ensure_part(s, (long long)(chunks + 1) * kOut * (W + 1)));
    k_out_grad<<<dim3((W + 1 + 31) / 32, chunks), dim3(32, 8), 0, s->stream>>>(s->dY, s->H[L - 1], rows, W, s->part);
    // sum the chunk partials into a [3][W + 1] block, then split weights and biases
    float *outBlock = s->part + (long long)chunks * kOut * (W + 1);
    k_sum_splits<<<sum_splits_grid((long long)kOut * (W + 1)), dim3(32, 8), 0, s->stream>>>(s->part, chunks, (long long)kOut * (W + 1), outBlock);
    for (int j = 0; j < kOut; ++j) {
        SCK(cudaMemcpyAsync(s->G + s->offWo + (long long)j * W, outBlock + (long long)j * (W + 1),
                            sizeof(float) * W, cudaMemcpyDeviceToDevice, s->stream));
        SCK(cudaMemcpyAsync(s->G + s->offBo + j, outBlock + (long long)j * (W + 1) + W, sizeof(float),
                            cudaMemcpyDeviceToDevice, s->stream));
    }
    bf16 *dZ = s->dZa, *dZn = s->dZb;
    k_out_bwd<<<dim3((unsigned)rows, (unsigned)((W + 255) / 256)), 256, 0, s->stream>>>(s->dY, s->P + s->offWo, s->Z[L - 1], rows, W, dZ);
    SCK(cudaGetLastError());
    // hidden layers, last to first
    for (int l = L - 1; l >= 0; --l) {
        const int K = s->Kl[l];
        const bf16 *in = l == 0 ? s->X0 : s->H[l - 1];
        // dW_l = dZ^T * in: both operands transposed to K-major [.][rows], split over rows
        k_transpose<<<dim3((W + kTrTile - 1) / kTrTile, (rows + kTrTile - 1) / kTrTile), 256, 0, s->stream>>>(dZ, rows, W, s->dZT);
        k_transpose<<<dim3((K + kTrTile - 1) / kTrTile, (rows + kTrTile - 1) / kTrTile), 256, 0, s->stream>>>(in, rows, K, s->inT);
        int splits = s->splits;
        while (splits > 1 && ((rows / 64) % splits)) splits >>= 1;
        STRY(ensure_part(s, (long long)splits * W * K));
        // columns of dW in tiles of 256 (then 128): rows n0.. of the K-major input
        for (int n0 = 0; n0 < K;) {
            const int bn = K - n0 >= 256 ? 256 : 128;
            GemmArgs g{};
            g.outF = s->part + n0;
            g.splitStride = (long long)W * K;
            g.ldo = K;
            STRY(gemm_n<EPI_F32>(s, bn, s->dZT, W, rows, s->inT + (long long)n0 * rows, splits, g));
            n0 += bn;
        }
        k_sum_splits<<<sum_splits_grid((long long)W * K), dim3(32, 8), 0, s->stream>>>(s->part, splits, (long long)W * K, s->G + s->offW[l]);
        // db_l = column sums of dZ
        STRY(ensure_part(s, (long long)chunks * W + W));
        k_colsum_bf16<<<dim3((W + 63) / 64, chunks), dim3(32, 8), 0, s->stream>>>(dZ, rows, W, s->part);
        k_sum_splits<<<sum_splits_grid(W), dim3(32, 8), 0, s->stream>>>(s->part, chunks, W, s->G + s->offB[l]);
        if (l > 0) {
            // dZ_{l-1} = (dZ_l * W_l) . SiLU'(Z_{l-1}); B operand W_l^T is [K_l][W]
            GemmArgs gd{};
            gd.outH = dZn;
            gd.zIn = s->Z[l - 1];
            gd.ldo = K;
            STRY(gemm_n<EPI_SILU_GRAD>(s, K, dZ, rows, W, s->WbT[l], 1, gd));
            std::swap(dZ, dZn);
        }
    }
    SCK(cudaGetLastError());
    return HIDEM_OK;
}

hidem_status read_loss(hidem_surrogate *s, int rows, double *loss) {
    const int nb = (rows + 255) / 256;
    SCK(cudaMemcpyAsync(s->lossHost, s->lossPart, sizeof(float) * nb, cudaMemcpyDeviceToHost, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    double t = 0;
    for (int i = 0; i < nb; ++i) t += s->lossHost[i];
    if (loss) *loss = t / ((double)rows * kOut);
    return HIDEM_OK;
}

hidem_status check_err(hidem_surrogate *s) {
    int flag = 0;
    SCK(cudaMemcpyAsync(&flag, s->dErr, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    if (flag) {
        SCK(cudaMemsetAsync(s->dErr, 0, sizeof(int), s->stream));
        return sfail(s, HIDEM_ERR_DEVICE, "tensor-core GEMM: %s",
                     flag == 1   ? "tile copies did not complete in time"
                     : flag == 2 ? "accumulator did not complete in time"
                                 : "pre-activation copies did not complete in time");
    }
    return HIDEM_OK;
}

}  // namespace

extern "C" {

void hidem_surrogate_config_default(hidem_surrogate_config *c) {
    if (!c) return;
    c->hidden_layers = 4;
    c->width = 256;
    c->fourier_bands = 8;
    c->batch = 16384;
    c->learning_rate = 1e-3;
    c->seed = 1;
    c->inputs = 5;
    c->cosine_decay = 0;
}

void hidem_surrogate_destroy(hidem_surrogate *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    void *bufs[] = {s->P, s->G, s->Mm, s->Vv, s->X0, s->Y, s->dY, s->dZa, s->dZb, s->dZT, s->inT,
                    s->part, s->lossPart, s->idx, s->dataIn, s->dataT, s->scratchIn, s->scratchT, s->dErr,
                    s->predIn, s->predY, s->predX};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (auto *p : s->Wb) if (p) cudaFree(p);
    for (auto *p : s->WbT) if (p) cudaFree(p);
    for (auto *p : s->Z) if (p) cudaFree(p);
    for (auto *p : s->H) if (p) cudaFree(p);
    if (s->lossHost) cudaFreeHost(s->lossHost);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

hidem_status hidem_surrogate_create(const hidem_surrogate_config *c, int device, hidem_surrogate **out) {
    std::string &err = hidem::g_nocontext_error;
    err.clear();
    if (!c || !out) {
        err = "config or out is NULL";
        return HIDEM_ERR_ARG;
    }
    *out = nullptr;
    if (c->hidden_layers < 1 || c->hidden_layers > kMlpMaxLayers || (c->width != 128 && c->width != 256) ||
        c->fourier_bands < 1 || c->fourier_bands > 12 || c->batch < 128 || c->batch % 128 ||
        c->batch > (1 << 20) || !(c->learning_rate > 0) || c->inputs < 1 || c->inputs > kMaxIn ||
        (c->cosine_decay != 0 && c->cosine_decay != 1)) {
        err = "surrogate config out of range (layers 1..8, width 128 | 256, bands 1..12, batch a "
              "multiple of 128, inputs 1..128, cosine_decay 0 | 1)";
        return HIDEM_ERR_ARG;
    }
    if (!encode_fn()) {
        err = "cuTensorMapEncodeTiled is not available from the driver";
        return HIDEM_ERR_CUDA;
    }
    hidem_surrogate *s = new hidem_surrogate();
    s->cfg = *c;
    s->device = device;
    s->L = c->hidden_layers;
    s->W = c->width;
    s->B = c->batch;
    s->nin = c->inputs;
    s->K0 = feature_width(c->inputs, c->fourier_bands);
    const int L = s->L, W = s->W, B = s->B, K0 = s->K0;
    long long off = 0;
    for (int l = 0; l < L; ++l) {
        const int K = l == 0 ? K0 : W;
        s->Kl.push_back(K);
        s->offW.push_back(off);
        off += (long long)W * K;
        s->offB.push_back(off);
        off += W;
    }
    s->offWo = off;
    off += (long long)kOut * W;
    s->offBo = off;
    off += kOut;
    s->np = off;
    const int chunks = (B + kChunk - 1) / kChunk;
    long long partNeed = std::max<long long>((long long)(chunks + 1) * kOut * (W + 1), (long long)chunks * W + W);
    partNeed = std::max<long long>(partNeed, (long long)s->splits * W * std::max(W, K0));
    auto fail = [&](cudaError_t e) {
        err = std::string("surrogate setup failed: ") + cudaGetErrorString(e);
        hidem_surrogate_destroy(s);
        return HIDEM_ERR_CUDA;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->smCount, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    auto dm = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    };
    dm((void **)&s->dErr, sizeof(int));
    dm((void **)&s->P, sizeof(float) * s->np);
    dm((void **)&s->G, sizeof(float) * s->np);
    dm((void **)&s->Mm, sizeof(float) * s->np);
    dm((void **)&s->Vv, sizeof(float) * s->np);
    s->Wb.assign(L, nullptr);
    s->WbT.assign(L, nullptr);
    s->Z.assign(L, nullptr);
    s->H.assign(L, nullptr);
    for (int l = 0; l < L; ++l) {
        dm((void **)&s->Wb[l], sizeof(bf16) * W * s->Kl[l]);
        dm((void **)&s->WbT[l], sizeof(bf16) * W * s->Kl[l]);
        dm((void **)&s->Z[l], sizeof(float) * (size_t)B * W);
        dm((void **)&s->H[l], sizeof(bf16) * (size_t)B * W);
    }
    dm((void **)&s->X0, sizeof(bf16) * (size_t)B * K0);
    dm((void **)&s->Y, sizeof(float) * (size_t)B * kOut);
    dm((void **)&s->dY, sizeof(float) * (size_t)B * kOut);
    dm((void **)&s->dZa, sizeof(bf16) * (size_t)B * W);
    dm((void **)&s->dZb, sizeof(bf16) * (size_t)B * W);
    dm((void **)&s->dZT, sizeof(bf16) * (size_t)B * W);
    dm((void **)&s->inT, sizeof(bf16) * (size_t)B * std::max(W, K0));
    dm((void **)&s->part, sizeof(float) * partNeed);
    s->partCap = partNeed;
    dm((void **)&s->lossPart, sizeof(float) * ((B + 255) / 256));
    dm((void **)&s->idx, sizeof(int) * B);
    dm((void **)&s->scratchIn, sizeof(float) * (size_t)B * s->nin);
    dm((void **)&s->scratchT, sizeof(float) * (size_t)B * kOut);
    // rows per predict chunk: with the persistent forward pass, 1,024 block pairs per chunk
    // keep the last round of pairs over the SMs a small share of a chunk
    s->PB = std::max(B, 262144);
    dm((void **)&s->predIn, sizeof(float) * (size_t)s->PB * s->nin);
    dm((void **)&s->predY, sizeof(float) * (size_t)s->PB * kOut);
    dm((void **)&s->predX, sizeof(bf16) * (size_t)s->PB * K0);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&s->lossHost, sizeof(float) * ((B + 255) / 256));
    if (e == cudaSuccess) e = cudaMemsetAsync(s->dErr, 0, sizeof(int), s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->Mm, 0, sizeof(float) * s->np, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->Vv, 0, sizeof(float) * s->np, s->stream);
    if (e != cudaSuccess) return fail(e);
    // initial weights: uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) from a seeded 64-bit
    // generator (splitmix64), biases zero
    std::vector<float> p(s->np, 0.f);
    unsigned long long st = c->seed * 0x9E3779B97F4A7C15ull + 12345;
    auto next = [&]() {
        unsigned long long z = (st += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < L; ++l) {
        const double a = 1.0 / std::sqrt((double)s->Kl[l]);
        for (long long q = 0; q < (long long)W * s->Kl[l]; ++q) p[s->offW[l] + q] = (float)((2 * next() - 1) * a);
    }
    const double ao = 1.0 / std::sqrt((double)W);
    for (long long q = 0; q < (long long)kOut * W; ++q) p[s->offWo + q] = (float)((2 * next() - 1) * ao);
    e = cudaMemcpy(s->P, p.data(), sizeof(float) * s->np, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(e);
    if (refresh_bf16(s) != HIDEM_OK || cudaStreamSynchronize(s->stream) != cudaSuccess) {
        err = s->err;
        hidem_surrogate_destroy(s);
        return HIDEM_ERR_CUDA;
    }
    *out = s;
    return HIDEM_OK;
}

const char *hidem_surrogate_last_error(const hidem_surrogate *s) { return s ? s->err.c_str() : "null surrogate"; }

int64_t hidem_surrogate_num_params(const hidem_surrogate *s) { return s ? s->np : 0; }

hidem_status hidem_surrogate_get_params(hidem_surrogate *s, float *out) {
    if (!s || !out) return HIDEM_ERR_ARG;
    SCK(cudaSetDevice(s->device));
    SCK(cudaMemcpyAsync(out, s->P, sizeof(float) * s->np, cudaMemcpyDeviceToHost, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    return HIDEM_OK;
}

hidem_status hidem_surrogate_set_params(hidem_surrogate *s, const float *in) {
    if (!s || !in) return HIDEM_ERR_ARG;
    SCK(cudaSetDevice(s->device));
    SCK(cudaMemcpyAsync(s->P, in, sizeof(float) * s->np, cudaMemcpyHostToDevice, s->stream));
    STRY(refresh_bf16(s));
    SCK(cudaStreamSynchronize(s->stream));
    return HIDEM_OK;
}

hidem_status hidem_surrogate_set_data(hidem_surrogate *s, const float *inputs, const float *targets,
                                      int64_t n) {
    if (!s) return HIDEM_ERR_ARG;
    if (!inputs || !targets || n <= 0 || n > 0x7fffffff) return sfail(s, HIDEM_ERR_ARG, "bad training set");
    SCK(cudaSetDevice(s->device));
    if (s->dataIn) cudaFree(s->dataIn);
    if (s->dataT) cudaFree(s->dataT);
    s->dataIn = s->dataT = nullptr;
    s->nData = 0;
    SCK(cudaMalloc((void **)&s->dataIn, sizeof(float) * s->nin * (size_t)n));
    SCK(cudaMalloc((void **)&s->dataT, sizeof(float) * kOut * (size_t)n));
    SCK(cudaMemcpyAsync(s->dataIn, inputs, sizeof(float) * s->nin * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    SCK(cudaMemcpyAsync(s->dataT, targets, sizeof(float) * kOut * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    s->nData = n;
    return HIDEM_OK;
}

hidem_status hidem_surrogate_train(hidem_surrogate *s, int32_t steps, double *loss) {
    if (!s) return HIDEM_ERR_ARG;
    if (steps < 0) return sfail(s, HIDEM_ERR_ARG, "negative step count");
    if (!s->nData) return sfail(s, HIDEM_ERR_STATE, "no training set");
    SCK(cudaSetDevice(s->device));
    const int B = s->B;
    for (int it = 0; it < steps; ++it) {
        k_sample<<<(B + 255) / 256, 256, 0, s->stream>>>(s->cfg.seed, (unsigned long long)s->steps, B, s->nData, s->idx);
        k_features<<<(B + 7) / 8, dim3(32, 8), 0, s->stream>>>(s->dataIn, s->idx, B, s->nin, s->cfg.fourier_bands, s->K0, s->X0);
        STRY(forward(s, B, true));
        STRY(backward(s, B, s->dataT, s->idx));
        s->steps += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)s->steps), c2 = 1.f - std::pow(b2, (float)s->steps);
        double lr = s->cfg.learning_rate;
        if (s->cfg.cosine_decay) lr *= 0.5 * (1.0 + std::cos(3.14159265358979 * it / (double)steps));
        k_adam<<<(unsigned)((s->np + 255) / 256), 256, 0, s->stream>>>(s->P, s->G, s->Mm, s->Vv, s->np,
                                                                      (float)lr, b1, b2, 1e-8f, c1, c2);
        STRY(refresh_bf16(s));
    }
    if (steps > 0 && loss) STRY(read_loss(s, B, loss));
    return check_err(s);
}

hidem_status hidem_surrogate_predict(hidem_surrogate *s, const float *inputs, int64_t n, float *out) {
    if (!s) return HIDEM_ERR_ARG;
    if (!inputs || !out || n < 0) return sfail(s, HIDEM_ERR_ARG, "bad arguments");
    SCK(cudaSetDevice(s->device));
    const int PB = s->PB;
    for (int64_t r0 = 0; r0 < n; r0 += PB) {
        const int rows = (int)std::min<int64_t>(PB, n - r0);
        const int padded = (rows + 127) / 128 * 128;
        if (padded > rows) SCK(cudaMemsetAsync(s->predIn, 0, sizeof(float) * s->nin * padded, s->stream));
        SCK(cudaMemcpyAsync(s->predIn, inputs + r0 * s->nin, sizeof(float) * s->nin * rows, cudaMemcpyHostToDevice, s->stream));
        k_features<<<(padded + 7) / 8, dim3(32, 8), 0, s->stream>>>(s->predIn, nullptr, padded, s->nin, s->cfg.fourier_bands, s->K0, s->predX);
        STRY(mlp_forward(s, s->predX, padded, s->predY, false));
        SCK(cudaMemcpyAsync(out + r0 * kOut, s->predY, sizeof(float) * kOut * rows, cudaMemcpyDeviceToHost, s->stream));
    }
    SCK(cudaStreamSynchronize(s->stream));
    return check_err(s);
}

hidem_status hidem_surrogate_predict_device(hidem_surrogate *s, const float *inputs, int64_t n, float *out) {
    if (!s) return HIDEM_ERR_ARG;
    if (!inputs || !out || n < 0) return sfail(s, HIDEM_ERR_ARG, "bad arguments");
    SCK(cudaSetDevice(s->device));
    const int PB = s->PB;
    for (int64_t r0 = 0; r0 < n; r0 += PB) {
        const int rows = (int)std::min<int64_t>(PB, n - r0);
        const int padded = (rows + 127) / 128 * 128;
        const float *in = inputs + r0 * s->nin;
        if (padded > rows) {
            // the ragged last chunk: zero rows up to the next multiple of 128
            SCK(cudaMemsetAsync(s->predIn, 0, sizeof(float) * s->nin * padded, s->stream));
            SCK(cudaMemcpyAsync(s->predIn, in, sizeof(float) * s->nin * rows, cudaMemcpyDeviceToDevice, s->stream));
            in = s->predIn;
        }
        k_features<<<(padded + 7) / 8, dim3(32, 8), 0, s->stream>>>(in, nullptr, padded, s->nin, s->cfg.fourier_bands,
                                                                  s->K0, s->predX);
        float *y = padded > rows ? s->predY : out + r0 * kOut;
        STRY(mlp_forward(s, s->predX, padded, y, false));
        if (padded > rows)
            SCK(cudaMemcpyAsync(out + r0 * kOut, s->predY, sizeof(float) * kOut * rows, cudaMemcpyDeviceToDevice,
                                s->stream));
    }
    SCK(cudaStreamSynchronize(s->stream));
    return check_err(s);
}

void *hidem_surrogate_get_stream(hidem_surrogate *s) { return s ? (void *)s->stream : nullptr; }

hidem_status hidem_surrogate_set_forward(hidem_surrogate *s, int32_t kind) {
    if (!s) return HIDEM_ERR_ARG;
    if (kind != HIDEM_SURROGATE_FORWARD_AUTO && kind != HIDEM_SURROGATE_FORWARD_BLOCK &&
        kind != HIDEM_SURROGATE_FORWARD_PINGPONG)
        return sfail(s, HIDEM_ERR_ARG, "forward kind %d (0 auto, 1 block, 2 ping-pong)", kind);
    if (kind == HIDEM_SURROGATE_FORWARD_PINGPONG && s->W != 256)
        return sfail(s, HIDEM_ERR_ARG, "the ping-pong forward pass needs width 256");
    s->forwardKind = kind;
    return HIDEM_OK;
}

hidem_status hidem_surrogate_gradients(hidem_surrogate *s, const float *inputs, const float *targets,
                                       int64_t n, float *grads, double *loss) {
    if (!s) return HIDEM_ERR_ARG;
    if (!inputs || !targets || !grads || n <= 0 || n % 128 || n > s->B)
        return sfail(s, HIDEM_ERR_ARG, "n must be a positive multiple of 128 up to the batch size");
    SCK(cudaSetDevice(s->device));
    const int rows = (int)n;
    SCK(cudaMemcpyAsync(s->scratchIn, inputs, sizeof(float) * s->nin * rows, cudaMemcpyHostToDevice, s->stream));
    SCK(cudaMemcpyAsync(s->scratchT, targets, sizeof(float) * kOut * rows, cudaMemcpyHostToDevice, s->stream));
    k_features<<<(rows + 7) / 8, dim3(32, 8), 0, s->stream>>>(s->scratchIn, nullptr, rows, s->nin, s->cfg.fourier_bands, s->K0, s->X0);
    STRY(forward(s, rows, true));
    STRY(backward(s, rows, s->scratchT, nullptr));
    STRY(read_loss(s, rows, loss));
    SCK(cudaMemcpyAsync(grads, s->G, sizeof(float) * s->np, cudaMemcpyDeviceToHost, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    return check_err(s);
}

}  // extern "C"
