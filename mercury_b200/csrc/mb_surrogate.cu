// Fitness surrogate for the evolutionary loop: a small 3-D convolutional
// network over voxel genomes, trained on (genome, simulated fitness) pairs
// and used to screen candidates before they are simulated.  There is no
// counterpart in the reference; its C ABI is in include/mercury_b200.h.
//
// Network (channels-last, one genome = 6x6x6 voxels of 5 classes):
//   x0   one-hot classes, 8 channels (classes 0..4, channels 5..7 zero)
//   a1 = relu(conv3x3x3(x0; W1 [32][27*8]) + b1)      same padding
//   a2 = relu(conv3x3x3(a1; W2 [32][27*32]) + b2)
//   a3 = relu(conv3x3x3(a2; W3 [32][27*32]) + b3)
//   h1 = relu(W4 [128][6912] flatten(a3) + b4)        flatten index v*32 + c
//   h2 = relu(W5 [128][128] h1 + b5)
//   y  = W6 [128] . h2 + b6
// Loss: mean squared error against the targets.  Optimiser: Adam on FP32
// master weights; the GEMMs read BF16 copies of weights and activations and
// accumulate in FP32 (mb_sg_kernels.cuh).  Every reduction runs in a fixed
// order, so predictions and gradients are reproducible to the bit.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mercury_b200.h"
#include "mb_sg_kernels.cuh"

namespace mb {
namespace sg {
namespace {

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------
// GEMM

__device__ __forceinline__ void ldsm_x4(uint32_t* r, const void* p) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t* r, const void* p) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}
__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int kLdK = kTileK + 8;   // row of a K-major tile (elements): 80 bytes
constexpr int kLdMN = kTileM + 8;  // row of an MN-major tile: 144 bytes
constexpr int kStage = kTileM * kLdK;  // >= kTileK * kLdMN

__device__ __forceinline__ float epilogue(const GemmArgs& g, int row, int col, float v) {
    if (g.bias) v += g.bias[col];
    if (g.relu) v = fmaxf(v, 0.0f);
    if (g.mask && !(__bfloat162float(g.mask[(size_t)row * g.ldc + col]) > 0.0f)) v = 0.0f;
    return v;
}

__device__ __forceinline__ void store(const GemmArgs& g, int row, int col, float v) {
    const size_t i = (size_t)row * g.ldc + col;
    if (g.c32) g.c32[i] = v;
    if (g.c16) g.c16[i] = __float2bfloat16_rn(v);
}

template <int AV, int BV>
__device__ __forceinline__ void load_stage(const GemmArgs& g, bf16* as, bf16* bs, int m0, int n0, int k0,
                                           int k_end) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int i = tid + t * kGemmThreads;
        if (AV == kDenseMN) {
            const int kr = i >> 3, ch = i & 7, gk = k0 + kr, gm = m0 + ch * 8;
            const bool ok = gk < k_end && gm < g.M;
            cp_async16(as + kr * kLdMN + ch * 8, ok ? g.A + (size_t)gk * g.lda + gm : g.A, ok);
        } else {
            const int row = i >> 2, ch = i & 3, gm = m0 + row, gk = k0 + ch * 8;
            const bf16* src = nullptr;
            if (gm < g.M && gk < k_end)
                src = AV == kIm2col ? im2col_chunk(g.A, g.lda, gm, gk, g.flip_a) : g.A + (size_t)gm * g.lda + gk;
            cp_async16(as + row * kLdK + ch * 8, src ? src : g.A, src != nullptr);
        }
        if (BV == kDenseK) {
            const int row = i >> 2, ch = i & 3, gn = n0 + row, gk = k0 + ch * 8;
            const bool ok = gn < g.N && gk < k_end;
            cp_async16(bs + row * kLdK + ch * 8, ok ? g.B + (size_t)gn * g.ldb + gk : g.B, ok);
        } else {
            const int kr = i >> 3, ch = i & 7, gk = k0 + kr, gn = n0 + ch * 8;
            const bf16* src = nullptr;
            if (gk < k_end && gn < g.N)
                src = BV == kIm2col ? im2col_chunk(g.B, g.ldb, gk, gn, g.flip_b) : g.B + (size_t)gk * g.ldb + gn;
            cp_async16(bs + kr * kLdMN + ch * 8, src ? src : g.B, src != nullptr);
        }
    }
}

template <int AV, int BV>
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(const GemmArgs g) {
    __shared__ __align__(16) bf16 As[2][kStage];
    __shared__ __align__(16) bf16 Bs[2][kStage];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m0 = blockIdx.y * kTileM, n0 = blockIdx.x * kTileN;
    const int k_begin = blockIdx.z * g.k_chunk;
    const int k_end = min(g.K, k_begin + g.k_chunk);
    const int nk = k_end > k_begin ? (k_end - k_begin + kTileK - 1) / kTileK : 0;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0f;

    if (nk > 0) {
        load_stage<AV, BV>(g, As[0], Bs[0], m0, n0, k_begin, k_end);
        cp_async_commit();
    }
    for (int t = 0; t < nk; ++t) {
        cp_async_wait_all();
        __syncthreads();
        if (t + 1 < nk) {
            load_stage<AV, BV>(g, As[(t + 1) & 1], Bs[(t + 1) & 1], m0, n0, k_begin + (t + 1) * kTileK, k_end);
            cp_async_commit();
        }
        const bf16* as = As[t & 1];
        const bf16* bs = Bs[t & 1];
#pragma unroll
        for (int kk = 0; kk < kTileK; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int mb = wm + 16 * i;
                if (AV == kDenseMN)
                    ldsm_x4_t(a[i], as + (kk + (lane & 7) + ((lane >> 4) << 3)) * kLdMN + mb + ((lane >> 3) & 1) * 8);
                else
                    ldsm_x4(a[i], as + (mb + (lane & 15)) * kLdK + kk + (lane >> 4) * 8);
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int nb = wn + 16 * j;
                uint32_t r[4];
                if (BV == kDenseK)
                    ldsm_x4(r, bs + (nb + (lane & 7) + ((lane >> 4) << 3)) * kLdK + kk + ((lane >> 3) & 1) * 8);
                else
                    ldsm_x4_t(r, bs + (kk + (lane & 7) + (((lane >> 3) & 1) << 3)) * kLdMN + nb + ((lane >> 4) << 3));
                b[2 * j][0] = r[0];
                b[2 * j][1] = r[1];
                b[2 * j + 1][0] = r[2];
                b[2 * j + 1][1] = r[3];
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], a[i], b[j]);
        }
    }
    // epilogue
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int row = m0 + wm + 16 * i + (lane >> 2) + (q >= 2 ? 8 : 0);
                const int col = n0 + wn + 8 * j + 2 * (lane & 3) + (q & 1);
                if (row >= g.M || col >= g.N) continue;
                if (gridDim.z > 1)
                    g.partial[((size_t)blockIdx.z * g.M + row) * g.N + col] = acc[i][j][q];
                else
                    store(g, row, col, epilogue(g, row, col, acc[i][j][q]));
            }
}

// ---------------------------------------------------------------------------
// tcgen05 GEMM (5th-generation tensor cores, accumulator in tensor memory)
// for the forward products: C[M,N] = A[M,K] B[N,K]^T with A dense K-major or
// an im2col view, B dense K-major (weights).  One warpgroup per 128 x BN
// tile.  Operands are staged by cp.async into the K-major, no-swizzle
// canonical layout of the UMMA shared-memory descriptor: 8-row x 16-byte
// core matrices, core matrix (row group g, 8-element k chunk c) at byte
// (c * ROWS/8 + g) * 128, so for one K=16 MMA the two k chunks are LBO =
// ROWS/8 * 128 bytes apart and row groups SBO = 128 bytes apart.  After a
// proxy fence and a barrier, one thread issues the 4 MMAs of a 64-deep
// k tile and commits them to the stage's mbarrier; the next tile loads while
// they run.  The epilogue reads the accumulator with tcgen05.ld (warp w owns
// rows 32w..32w+31).  Every wait is bounded: on timeout the kernel records
// an error and leaves the tile.
constexpr int kTcM = 128, kTcK = 64, kTcThreads = 128, kTcStages = 3;

template <int BN>
__host__ __device__ constexpr uint32_t tc_stage_bytes() { return (uint32_t)(kTcM + BN) * kTcK * 2; }
template <int BN>
__host__ __device__ constexpr uint32_t tc_smem_bytes() { return kTcStages * tc_stage_bytes<BN>(); }
template <int BN>
__host__ __device__ constexpr uint32_t tc_tmem_cols() { return BN < 32 ? 32u : (uint32_t)BN; }  // a power of 2, >= 32

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <int AV, int BN>
__device__ __forceinline__ void tc_load(const GemmArgs& g, uint8_t* as, uint8_t* bs, int m0, int k0, int k_stop) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int t = 0; t < kTcM * (kTcK / 8) / kTcThreads; ++t) {
        const int i = tid + t * kTcThreads, row = i % kTcM, c = i / kTcM;
        const int gm = m0 + row, gk = k0 + c * 8;
        const bf16* src = nullptr;
        if (gm < g.M && gk < k_stop)
            src = AV == kIm2col ? im2col_chunk(g.A, g.lda, gm, gk, g.flip_a) : g.A + (size_t)gm * g.lda + gk;
        cp_async16(as + (c * (kTcM / 8) + row / 8) * 128 + (row % 8) * 16, src ? src : g.A, src != nullptr);
    }
#pragma unroll
    for (int t = 0; t < (BN * (kTcK / 8) + kTcThreads - 1) / kTcThreads; ++t) {
        const int i = tid + t * kTcThreads;
        if (i >= BN * (kTcK / 8)) break;
        const int row = i % BN, c = i / BN;
        const int gk = k0 + c * 8;
        const bool ok = row < g.N && gk < k_stop;
        cp_async16(bs + (c * (BN / 8) + row / 8) * 128 + (row % 8) * 16,
                   ok ? g.B + (size_t)row * g.ldb + gk : g.B, ok);
    }
}

template <int AV, int BN>
__global__ void __launch_bounds__(kTcThreads) gemm_tc_kernel(const GemmArgs g, uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ __align__(8) uint64_t bars[kTcStages];
    __shared__ uint32_t tmem_slot;
    constexpr int kA = kTcM * kTcK * 2;
    constexpr uint32_t kStageBytes = tc_stage_bytes<BN>(), kCols = tc_tmem_cols<BN>();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kTcM;
    // split K: this CTA adds k in [k_begin, k_begin + k_chunk)
    const int k_begin = blockIdx.y * g.k_chunk;
    const int k_stop = min(g.K, k_begin + g.k_chunk);
    const int nk = k_stop > k_begin ? (k_stop - k_begin + kTcK - 1) / kTcK : 0;
    if (tid == 0)
        for (int i = 0; i < kTcStages; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bars[i])));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const uint32_t tmem = tmem_slot;
    // instruction descriptor: D f32, A and B bf16, both K-major, N, M = 128
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
    auto stage = [&](int kt) { return tc_smem + (kt % kTcStages) * kStageBytes; };
    // the j-th commit on a stage completes phase j; tile kt is commit kt / kTcStages of stage kt % kTcStages
    auto wait_tile = [&](int kt) {
        return mbar_wait(smem_u32(&bars[kt % kTcStages]), (uint32_t)(kt / kTcStages) & 1u);
    };
    // prologue: tiles 0 .. kTcStages-2 in flight
    for (int kt = 0; kt < kTcStages - 1; ++kt) {
        if (kt < nk) tc_load<AV, BN>(g, stage(kt), stage(kt) + kA, m0, k_begin + kt * kTcK, k_stop);
        cp_async_commit();
    }
    bool ok = true;
    int issued = 0;  // k tiles whose MMAs were committed
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait_group<kTcStages - 2>();  // this thread's copies of tile kt landed
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
            const uint32_t a0 = smem_u32(stage(kt)), b0 = a0 + kA;
#pragma unroll
            for (int s = 0; s < kTcK / 16; ++s) {
                const uint64_t da = umma_desc(a0 + 2 * s * (kTcM / 8) * 128, (kTcM / 8) * 128, 128);
                const uint64_t db = umma_desc(b0 + 2 * s * (BN / 8) * 128, (BN / 8) * 128, 128);
                const uint32_t acc = (kt > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                smem_u32(&bars[kt % kTcStages])));
        }
        issued = kt + 1;
        // refill the stage of tile kt - 1 with tile kt + kTcStages - 1 once
        // its MMAs are done reading it
        const int nt = kt + kTcStages - 1;
        if (nt < nk) {
            const bool w = kt >= 1 ? wait_tile(kt - 1) : true;
            if (!__syncthreads_and(w)) {
                ok = false;
                break;
            }
            tc_load<AV, BN>(g, stage(nt), stage(nt) + kA, m0, k_begin + nt * kTcK, k_stop);
        }
        cp_async_commit();
    }
    cp_async_wait_group<0>();
    // the last committed tile (MMAs complete in issue order); on failure too,
    // before the tensor memory is released
    if (issued > 0) {
        const bool w = wait_tile(issued - 1);
        ok = ok && w;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicAdd(err, 1u);
    } else {
        const int row = m0 + warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 8) {
            uint32_t r[8];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (row < g.M) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int col = c0 + j;
                    if (col >= g.N) continue;
                    if (gridDim.y > 1)
                        g.partial[((size_t)blockIdx.y * g.M + row) * g.N + col] = __uint_as_float(r[j]);
                    else
                        store(g, row, col, epilogue(g, row, col, __uint_as_float(r[j])));
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols));
    }
}

// ---------------------------------------------------------------------------
// Planar implicit-GEMM convolution on tcgen05 (the forward 3x3x3 layers).
//
// Activations are stored as planes of 8 channels over the genomes' 7x7x7
// grids laid end to end: the 6x6x6 cells of genome b at padded row
// p = 343 b + x + 7y + 49z, and the rows with x, y or z = 6 zero.  That zero
// layer is the halo of both sides: x = -1 of a row is x = 6 of the row
// before, y = -1 of a plane is y = 6 of the plane before, z = -1 of a genome
// is z = 6 of the genome before.  Element (plane c/8, row p, channel c%8)
// at (c/8 * rows + p) 8 + c%8 (rows = the plane stride, a whole number of
// tiles), so one row of one plane is 16 bytes and consecutive rows are 16
// bytes apart -- exactly the K-major no-swizzle UMMA layout with SBO = 128
// bytes.  The input of output row p at offset o is row p + delta(o),
// delta = dx + 7 dy + 49 dz: a shift of the descriptor's start address.  A
// CTA loads, for an output tile of 128 rows, its 248-row input window
// (tile - 57 .. tile + 191, zero outside the genomes) once and issues all
// the tile's MMAs from it: 27 offsets x 2 channel halves (K = 16 each, LBO =
// the plane stride) for 32 input channels; for 8 input channels two offsets
// share one K = 16 MMA (LBO = the row distance between them).  The weights
// stay in shared memory for the CTA's whole run (persistent CTAs).  Halo
// rows are computed and discarded: the epilogue writes zeros there, so the
// next layer's halo is zero.  216 of every 343 rows are cells (an 8x8x8 grid
// per genome would have 216 of 512).
constexpr int kCvRows = 248, kCvLead = 57, kCvTile = 128, kCvSide = 7, kCvGenome = 343;

__host__ __device__ constexpr int cv_delta(int o) {
    return (o % 3 - 1) + kCvSide * ((o / 3) % 3 - 1) + kCvSide * kCvSide * (o / 9 - 1);
}
// rows of the planar layout of n genomes: whole tiles
__host__ __device__ constexpr uint32_t cv_rows(uint32_t n) {
    return (n * (uint32_t)kCvGenome + kCvTile - 1) / kCvTile * kCvTile;
}

struct ConvTcArgs {
    const bf16* in;        // planar input [p_in][cv_rows(n)][8]
    int p_in;              // input planes: 1 (8 channels) or 4 (32)
    const bf16* w;         // [32][27 * 8 * p_in], k = offset * 8 p_in + channel
    const float* bias;     // [32]
    int n;                 // genomes
    bf16* out_planar;      // [4][cv_rows(n)][8] or null
    bf16* out_compact;     // [n][216][32] (voxel x + 6y + 36z) or null
    uint32_t* err;
    // input gradient of a layer (the backward): no bias and no ReLU; the
    // output keeps the product where the forward activation mask[n][216][32]
    // (compact) is positive and is zero elsewhere
    const bf16* mask;
};

template <int P>
__global__ void __launch_bounds__(128) conv_tc_kernel(const ConvTcArgs g) {
    extern __shared__ __align__(1024) uint8_t cv_smem[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_slot;
    constexpr int K = 27 * 8 * P;
    constexpr int kWChunks = P == 1 ? 28 : K / 8;           // 8-element k chunks (one zero chunk pads K = 216)
    constexpr uint32_t kWBytes = kWChunks * 512;             // 32 rows = 4 row groups x 128 B per chunk
    constexpr uint32_t kABytes = P * kCvRows * 16;
    constexpr uint32_t kPlane = kCvRows * 16;                // plane stride inside an A buffer
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint8_t* sw = cv_smem;
    uint8_t* sa[2] = {cv_smem + kWBytes, cv_smem + kWBytes + kABytes};
    const int rows = (int)cv_rows((uint32_t)g.n), tiles = rows / kCvTile, real_rows = g.n * kCvGenome;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bars[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bars[1])));
    }
    if (warp == 0) {  // two 32-column accumulators: tile i uses columns 32 (i & 1)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(64u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    // weights, in the K-major core-matrix layout: chunk c of row n at (c*4 + n/8)*128 + (n%8)*16
    for (int i = tid; i < kWChunks * 32; i += 128) {
        const int c = i >> 5, row = i & 31;
        const bool ok = c * 8 < K;
        cp_async16(sw + (c * 4 + row / 8) * 128 + (row % 8) * 16, ok ? g.w + (size_t)row * K + c * 8 : g.w, ok);
    }
    auto load_a = [&](int t, uint8_t* dst) {
        const int r0 = t * kCvTile;
        for (int i = tid; i < P * kCvRows; i += 128) {
            const int plane = i / kCvRows, rr = i - plane * kCvRows, row = r0 - kCvLead + rr;
            const bool ok = row >= 0 && row < real_rows;
            cp_async16(dst + plane * kPlane + rr * 16, ok ? g.in + ((size_t)plane * rows + row) * 8 : g.in, ok);
        }
    };
    // epilogue of tile t from accumulator `acc`: row p from TMEM lane 32*warp + lane
    auto epilogue = [&](int t, uint32_t acc) {
        const int p = t * kCvTile + warp * 32 + lane, b = p / kCvGenome, loc = p - b * kCvGenome;
        const int x = loc % kCvSide, y = (loc / kCvSide) % kCvSide, z = loc / (kCvSide * kCvSide);
        const bool real = b < g.n && x < 6 && y < 6 && z < 6;
        const int v = x + 6 * y + 36 * z;
#pragma unroll
        for (int c0 = 0; c0 < 32; c0 += 8) {
            uint32_t r[8];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(acc + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            alignas(16) bf16 h[8];
            if (g.mask) {
                alignas(16) bf16 mk[8];
                *reinterpret_cast<uint4*>(mk) =
                    real ? *reinterpret_cast<const uint4*>(g.mask + ((size_t)b * 216 + v) * 32 + c0) : make_uint4(0, 0, 0, 0);
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    h[j] = __float2bfloat16_rn(__bfloat162float(mk[j]) > 0.0f ? __uint_as_float(r[j]) : 0.0f);
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    h[j] = __float2bfloat16_rn(real ? fmaxf(__uint_as_float(r[j]) + g.bias[c0 + j], 0.0f) : 0.0f);
            }
            const uint4 pk = *reinterpret_cast<const uint4*>(h);
            if (g.out_planar) *reinterpret_cast<uint4*>(g.out_planar + ((size_t)(c0 / 8) * rows + p) * 8) = pk;
            if (g.out_compact && real)
                *reinterpret_cast<uint4*>(g.out_compact + ((size_t)b * 216 + v) * 32 + c0) = pk;
        }
    };
    int t = blockIdx.x;
    if (t < tiles) load_a(t, sa[0]);
    cp_async_commit();
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (4u << 17) | (8u << 24);  // f32 <- bf16 x bf16, N 32, M 128
    // Tile i: MMAs into accumulator i & 1 (commit on bars[i & 1], its
    // (i >> 1)-th phase); meanwhile the epilogue of tile i - 1 and the load
    // of tile i + 1 (into the A buffer tile i - 1 used).
    bool ok = true;
    int prev = -1;  // tile of the previous iteration, its epilogue pending
    int i = 0;
    for (; t < tiles; t += gridDim.x, ++i) {
        const int s = i & 1;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
            const uint32_t a0 = smem_u32(sa[s]), w0 = smem_u32(sw), d = tmem + 32u * (uint32_t)s;
            auto mma = [&](uint64_t da, uint64_t db, uint32_t acc) {
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            };
            // descriptors are linear in the start-address field (address >> 4):
            // each MMA adds a compile-time byte offset >> 4 to a base
            if (P == 4) {
                const uint64_t da0 = umma_desc(a0, kPlane, 128), db0 = umma_desc(w0, 512, 128);
#pragma unroll
                for (int o = 0; o < 27; ++o) {
#pragma unroll
                    for (int q = 0; q < 2; ++q)
                        mma(da0 + ((2 * q * kPlane + (kCvLead + cv_delta(o)) * 16) >> 4),
                            db0 + (((o * 4 + 2 * q) * 512) >> 4), (o | q) ? 1u : 0u);
                }
            } else {
                const uint64_t da0 = umma_desc(a0, 0, 128), db0 = umma_desc(w0, 512, 128);
#pragma unroll
                for (int pr = 0; pr < 14; ++pr) {
                    const int o1 = 2 * pr, o2 = 2 * pr + 1;
                    const int d1 = cv_delta(o1), d2 = o2 < 27 ? cv_delta(o2) : d1 + 1;  // offset 27: zero weights
                    mma(da0 + ((uint64_t)(kCvLead + d1) * 16 >> 4) + ((uint64_t)(d2 - d1) << 16),
                        db0 + ((2 * pr * 512) >> 4), pr ? 1u : 0u);
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                smem_u32(&bars[s])));
        }
        if (prev >= 0) {
            // the previous tile's MMAs: done reading its A buffer, accumulator ready
            const bool w = mbar_wait(smem_u32(&bars[s ^ 1]), (uint32_t)((i - 1) >> 1) & 1u);
            if (!__syncthreads_and(w)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        }
        // the next tile's input into the freed buffer, in flight during the
        // previous tile's epilogue
        const int nt = t + gridDim.x;
        if (nt < tiles) load_a(nt, sa[s ^ 1]);
        cp_async_commit();
        if (prev >= 0) epilogue(prev, tmem + 32u * (uint32_t)(s ^ 1));
        cp_async_wait_all();
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
        __syncthreads();
        prev = t;
    }
    if (ok && prev >= 0) {  // the last tile
        const bool w = mbar_wait(smem_u32(&bars[(i - 1) & 1]), (uint32_t)((i - 1) >> 1) & 1u);
        ok = __syncthreads_and(w);
        if (ok) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
            epilogue(prev, tmem + 32u * (uint32_t)((i - 1) & 1));
        }
    } else if (!ok) {
        // drain: the tile issued in the iteration that failed
        mbar_wait(smem_u32(&bars[i & 1]), (uint32_t)(i >> 1) & 1u);
    }
    cp_async_wait_all();
    if (!ok && tid == 0) atomicAdd(g.err, 1u);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(64u));
    }
}

// Compact [n][216][32] (voxel x + 6y + 36z) to the planar layout
// [4][cv_rows(n)][8] with zero halo rows: the layout conv_tc_kernel reads.
__global__ void planar_from_compact_kernel(const bf16* __restrict__ c, uint32_t n, bf16* __restrict__ x) {
    const uint32_t rows = cv_rows(n);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * rows; i += gridDim.x * blockDim.x) {
        const uint32_t plane = i / rows, p = i % rows, b = p / kCvGenome, loc = p % kCvGenome;
        const uint32_t xx = loc % kCvSide, yy = (loc / kCvSide) % kCvSide, zz = loc / (kCvSide * kCvSide);
        uint4 v = make_uint4(0, 0, 0, 0);
        if (b < n && xx < 6 && yy < 6 && zz < 6)
            v = *reinterpret_cast<const uint4*>(c + ((size_t)b * 216 + xx + 6 * yy + 36 * zz) * 32 + plane * 8);
        *reinterpret_cast<uint4*>(x + (size_t)i * 8) = v;
    }
}

// Weights of the input-gradient convolution of a 32 -> 32 layer:
// wf[ci][o * 32 + co] = w[co][(26 - o) * 32 + ci] (the transposed kernel,
// offsets mirrored: offset 26 - o is offset o reflected through the centre).
__global__ void conv_weight_flip_kernel(const bf16* __restrict__ w, bf16* __restrict__ wf) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 32 * 27 * 32; i += gridDim.x * blockDim.x) {
        const uint32_t ci = i / 864, k = i % 864, o = k / 32, co = k % 32;
        wf[i] = w[co * 864 + (26 - o) * 32 + ci];
    }
}

// One-hot classes in the planar layout (8 channels, zero halo rows).
__global__ void onehot_planar_kernel(const uint8_t* __restrict__ cls, uint32_t n, bf16* __restrict__ x) {
    const uint32_t rows = cv_rows(n);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        const uint32_t b = i / kCvGenome, loc = i % kCvGenome;
        const uint32_t xx = loc % kCvSide, yy = (loc / kCvSide) % kCvSide, zz = loc / (kCvSide * kCvSide);
        uint32_t c = 0xFFu;
        if (b < n && xx < 6 && yy < 6 && zz < 6) c = cls[b * 216 + xx + 6 * yy + 36 * zz];
        alignas(16) bf16 h[8];
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) h[k] = __float2bfloat16_rn(c == k && c < 5 ? 1.0f : 0.0f);
        *reinterpret_cast<uint4*>(x + (size_t)i * 8) = *reinterpret_cast<const uint4*>(h);
    }
}

// Split-K: partial sums added in split order, then the epilogue.
__global__ void splitk_reduce_kernel(const GemmArgs g, int splits) {
    const size_t n = (size_t)g.M * g.N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int z = 0; z < splits; ++z) s += g.partial[(size_t)z * n + i];
        const int row = (int)(i / g.N), col = (int)(i % g.N);
        store(g, row, col, epilogue(g, row, col, s));
    }
}

// ---------------------------------------------------------------------------
// Small kernels

// One-hot classes, 8 channels per voxel.
__global__ void onehot_kernel(const uint8_t* __restrict__ cls, uint32_t n_vox, bf16* __restrict__ x) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_vox; i += gridDim.x * blockDim.x) {
        const uint32_t c = cls[i];
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) x[(size_t)i * 8 + k] = __float2bfloat16_rn(c == k && c < 5 ? 1.0f : 0.0f);
    }
}

// y[b] = b6 + sum_j h2[b, j] w6[j]: lane l adds j = l, l+32, l+64, l+96 in
// order, then an xor butterfly.
__global__ void head_kernel(const bf16* __restrict__ h2, const bf16* __restrict__ w6, const float* __restrict__ b6,
                            uint32_t n, float* __restrict__ y) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t b = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (b >= n) return;
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t j = lane + 32 * i;
        s = fmaf(__bfloat162float(h2[(size_t)b * 128 + j]), __bfloat162float(w6[j]), s);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[b] = s + b6[0];
}

// Loss and the gradients of the head: dy = 2 (y - t) / n; dW6[j] = sum_b dy
// h2[b, j] (thread j, samples in order); db6 = sum_b dy; dz2 = dy w6 where
// h2 > 0.  One block of 128 threads.
__global__ void head_backward_kernel(const float* __restrict__ y, const float* __restrict__ t,
                                     const bf16* __restrict__ h2, const bf16* __restrict__ w6, uint32_t n,
                                     float* __restrict__ dw6, float* __restrict__ db6, bf16* __restrict__ dz2,
                                     float* __restrict__ loss) {
    const uint32_t j = threadIdx.x;
    const float inv = 1.0f / (float)n;
    float g = 0.0f;
    for (uint32_t b = 0; b < n; ++b) {
        const float dy = 2.0f * (y[b] - t[b]) * inv;
        const float hv = __bfloat162float(h2[(size_t)b * 128 + j]);
        g = fmaf(dy, hv, g);
        dz2[(size_t)b * 128 + j] = __float2bfloat16_rn(hv > 0.0f ? dy * __bfloat162float(w6[j]) : 0.0f);
    }
    dw6[j] = g;
    if (j == 0) {
        float s = 0.0f, l = 0.0f;
        for (uint32_t b = 0; b < n; ++b) {
            const float e = y[b] - t[b];
            s += 2.0f * e * inv;
            l = fmaf(e, e, l);
        }
        db6[0] = s;
        loss[0] = l * inv;
    }
}

// Column sums in two fixed-order stages (coalesced rows): block b sums rows
// [b chunk, (b+1) chunk); thread t takes column t % cols and every
// (256 / cols)-th row from phase t / cols, the phases are added in order;
// colsum_final_kernel then adds the blocks' partial sums in contiguous
// ranges of blocks and the ranges in order.
constexpr int kColsumBlocks = 256;
__global__ void __launch_bounds__(256) colsum_partial_kernel(const bf16* __restrict__ a, uint32_t rows, uint32_t cols,
                                                             uint32_t chunk, float* __restrict__ partial) {
    __shared__ float red[256];
    const uint32_t t = threadIdx.x, phases = 256 / cols, c = t % cols, ph = t / cols;
    const uint32_t r0 = blockIdx.x * chunk, r1 = min(rows, r0 + chunk);
    float s = 0.0f;
    if (ph < phases)
        for (uint32_t r = r0 + ph; r < r1; r += phases) s += __bfloat162float(a[(size_t)r * cols + c]);
    red[t] = s;
    __syncthreads();
    if (t < cols) {
        float v = 0.0f;
        for (uint32_t q = 0; q < phases; ++q) v += red[q * cols + t];
        partial[(size_t)blockIdx.x * cols + t] = v;
    }
}

// 1,024 threads: thread t adds, for column t % cols, the partial sums of a
// contiguous range of blocks (part t / cols of 1024 / cols); the parts are
// then added in order.  Every load of a thread is independent of the others,
// so the stage costs about one memory latency.
__global__ void __launch_bounds__(1024) colsum_final_kernel(const float* __restrict__ partial, uint32_t blocks,
                                                            uint32_t cols, float* __restrict__ out) {
    __shared__ float red[1024];
    const uint32_t t = threadIdx.x, parts = 1024 / cols, c = t % cols, p = t / cols;
    const uint32_t per = (blocks + parts - 1) / parts, b0 = p * per, b1 = min(blocks, b0 + per);
    float v = 0.0f;
    for (uint32_t b = b0; b < b1; ++b) v += partial[(size_t)b * cols + c];
    red[t] = v;
    __syncthreads();
    if (t < cols) {
        float s = 0.0f;
        for (uint32_t q = 0; q < parts; ++q) s += red[q * cols + t];
        out[t] = s;
    }
}

// wt[(o*32 + co) * cin + ci] = w[co * 27*cin + o*cin + ci]: the weights of
// the input-gradient convolution as a K x N (MN-major) operand.
__global__ void conv_weight_t_kernel(const bf16* __restrict__ w, uint32_t cin, bf16* __restrict__ wt) {
    const uint32_t n = 27 * 32 * cin;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t ci = i % cin, k = i / cin, o = k / 32, co = k % 32;
        wt[i] = w[(size_t)co * 27 * cin + o * cin + ci];
    }
}

// Adam on the FP32 master weights, then their BF16 copies.
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, bf16* __restrict__ wb, uint32_t n, float lr, float b1,
                            float b2, float eps, float c1, float c2, float wd) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * w[i]);
        w[i] = wi;
        wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void to_bf16_kernel(const float* __restrict__ w, bf16* __restrict__ wb, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

template <int AV, int BV>
cudaError_t gemm(GemmArgs g, int splits, cudaStream_t s) {
    if (g.M <= 0 || g.N <= 0) return cudaSuccess;
    splits = std::max(1, std::min<int>(splits, (int)(g.partial_cap / ((size_t)g.M * g.N))));
    g.k_chunk = ((g.K + splits - 1) / splits + kTileK - 1) / kTileK * kTileK;
    splits = std::max(1, (g.K + g.k_chunk - 1) / g.k_chunk);
    const dim3 grid((g.N + kTileN - 1) / kTileN, (g.M + kTileM - 1) / kTileM, splits);
    gemm_kernel<AV, BV><<<grid, kGemmThreads, 0, s>>>(g);
    if (splits > 1) {
        const size_t n = (size_t)g.M * g.N;
        splitk_reduce_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, s>>>(g, splits);
    }
    return cudaGetLastError();
}

template <int P>
cudaError_t conv_tc(const ConvTcArgs& g, int num_sms, cudaStream_t s) {
    constexpr uint32_t smem = (P == 1 ? 28 : 27 * P) * 512 + 2 * P * kCvRows * 16;
    static bool prepared = false;
    if (!prepared) {
        cudaError_t e = cudaFuncSetAttribute(conv_tc_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        prepared = true;
    }
    const int tiles = (int)(cv_rows((uint32_t)g.n) / kCvTile);
    if (tiles == 0) return cudaSuccess;
    const int grid = std::min(tiles, (P == 1 ? 4 : 2) * num_sms);
    conv_tc_kernel<P><<<grid, 128, smem, s>>>(g);
    return cudaGetLastError();
}

template <int AV, int BN>
cudaError_t gemm_tc(GemmArgs g, uint32_t* err, cudaStream_t s, int splits = 1) {
    static bool prepared = false;
    if (!prepared) {
        cudaError_t e = cudaFuncSetAttribute(gemm_tc_kernel<AV, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)tc_smem_bytes<BN>());
        if (e != cudaSuccess) return e;
        prepared = true;
    }
    if (g.M <= 0 || g.N <= 0) return cudaSuccess;
    splits = std::max(1, std::min<int>(splits, (int)(g.partial_cap / ((size_t)g.M * g.N))));
    g.k_chunk = ((g.K + splits - 1) / splits + kTcK - 1) / kTcK * kTcK;
    splits = std::max(1, (g.K + g.k_chunk - 1) / g.k_chunk);
    const dim3 grid((g.M + kTcM - 1) / kTcM, splits);
    gemm_tc_kernel<AV, BN><<<grid, kTcThreads, tc_smem_bytes<BN>(), s>>>(g, err);
    if (splits > 1) {
        const size_t n = (size_t)g.M * g.N;
        splitk_reduce_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, s>>>(g, splits);
    }
    return cudaGetLastError();
}

}  // namespace
}  // namespace sg
}  // namespace mb

// ---------------------------------------------------------------------------
// Host driver

namespace {

using bf16 = __nv_bfloat16;
using namespace mb::sg;

// Flat parameter layout: tensors in order, each padded to 8 elements.
enum Tensor { kW1, kB1, kW2, kB2, kW3, kB3, kW4, kB4, kW5, kB5, kW6, kB6, kTensors };
constexpr uint32_t kSize[kTensors] = {32 * 27 * 8, 32, 32 * 27 * 32, 32, 32 * 27 * 32, 32,
                                      128 * 6912, 128, 128 * 128, 128, 128, 1};
constexpr uint32_t kFanIn[kTensors] = {27 * 5, 0, 27 * 32, 0, 27 * 32, 0, 6912, 0, 128, 0, 128, 0};

struct Layout {
    uint32_t off[kTensors + 1];
    Layout() {
        uint32_t o = 0;
        for (int i = 0; i < kTensors; ++i) {
            off[i] = o;
            o += (kSize[i] + 7) / 8 * 8;
        }
        off[kTensors] = o;
    }
};
const Layout kLayout;

template <typename T>
struct Buf {
    T* p = nullptr;
    ~Buf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) {
        if (p) cudaFree(p);
        p = nullptr;
        return cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
    }
};

uint64_t mix64(uint64_t z) {
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

}  // namespace

struct mb_surrogate {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t max_batch = 0;
    std::string err;
    uint64_t step = 0;
    float weight_decay = 0.0f;
    bool tcgen05 = true;   // forward GEMMs on the 5th-generation tensor cores
    int num_sms = 148;
    Buf<uint32_t> tc_err;
    Buf<bf16> x0p, a1p, a2p;  // padded planar activations of the tcgen05 convolutions
    Buf<bf16> dz3p, dz2p, wf2, wf3;  // backward on tcgen05: planar gradients, mirrored weights
    Buf<float> w, m, v, g, loss, y, t, partial;
    Buf<bf16> wb, wt2, wt3, x0, a1, a2, a3, h1, h2, dz2h, dz1h, dz3, dz2c, dz1c;
    Buf<uint8_t> cls;
    ~mb_surrogate() {
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

mb_status sfail(mb_surrogate* s, mb_status st, const char* msg) {
    if (s) s->err = msg;
    return st;
}

#define SG_CUDA(s, call)                                                                  \
    do {                                                                                  \
        cudaError_t _e = (call);                                                          \
        if (_e != cudaSuccess) {                                                          \
            if (s) s->err = std::string(#call) + ": " + cudaGetErrorString(_e);           \
            return MB_ERR_CUDA;                                                           \
        }                                                                                 \
    } while (0)

const float* P(const mb_surrogate* s, Tensor i) { return s->w.p + kLayout.off[i]; }
const bf16* PB(const mb_surrogate* s, Tensor i) { return s->wb.p + kLayout.off[i]; }
float* G(mb_surrogate* s, Tensor i) { return s->g.p + kLayout.off[i]; }

constexpr size_t kPartialFloats = 64 * 32 * 27 * 32;

GemmArgs args(mb_surrogate* s, const bf16* A, int lda, const bf16* B, int ldb, int M, int N, int K) {
    GemmArgs a{};
    a.partial = s->partial.p;
    a.partial_cap = kPartialFloats;
    a.A = A;
    a.B = B;
    a.M = M;
    a.N = N;
    a.K = K;
    a.lda = lda;
    a.ldb = ldb;
    a.ldc = N;
    return a;
}

// Forward of n samples already one-hot in s->x0; leaves a1..a3, h1, h2, y.
// The products run on tcgen05 (or, when switched off, on mma.sync).
cudaError_t forward(mb_surrogate* s, uint32_t n) {
    cudaStream_t st = s->stream;
    const int R = (int)n * kVox;
    cudaError_t e;
    auto conv = [&](const bf16* x, int cin, Tensor w, Tensor b, bf16* out) {
        GemmArgs a = args(s, x, cin, PB(s, w), 27 * cin, R, 32, 27 * cin);
        a.bias = P(s, b);
        a.relu = 1;
        a.c16 = out;
        return s->tcgen05 ? gemm_tc<kIm2col, 32>(a, s->tc_err.p, st) : gemm<kIm2col, kDenseK>(a, 1, st);
    };
    // the flatten layer: K = 6912 split over CTAs (M is only the batch);
    // the 128 x 128 layer is too small for the tensor-memory set-up to pay
    auto fc = [&](const bf16* x, int k, Tensor w, Tensor b, bf16* out) {
        GemmArgs a = args(s, x, k, PB(s, w), k, (int)n, 128, k);
        a.bias = P(s, b);
        a.relu = 1;
        a.c16 = out;
        if (s->tcgen05 && k > 1024) {
            const int mt = ((int)n + kTcM - 1) / kTcM;
            return gemm_tc<kDenseK, 128>(a, s->tc_err.p, st, std::max(1, std::min(k / kTcK / 4, 2 * s->num_sms / mt)));
        }
        return gemm<kDenseK, kDenseK>(a, 1, st);
    };
    if (s->tcgen05) {
        onehot_planar_kernel<<<std::min<uint32_t>((cv_rows(n) + 255) / 256, 4096), 256, 0, st>>>(s->cls.p, n, s->x0p.p);
        const ConvTcArgs c1{s->x0p.p, 1, PB(s, kW1), P(s, kB1), (int)n, s->a1p.p, s->a1.p, s->tc_err.p};
        const ConvTcArgs c2{s->a1p.p, 4, PB(s, kW2), P(s, kB2), (int)n, s->a2p.p, s->a2.p, s->tc_err.p};
        const ConvTcArgs c3{s->a2p.p, 4, PB(s, kW3), P(s, kB3), (int)n, nullptr, s->a3.p, s->tc_err.p};
        if ((e = conv_tc<1>(c1, s->num_sms, st)) != cudaSuccess) return e;
        if ((e = conv_tc<4>(c2, s->num_sms, st)) != cudaSuccess) return e;
        if ((e = conv_tc<4>(c3, s->num_sms, st)) != cudaSuccess) return e;
    } else {
        if ((e = conv(s->x0.p, 8, kW1, kB1, s->a1.p)) != cudaSuccess) return e;
        if ((e = conv(s->a1.p, 32, kW2, kB2, s->a2.p)) != cudaSuccess) return e;
        if ((e = conv(s->a2.p, 32, kW3, kB3, s->a3.p)) != cudaSuccess) return e;
    }
    if ((e = fc(s->a3.p, 6912, kW4, kB4, s->h1.p)) != cudaSuccess) return e;
    if ((e = fc(s->h1.p, 128, kW5, kB5, s->h2.p)) != cudaSuccess) return e;
    head_kernel<<<(n + 7) / 8, 256, 0, st>>>(s->h2.p, PB(s, kW6), P(s, kB6), n, s->y.p);
    return cudaGetLastError();
}

// Reads and clears the tensor-core GEMM error count (after a synchronise).
mb_status check_tc(mb_surrogate* s) {
    uint32_t err = 0;
    SG_CUDA(s, cudaMemcpyAsync(&err, s->tc_err.p, sizeof(err), cudaMemcpyDeviceToHost, s->stream));
    SG_CUDA(s, cudaStreamSynchronize(s->stream));
    if (err) {
        SG_CUDA(s, cudaMemsetAsync(s->tc_err.p, 0, sizeof(uint32_t), s->stream));
        return sfail(s, MB_ERR_CUDA, "tensor-core GEMM wait timed out");
    }
    return MB_OK;
}

int splits_for(int K) { return std::max(1, std::min(64, K / 1024)); }

// Bias gradients: column sums of a [rows][cols] gradient (cols 32 or 128),
// in a fixed order (partial sums in the split-K scratch).
void colsum(mb_surrogate* s, const bf16* a, uint32_t rows, uint32_t cols, float* out) {
    assert(cols <= 256 && 256 % cols == 0);  // both stages split 256 / 1024 threads into whole columns
    const uint32_t chunk = std::max<uint32_t>(1, (rows + kColsumBlocks - 1) / kColsumBlocks);
    const uint32_t blocks = (rows + chunk - 1) / chunk;
    colsum_partial_kernel<<<blocks, 256, 0, s->stream>>>(a, rows, cols, chunk, s->partial.p);
    colsum_final_kernel<<<1, 1024, 0, s->stream>>>(s->partial.p, blocks, cols, out);
}

// Backward of the last forward against targets s->t; gradients into s->g.
cudaError_t backward(mb_surrogate* s, uint32_t n) {
    cudaStream_t st = s->stream;
    const int R = (int)n * kVox;
    cudaError_t e;
    head_backward_kernel<<<1, 128, 0, st>>>(s->y.p, s->t.p, s->h2.p, PB(s, kW6), n, G(s, kW6), G(s, kB6),
                                            s->dz2h.p, s->loss.p);
    // fc2: dW5 = dz2^T h1, db5, dz1 = (dz2 W5) where h1 > 0
    {
        GemmArgs a = args(s, s->dz2h.p, 128, s->h1.p, 128, 128, 128, (int)n);
        a.c32 = G(s, kW5);
        if ((e = gemm<kDenseMN, kDenseMN>(a, splits_for((int)n), st)) != cudaSuccess) return e;
    }
    colsum(s, s->dz2h.p, n, 128, G(s, kB5));
    {
        GemmArgs a = args(s, s->dz2h.p, 128, PB(s, kW5), 128, (int)n, 128, 128);
        a.mask = s->h1.p;
        a.c16 = s->dz1h.p;
        if ((e = gemm<kDenseK, kDenseMN>(a, 1, st)) != cudaSuccess) return e;
    }
    // fc1: dW4 = dz1^T flatten(a3), db4, dz3 = (dz1 W4) where a3 > 0
    {
        GemmArgs a = args(s, s->dz1h.p, 128, s->a3.p, 6912, 128, 6912, (int)n);
        a.c32 = G(s, kW4);
        if ((e = gemm<kDenseMN, kDenseMN>(a, splits_for((int)n), st)) != cudaSuccess) return e;
    }
    colsum(s, s->dz1h.p, n, 128, G(s, kB4));
    {
        GemmArgs a = args(s, s->dz1h.p, 128, PB(s, kW4), 6912, (int)n, 6912, 128);
        a.mask = s->a3.p;
        a.c16 = s->dz3.p;
        if ((e = gemm<kDenseK, kDenseMN>(a, 1, st)) != cudaSuccess) return e;
    }
    // conv3: dW3 = dz3^T im2col(a2), db3, dz2 = conv^T(dz3; W3) where a2 > 0
    {
        GemmArgs a = args(s, s->dz3.p, 32, s->a2.p, 32, 32, 27 * 32, R);
        a.c32 = G(s, kW3);
        if ((e = gemm<kDenseMN, kIm2col>(a, splits_for(R), st)) != cudaSuccess) return e;
    }
    colsum(s, s->dz3.p, (uint32_t)R, 32, G(s, kB3));
    if (s->tcgen05) {
        // input gradient as the forward convolution of the gradient with the
        // mirrored, transposed kernel, on tcgen05; masked by a2 > 0
        planar_from_compact_kernel<<<std::min<uint32_t>((4 * cv_rows(n) + 255) / 256, 4096), 256, 0, st>>>(s->dz3.p, n,
                                                                                                      s->dz3p.p);
        conv_weight_flip_kernel<<<108, 256, 0, st>>>(PB(s, kW3), s->wf3.p);
        ConvTcArgs c{s->dz3p.p, 4, s->wf3.p, nullptr, (int)n, s->dz2p.p, s->dz2c.p, s->tc_err.p};
        c.mask = s->a2.p;
        if ((e = conv_tc<4>(c, s->num_sms, st)) != cudaSuccess) return e;
    } else {
        conv_weight_t_kernel<<<108, 256, 0, st>>>(PB(s, kW3), 32, s->wt3.p);
        GemmArgs a = args(s, s->dz3.p, 32, s->wt3.p, 32, R, 32, 27 * 32);
        a.flip_a = 1;
        a.mask = s->a2.p;
        a.c16 = s->dz2c.p;
        if ((e = gemm<kIm2col, kDenseMN>(a, 1, st)) != cudaSuccess) return e;
    }
    // conv2
    {
        GemmArgs a = args(s, s->dz2c.p, 32, s->a1.p, 32, 32, 27 * 32, R);
        a.c32 = G(s, kW2);
        if ((e = gemm<kDenseMN, kIm2col>(a, splits_for(R), st)) != cudaSuccess) return e;
    }
    colsum(s, s->dz2c.p, (uint32_t)R, 32, G(s, kB2));
    if (s->tcgen05) {
        conv_weight_flip_kernel<<<108, 256, 0, st>>>(PB(s, kW2), s->wf2.p);
        ConvTcArgs c{s->dz2p.p, 4, s->wf2.p, nullptr, (int)n, nullptr, s->dz1c.p, s->tc_err.p};
        c.mask = s->a1.p;
        if ((e = conv_tc<4>(c, s->num_sms, st)) != cudaSuccess) return e;
    } else {
        conv_weight_t_kernel<<<108, 256, 0, st>>>(PB(s, kW2), 32, s->wt2.p);
        GemmArgs a = args(s, s->dz2c.p, 32, s->wt2.p, 32, R, 32, 27 * 32);
        a.flip_a = 1;
        a.mask = s->a1.p;
        a.c16 = s->dz1c.p;
        if ((e = gemm<kIm2col, kDenseMN>(a, 1, st)) != cudaSuccess) return e;
    }
    // conv1: dW1 = dz1^T im2col(x0), db1
    {
        GemmArgs a = args(s, s->dz1c.p, 32, s->x0.p, 8, 32, 27 * 8, R);
        a.c32 = G(s, kW1);
        if ((e = gemm<kDenseMN, kIm2col>(a, splits_for(R), st)) != cudaSuccess) return e;
    }
    colsum(s, s->dz1c.p, (uint32_t)R, 32, G(s, kB1));
    return cudaGetLastError();
}

mb_status upload_batch(mb_surrogate* s, const uint8_t* genomes, const float* targets, uint32_t n) {
    cudaStream_t st = s->stream;
    SG_CUDA(s, cudaMemcpyAsync(s->cls.p, genomes, (size_t)n * kVox, cudaMemcpyHostToDevice, st));
    if (targets) SG_CUDA(s, cudaMemcpyAsync(s->t.p, targets, n * sizeof(float), cudaMemcpyHostToDevice, st));
    onehot_kernel<<<std::min<uint32_t>((n * kVox + 255) / 256, 4096), 256, 0, st>>>(s->cls.p, n * kVox, s->x0.p);
    SG_CUDA(s, cudaGetLastError());
    return MB_OK;
}

}  // namespace

extern "C" {

uint32_t mb_surrogate_param_count(void) { return kLayout.off[kTensors]; }

void mb_surrogate_layout(uint32_t* offsets) {
    if (!offsets) return;
    for (int i = 0; i <= kTensors; ++i) offsets[i] = kLayout.off[i];
}

mb_status mb_surrogate_create(int device, uint32_t max_batch, uint64_t seed, mb_surrogate** out) {
    if (!out || max_batch == 0 || max_batch > 65536) return MB_ERR_ARGUMENT;
    *out = nullptr;
    std::unique_ptr<mb_surrogate> s(new mb_surrogate());
    s->device = device;
    s->max_batch = max_batch;
    if (cudaSetDevice(device) != cudaSuccess) return MB_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return MB_ERR_CUDA;
    const size_t np = kLayout.off[kTensors], R = (size_t)max_batch * kVox;
    auto ok = [](cudaError_t e) { return e == cudaSuccess; };
    if (!(ok(s->w.alloc(np)) && ok(s->m.alloc(np)) && ok(s->v.alloc(np)) && ok(s->g.alloc(np)) &&
          ok(s->wb.alloc(np)) && ok(s->loss.alloc(1)) && ok(s->y.alloc(max_batch)) && ok(s->t.alloc(max_batch)) &&
          ok(s->partial.alloc(kPartialFloats)) && ok(s->wt2.alloc(27 * 32 * 32)) &&
          ok(s->wt3.alloc(27 * 32 * 32)) && ok(s->x0.alloc(R * 8)) && ok(s->a1.alloc(R * 32)) &&
          ok(s->a2.alloc(R * 32)) && ok(s->a3.alloc(R * 32)) && ok(s->h1.alloc((size_t)max_batch * 128)) &&
          ok(s->h2.alloc((size_t)max_batch * 128)) && ok(s->dz2h.alloc((size_t)max_batch * 128)) &&
          ok(s->dz1h.alloc((size_t)max_batch * 128)) && ok(s->dz3.alloc(R * 32)) && ok(s->dz2c.alloc(R * 32)) &&
          ok(s->dz1c.alloc(R * 32)) && ok(s->cls.alloc(R)) && ok(s->tc_err.alloc(1)) &&
          ok(s->x0p.alloc((size_t)cv_rows(max_batch) * 8)) && ok(s->a1p.alloc((size_t)cv_rows(max_batch) * 4 * 8)) &&
          ok(s->a2p.alloc((size_t)cv_rows(max_batch) * 4 * 8)) && ok(s->dz3p.alloc((size_t)cv_rows(max_batch) * 4 * 8)) &&
          ok(s->dz2p.alloc((size_t)cv_rows(max_batch) * 4 * 8)) && ok(s->wf2.alloc(32 * 864)) &&
          ok(s->wf3.alloc(32 * 864))))
        return MB_ERR_CUDA;
    if (cudaMemset(s->tc_err.p, 0, sizeof(uint32_t)) != cudaSuccess) return MB_ERR_CUDA;
    if (cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return MB_ERR_CUDA;
    // He-normal weights (fan-in of the real inputs), zero biases, zero
    // weights on the padding channels of W1; Box-Muller over SplitMix64.
    std::vector<float> w(np, 0.0f);
    uint64_t state = seed;
    auto uniform = [&]() { return ((mix64(state += 0x9E3779B97F4A7C15ULL) >> 11) + 0.5) * (1.0 / 9007199254740992.0); };
    for (int t = 0; t < kTensors; ++t) {
        if (!kFanIn[t]) continue;
        const double sd = std::sqrt((t == kW6 ? 1.0 : 2.0) / kFanIn[t]);
        for (uint32_t i = 0; i < kSize[t]; ++i) {
            if (t == kW1 && i % 8 >= 5) continue;
            const double u1 = uniform(), u2 = uniform();
            w[kLayout.off[t] + i] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
        }
    }
    const mb_status st = mb_surrogate_set_params(s.get(), w.data());
    if (st != MB_OK) return st;
    *out = s.release();
    return MB_OK;
}

void mb_surrogate_destroy(mb_surrogate* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    delete s;
}

const char* mb_surrogate_last_error(const mb_surrogate* s) { return s ? s->err.c_str() : "null surrogate"; }

mb_status mb_surrogate_set_params(mb_surrogate* s, const float* params) {
    if (!s || !params) return sfail(s, MB_ERR_ARGUMENT, "null argument");
    cudaSetDevice(s->device);
    const size_t np = kLayout.off[kTensors];
    cudaStream_t st = s->stream;
    SG_CUDA(s, cudaMemcpyAsync(s->w.p, params, np * sizeof(float), cudaMemcpyHostToDevice, st));
    SG_CUDA(s, cudaMemsetAsync(s->m.p, 0, np * sizeof(float), st));
    SG_CUDA(s, cudaMemsetAsync(s->v.p, 0, np * sizeof(float), st));
    to_bf16_kernel<<<1024, 256, 0, st>>>(s->w.p, s->wb.p, (uint32_t)np);
    SG_CUDA(s, cudaGetLastError());
    SG_CUDA(s, cudaStreamSynchronize(st));
    s->step = 0;
    return MB_OK;
}

mb_status mb_surrogate_use_tcgen05(mb_surrogate* s, int on) {
    if (!s) return MB_ERR_ARGUMENT;
    s->tcgen05 = on != 0;
    return MB_OK;
}

mb_status mb_surrogate_set_weight_decay(mb_surrogate* s, float weight_decay) {
    if (!s || !(weight_decay >= 0.0f)) return sfail(s, MB_ERR_ARGUMENT, "weight decay must be >= 0");
    s->weight_decay = weight_decay;
    return MB_OK;
}

mb_status mb_surrogate_get_params(mb_surrogate* s, float* params) {
    if (!s || !params) return sfail(s, MB_ERR_ARGUMENT, "null argument");
    cudaSetDevice(s->device);
    SG_CUDA(s, cudaMemcpyAsync(params, s->w.p, kLayout.off[kTensors] * sizeof(float), cudaMemcpyDeviceToHost,
                               s->stream));
    SG_CUDA(s, cudaStreamSynchronize(s->stream));
    return MB_OK;
}

mb_status mb_surrogate_predict(mb_surrogate* s, const uint8_t* genomes, uint32_t n, float* out) {
    if (!s || !genomes || !out) return sfail(s, MB_ERR_ARGUMENT, "null argument");
    cudaSetDevice(s->device);
    for (uint32_t b0 = 0; b0 < n; b0 += s->max_batch) {
        const uint32_t nb = std::min(s->max_batch, n - b0);
        const mb_status st = upload_batch(s, genomes + (size_t)b0 * kVox, nullptr, nb);
        if (st != MB_OK) return st;
        SG_CUDA(s, forward(s, nb));
        SG_CUDA(s, cudaMemcpyAsync(out + b0, s->y.p, nb * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    }
    SG_CUDA(s, cudaStreamSynchronize(s->stream));
    return check_tc(s);
}

mb_status mb_surrogate_gradients(mb_surrogate* s, const uint8_t* genomes, const float* targets, uint32_t n,
                                 float* grads, float* loss) {
    if (!s || !genomes || !targets) return sfail(s, MB_ERR_ARGUMENT, "null argument");
    if (n == 0 || n > s->max_batch) return sfail(s, MB_ERR_ARGUMENT, "batch must be 1..max_batch");
    cudaSetDevice(s->device);
    mb_status st = upload_batch(s, genomes, targets, n);
    if (st != MB_OK) return st;
    SG_CUDA(s, cudaMemsetAsync(s->g.p, 0, kLayout.off[kTensors] * sizeof(float), s->stream));
    SG_CUDA(s, forward(s, n));
    SG_CUDA(s, backward(s, n));
    if (grads)
        SG_CUDA(s, cudaMemcpyAsync(grads, s->g.p, kLayout.off[kTensors] * sizeof(float), cudaMemcpyDeviceToHost,
                                   s->stream));
    if (loss) SG_CUDA(s, cudaMemcpyAsync(loss, s->loss.p, sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    SG_CUDA(s, cudaStreamSynchronize(s->stream));
    return check_tc(s);
}

mb_status mb_surrogate_train_step(mb_surrogate* s, const uint8_t* genomes, const float* targets, uint32_t n,
                                  float lr, float* loss) {
    const mb_status st = mb_surrogate_gradients(s, genomes, targets, n, nullptr, loss);
    if (st != MB_OK) return st;
    const float b1 = 0.9f, b2 = 0.999f;
    ++s->step;
    const float c1 = 1.0f - std::pow(b1, (float)s->step), c2 = 1.0f - std::pow(b2, (float)s->step);
    adam_kernel<<<1024, 256, 0, s->stream>>>(s->w.p, s->m.p, s->v.p, s->g.p, s->wb.p, kLayout.off[kTensors], lr, b1,
                                             b2, 1e-8f, c1, c2, s->weight_decay);
    SG_CUDA(s, cudaGetLastError());
    SG_CUDA(s, cudaStreamSynchronize(s->stream));
    return MB_OK;
}

}  // extern "C"
