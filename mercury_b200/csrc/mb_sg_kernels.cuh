// BF16 tensor-core kernels of the fitness surrogate (mb_surrogate.cu).
//
// One GEMM kernel does every product of the network, forward and backward:
// C[M,N] = sum_k A[m,k] B[k,n], BF16 operands, FP32 accumulation on the
// tensor cores (mma.sync m16n8k16), 64x64x32 tiles, 4 warps of 32x32, two
// shared-memory stages filled by cp.async.  Operands are read through one of
// three views:
//   dense K-major   element (i, k) at ptr[i * ld + k]
//   dense MN-major  element (i, k) at ptr[k * ld + i]
//   im2col          the 3x3x3 neighbourhood of a channels-last 6x6x6 grid:
//                   row r = b * 216 + v (sample b, voxel v), column
//                   j = o * C + c (offset o of 27, channel c) is
//                   act[(b * 216 + u) * C + c] with u = v + d(o) (or v - d(o)
//                   with `flip`), 0 outside the grid.  For A it is the M x K
//                   matrix (rows r); for B the K x N one (rows r = k).
// Every view moves 16-byte chunks of 8 consecutive elements along its
// contiguous dimension, so that dimension and every leading dimension are
// multiples of 8 and pointers 16-byte aligned (the host checks).
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace mb {
namespace sg {

enum View : int { kDenseK = 0, kDenseMN = 1, kIm2col = 2 };

struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    int M, N, K;
    int lda, ldb;         // dense views: leading dimension; im2col: channels C
    int flip_a, flip_b;   // im2col: u = v - d(o)
    // epilogue
    const float* bias;              // per column, or null
    int relu;
    const __nv_bfloat16* mask;      // keep C[m,n] where mask[m*ldc+n] > 0, or null
    float* c32;                     // fp32 output or null
    __nv_bfloat16* c16;             // bf16 output or null
    int ldc;
    // split K: partial sums [splits][M][N] when splits > 1
    float* partial;
    size_t partial_cap;             // floats in `partial`
    int k_chunk;                    // K per split, multiple of 32
};

constexpr int kTileM = 64, kTileN = 64, kTileK = 32, kGemmThreads = 128;
constexpr int kGrid = 6, kVox = 216;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Address of the 8-element chunk (row r, columns j..j+7) of an im2col view;
// null when the neighbour is outside the grid.
__device__ __forceinline__ const __nv_bfloat16* im2col_chunk(const __nv_bfloat16* act, int C, int r, int j,
                                                            int flip) {
    const int b = r / kVox, v = r - b * kVox;
    const int o = j / C, c = j - o * C;
    int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
    if (flip) {
        dx = -dx;
        dy = -dy;
        dz = -dz;
    }
    const int x = v % kGrid + dx, y = (v / kGrid) % kGrid + dy, z = v / (kGrid * kGrid) + dz;
    if (x < 0 || x >= kGrid || y < 0 || y >= kGrid || z < 0 || z >= kGrid) return nullptr;
    return act + ((size_t)(b * kVox + x + kGrid * y + kGrid * kGrid * z) * C + c);
}

}  // namespace sg
}  // namespace mb
