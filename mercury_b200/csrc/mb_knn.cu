// k-nearest-neighbour springs of point-cloud robots, built on the device
// (the springs of the reference's NNRobot, common/evolvables/knn.cu:62-145
// with knn_kernel.cu:34-60, as the third benchmark configuration uses them:
// every mass joined to its k nearest masses, each unordered pair once).
//
// Per robot:
//   select_kernel  one thread per mass scans the robot's positions (shared
//                  memory) and keeps its k nearest in registers, ordered by
//                  (squared distance, index) -- the order of a stable sort of
//                  the distance row; squared distances are the float32 sum
//                  (dx*dx + dy*dy) + dz*dz;
//   mark_kernel    sets bit (min, max) of an upper-triangular bitset for
//                  every neighbour pair;
//   count_kernel   popcounts each row; the host adds them up;
//   emit_kernel    writes the pairs row by row, partners ascending (the
//                  lexicographic order of the unique pairs), with the float32
//                  distance as mean length and the composite material of the
//                  two masses.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/mercury_b200.h"

namespace mb {
namespace {

constexpr uint32_t kKnnMaxK = 32;
constexpr uint32_t kKnnMaxMasses = 4096;
constexpr uint32_t kKnnThreads = 256;

__device__ __forceinline__ float sqdist(float3 a, float3 b) {
    const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

__device__ __forceinline__ int composite_knn(int m1, int m2) {
    if (m1 == 0 || m2 == 0) return 0;
    const int i = min(m1, m2) - 1, j = max(m1, m2) - 1;
    if (i == j) return i + 1;
    return 23 + i * 21 - i * (i - 1) / 2 + (j - i - 1);
}

struct KnnArgs {
    const float* pos;         // 3 per mass
    const int64_t* mass_off;  // n_robots + 1
    uint32_t k;
    uint16_t* nn;             // per mass: k neighbours (scratch), ascending (d2, index)
    uint32_t* bits;           // per robot: rows of ceil(m / 32) words
    const uint64_t* bit_off;  // per robot: first word
    uint32_t* row_count;      // per mass
};

__global__ void __launch_bounds__(kKnnThreads) select_kernel(const KnnArgs a) {
    extern __shared__ float3 pts[];
    const uint32_t r = blockIdx.y;
    const int64_t m0 = a.mass_off[r];
    const uint32_t m = (uint32_t)(a.mass_off[r + 1] - m0);
    for (uint32_t j = threadIdx.x; j < m; j += blockDim.x)
        pts[j] = make_float3(a.pos[3 * (m0 + j)], a.pos[3 * (m0 + j) + 1], a.pos[3 * (m0 + j) + 2]);
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t k = min(a.k, m - 1);
    float kd[kKnnMaxK];
    uint32_t kj[kKnnMaxK];
    uint32_t n = 0;
    const float3 pi = pts[i];
    for (uint32_t j = 0; j < m; ++j) {
        if (j == i) continue;
        const float d = sqdist(pi, pts[j]);
        // j ascends: an equal distance never displaces an earlier index
        if (n == k && !(d < kd[k - 1])) continue;
        uint32_t p = n < k ? n++ : k - 1;
        while (p > 0 && d < kd[p - 1]) {
            kd[p] = kd[p - 1];
            kj[p] = kj[p - 1];
            --p;
        }
        kd[p] = d;
        kj[p] = j;
    }
    uint16_t* out = a.nn + (size_t)(m0 + i) * a.k;
    for (uint32_t q = 0; q < a.k; ++q) out[q] = q < n ? (uint16_t)kj[q] : (uint16_t)0xFFFFu;
}

__global__ void mark_kernel(const KnnArgs a) {
    const uint32_t r = blockIdx.y;
    const int64_t m0 = a.mass_off[r];
    const uint32_t m = (uint32_t)(a.mass_off[r + 1] - m0), words = (m + 31) / 32;
    uint32_t* bits = a.bits + a.bit_off[r];
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m * a.k; e += gridDim.x * blockDim.x) {
        const uint32_t i = e / a.k, j = a.nn[(size_t)m0 * a.k + e];
        if (j == 0xFFFFu) continue;
        const uint32_t lo = min(i, j), hi = max(i, j);
        atomicOr(&bits[(size_t)lo * words + hi / 32], 1u << (hi % 32));
    }
}

__global__ void count_kernel(const KnnArgs a) {
    const uint32_t r = blockIdx.y;
    const int64_t m0 = a.mass_off[r];
    const uint32_t m = (uint32_t)(a.mass_off[r + 1] - m0), words = (m + 31) / 32;
    const uint32_t* bits = a.bits + a.bit_off[r];
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < m; row += gridDim.x * blockDim.x) {
        uint32_t c = 0;
        for (uint32_t w = 0; w < words; ++w) c += __popc(bits[(size_t)row * words + w]);
        a.row_count[m0 + row] = c;
    }
}

struct EmitArgs {
    const float* pos;
    const uint8_t* mass_mat;
    const int64_t* mass_off;
    const uint32_t* bits;
    const uint64_t* bit_off;
    const uint64_t* row_first;  // per mass: first spring of its row (global)
    uint16_t* pairs;            // robot-local indices
    uint8_t* mat;
    float* lbar;
};

__global__ void emit_kernel(const EmitArgs a) {
    const uint32_t r = blockIdx.y;
    const int64_t m0 = a.mass_off[r];
    const uint32_t m = (uint32_t)(a.mass_off[r + 1] - m0), words = (m + 31) / 32;
    const uint32_t* bits = a.bits + a.bit_off[r];
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < m; row += gridDim.x * blockDim.x) {
        uint64_t s = a.row_first[m0 + row];
        const float3 p = make_float3(a.pos[3 * (m0 + row)], a.pos[3 * (m0 + row) + 1], a.pos[3 * (m0 + row) + 2]);
        for (uint32_t w = 0; w < words; ++w) {
            uint32_t v = bits[(size_t)row * words + w];
            while (v) {
                const uint32_t b = w * 32 + (uint32_t)(__ffs(v) - 1);
                v &= v - 1;
                const int64_t g = m0 + b;
                const float3 q = make_float3(a.pos[3 * g], a.pos[3 * g + 1], a.pos[3 * g + 2]);
                a.pairs[2 * s] = (uint16_t)row;
                a.pairs[2 * s + 1] = (uint16_t)b;
                a.lbar[s] = __fsqrt_rn(sqdist(p, q));
                a.mat[s] = (uint8_t)composite_knn(a.mass_mat[m0 + row], a.mass_mat[g]);
                ++s;
            }
        }
    }
}

// Grow-only device buffer, kept between calls.
template <typename T>
struct Dev {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count) {
        if (count <= n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        const size_t c = std::max<size_t>(count, 1);
        const cudaError_t e = cudaMalloc(&p, c * sizeof(T));
        if (e == cudaSuccess) n = c;
        return e;
    }
};

// Scratch and stream of one device, kept for the process: calls reuse them
// (one call at a time per device, under the lock), so a call allocates only
// when it needs more than any earlier one.
struct KnnScratch {
    std::mutex lock;
    cudaStream_t stream = nullptr;
    Dev<float> pos, lbar;
    Dev<uint8_t> mm, mat;
    Dev<int64_t> off;
    Dev<uint16_t> nn, pairs;
    Dev<uint32_t> bits, rc;
    Dev<uint64_t> boff, first;
};

KnnScratch& knn_scratch(int device) {
    static std::mutex registry_lock;
    static std::vector<std::unique_ptr<KnnScratch>> per_device;
    std::lock_guard<std::mutex> g(registry_lock);
    if ((size_t)device >= per_device.size()) per_device.resize(device + 1);
    if (!per_device[device]) per_device[device] = std::make_unique<KnnScratch>();
    return *per_device[device];
}

}  // namespace
}  // namespace mb

extern "C" mb_status mb_knn_springs(int device, uint32_t n_robots, const int64_t* mass_offsets, const float* pos,
                                    const uint8_t* mass_material, uint32_t k, int64_t* spring_offsets,
                                    uint16_t* pairs, uint8_t* spring_material, float* lbar, uint64_t capacity) {
    using namespace mb;
    if (!mass_offsets || !pos || !mass_material || !spring_offsets || n_robots == 0) return MB_ERR_ARGUMENT;
    if (k == 0 || k > kKnnMaxK || mass_offsets[0] != 0) return MB_ERR_ARGUMENT;
    uint32_t max_m = 0;
    std::vector<uint64_t> bit_off(n_robots + 1, 0);
    for (uint32_t r = 0; r < n_robots; ++r) {
        if (mass_offsets[r + 1] < mass_offsets[r]) return MB_ERR_ARGUMENT;
        const uint64_t m = (uint64_t)(mass_offsets[r + 1] - mass_offsets[r]);
        if (m > kKnnMaxMasses) return MB_ERR_CAPACITY;
        max_m = std::max<uint32_t>(max_m, (uint32_t)m);
        bit_off[r + 1] = bit_off[r] + m * ((m + 31) / 32);
    }
    const uint64_t M = (uint64_t)mass_offsets[n_robots];
    if (device < 0 || cudaSetDevice(device) != cudaSuccess) return MB_ERR_CUDA;
    KnnScratch& sc = knn_scratch(device);
    std::lock_guard<std::mutex> held(sc.lock);
    if (!sc.stream && cudaStreamCreateWithFlags(&sc.stream, cudaStreamNonBlocking) != cudaSuccess) {
        sc.stream = nullptr;
        return MB_ERR_CUDA;
    }
    cudaStream_t st = sc.stream;
    auto& d_pos = sc.pos;
    auto& d_lbar = sc.lbar;
    auto& d_mm = sc.mm;
    auto& d_mat = sc.mat;
    auto& d_off = sc.off;
    auto& d_nn = sc.nn;
    auto& d_pairs = sc.pairs;
    auto& d_bits = sc.bits;
    auto& d_rc = sc.rc;
    auto& d_boff = sc.boff;
    auto& d_first = sc.first;
#define KNN_CUDA(x)                               \
    do {                                          \
        if ((x) != cudaSuccess) return MB_ERR_CUDA; \
    } while (0)
    KNN_CUDA(d_pos.alloc(3 * M));
    KNN_CUDA(d_mm.alloc(M));
    KNN_CUDA(d_off.alloc(n_robots + 1));
    KNN_CUDA(d_nn.alloc(M * k));
    KNN_CUDA(d_bits.alloc(bit_off[n_robots]));
    KNN_CUDA(d_boff.alloc(n_robots + 1));
    KNN_CUDA(d_rc.alloc(M));
    KNN_CUDA(cudaMemcpyAsync(d_pos.p, pos, 3 * M * sizeof(float), cudaMemcpyHostToDevice, st));
    KNN_CUDA(cudaMemcpyAsync(d_mm.p, mass_material, M, cudaMemcpyHostToDevice, st));
    KNN_CUDA(cudaMemcpyAsync(d_off.p, mass_offsets, (n_robots + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    KNN_CUDA(cudaMemcpyAsync(d_boff.p, bit_off.data(), (n_robots + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    KNN_CUDA(cudaMemsetAsync(d_bits.p, 0, bit_off[n_robots] * sizeof(uint32_t), st));
    const KnnArgs ka{d_pos.p, d_off.p, k, d_nn.p, d_bits.p, d_boff.p, d_rc.p};
    const dim3 grid((max_m + kKnnThreads - 1) / kKnnThreads, n_robots);
    select_kernel<<<grid, kKnnThreads, max_m * sizeof(float3), st>>>(ka);
    mark_kernel<<<grid, kKnnThreads, 0, st>>>(ka);
    count_kernel<<<grid, kKnnThreads, 0, st>>>(ka);
    KNN_CUDA(cudaGetLastError());
    std::vector<uint32_t> rc(M);
    KNN_CUDA(cudaMemcpyAsync(rc.data(), d_rc.p, M * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    KNN_CUDA(cudaStreamSynchronize(st));
    std::vector<uint64_t> first(M);
    uint64_t total = 0;
    spring_offsets[0] = 0;
    for (uint32_t r = 0; r < n_robots; ++r) {
        for (int64_t i = mass_offsets[r]; i < mass_offsets[r + 1]; ++i) {
            first[i] = total;
            total += rc[i];
        }
        spring_offsets[r + 1] = (int64_t)total;
    }
    if (!pairs) return MB_OK;  // counting call
    if (total > capacity || !spring_material || !lbar) return MB_ERR_CAPACITY;
    KNN_CUDA(d_first.alloc(M));
    KNN_CUDA(d_pairs.alloc(2 * total));
    KNN_CUDA(d_mat.alloc(total));
    KNN_CUDA(d_lbar.alloc(total));
    KNN_CUDA(cudaMemcpyAsync(d_first.p, first.data(), M * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    const EmitArgs ea{d_pos.p, d_mm.p, d_off.p, d_bits.p, d_boff.p, d_first.p, d_pairs.p, d_mat.p, d_lbar.p};
    emit_kernel<<<grid, kKnnThreads, 0, st>>>(ea);
    KNN_CUDA(cudaGetLastError());
    KNN_CUDA(cudaMemcpyAsync(pairs, d_pairs.p, 2 * total * sizeof(uint16_t), cudaMemcpyDeviceToHost, st));
    KNN_CUDA(cudaMemcpyAsync(spring_material, d_mat.p, total, cudaMemcpyDeviceToHost, st));
    KNN_CUDA(cudaMemcpyAsync(lbar, d_lbar.p, total * sizeof(float), cudaMemcpyDeviceToHost, st));
    KNN_CUDA(cudaStreamSynchronize(st));
#undef KNN_CUDA
    return MB_OK;
}
