// Development ("Devo") on the device: per robot, the springs of stress ranks
// [lo, hi) are rewired to random mass pairs (Simulator::Devo,
// Simulator.cu:640-668; replaceSprings, devo_kernel.cu:81-168).
//
// One CTA per robot.  The reference sorts every robot's stresses with a CUB
// segmented radix sort (Simulator.cu:597-631) to use its first k entries;
// here the rank window is found by radix *selection*: every spring gets the
// unique 64-bit key (stress key << 32 | spring index), whose ascending order
// is descending stress with ties by ascending index (the stable sort's
// order), and eight 8-bit histogram passes over the robot's keys find the
// key of a given rank.  The window's keys are then gathered into shared
// memory and ranked among themselves.  Work per robot: 16 passes over its
// stresses (L2-resident) plus O(k^2 / threads) for the final ranking.
//
// Random pairs come from a counter-based generator (SplitMix64's output
// function over seed, robot, rank, draw; Lemire's multiply-shift to [0, m)),
// so the result does not depend on the launch shape.  The arithmetic of the
// new mean length is written with explicit round-to-nearest intrinsics so
// that it is the same on every device and in the CPU restatement.
#include "mb_devo.h"
#include "mb_sin.cuh"

namespace mb {
namespace {

constexpr uint32_t kDevoThreads = 512;

__device__ __forceinline__ uint32_t stress_key(float s) {
    uint32_t u = __float_as_uint(s);
    if (u == 0x80000000u) u = 0;  // -0 ranks with +0
    const uint32_t ord = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ~ord;
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint32_t draw(uint64_t key, uint32_t j, uint32_t n, uint32_t m) {
    const uint64_t u = mix64(key + 0xD1B54A32D192ED03ULL * ((((uint64_t)j << 8) | n) + 1));
    return (uint32_t)(((u >> 32) * (uint64_t)m) >> 32);
}

__device__ __forceinline__ int composite(int m1, int m2) {
    if (m1 == 0 || m2 == 0) return 0;
    const int i = min(m1, m2) - 1, j = max(m1, m2) - 1;
    if (i == j) return i + 1;
    return 23 + i * 21 - i * (i - 1) / 2 + (j - i - 1);
}

struct SelectShared {
    uint32_t hist[256];
    uint64_t prefix;
    uint32_t want;
};

// Key of rank q (0-based, q < n) among the robot's n keys.
__device__ uint64_t select_rank(const float* __restrict__ st, uint32_t n, uint32_t q, SelectShared& sh) {
    uint64_t prefix = 0;
    uint32_t want = q;
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (uint32_t i = tid; i < 256; i += blockDim.x) sh.hist[i] = 0;
        __syncthreads();
        const uint64_t hi_mask = shift == 56 ? 0ull : (~0ull << (shift + 8));
        for (uint32_t i = tid; i < n; i += blockDim.x) {
            const uint64_t key = ((uint64_t)stress_key(__ldg(&st[i])) << 32) | i;
            if ((key & hi_mask) == prefix) atomicAdd(&sh.hist[(key >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (tid < 32) {
            // lane l owns buckets 8l .. 8l+7
            uint32_t c[8], sum = 0;
            for (int b = 0; b < 8; ++b) {
                c[b] = sh.hist[8 * lane + b];
                sum += c[b];
            }
            uint32_t incl = sum;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += v;
            }
            const uint32_t excl = incl - sum;
            const bool mine = excl <= want && want < incl;
            if (mine) {
                uint32_t cum = excl;
                for (int b = 0; b < 8; ++b) {
                    if (want < cum + c[b]) {
                        sh.prefix = prefix | ((uint64_t)(8 * lane + b) << shift);
                        sh.want = want - cum;
                        break;
                    }
                    cum += c[b];
                }
            }
        }
        __syncthreads();
        prefix = sh.prefix;
        want = sh.want;
        __syncthreads();
    }
    return prefix;
}

__global__ void __launch_bounds__(kDevoThreads) devo_kernel(DevoParams p) {
    __shared__ SelectShared sh;
    __shared__ uint64_t sel[kDevoMaxReplaced];
    __shared__ uint32_t order[kDevoMaxReplaced];
    __shared__ uint32_t n_sel;
    const uint32_t r = blockIdx.x, tid = threadIdx.x;
    const int64_t m0 = p.mass_off[r], s0 = p.spring_off[r];
    const uint32_t m = (uint32_t)(p.mass_off[r + 1] - m0), n = (uint32_t)(p.spring_off[r + 1] - s0);
    uint64_t lo = 0, hi = p.k < n ? p.k : n;
    if (p.flags & kDevoReferenceRanks) {
        lo = (uint64_t)r * p.k;
        hi = lo + p.k;
        if (lo > n) lo = n;
        if (hi > n) hi = n;
    }
    if (m < 2) hi = lo;
    const uint32_t cnt = (uint32_t)(hi - lo);
    DevoRecord* out = p.out + (size_t)r * p.k;
    for (uint32_t j = cnt + tid; j < p.k; j += blockDim.x) out[j] = DevoRecord{0xFFFFFFFFu, 0u, 0u, 0.0f};
    if (cnt == 0) return;
    const float* st = p.stress + s0;
    const uint64_t key_hi = select_rank(st, n, (uint32_t)hi - 1, sh);
    const uint64_t key_lo = lo ? select_rank(st, n, (uint32_t)lo - 1, sh) : 0ull;
    if (tid == 0) n_sel = 0;
    __syncthreads();
    for (uint32_t i = tid; i < n; i += blockDim.x) {
        const uint64_t key = ((uint64_t)stress_key(__ldg(&st[i])) << 32) | i;
        if (key <= key_hi && (lo == 0 || key > key_lo)) sel[atomicAdd(&n_sel, 1u)] = key;
    }
    __syncthreads();
    for (uint32_t x = tid; x < cnt; x += blockDim.x) {
        const uint64_t kx = sel[x];
        uint32_t rank = 0;
        for (uint32_t y = 0; y < cnt; ++y) rank += sel[y] < kx;
        order[rank] = (uint32_t)kx;
    }
    __syncthreads();
    const uint64_t rkey = mix64(p.seed + 0x9E3779B97F4A7C15ULL * ((uint64_t)r + 1));
    for (uint32_t j = tid; j < cnt; j += blockDim.x) {
        uint32_t a = draw(rkey, j, 0, m), b = draw(rkey, j, 1, m);
        for (uint32_t d = 2; b == a && d < 64; ++d) b = draw(rkey, j, d, m);
        if (b == a) b = (a + 1) % m;
        const int id = composite(p.mass_mat[m0 + a], p.mass_mat[m0 + b]);
        const float4 pa = p.pos[m0 + a], pb = p.pos[m0 + b];
        const float dx = __fsub_rn(pa.x, pb.x), dy = __fsub_rn(pa.y, pb.y), dz = __fsub_rn(pa.z, pb.z);
        const float d = __fsqrt_rn(__fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz))));
        const float4 mat = p.table[id];
        const float arg = __fmaf_rn(mat.z, p.t, mat.w);
        const float sn = (float)sin_cw((double)arg);
        const float den = __fadd_rn(1.0f, __fmul_rn(mat.y, sn));
        out[j] = DevoRecord{(uint32_t)(s0 + order[j]), a | (b << 16), (uint32_t)id, __fdiv_rn(d, den)};
    }
}

}  // namespace

cudaError_t launch_devo(const DevoParams& p, uint32_t n_robots, cudaStream_t s) {
    if (n_robots == 0 || p.k == 0) return cudaSuccess;
    devo_kernel<<<n_robots, kDevoThreads, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace mb
