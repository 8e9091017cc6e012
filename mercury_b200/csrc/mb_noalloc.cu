// Entry point for callers that cannot allocate device memory.
//
// Some hosts of this library may not call cudaMalloc at all: an engine that
// owns every device allocation through its own pool, or a plugin sandbox
// whose memory budget is fixed up front.  mb_simulate_robot_noalloc serves them: the
// caller passes the robot's arrays already on the device, and the packed
// topology the step kernel needs (bin descriptor, packed springs, incidence
// rows) is built on the device inside one fixed scratch array that is part of
// this library's image -- a file-scope __device__ array loaded with the
// module, so it lives on every GPU that loads the library until the process
// exits.  No cudaMalloc, cudaFree or allocating library routine is called.
//
// The scratch array is shared by every call on a device and keeps the last
// call's contents; the build kernel clears what has to start at zero.  Calls
// that overlap on the GPU (two streams, or two host threads) race on it: the
// caller must serialise them.
#include <cstdint>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/mercury_b200.h"
#include "mb_internal.h"

namespace mb {
namespace {

constexpr uint32_t kNaMaxMasses = MB_NOALLOC_MAX_MASSES;
constexpr uint32_t kNaMaxSprings = MB_NOALLOC_MAX_SPRINGS;
constexpr uint32_t kNaMaxIncidence = MB_NOALLOC_MAX_INCIDENCE;
constexpr uint32_t kNaSlices = kNaMaxMasses / kSliceWidth;
constexpr uint32_t kBuildThreads = 1024;
constexpr uint32_t kNaChunk = 128;  // steps per launch: bounds the actuation table

// The step kernel shape used below (1,024 threads x 8 springs x 2 masses)
// must hold the largest robot accepted, and the packed spring word has
// 12-bit mass indices.
static_assert(1024u * 8u >= kNaMaxSprings, "step shape must hold MB_NOALLOC_MAX_SPRINGS springs");
static_assert(1024u * 2u >= kNaMaxMasses, "step shape must hold MB_NOALLOC_MAX_MASSES masses");
static_assert(kNaMaxMasses <= 4096u, "mass indices of packed springs have 12 bits");
static_assert(kNaMaxMasses % kSliceWidth == 0, "whole slices");
// the largest robot accepted fits the 227 KB of shared memory a CTA may use
static_assert(bin_smem_bytes_dev(kNaMaxMasses, kNaMaxSprings, kNaMaxIncidence) <= 227u * 1024u,
              "the step kernel's shared memory at the limits");

// Status bits written by the build kernel.
constexpr uint32_t kNaBadTopology = 1u;  // index or material out of range
constexpr uint32_t kNaTooWide = 2u;      // incidence rows exceed kNaMaxIncidence

// Scratch layout (byte offsets, every region 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffBin = 0;
constexpr size_t kOffStatus = align256(kOffBin + sizeof(BinDesc));
constexpr size_t kOffFlag = align256(kOffStatus + sizeof(uint32_t));
constexpr size_t kOffMassGidx = align256(kOffFlag + sizeof(uint32_t));
constexpr size_t kOffSpringGidx = align256(kOffMassGidx + 4 * kNaMaxMasses);
constexpr size_t kOffSpringPair = align256(kOffSpringGidx + 4 * kNaMaxSprings);
constexpr size_t kOffLbar = align256(kOffSpringPair + 4 * kNaMaxSprings);
constexpr size_t kOffSliceOff = align256(kOffLbar + 4 * kNaMaxSprings);
constexpr size_t kOffSliceWidth = align256(kOffSliceOff + 4 * kNaSlices);
constexpr size_t kOffMatIds = align256(kOffSliceWidth + 4 * kNaSlices);
constexpr size_t kOffNMat = align256(kOffMatIds + kMaxMaterialSlots);
constexpr size_t kOffInvK = align256(kOffNMat + sizeof(uint32_t));
constexpr size_t kOffRates = align256(kOffInvK + 4 * kMaxMaterialSlots);
constexpr size_t kOffRowStart = align256(kOffRates + 4 * kMaxMaterialSlots * kNaChunk);
constexpr size_t kOffRows = align256(kOffRowStart + 4 * (kNaMaxMasses + 1));
constexpr size_t kOffInc = align256(kOffRows + 4 * 2 * kNaMaxSprings);
constexpr size_t kScratchBytes = align256(kOffInc + 2 * kNaMaxIncidence);

// The scratch array itself.  In host code `g_noalloc_scratch` names a host
// shadow, not device memory; its device address comes from
// cudaGetSymbolAddress (scratch_address below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct BuildArgs {
    uint32_t n_mass;
    uint32_t n_spring;
    const uint16_t* pairs;
    const uint8_t* mat;
    const float* lbar;
    unsigned char* scratch;
};

// Exclusive block scan of one value per thread (kBuildThreads threads);
// returns the exclusive prefix and writes the total to *total.
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_tmp, uint32_t* total) {
    const uint32_t tid = threadIdx.x;
    s_tmp[tid] = v;
    __syncthreads();
    for (uint32_t off = 1; off < kBuildThreads; off <<= 1) {
        const uint32_t add = tid >= off ? s_tmp[tid - off] : 0u;
        __syncthreads();
        s_tmp[tid] += add;
        __syncthreads();
    }
    const uint32_t incl = s_tmp[tid];
    *total = s_tmp[kBuildThreads - 1];
    __syncthreads();
    return incl - v;
}

// Builds the one-bin packed topology of a robot in the scratch array, in
// the layout and summation order the step kernel expects: non-air springs
// in their original order, per-mass rows sorted by (other end, spring index,
// a end first), rows stored 32 masses per slice (SELL-32).  On a bad input
// the bin descriptor is left empty, so the step kernel does nothing.
__global__ void __launch_bounds__(kBuildThreads) noalloc_build(const BuildArgs a) {
    __shared__ uint32_t s_deg[kNaMaxMasses];
    __shared__ uint32_t s_slot[kMaxMaterialSlots];
    __shared__ uint32_t s_tmp[kBuildThreads];
    __shared__ uint32_t s_status, s_nmat, s_ninc;
    const uint32_t tid = threadIdx.x;
    unsigned char* sc = a.scratch;
    BinDesc* bin = reinterpret_cast<BinDesc*>(sc + kOffBin);
    uint32_t* status = reinterpret_cast<uint32_t*>(sc + kOffStatus);
    uint32_t* flag = reinterpret_cast<uint32_t*>(sc + kOffFlag);
    uint32_t* mass_gidx = reinterpret_cast<uint32_t*>(sc + kOffMassGidx);
    uint32_t* spring_gidx = reinterpret_cast<uint32_t*>(sc + kOffSpringGidx);
    uint32_t* spring_pair = reinterpret_cast<uint32_t*>(sc + kOffSpringPair);
    float* lbar = reinterpret_cast<float*>(sc + kOffLbar);
    uint32_t* slice_off = reinterpret_cast<uint32_t*>(sc + kOffSliceOff);
    uint32_t* slice_width = reinterpret_cast<uint32_t*>(sc + kOffSliceWidth);
    uint8_t* mat_ids = reinterpret_cast<uint8_t*>(sc + kOffMatIds);
    uint32_t* row_start = reinterpret_cast<uint32_t*>(sc + kOffRowStart);
    uint32_t* rows = reinterpret_cast<uint32_t*>(sc + kOffRows);
    uint16_t* inc = reinterpret_cast<uint16_t*>(sc + kOffInc);
    uint32_t* n_mat = reinterpret_cast<uint32_t*>(sc + kOffNMat);

    // clear what must start at zero (the scratch keeps the previous call)
    for (uint32_t i = tid; i < kNaMaxMasses; i += kBuildThreads) s_deg[i] = 0;
    for (uint32_t i = tid; i < kMaxMaterialSlots; i += kBuildThreads) s_slot[i] = 0;
    if (tid == 0) {
        s_status = 0;
        s_nmat = 0;
        s_ninc = 0;
    }
    __syncthreads();

    // validate; mark materials; count non-air springs and degrees
    const uint32_t per = (a.n_spring + kBuildThreads - 1) / kBuildThreads;
    const uint32_t lo = min(tid * per, a.n_spring), hi = min(lo + per, a.n_spring);
    uint32_t cnt = 0;
    for (uint32_t s = lo; s < hi; ++s) {
        const uint32_t p = a.pairs[2 * s], q = a.pairs[2 * s + 1], m = a.mat[s];
        if (p >= a.n_mass || q >= a.n_mass || m >= MB_COMPOSITE_COUNT) {
            atomicOr(&s_status, kNaBadTopology);
            continue;
        }
        if (m == 0) continue;  // air springs never act
        ++cnt;
        s_slot[m] = 1;
        atomicAdd(&s_deg[p], 1u);
        atomicAdd(&s_deg[q], 1u);
    }
    uint32_t n_act = 0;
    const uint32_t base = block_exclusive_scan(cnt, s_tmp, &n_act);
    if (tid == 0) {  // material slots in ascending composite id
        uint32_t n = 0;
        for (uint32_t m = 0; m < MB_COMPOSITE_COUNT; ++m)
            if (s_slot[m]) {
                mat_ids[n] = (uint8_t)m;
                s_slot[m] = n++;
            }
        s_nmat = n;
        *n_mat = n;
    }
    __syncthreads();

    // packed springs: non-air, original order
    uint32_t k = base;
    for (uint32_t s = lo; s < hi; ++s) {
        const uint32_t p = a.pairs[2 * s], q = a.pairs[2 * s + 1], m = a.mat[s];
        if (p >= a.n_mass || q >= a.n_mass || m >= MB_COMPOSITE_COUNT || m == 0) continue;
        spring_gidx[k] = s;
        spring_pair[k] = p | (q << 12) | (s_slot[m] << 24);
        lbar[k] = a.lbar[s];
        ++k;
    }
    // row starts: two masses per thread
    {
        const uint32_t i0 = 2 * tid, i1 = 2 * tid + 1;
        const uint32_t d0 = i0 < a.n_mass ? s_deg[i0] : 0u, d1 = i1 < a.n_mass ? s_deg[i1] : 0u;
        uint32_t tot = 0;
        const uint32_t b0 = block_exclusive_scan(d0 + d1, s_tmp, &tot);
        if (i0 < a.n_mass) row_start[i0] = b0;
        if (i1 < a.n_mass) row_start[i1] = b0 + d0;
        if (tid == 0) row_start[a.n_mass] = tot;
    }
    for (uint32_t i = tid; i < kNaMaxMasses; i += kBuildThreads) s_deg[i] = 0;  // reuse as fill counters
    __syncthreads();

    // fill rows (arbitrary order), then sort each row by its summation key
    for (uint32_t j = tid; j < n_act; j += kBuildThreads) {
        const uint32_t w = spring_pair[j], p = w & 0xFFFu, q = (w >> 12) & 0xFFFu;
        rows[row_start[p] + atomicAdd(&s_deg[p], 1u)] = j << 1;
        rows[row_start[q] + atomicAdd(&s_deg[q], 1u)] = (j << 1) | 1u;
    }
    __syncthreads();
    for (uint32_t i = tid; i < a.n_mass; i += kBuildThreads) {
        const uint32_t r0 = row_start[i], r1 = row_start[i + 1];
        for (uint32_t x = r0 + 1; x < r1; ++x) {
            const uint32_t e = rows[x];
            const uint32_t we = spring_pair[e >> 1];
            const uint32_t oe = (e & 1u) ? (we & 0xFFFu) : ((we >> 12) & 0xFFFu);
            const uint32_t ge = spring_gidx[e >> 1];
            uint32_t y = x;
            while (y > r0) {
                const uint32_t f = rows[y - 1];
                const uint32_t wf = spring_pair[f >> 1];
                const uint32_t of = (f & 1u) ? (wf & 0xFFFu) : ((wf >> 12) & 0xFFFu);
                const uint32_t gf = spring_gidx[f >> 1];
                const bool after = of != oe ? of > oe : (gf != ge ? gf > ge : (f & 1u) > (e & 1u));
                if (!after) break;
                rows[y] = f;
                --y;
            }
            rows[y] = e;
        }
    }
    __syncthreads();

    // slices: width = longest row of the 32 masses; offsets by prefix sum
    const uint32_t n_slices = (a.n_mass + kSliceWidth - 1) / kSliceWidth;
    if (tid < n_slices) {
        uint32_t w = 0;
        for (uint32_t i = tid * kSliceWidth; i < min(a.n_mass, (tid + 1) * kSliceWidth); ++i)
            w = max(w, row_start[i + 1] - row_start[i]);
        slice_width[tid] = w;
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t off = 0;
        for (uint32_t sl = 0; sl < n_slices; ++sl) {
            slice_off[sl] = off;
            off += kSliceWidth * slice_width[sl];
        }
        s_ninc = off;
        if (off > kNaMaxIncidence) s_status |= kNaTooWide;
    }
    __syncthreads();
    const bool ok = s_status == 0;
    if (ok) {
        for (uint32_t x = tid; x < s_ninc; x += kBuildThreads) inc[x] = kPadEntry;
        __syncthreads();
        for (uint32_t i = tid; i < a.n_mass; i += kBuildThreads) {
            const uint32_t o = slice_off[i / kSliceWidth] + (i % kSliceWidth);
            for (uint32_t x = row_start[i]; x < row_start[i + 1]; ++x)
                inc[o + (x - row_start[i]) * kSliceWidth] = (uint16_t)rows[x];
            mass_gidx[i] = i;
        }
    }
    if (tid == 0) {
        BinDesc d;
        memset(&d, 0, sizeof(d));
        if (ok) {
            d.n_mass = a.n_mass;
            d.n_spring = n_act;
            d.n_inc = s_ninc;
        }
        *bin = d;
        *status = s_status;
        *flag = 0;  // the step kernel ORs bit 0 on a non-finite position
    }
}

// Device address of the scratch array, looked up once per device with the
// device current (the first call on a device).  The address is kept for the
// life of the process, so a device must not be reset (cudaDeviceReset)
// after the first call on it.
std::mutex g_addr_mutex;
unsigned char* g_addr[64] = {};

cudaError_t scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[device];
    return cudaSuccess;
}

}  // namespace
}  // namespace mb

extern "C" mb_status mb_simulate_robot_noalloc(void* stream, const float* table, uint32_t n_masses,
                                               float* pos, float* vel, uint32_t n_springs,
                                               const uint16_t* pairs, const uint8_t* spring_material,
                                               const float* lbar, float* stress, float dt, float t0,
                                               uint32_t steps, int track_stresses, float* t_end) {
    using namespace mb;
    if (!table || !pos || !vel || (n_springs && (!pairs || !spring_material || !lbar)) ||
        (track_stresses && !stress) || !(dt > 0.0f))
        return MB_ERR_ARGUMENT;
    if (n_masses == 0 || n_masses > kNaMaxMasses || n_springs > kNaMaxSprings) return MB_ERR_CAPACITY;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return MB_ERR_CUDA;
    unsigned char* sc = nullptr;
    if (scratch_address(device, &sc) != cudaSuccess) return MB_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    BuildArgs ba{n_masses, n_springs, pairs, spring_material, lbar, sc};
    noalloc_build<<<1, kBuildThreads, 0, st>>>(ba);
    if (cudaGetLastError() != cudaSuccess) return MB_ERR_CUDA;

    // the step kernel of the batched path, on one bin that lives in the scratch
    const KernelShape shape{1024, 8, 2};  // holds kNaMaxSprings springs, kNaMaxMasses masses (asserted above)
    StepParams p{};
    p.bins = reinterpret_cast<const BinDesc*>(sc + kOffBin);
    p.n_bins = 1;
    p.pos = reinterpret_cast<float4*>(pos);
    p.vel = reinterpret_cast<float4*>(vel);
    p.stress = stress;
    p.mass_gidx = reinterpret_cast<const uint32_t*>(sc + kOffMassGidx);
    p.spring_gidx = reinterpret_cast<const uint32_t*>(sc + kOffSpringGidx);
    p.spring_pair = reinterpret_cast<const uint32_t*>(sc + kOffSpringPair);
    p.spring_lbar = reinterpret_cast<const float*>(sc + kOffLbar);
    p.slice_off = reinterpret_cast<const uint32_t*>(sc + kOffSliceOff);
    p.slice_width = reinterpret_cast<const uint32_t*>(sc + kOffSliceWidth);
    p.inc = reinterpret_cast<const uint16_t*>(sc + kOffInc);
    p.n_mat = reinterpret_cast<const uint32_t*>(sc + kOffNMat);
    p.rates = reinterpret_cast<const float*>(sc + kOffRates);
    p.invk = reinterpret_cast<const float*>(sc + kOffInvK);
    p.bin_flags = reinterpret_cast<uint32_t*>(sc + kOffFlag);
    p.dt = dt;
    p.track = track_stresses ? 1u : 0u;
    p.smem_bytes = bin_smem_bytes(n_masses, n_springs, kNaMaxIncidence);
    if (p.smem_bytes > max_step_smem(device)) return MB_ERR_CAPACITY;
    p.mode = kModeXpbd;
    if (prepare_step(shape, kModeXpbd, p.track != 0, p.smem_bytes) != cudaSuccess) return MB_ERR_CUDA;
    float t = t0;
    uint32_t done = 0;
    while (done < steps) {
        const uint32_t n = steps - done < kNaChunk ? steps - done : kNaChunk;
        if (launch_actuation(reinterpret_cast<const float4*>(table),
                             reinterpret_cast<const uint8_t*>(sc + kOffMatIds), p.n_mat, t, dt, n,
                             kModeXpbd, reinterpret_cast<float*>(sc + kOffRates),
                             reinterpret_cast<float*>(sc + kOffInvK), st) != cudaSuccess)
            return MB_ERR_CUDA;
        p.t0 = t;
        p.steps = n;
        if (launch_step(p, shape, st) != cudaSuccess) return MB_ERR_CUDA;
        volatile float v = t;
        for (uint32_t i = 0; i < n; ++i) v = v + dt;
        t = v;
        done += n;
    }
    uint32_t status[2] = {0, 0};
    if (cudaMemcpyAsync(&status[0], sc + kOffStatus, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&status[1], sc + kOffFlag, sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return MB_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MB_ERR_CUDA;
    if (t_end) *t_end = t;
    if (status[0] & kNaBadTopology) return MB_ERR_ARGUMENT;
    if (status[0] & kNaTooWide) return MB_ERR_CAPACITY;
    if (status[1] & 1u) return MB_ERR_NONFINITE;
    return MB_OK;
}
