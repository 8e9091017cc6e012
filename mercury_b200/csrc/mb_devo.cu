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

// ---------------------------------------------------------------------------
// Re-packing on the device (see mb_devo.h).

namespace mb {
namespace {

constexpr uint32_t kRebuildThreads = 512;
constexpr uint32_t kRebuildMaxMass = 4096;
constexpr uint32_t kRebuildMaxSlices = kRebuildMaxMass / kSliceWidth;
constexpr uint32_t kRowLocal = 48;  // rows up to this length are sorted in registers/local memory

__global__ void pslot_kernel(const uint32_t* __restrict__ gidx, uint32_t n_packed, uint32_t n_springs,
                             uint32_t* __restrict__ pslot) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n_packed; q += gridDim.x * blockDim.x) {
        const uint32_t g = gidx[q];
        if (g < n_springs) pslot[g] = q;
    }
}

__global__ void apply_kernel(const DevoApplyParams p, int pass) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n_rec) return;
    const DevoRecord rec = p.rec[i];
    if (rec.spring == 0xFFFFFFFFu) return;
    const uint32_t g = rec.spring, r = i / p.k;
    const uint32_t old_mat = p.spring_mat[g], new_mat = rec.material;
    const bool take = old_mat == 0 && new_mat != 0;  // an air spring stops being air
    if ((pass == 1) != take) return;
    const uint32_t a = rec.pair & 0xFFFFu, b = rec.pair >> 16;
    p.pairs[2 * (size_t)g] = (uint16_t)a;
    p.pairs[2 * (size_t)g + 1] = (uint16_t)b;
    p.spring_mat[g] = (uint8_t)new_mat;
    p.lbar[g] = rec.lbar;
    const uint32_t bin = p.robot_bin[r];
    const uint32_t first = p.bins[bin].spring_begin;
    uint32_t slot = p.pslot[g];
    if (new_mat == 0) {  // becomes (or stays) air: its slot turns inert
        if (slot != kNoSlot) {
            p.spring_gidx[slot] = p.inert;
            p.pslot[g] = kNoSlot;
            const uint32_t c = atomicAdd(&p.free_count[bin], 1u);
            p.free_slots[first + c] = slot;
        }
        return;
    }
    if (take) {
        const uint32_t t = atomicAdd(&p.free_taken[bin], 1u), c = p.free_count[bin];
        if (t >= c) {
            atomicAdd(&p.status[0], 1u);
            return;
        }
        slot = p.free_slots[first + c - 1 - t];
        p.spring_gidx[slot] = g;
        p.pslot[g] = slot;
    }
    const uint32_t ms = p.slot_of[new_mat];
    if (ms == kNoMatSlot || slot == kNoSlot) {
        atomicAdd(&p.status[0], 1u);
        return;
    }
    const uint32_t base = p.robot_mass_base[r];
    p.spring_pair[slot] = (base + a) | ((base + b) << 12) | (ms << 24);
    p.spring_lbar[slot] = rec.lbar;
}

__global__ void relayout_kernel(const BinDesc* __restrict__ old_bins, const uint32_t* __restrict__ new_begin,
                                const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, uint32_t eb) {
    const BinDesc bd = old_bins[blockIdx.x];
    const size_t from = (size_t)bd.inc_begin * eb, to = (size_t)new_begin[blockIdx.x] * eb;
    for (size_t i = threadIdx.x; i < (size_t)bd.n_inc * eb; i += blockDim.x) dst[to + i] = src[from + i];
}

// Row entries while rebuilding: key of the other end << 47 | spring index
// (upload order) << 16 | (1 at the b end) << 15 | packed slot in the bin.
// The key is the bin-local index of a resident bin's mass (robots are
// contiguous and in order inside a bin) and the robot-local index in a split
// part (whose halo masses are numbered after its own), so sorting entries
// sorts every row into the summation order (other end, spring, a end first).
constexpr uint32_t kKeyOffset = 1u << 16;  // keys are < 65536
__device__ __forceinline__ uint32_t row_other(unsigned long long e) { return (uint32_t)(e >> 47); }

// Exclusive scan of v[0..n) in place (n <= kRebuildMaxMass); returns the total.
__device__ uint32_t block_scan(uint32_t* v, uint32_t n, uint32_t* warp_tot) {
    constexpr uint32_t kPer = kRebuildMaxMass / kRebuildThreads;  // 8 entries per thread
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t loc[kPer], sum = 0;
#pragma unroll
    for (uint32_t j = 0; j < kPer; ++j) {
        const uint32_t i = tid * kPer + j;
        loc[j] = i < n ? v[i] : 0u;
        sum += loc[j];
    }
    uint32_t incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += x;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t nw = kRebuildThreads / 32;
        uint32_t t = lane < nw ? warp_tot[lane] : 0u, ti = t;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= (uint32_t)o) ti += x;
        }
        if (lane < nw) warp_tot[lane] = ti - t;  // exclusive
        if (lane == nw - 1) warp_tot[nw] = ti;   // total
    }
    __syncthreads();
    uint32_t run = warp_tot[warp] + incl - sum;
#pragma unroll
    for (uint32_t j = 0; j < kPer; ++j) {
        const uint32_t i = tid * kPer + j;
        if (i < n) v[i] = run;
        run += loc[j];
    }
    const uint32_t total = warp_tot[kRebuildThreads / 32];
    __syncthreads();
    return total;
}

__global__ void __launch_bounds__(kRebuildThreads) rebuild_kernel(const RebuildParams p) {
    __shared__ uint32_t start[kRebuildMaxMass + 1];
    __shared__ uint32_t cur[kRebuildMaxMass];
    __shared__ uint32_t swidth[kRebuildMaxSlices], soff[kRebuildMaxSlices];
    __shared__ uint32_t warp_tot[kRebuildThreads / 32 + 1];
    __shared__ uint32_t s_total;
    const uint32_t b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const BinDesc bd = p.bins[b];
    const uint32_t nm = bd.n_mass, ns = bd.n_spring, cap = bd.row_cap;
    // split parts: keys of their local masses (own, then halo); resident
    // bins: the local index itself
    const uint32_t* keys = p.keys ? p.keys + p.key_begin[b] : nullptr;
    auto key_of = [&](uint32_t local) { return keys ? keys[local] : local; };
    if (tid == 0) {  // the free list after this call's takes
        const uint32_t c = p.free_count[b], t = p.free_taken[b];
        p.free_count[b] = c - min(t, c);
        p.free_taken[b] = 0;
    }
    if (nm > kRebuildMaxMass || ns > kMaxBinSprings) {
        if (tid == 0) atomicAdd(&p.status[0], 1u);
        return;
    }
    // 1. degrees (rows exist for the bin's own masses only)
    for (uint32_t i = tid; i < nm; i += kRebuildThreads) start[i] = 0;
    __syncthreads();
    for (uint32_t j = tid; j < ns; j += kRebuildThreads) {
        const uint32_t q = bd.spring_begin + j;
        if (p.spring_gidx[q] == p.inert) continue;
        const uint32_t w = p.spring_pair[q], a = w & 0xFFFu, c = (w >> 12) & 0xFFFu;
        if (a < nm) atomicAdd(&start[a], 1u);
        if (c < nm) atomicAdd(&start[c], 1u);
    }
    __syncthreads();
    // 2. row starts
    const uint32_t n_ent = block_scan(start, nm, warp_tot);
    if (tid == 0) start[nm] = n_ent;
    for (uint32_t i = tid; i < nm; i += kRebuildThreads) cur[i] = start[i];
    __syncthreads();
    // 3. entries: key of the other end << 47 | spring << 16 | (b end) << 15 | packed slot
    unsigned long long* rows = p.rows + 2ull * bd.spring_begin;
    for (uint32_t j = tid; j < ns; j += kRebuildThreads) {
        const uint32_t q = bd.spring_begin + j, gw = p.spring_gidx[q];
        if (gw == p.inert) continue;
        const uint32_t w = p.spring_pair[q], a = w & 0xFFFu, c = (w >> 12) & 0xFFFu;
        const unsigned long long sg = (unsigned long long)(gw & 0x7FFFFFFFu) << 16;  // bit 31: a split copy
        if (a < nm) rows[atomicAdd(&cur[a], 1u)] = ((unsigned long long)key_of(c) << 47) | sg | j;
        if (c < nm) rows[atomicAdd(&cur[c], 1u)] = ((unsigned long long)key_of(a) << 47) | sg | (1ull << 15) | j;
    }
    __syncthreads();
    // 4. summation order within each row
    for (uint32_t i = tid; i < nm; i += kRebuildThreads) {
        unsigned long long* r = rows + start[i];
        const uint32_t len = start[i + 1] - start[i];
        if (len <= kRowLocal) {
            unsigned long long loc[kRowLocal];
            for (uint32_t x = 0; x < len; ++x) {
                const unsigned long long e = r[x];
                uint32_t y = x;
                while (y > 0 && loc[y - 1] > e) {
                    loc[y] = loc[y - 1];
                    --y;
                }
                loc[y] = e;
            }
            for (uint32_t x = 0; x < len; ++x) r[x] = loc[x];
        } else {
            for (uint32_t x = 1; x < len; ++x) {
                const unsigned long long e = r[x];
                uint32_t y = x;
                while (y > 0 && r[y - 1] > e) {
                    r[y] = r[y - 1];
                    --y;
                }
                r[y] = e;
            }
        }
    }
    __syncthreads();
    // 5. slice widths: aligned by neighbour offset when every row of the
    //    slice has distinct other ends and the union of offsets is at most 4
    //    columns wider than the longest row (the host packer's rule)
    const uint32_t n_sl = (nm + kSliceWidth - 1) / kSliceWidth;
    for (uint32_t sl = warp; sl < n_sl; sl += kRebuildThreads / 32) {
        const uint32_t i = sl * kSliceWidth + lane;
        const uint32_t r0 = i < nm ? start[i] : 0u, r1 = i < nm ? start[i + 1] : 0u;
        uint32_t w_rank = r1 - r0;
        for (int o = 16; o; o >>= 1) w_rank = max(w_rank, __shfl_xor_sync(0xffffffffu, w_rank, o));
        bool mine = true;
        for (uint32_t q = r0 + 1; q < r1; ++q) mine &= row_other(rows[q]) != row_other(rows[q - 1]);
        bool aligned = __all_sync(0xffffffffu, mine);
        uint32_t u = 0;
        if (aligned) {
            uint32_t h = r0;
            while (true) {
                const uint32_t head =
                    h < r1 ? row_other(rows[h]) + kKeyOffset - (i < nm ? key_of(i) : 0u) : 0xFFFFFFFFu;
                const uint32_t m = __reduce_min_sync(0xffffffffu, head);
                if (m == 0xFFFFFFFFu) break;
                if (head == m) ++h;
                if (++u > w_rank + 4) break;
            }
            aligned = u <= w_rank + 4;
        }
        if (lane == 0) swidth[sl] = aligned ? (u | 0x80000000u) : w_rank;
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t off = 0;
        for (uint32_t sl = 0; sl < n_sl; ++sl) {
            soff[sl] = off;
            off += kSliceWidth * (swidth[sl] & 0x7FFFFFFFu);
        }
        s_total = off;
    }
    __syncthreads();
    const uint32_t n_inc = s_total;
    if (n_inc > cap) {
        if (tid == 0) atomicAdd(&p.status[0], 1u);
        return;
    }
    // 6. write the slices
    for (uint32_t sl = tid; sl < n_sl; sl += kRebuildThreads) {
        p.slice_off[bd.slice_begin + sl] = soff[sl];
        p.slice_width[bd.slice_begin + sl] = swidth[sl] & 0x7FFFFFFFu;
    }
    for (uint32_t e = tid; e < n_inc; e += kRebuildThreads) {
        if (p.streamed)
            p.inc32[bd.inc_begin + e] = kPadEntry32;
        else
            p.inc[bd.inc_begin + e] = kPadEntry;
    }
    __syncthreads();
    for (uint32_t sl = warp; sl < n_sl; sl += kRebuildThreads / 32) {
        const uint32_t i = sl * kSliceWidth + lane;
        const uint32_t r0 = i < nm ? start[i] : 0u, r1 = i < nm ? start[i + 1] : 0u;
        const bool aligned = (swidth[sl] & 0x80000000u) != 0;
        const uint32_t base = bd.inc_begin + soff[sl] + lane;
        auto put = [&](uint32_t col, unsigned long long e) {
            const uint32_t v = ((uint32_t)(e & 0x7FFFu) << 1) | (uint32_t)((e >> 15) & 1u);
            if (p.streamed)
                p.inc32[base + col * kSliceWidth] = v;
            else
                p.inc[base + col * kSliceWidth] = (uint16_t)v;
        };
        if (aligned) {
            uint32_t h = r0, col = 0;
            while (true) {
                const unsigned long long e = h < r1 ? rows[h] : 0ull;
                const uint32_t head = h < r1 ? row_other(e) + kKeyOffset - key_of(i) : 0xFFFFFFFFu;
                const uint32_t m = __reduce_min_sync(0xffffffffu, head);
                if (m == 0xFFFFFFFFu) break;
                if (head == m) {
                    put(col, e);
                    ++h;
                }
                ++col;
            }
        } else {
            for (uint32_t q = r0; q < r1; ++q) put(q - r0, rows[q]);
        }
    }
    if (tid == 0) {
        p.bins[b].n_inc = n_inc;
        if (keys)
            atomicMax(&p.status[1], split_smem_bytes(bd.x_stride, ns, n_inc, bd.n_export));
        else if (!p.streamed)
            atomicMax(&p.status[1], bin_smem_bytes_dev(nm, ns, n_inc) + face_smem_bytes(nm, bd.n_face, bd.n_face_inc));
    }
}

// --- development of split robots -------------------------------------------

constexpr uint32_t kPending = 0xFFFFFFFEu;  // map: a halo mass a part needs, not numbered yet
constexpr uint32_t kSplitThreads = 256;

__device__ __forceinline__ uint32_t part_of_mass(const SplitDevoParams& p, uint32_t r, uint32_t m) {
    return p.part_of[p.mass_off[r] + m];
}

// Own masses of each bin into its map and keys; the spring slots beyond the
// packed ones become the free list (the lowest slot last, so taken first).
__global__ void __launch_bounds__(kSplitThreads) split_setup_bins_kernel(const SplitDevoParams p) {
    const uint32_t b = blockIdx.x, tid = threadIdx.x;
    const uint32_t r = p.bin_robot[b];
    const BinDesc bd = p.bins[b];
    const uint32_t cap = p.spring_cap[b];
    const uint32_t n_free = cap - bd.n_spring;
    for (uint32_t i = tid; i < n_free; i += kSplitThreads) {
        const uint32_t slot = cap - 1 - i, q = bd.spring_begin + slot;
        p.free_slots[bd.spring_begin + i] = slot;
        p.spring_gidx[q] = p.inert;
        p.spring_pair[q] = 0;
        p.spring_lbar[q] = 0.0f;
    }
    if (tid == 0) {
        p.free_count[b] = n_free;
        p.free_taken[b] = 0;
    }
    if (r == kNoSlot) return;
    const int64_t m0 = p.mass_off[r];
    uint32_t* map = p.map + p.map_begin[b];
    uint32_t* keys = p.keys + p.key_begin[b];
    for (uint32_t i = tid; i < bd.n_mass; i += kSplitThreads) {
        const uint32_t m = (uint32_t)(p.mass_gidx[bd.mass_begin + i] - m0);
        map[m] = i;
        keys[i] = m;
    }
}

// Halo masses of every bin from the export lists of the parts that own them.
__global__ void __launch_bounds__(kSplitThreads) split_setup_halo_kernel(const SplitDevoParams p) {
    const uint32_t q = blockIdx.x, tid = threadIdx.x;
    const uint32_t r = p.bin_robot[q];
    if (r == kNoSlot) return;
    const BinDesc bd = p.bins[q];
    const int64_t m0 = p.mass_off[r];
    const uint32_t cluster_first = p.robot_bin[r] - p.robot_slot0[r];
    for (uint32_t i = tid; i < bd.n_export; i += kSplitThreads) {
        const uint32_t e = p.exports[bd.export_begin + i];
        const uint32_t li = e & 0xFFFu, rank = (e >> 12) & 7u, slot = e >> 15;
        const uint32_t dst = cluster_first + rank;
        if (dst >= p.n_bins || p.bin_robot[dst] != r || li >= bd.n_mass) {
            atomicAdd(&p.status[0], 1u);
            continue;
        }
        const uint32_t m = (uint32_t)(p.mass_gidx[bd.mass_begin + li] - m0);
        p.map[p.map_begin[dst] + m] = slot;
        p.keys[p.key_begin[dst] + slot] = m;
    }
}

// The slot of every spring in the part of each of its ends.
__global__ void __launch_bounds__(kSplitThreads) split_setup_slots_kernel(const SplitDevoParams p) {
    const uint32_t b = blockIdx.x, tid = threadIdx.x;
    const uint32_t r = p.bin_robot[b];
    if (r == kNoSlot) return;
    const BinDesc bd = p.bins[b];
    const uint32_t part = b - p.robot_bin[r];
    for (uint32_t j = tid; j < bd.n_spring; j += kSplitThreads) {
        const uint32_t gw = p.spring_gidx[bd.spring_begin + j];
        if (gw == p.inert) continue;
        const uint32_t g = gw & 0x7FFFFFFFu;
        const uint32_t a = p.pairs[2 * (size_t)g], c = p.pairs[2 * (size_t)g + 1];
        if (part_of_mass(p, r, a) == part) p.slot_a[g] = j;
        if (part_of_mass(p, r, c) == part) p.slot_b[g] = j;
    }
}

// Pass 0 frees the slots of parts a spring leaves (it becomes air, or no end
// stays in the part); pass 1 keeps or takes a slot in every part that holds
// one of its new ends and marks the halo masses those parts now need.
__global__ void split_apply_kernel(const SplitDevoParams p, int pass) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n_rec) return;
    const DevoRecord rec = p.rec[i];
    if (rec.spring == 0xFFFFFFFFu) return;
    const uint32_t g = rec.spring, r = i / p.k, fb = p.robot_bin[r];
    const uint32_t a0 = p.pairs[2 * (size_t)g], b0 = p.pairs[2 * (size_t)g + 1], mo = p.spring_mat[g];
    const uint32_t a1 = rec.pair & 0xFFFFu, b1 = rec.pair >> 16, mn = rec.material;
    const uint32_t pa0 = part_of_mass(p, r, a0), pb0 = part_of_mass(p, r, b0);
    const uint32_t pa1 = part_of_mass(p, r, a1), pb1 = part_of_mass(p, r, b1);
    const uint32_t sa = p.slot_a[g], sb = p.slot_b[g];
    auto in_old = [&](uint32_t q) { return mo != 0 && (q == pa0 || q == pb0); };
    auto in_new = [&](uint32_t q) { return mn != 0 && (q == pa1 || q == pb1); };
    auto old_slot = [&](uint32_t q) { return q == pa0 ? sa : sb; };
    if (pass == 0) {
        const uint32_t qs[2] = {pa0, pb0};
        for (int k = 0; k < 2; ++k) {
            const uint32_t q = qs[k];
            if (mo == 0 || (k == 1 && q == pa0) || in_new(q)) continue;
            const uint32_t slot = old_slot(q), bin = fb + q;
            if (slot == kNoSlot) {
                atomicAdd(&p.status[0], 1u);
                continue;
            }
            const uint32_t first = p.bins[bin].spring_begin;
            p.spring_gidx[first + slot] = p.inert;
            p.free_slots[first + atomicAdd(&p.free_count[bin], 1u)] = slot;
        }
        return;
    }
    uint32_t nsa = kNoSlot, nsb = kNoSlot;
    if (mn != 0) {
        const uint32_t qs[2] = {pa1, pb1};
        for (int k = 0; k < 2; ++k) {
            const uint32_t q = qs[k];
            if (k == 1 && q == pa1) {
                nsb = nsa;
                continue;
            }
            const uint32_t bin = fb + q;
            uint32_t slot;
            if (in_old(q)) {
                slot = old_slot(q);
            } else {
                const uint32_t t = atomicAdd(&p.free_taken[bin], 1u), c = p.free_count[bin];
                if (t >= c) {
                    atomicAdd(&p.status[0], 1u);
                    slot = kNoSlot;
                } else {
                    slot = p.free_slots[p.bins[bin].spring_begin + c - 1 - t];
                }
            }
            (k == 0 ? nsa : nsb) = slot;
            // ends the part does not own join its halo
            uint32_t* map = p.map + p.map_begin[bin];
            if (pa1 != q) atomicCAS(&map[a1], kNoSlot, kPending);
            if (pb1 != q) atomicCAS(&map[b1], kNoSlot, kPending);
        }
    }
    p.slot_a[g] = nsa;
    p.slot_b[g] = nsb;
}

// Numbers the halo masses each bin now needs (after its local masses, in
// robot order) and appends their export entries to the parts that own them.
__global__ void __launch_bounds__(kSplitThreads) split_halo_kernel(const SplitDevoParams p) {
    __shared__ uint32_t warp_cnt[kSplitThreads / 32];
    __shared__ uint32_t s_base;
    const uint32_t b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t r = p.bin_robot[b];
    if (r == kNoSlot) return;
    const uint32_t fb = p.robot_bin[r], rank = p.robot_slot0[r] + (b - fb);
    const uint32_t nm = (uint32_t)(p.mass_off[r + 1] - p.mass_off[r]);
    const uint32_t cap_x = p.bins[b].x_stride;
    uint32_t* map = p.map + p.map_begin[b];
    uint32_t* keys = p.keys + p.key_begin[b];
    if (tid == 0) s_base = p.bins[b].n_all;
    __syncthreads();
    for (uint32_t base = 0; base < nm; base += kSplitThreads) {
        const uint32_t m = base + tid;
        const bool need = m < nm && map[m] == kPending;
        const uint32_t bal = __ballot_sync(0xffffffffu, need);
        if (lane == 0) warp_cnt[warp] = __popc(bal);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t w = 0; w < kSplitThreads / 32; ++w) {
            before += w < warp ? warp_cnt[w] : 0u;
            total += warp_cnt[w];
        }
        const uint32_t local = s_base + before + __popc(bal & ((1u << lane) - 1u));
        if (need) {
            if (local >= cap_x) {
                atomicAdd(&p.status[0], 1u);
                map[m] = kNoSlot;
            } else {
                map[m] = local;
                keys[local] = m;
                const uint32_t ob = fb + part_of_mass(p, r, m);
                const uint32_t li = p.map[p.map_begin[ob] + m];
                const uint32_t x = atomicAdd(&p.bins[ob].n_export, 1u);
                if (li >= 4096u || x >= p.export_cap[ob])
                    atomicAdd(&p.status[0], 1u);
                else
                    p.exports[p.bins[ob].export_begin + x] = li | (rank << 12) | (local << 15);
            }
        }
        __syncthreads();
        if (tid == 0) s_base += total;
        __syncthreads();
    }
    if (tid == 0) p.bins[b].n_all = min(s_base, cap_x);
}

// Writes the packed springs of every part holding a new end, then the
// canonical topology.
__global__ void split_write_kernel(const SplitDevoParams p) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n_rec) return;
    const DevoRecord rec = p.rec[i];
    if (rec.spring == 0xFFFFFFFFu) return;
    const uint32_t g = rec.spring, r = i / p.k, fb = p.robot_bin[r];
    const uint32_t a1 = rec.pair & 0xFFFFu, b1 = rec.pair >> 16, mn = rec.material;
    if (mn != 0) {
        const uint32_t pa1 = part_of_mass(p, r, a1), pb1 = part_of_mass(p, r, b1);
        const uint32_t ms = p.slot_of[mn];
        const uint32_t qs[2] = {pa1, pb1}, slots[2] = {p.slot_a[g], p.slot_b[g]};
        for (int k = 0; k < 2; ++k) {
            const uint32_t q = qs[k];
            if (k == 1 && q == pa1) continue;
            const uint32_t bin = fb + q, slot = slots[k];
            const uint32_t* map = p.map + p.map_begin[bin];
            const uint32_t la = map[a1], lb = map[b1], cap_x = p.bins[bin].x_stride;
            if (slot == kNoSlot || ms == kNoMatSlot || la >= cap_x || lb >= cap_x) {
                atomicAdd(&p.status[0], 1u);
                continue;
            }
            const uint32_t at = p.bins[bin].spring_begin + slot;
            p.spring_pair[at] = la | (lb << 12) | (ms << 24);
            p.spring_lbar[at] = rec.lbar;
            p.spring_gidx[at] = g | (q != pa1 ? 0x80000000u : 0u);  // the part of the a end writes the stress
            atomicMax(&p.bins[bin].n_spring, slot + 1);
        }
    }
    p.pairs[2 * (size_t)g] = (uint16_t)a1;
    p.pairs[2 * (size_t)g + 1] = (uint16_t)b1;
    p.spring_mat[g] = (uint8_t)mn;
    p.lbar[g] = rec.lbar;
}

__global__ void relayout_ranges_kernel(const uint32_t* __restrict__ old_begin, const uint32_t* __restrict__ count,
                                       const uint32_t* __restrict__ new_begin, const uint8_t* __restrict__ src,
                                       uint8_t* __restrict__ dst, uint32_t eb) {
    const size_t from = (size_t)old_begin[blockIdx.x] * eb, to = (size_t)new_begin[blockIdx.x] * eb;
    for (size_t i = threadIdx.x; i < (size_t)count[blockIdx.x] * eb; i += blockDim.x) dst[to + i] = src[from + i];
}

}  // namespace

cudaError_t launch_split_devo_setup(const SplitDevoParams& p, uint32_t n_bins, uint32_t n_springs, cudaStream_t s) {
    if (n_bins == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(p.slot_a, 0xFF, (size_t)n_springs * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(p.slot_b, 0xFF, (size_t)n_springs * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    split_setup_bins_kernel<<<n_bins, kSplitThreads, 0, s>>>(p);
    split_setup_halo_kernel<<<n_bins, kSplitThreads, 0, s>>>(p);
    split_setup_slots_kernel<<<n_bins, kSplitThreads, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_split_devo_apply(const SplitDevoParams& p, uint32_t n_bins, cudaStream_t s) {
    if (p.n_rec == 0) return cudaSuccess;
    const uint32_t grid = (p.n_rec + 255) / 256;
    split_apply_kernel<<<grid, 256, 0, s>>>(p, 0);
    split_apply_kernel<<<grid, 256, 0, s>>>(p, 1);
    split_halo_kernel<<<n_bins, kSplitThreads, 0, s>>>(p);
    split_write_kernel<<<grid, 256, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_relayout_ranges(const uint32_t* old_begin, const uint32_t* count, const uint32_t* new_begin,
                                   uint32_t n_bins, const void* src, void* dst, uint32_t entry_bytes,
                                   cudaStream_t s) {
    if (n_bins == 0) return cudaSuccess;
    relayout_ranges_kernel<<<n_bins, 256, 0, s>>>(old_begin, count, new_begin, static_cast<const uint8_t*>(src),
                                                  static_cast<uint8_t*>(dst), entry_bytes);
    return cudaGetLastError();
}

cudaError_t launch_build_pslot(const uint32_t* spring_gidx, uint32_t n_packed, uint32_t n_springs,
                               uint32_t* pslot, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(pslot, 0xFF, (size_t)n_springs * sizeof(uint32_t), s);
    if (e != cudaSuccess || n_packed == 0) return e;
    pslot_kernel<<<(n_packed + 255) / 256, 256, 0, s>>>(spring_gidx, n_packed, n_springs, pslot);
    return cudaGetLastError();
}

cudaError_t launch_devo_apply(const DevoApplyParams& p, int pass, cudaStream_t s) {
    if (p.n_rec == 0) return cudaSuccess;
    apply_kernel<<<(p.n_rec + 255) / 256, 256, 0, s>>>(p, pass);
    return cudaGetLastError();
}

cudaError_t launch_relayout(const BinDesc* old_bins, const uint32_t* new_begin, uint32_t n_bins,
                            const void* src, void* dst, uint32_t entry_bytes, cudaStream_t s) {
    if (n_bins == 0) return cudaSuccess;
    relayout_kernel<<<n_bins, 256, 0, s>>>(old_bins, new_begin, static_cast<const uint8_t*>(src),
                                           static_cast<uint8_t*>(dst), entry_bytes);
    return cudaGetLastError();
}

// Placement of a resident bin's springs (one warp per bin), the rule of the
// host packer's bank_order: lanes 8q .. 8q + 7 of a warp form one shared-
// memory wavefront of the step kernel's 16-byte endpoint loads, conflict-
// free when their masses differ mod 8.  Each group of 8 slots takes, in
// order, the earliest springs of a window of the next 64 unplaced ones whose
// a and b are both new mod 8 in the group (the first such spring under the
// group's used residues, repeatedly: a spring passed over stays blocked,
// since the used sets only grow), then fills any slot left with the earliest
// unplaced spring.  The window holds positions 0..63 as two per lane
// (lane, lane + 32); picks are found by ballot.  Each chunk of kPlaceChunk
// springs is placed on its own, by one warp (chunks w, w + 16, ... by warp
// w); the loop touches shared memory only (the bin's packed words and the
// slot order); the whole CTA copies the bin in before and permutes the
// three arrays in place after it, gidx and lbar read from the scratch copy.
constexpr uint32_t kPlaceThreads = 512;

__global__ void __launch_bounds__(kPlaceThreads) bank_place_kernel(const BinDesc* __restrict__ bins,
                                                                    uint32_t* pair, uint32_t* gidx, float* lbar,
                                                                    unsigned long long* scratch) {
    extern __shared__ uint32_t sword[];  // the bin's packed words, in upload order; then the slot order (u16)
    __shared__ uint32_t swin[kPlaceThreads / 32][64];  // per warp: bin-local spring indices, window order
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    uint32_t* win = swin[tid >> 5];
    const uint32_t s0 = bins[blockIdx.x].spring_begin, n = bins[blockIdx.x].n_spring;
    uint16_t* sorder = reinterpret_cast<uint16_t*>(sword + n);  // slot -> upload index (n <= kMaxBinSprings)
    uint32_t dyn;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if (n > kMaxBinSprings || (size_t)n * 6u > dyn) return;  // the launch was sized for fewer: left as it is
    for (uint32_t i = tid; i < n; i += kPlaceThreads) {
        sword[i] = pair[s0 + i];
        scratch[s0 + i] = (unsigned long long)gidx[s0 + i] | (unsigned long long)__float_as_uint(lbar[s0 + i]) << 32;
    }
    __syncthreads();
    for (uint32_t c0 = (tid >> 5) * kPlaceChunk; c0 < n; c0 += kPlaceThreads / 32u * kPlaceChunk) {
        const uint32_t c1 = min(n, c0 + kPlaceChunk);
        uint32_t len = 0, next = c0, placed = c0;
        while (placed < c1) {
            const uint32_t add = min(64u - len, c1 - next);
            for (uint32_t k = lane; k < add; k += 32) win[len + k] = next + k;
            __syncwarp();
            len += add;
            next += add;
            const uint32_t want = min(8u, c1 - placed);  // <= len
            const bool v0 = lane < len, v1 = lane + 32u < len;
            const uint32_t i0 = v0 ? win[lane] : 0u, i1 = v1 ? win[lane + 32] : 0u;
            const uint32_t w0 = v0 ? sword[i0] : 0u, w1 = v1 ? sword[i1] : 0u;
            const uint32_t a0 = w0 & 7u, b0 = (w0 >> 12) & 7u, a1 = w1 & 7u, b1 = (w1 >> 12) & 7u;
            // the longest prefix of the window whose residues are pairwise new
            // is what the greedy picks first, one after another: taken at once
            // (both matches run on every lane: a short-circuit would leave lanes
            // out of a full-warp match)
            const uint32_t below_lane = (1u << lane) - 1u;
            const uint32_t same_a = __match_any_sync(0xFFFFFFFFu, a0);
            const uint32_t same_b = __match_any_sync(0xFFFFFFFFu, b0);
            const uint32_t cm = __ballot_sync(0xFFFFFFFFu, lane < want && ((same_a | same_b) & below_lane) != 0u);
            uint32_t got = cm ? (uint32_t)__ffs(cm) - 1u : want;  // >= 1: lane 0 never clashes
            uint32_t ua = __reduce_or_sync(0xFFFFFFFFu, lane < got ? 1u << a0 : 0u);  // residues used, mod 8
            uint32_t ub = __reduce_or_sync(0xFFFFFFFFu, lane < got ? 1u << b0 : 0u);
            unsigned long long picked = (1ull << got) - 1ull;  // bit p: window position p placed in this group
            while (got < want) {
                const uint32_t m0 = __ballot_sync(0xFFFFFFFFu, v0 && !((ua >> a0) & 1u) && !((ub >> b0) & 1u));
                uint32_t p;
                if (m0) {
                    p = (uint32_t)__ffs(m0) - 1u;
                } else {
                    const uint32_t m1 = __ballot_sync(0xFFFFFFFFu, v1 && !((ua >> a1) & 1u) && !((ub >> b1) & 1u));
                    if (!m1) break;
                    p = 31u + (uint32_t)__ffs(m1);
                }
                const uint32_t wp = __shfl_sync(0xFFFFFFFFu, p < 32u ? w0 : w1, p & 31u);
                ua |= 1u << (wp & 7u);
                ub |= 1u << ((wp >> 12) & 7u);
                picked |= 1ull << p;
                ++got;
            }
            const unsigned long long valid = len >= 64u ? ~0ull : (1ull << len) - 1ull;
            for (unsigned long long rest = valid & ~picked; got < want; rest &= rest - 1ull, ++got)
                picked |= rest & (~rest + 1ull);
            // the group in window order into slots placed.., the rest compacted
            const unsigned long long kept = valid & ~picked;
            __syncwarp();  // every lane has read its window entries
            if (v0) {
                const unsigned long long below = (1ull << lane) - 1ull;
                if ((picked >> lane) & 1ull)
                    sorder[placed + (uint32_t)__popcll(picked & below)] = (uint16_t)i0;
                else
                    win[__popcll(kept & below)] = i0;
            }
            if (v1) {
                const unsigned long long below = (1ull << (lane + 32u)) - 1ull;
                if ((picked >> (lane + 32u)) & 1ull)
                    sorder[placed + (uint32_t)__popcll(picked & below)] = (uint16_t)i1;
                else
                    win[__popcll(kept & below)] = i1;
            }
            __syncwarp();
            len -= got;
            placed += got;
        }
    }
    __syncthreads();
    for (uint32_t d = tid; d < n; d += kPlaceThreads) {
        const uint32_t i = sorder[d];
        const unsigned long long x = scratch[s0 + i];
        pair[s0 + d] = sword[i];
        gidx[s0 + d] = (uint32_t)x;
        lbar[s0 + d] = __uint_as_float((uint32_t)(x >> 32));
    }
}

cudaError_t launch_bank_place(const BinDesc* bins, uint32_t n_bins, uint32_t max_springs, uint32_t* pair,
                              uint32_t* gidx, float* lbar, unsigned long long* scratch, cudaStream_t s) {
    if (n_bins == 0 || max_springs == 0) return cudaSuccess;
    if (max_springs > kMaxBinSprings) return cudaErrorInvalidValue;
    // the opt-in covers the static windows too: static + dynamic above 48 KB
    // needs it, so it is set on every launch
    const size_t smem = (size_t)max_springs * (sizeof(uint32_t) + sizeof(uint16_t)) + 4u;
    cudaError_t e = cudaFuncSetAttribute(bank_place_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    bank_place_kernel<<<n_bins, kPlaceThreads, smem, s>>>(bins, pair, gidx, lbar, scratch);
    return cudaGetLastError();
}

cudaError_t launch_rebuild(const RebuildParams& p, cudaStream_t s) {
    if (p.n_bins == 0) return cudaSuccess;
    rebuild_kernel<<<p.n_bins, kRebuildThreads, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace mb
