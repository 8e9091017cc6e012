// Packing of a population into bins (host only; see mb_pack.h).
//
// The reference gives every robot one CTA and pads every robot to the
// largest mass and spring count (Simulator.cu:231-239, 489-494).  Here
// robots keep their own sizes and are grouped into bins, each simulated by
// one CTA; bins are filled largest-robot-first onto the least loaded bin
// (LPT), and the bin count is a whole number of waves (SMs x resident CTAs
// per SM) so that every SM gets the same work.  With two or more waves the
// launch has one CTA per group of bins that runs them one after another,
// and robots are balanced over the groups first (plan_bins_grouped): a
// group's load is what sets its SM's time.  Inside a bin:
//   - masses keep robot order (robot r's masses, then robot r+1's ...);
//   - non-air springs of each robot are sorted by (b - a, a) (for a lattice:
//     one direction, consecutive a), then placed so that the 8 springs of a
//     quarter-warp read distinct bank groups at both ends (bank_order);
//   - every mass gets a row of incident springs sorted by (other end,
//     spring index, a end before b end) -- the fixed summation order -- and
//     rows are stored 32 masses per slice, column-major (SELL-32), with
//     columns aligned by the offset of the other end where possible.
// Robots are preprocessed and bins built in parallel over host threads; the
// result does not depend on the number of threads.
#include "mb_pack.h"

#include <algorithm>
#include <tuple>
#include <climits>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <unistd.h>

namespace mb {

// ---- worker pool ----
//
// Host threads are started once per process and reused: an upload runs
// several parallel loops, and starting 16 threads costs about as much as
// a loop's work.  One loop runs at a time (callers on other host threads
// wait); a loop started from inside a worker, or in a child process
// forked after the pool started (it has no workers), runs on the calling
// thread.  The pool is never torn down: its threads wait on a condition
// variable until the process ends.
namespace {

thread_local bool t_in_pool = false;

class WorkerPool {
  public:
    explicit WorkerPool(unsigned n) : pid_(getpid()) {
        for (unsigned k = 0; k < n; ++k) workers_.emplace_back([this, k] { work(k); });
    }
    unsigned size() const { return (unsigned)workers_.size(); }
    bool usable() const { return getpid() == pid_; }

    void run(uint32_t n, unsigned threads, const std::function<void(uint32_t)>& f) {
        std::lock_guard<std::mutex> one(run_mu_);
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &f;
            n_ = n;
            next_.store(0);
            want_ = std::min<unsigned>(threads - 1, size());
            active_ = want_;
            ++generation_;
        }
        cv_.notify_all();
        t_in_pool = true;
        for (uint32_t i = next_++; i < n; i = next_++) f(i);
        t_in_pool = false;
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [this] { return active_ == 0; });
        job_ = nullptr;
    }

  private:
    void work(unsigned index) {
        t_in_pool = true;
        uint64_t seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return generation_ != seen; });
            seen = generation_;
            if (index >= want_) continue;  // not needed by this loop
            const std::function<void(uint32_t)>& f = *job_;
            const uint32_t n = n_;
            lk.unlock();
            for (uint32_t i = next_++; i < n; i = next_++) f(i);
            lk.lock();
            if (--active_ == 0) done_.notify_one();
        }
    }

    const pid_t pid_;
    std::vector<std::thread> workers_;
    std::mutex run_mu_, mu_;
    std::condition_variable cv_, done_;
    const std::function<void(uint32_t)>* job_ = nullptr;
    std::atomic<uint32_t> next_{0};
    uint32_t n_ = 0;
    unsigned want_ = 0, active_ = 0;
    uint64_t generation_ = 0;
};

WorkerPool& worker_pool() {
    static WorkerPool* pool =
        new WorkerPool(std::max(1u, std::thread::hardware_concurrency()) - 1);  // the caller is the last
    return *pool;
}

}  // namespace

void parallel_for(uint32_t n, unsigned threads, const std::function<void(uint32_t)>& f) {
    if (threads <= 1 || n <= 1 || t_in_pool) {
        for (uint32_t i = 0; i < n; ++i) f(i);
        return;
    }
    WorkerPool& pool = worker_pool();
    if (!pool.usable() || pool.size() == 0) {
        for (uint32_t i = 0; i < n; ++i) f(i);
        return;
    }
    pool.run(n, std::min<unsigned>(threads, n), f);
}

namespace {

struct RobotPack {
    std::vector<uint32_t> springs;  // robot-local indices of non-air springs, packed order
    uint32_t n_mass = 0;
    uint64_t cost = 0;
    uint64_t inc_estimate = 0;
    uint32_t n_face = 0;     // faces with three distinct corners
    uint32_t face_smem = 0;  // shared memory of the face drag, bytes (upper bound)
    uint32_t max_degree = 0;  // most non-air springs at one mass
    uint64_t mats[4] = {0, 0, 0, 0};  // composite ids of its non-air springs (bit set)
    std::string error;
    mb_status status = MB_OK;
};

// Shapes the automatic choice considers, in order of preference: 32 warps
// per SM with about 8-10 springs per thread first.
const KernelShape kAuto[] = {
    {1024, 10, 2}, {1024, 12, 2}, {1024, 8, 2}, {512, 16, 4}, {512, 8, 2},
    {1024, 6, 2},  {1024, 4, 1},  {512, 4, 1},  {256, 8, 2},
};

// Shapes for the parts of split robots, in order of preference: one own mass
// per thread first (fewer registers, no spills at the 64-register cap).
const KernelShape kSplit[] = {{1024, 8, 1}, {1024, 10, 1}, {1024, 8, 2}, {1024, 10, 2}, {1024, 12, 2}};

void preprocess(const mb_batch_desc* b, uint32_t r, RobotPack& p) {
    const int64_t m0 = b->mass_offsets[r], m1 = b->mass_offsets[r + 1];
    const int64_t s0 = b->spring_offsets[r], s1 = b->spring_offsets[r + 1];
    char buf[256];
    if (m1 < m0 || s1 < s0) {
        std::snprintf(buf, sizeof(buf), "offsets decrease at robot %u", r);
        p.error = buf;
        p.status = MB_ERR_ARGUMENT;
        return;
    }
    const int64_t cm = m1 - m0;
    if (cm > 4096) {
        std::snprintf(buf, sizeof(buf), "robot %u has %lld masses (max 4096)", r, (long long)cm);
        p.error = buf;
        p.status = MB_ERR_CAPACITY;
        return;
    }
    for (int64_t i = m0; i < m1; ++i)
        if (b->mass_material[i] > 22) {
            std::snprintf(buf, sizeof(buf), "mass material %u of robot %u out of range", b->mass_material[i], r);
            p.error = buf;
            p.status = MB_ERR_ARGUMENT;
            return;
        }
    std::vector<uint32_t> deg((size_t)cm, 0);
    auto& sp = p.springs;
    sp.reserve((size_t)(s1 - s0));
    for (int64_t s = s0; s < s1; ++s) {
        const uint16_t a = b->pairs[2 * s], c = b->pairs[2 * s + 1];
        if (a >= cm || c >= cm) {
            std::snprintf(buf, sizeof(buf), "spring %lld of robot %u joins mass %u/%u of %lld",
                          (long long)(s - s0), r, a, c, (long long)cm);
            p.error = buf;
            p.status = MB_ERR_ARGUMENT;
            return;
        }
        if (b->spring_material[s] >= MB_COMPOSITE_COUNT) {
            std::snprintf(buf, sizeof(buf), "spring material %u out of range", b->spring_material[s]);
            p.error = buf;
            p.status = MB_ERR_ARGUMENT;
            return;
        }
        if (!std::isfinite(b->lbar[s])) {
            p.error = "non-finite mean length";
            p.status = MB_ERR_ARGUMENT;
            return;
        }
        if (b->spring_material[s] == 0) continue;  // air springs never act (sim_kernel.cu:211)
        p.mats[b->spring_material[s] >> 6] |= 1ull << (b->spring_material[s] & 63);
        sp.push_back((uint32_t)(s - s0));
        deg[a]++;
        deg[c]++;
    }
    // order (b - a, a), ties by spring index: sp is in index order, so two
    // stable counting passes -- by a, then by b - a -- give exactly that
    {
        const size_t n = sp.size();
        const uint32_t nm = (uint32_t)cm;  // a, b < nm, so |b - a| < nm
        std::vector<uint32_t> tmp(n), cnt(2 * (size_t)nm + 1);
        auto pass = [&](const std::vector<uint32_t>& src, std::vector<uint32_t>& dst, uint32_t buckets,
                        auto key) {
            std::fill(cnt.begin(), cnt.begin() + buckets + 1, 0u);
            for (uint32_t x : src) cnt[key(x) + 1]++;
            for (uint32_t k = 0; k < buckets; ++k) cnt[k + 1] += cnt[k];
            for (uint32_t x : src) dst[cnt[key(x)]++] = x;
        };
        auto key_a = [&](uint32_t ls) { return (uint32_t)b->pairs[2 * (s0 + ls)]; };
        auto key_dx = [&](uint32_t ls) {
            return (uint32_t)((int)b->pairs[2 * (s0 + ls) + 1] - (int)b->pairs[2 * (s0 + ls)] + (int)nm);
        };
        pass(sp, tmp, nm, key_a);
        pass(tmp, sp, 2 * nm, key_dx);
    }
    // faces: corners in range, at most kMaxFacesPerMass faces per mass;
    // faces with two equal corners are skipped (sim_kernel.cu:99)
    if (b->faces && b->face_offsets && b->face_offsets[b->n_robots] > 0) {
        const int64_t f0 = b->face_offsets[r], f1 = b->face_offsets[r + 1];
        if (f1 < f0) {
            std::snprintf(buf, sizeof(buf), "face offsets decrease at robot %u", r);
            p.error = buf;
            p.status = MB_ERR_ARGUMENT;
            return;
        }
        std::vector<uint32_t> fdeg((size_t)cm, 0);
        uint32_t nf = 0;
        for (int64_t f = f0; f < f1; ++f) {
            const uint16_t* c = b->faces + 3 * f;
            if (c[0] >= cm || c[1] >= cm || c[2] >= cm) {
                std::snprintf(buf, sizeof(buf), "face %lld of robot %u has a corner out of %lld masses",
                              (long long)(f - f0), r, (long long)cm);
                p.error = buf;
                p.status = MB_ERR_ARGUMENT;
                return;
            }
            if (c[0] == c[1] || c[0] == c[2] || c[1] == c[2]) continue;
            ++nf;
            for (int k = 0; k < 3; ++k)
                if (++fdeg[c[k]] > kMaxFacesPerMass) {
                    std::snprintf(buf, sizeof(buf), "mass %u of robot %u is a corner of more than %u faces",
                                  c[k], r, kMaxFacesPerMass);
                    p.error = buf;
                    p.status = MB_ERR_CAPACITY;
                    return;
                }
        }
        if (nf > kMaxRobotFaces) {
            std::snprintf(buf, sizeof(buf), "robot %u has %u faces (max %u)", r, nf, kMaxRobotFaces);
            p.error = buf;
            p.status = MB_ERR_CAPACITY;
            return;
        }
        p.n_face = nf;
        // velocities and face rows of every mass of a bin that has faces,
        // alignment, the faces (force, corners) and their three incidence
        // entries
        p.face_smem = 16u + 20u * (uint32_t)cm + 30u * nf;
    }
    p.n_mass = (uint32_t)cm;
    p.cost = (uint64_t)sp.size() * 4 + (uint64_t)cm + 2ull * p.n_face;
    uint64_t est = 0;  // incidence entries with rows padded to the slice maximum
    for (int64_t i = 0; i < cm; i += 32) {
        uint32_t w = 0;
        for (int64_t k = i; k < std::min<int64_t>(i + 32, cm); ++k) w = std::max(w, deg[k]);
        est += 32ull * w;
        p.max_degree = std::max(p.max_degree, w);
    }
    p.inc_estimate = est + 64;  // slack for slices straddling robots
}

// LPT assignment of robots to `nb` bins by cost, within the shape's and the
// shared memory's capacity.
// spring_extra (the register-row kernel, when nonzero): the bin must also
// fit that kernel's layout -- the usual one without the rows, 8 bytes of
// alignment, spring_extra bytes per spring.
bool plan_bins(const std::vector<RobotPack>& packs, uint32_t nb, const KernelShape& sh,
               uint32_t smem_cap, std::vector<std::vector<uint32_t>>& plan, uint32_t spring_extra = 0) {
    const uint32_t n = (uint32_t)packs.size();
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return packs[a].cost > packs[b].cost; });
    std::vector<uint64_t> load(nb, 0), bm(nb, 0), bs(nb, 0), bi(nb, 0), bx(nb, 0);
    plan.assign(nb, {});
    const uint64_t cap_s = std::min<uint64_t>((uint64_t)sh.threads * sh.spt, kMaxBinSprings);
    const uint64_t cap_m = std::min<uint64_t>((uint64_t)sh.threads * sh.mpt, 4096);
    for (uint32_t r : order) {
        const auto& p = packs[r];
        int best = -1;
        for (uint32_t b = 0; b < nb; ++b) {
            if (bm[b] + p.n_mass > cap_m || bs[b] + p.springs.size() > cap_s) continue;
            const uint32_t m1 = (uint32_t)(bm[b] + p.n_mass), s1 = (uint32_t)(bs[b] + p.springs.size());
            if (bin_smem_bytes(m1, s1, (uint32_t)(bi[b] + p.inc_estimate)) + bx[b] + p.face_smem > smem_cap ||
                (spring_extra && bin_smem_bytes(m1, s1, 0) + 8u + spring_extra * s1 > smem_cap))
                continue;
            if (best < 0 || load[b] < load[best]) best = (int)b;
        }
        if (best < 0) return false;
        load[best] += p.cost;
        bm[best] += p.n_mass;
        bs[best] += p.springs.size();
        bi[best] += p.inc_estimate;
        bx[best] += p.face_smem;
        plan[best].push_back(r);
    }
    for (auto& v : plan) std::sort(v.begin(), v.end());
    return true;
}

// Two-level LPT for launches of more than one wave.  A launch of `groups`
// CTAs runs bins g, g + groups, g + 2 groups ... one after another on CTA g,
// so what has to be even is the load of a group, not of a bin: robots are
// first spread over the groups by LPT (a group holds nb / groups bins'
// capacity), then each group's robots are spread over its own bins by LPT
// under the per-bin limits.  Returns false when a group cannot be split,
// and the caller falls back to plan_bins.
bool plan_bins_grouped(const std::vector<RobotPack>& packs, uint32_t nb, uint32_t groups,
                       const KernelShape& sh, uint32_t smem_cap,
                       std::vector<std::vector<uint32_t>>& plan, uint32_t spring_extra = 0) {
    if (groups == 0 || nb <= groups || nb % groups) return false;
    const uint32_t per = nb / groups;
    const uint32_t n = (uint32_t)packs.size();
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return packs[a].cost > packs[b].cost; });
    const uint64_t cap_s = std::min<uint64_t>((uint64_t)sh.threads * sh.spt, kMaxBinSprings);
    const uint64_t cap_m = std::min<uint64_t>((uint64_t)sh.threads * sh.mpt, 4096);
    std::vector<uint64_t> gload(groups, 0), gm(groups, 0), gs(groups, 0);
    std::vector<std::vector<uint32_t>> members(groups);
    for (uint32_t r : order) {
        const auto& p = packs[r];
        int best = -1;
        for (uint32_t g = 0; g < groups; ++g) {
            if (gm[g] + p.n_mass > per * cap_m || gs[g] + p.springs.size() > per * cap_s) continue;
            if (best < 0 || gload[g] < gload[best]) best = (int)g;
        }
        if (best < 0) return false;
        gload[best] += p.cost;
        gm[best] += p.n_mass;
        gs[best] += p.springs.size();
        members[best].push_back(r);  // descending cost within the group
    }
    plan.assign(nb, {});
    for (uint32_t g = 0; g < groups; ++g) {
        std::vector<uint64_t> load(per, 0), bm(per, 0), bs(per, 0), bi(per, 0), bx(per, 0);
        for (uint32_t r : members[g]) {
            const auto& p = packs[r];
            int best = -1;
            for (uint32_t j = 0; j < per; ++j) {
                if (bm[j] + p.n_mass > cap_m || bs[j] + p.springs.size() > cap_s) continue;
                const uint32_t m1 = (uint32_t)(bm[j] + p.n_mass), s1 = (uint32_t)(bs[j] + p.springs.size());
                if (bin_smem_bytes(m1, s1, (uint32_t)(bi[j] + p.inc_estimate)) + bx[j] + p.face_smem > smem_cap ||
                    (spring_extra && bin_smem_bytes(m1, s1, 0) + 8u + spring_extra * s1 > smem_cap))
                    continue;
                if (best < 0 || load[j] < load[best]) best = (int)j;
            }
            if (best < 0) return false;
            load[best] += p.cost;
            bm[best] += p.n_mass;
            bs[best] += p.springs.size();
            bi[best] += p.inc_estimate;
            bx[best] += p.face_smem;
            plan[(size_t)best * groups + g].push_back(r);
        }
    }
    for (auto& v : plan) std::sort(v.begin(), v.end());
    return true;
}

struct BinLocal {
    std::vector<uint32_t> mass_gidx, spring_gidx, pair, slice_off, slice_width, inc32;
    std::vector<uint16_t> inc;
    std::vector<uint32_t> faces, face_row;  // face drag: corners (2 words per face), rows per mass
    std::vector<uint16_t> face_inc;
    uint32_t n_face = 0;
    std::vector<float> lbar;
    uint32_t n_mass = 0, n_spring = 0, n_inc = 0, smem = 0, aligned = 0, ranked = 0;
    uint64_t padding = 0;
};

struct Ent {
    uint32_t other, orig, sign, packed;
    // index of the other end used for column alignment; its order within a
    // row must be the order of `other`, since aligned columns follow it
    uint32_t align;
};

inline bool ent_less(const Ent& x, const Ent& y) {
    if (x.other != y.other) return x.other < y.other;
    if (x.orig != y.orig) return x.orig < y.orig;
    return x.sign < y.sign;
}

// Every row in summation order: (other end, spring index, a end first).
void sort_rows(uint32_t nm, const std::vector<uint32_t>& row_start, raw_vector<Ent>& ents) {
    for (uint32_t i = 0; i < nm; ++i) {
        Ent* first = ents.data() + row_start[i];
        Ent* last = ents.data() + row_start[i + 1];
        if (last - first > 24) {
            std::sort(first, last, ent_less);
        } else {
            for (Ent* x = first + 1; x < last; ++x) {
                const Ent e = *x;
                Ent* y = x;
                while (y > first && ent_less(e, *(y - 1))) {
                    *y = *(y - 1);
                    --y;
                }
                *y = e;
            }
        }
    }
}

// SELL-32 rows of masses 0..nm-1 from their sorted entries (row_start:
// CSR offsets into ents); fills L's slices and incidence arrays.
void slice_rows(uint32_t nm, const std::vector<uint32_t>& row_start, const raw_vector<Ent>& ents,
                bool streamed, BinLocal& L) {
    // SELL-32: columns aligned by the offset of the other end (other - i)
    // when every row of the slice has distinct offsets -- then the k-th
    // entries of a warp's 32 masses are springs of one direction with
    // consecutive packed indices (conflict-free gather) -- otherwise, or
    // when alignment would widen the slice by more than 4 columns, ranks.
    // the union of a slice's offsets as a bitset over [lo, hi]: an entry's
    // aligned column is the rank of its offset (prefix popcounts per word)
    std::vector<uint64_t> bits;
    std::vector<uint32_t> before;
    for (uint32_t i0 = 0; i0 < nm; i0 += kSliceWidth) {
        const uint32_t i1 = std::min<uint32_t>(i0 + kSliceWidth, nm);
        uint32_t w_rank = 0;
        bool distinct = true;
        int lo = INT32_MAX, hi = INT32_MIN;
        for (uint32_t i = i0; i < i1; ++i) {
            const uint32_t r0 = row_start[i], r1 = row_start[i + 1];
            w_rank = std::max(w_rank, r1 - r0);
            for (uint32_t q = r0; q < r1; ++q) {
                if (q > r0 && ents[q].other == ents[q - 1].other) distinct = false;
                const int o = (int)ents[q].align - (int)i;
                lo = std::min(lo, o);
                hi = std::max(hi, o);
            }
        }
        uint32_t n_union = 0;
        if (distinct && lo <= hi) {
            const size_t words = (size_t)(hi - lo) / 64 + 1;
            bits.assign(words, 0);
            for (uint32_t i = i0; i < i1; ++i)
                for (uint32_t q = row_start[i]; q < row_start[i + 1]; ++q) {
                    const int o = (int)ents[q].align - (int)i - lo;
                    bits[o >> 6] |= 1ull << (o & 63);
                }
            before.assign(words, 0);
            for (size_t wd = 0; wd < words; ++wd) {
                before[wd] = n_union;
                n_union += (uint32_t)__builtin_popcountll(bits[wd]);
            }
        }
        const bool aligned = distinct && n_union <= w_rank + 4;
        const uint32_t w = aligned ? n_union : w_rank;
        aligned ? ++L.aligned : ++L.ranked;
        const size_t base = streamed ? L.inc32.size() : L.inc.size();
        L.slice_off.push_back((uint32_t)base);
        L.slice_width.push_back(w);
        if (streamed)
            L.inc32.resize(base + (size_t)w * kSliceWidth, kPadEntry32);
        else
            L.inc.resize(base + (size_t)w * kSliceWidth, kPadEntry);
        for (uint32_t i = i0; i < i1; ++i)
            for (uint32_t q = row_start[i]; q < row_start[i + 1]; ++q) {
                const Ent& e = ents[q];
                uint32_t col = q - row_start[i];
                if (aligned) {
                    const int o = (int)e.align - (int)i - lo;
                    const uint64_t below = bits[o >> 6] & ((1ull << (o & 63)) - 1ull);
                    col = before[o >> 6] + (uint32_t)__builtin_popcountll(below);
                }
                const size_t at = base + (size_t)col * kSliceWidth + (i - i0);
                if (streamed)
                    L.inc32[at] = (e.packed << 1) | e.sign;
                else
                    L.inc[at] = (uint16_t)((e.packed << 1) | e.sign);
            }
    }
    L.n_inc = (uint32_t)(streamed ? L.inc32.size() : L.inc.size());
    L.padding = L.n_inc - (uint64_t)row_start[nm];
}

// Faces of a resident bin: the bin-local corners {c0 | c1 << 16, c2} of
// every face with three distinct corners, robot by robot in face order,
// and per mass the faces it is a corner of in ascending order -- the
// summation order of the face drag -- as incidence entries (bin-local face
// index) and a row per mass: first entry | count << 24.
void build_faces(const mb_batch_desc* b, const std::vector<RobotPack>& packs,
                 const std::vector<uint32_t>& robots, uint32_t nm, BinLocal& L) {
    uint32_t nf = 0;
    for (uint32_t r : robots) nf += packs[r].n_face;
    if (!nf) return;
    // the bin's faces in robot face order (bin-local corners)
    std::vector<uint32_t> c0s(nf), c1s(nf), c2s(nf);
    {
        uint32_t mbase = 0, f = 0;
        for (uint32_t r : robots) {
            for (int64_t g = b->face_offsets[r]; g < b->face_offsets[r + 1]; ++g) {
                const uint16_t* c = b->faces + 3 * g;
                if (c[0] == c[1] || c[0] == c[2] || c[1] == c[2]) continue;
                c0s[f] = mbase + c[0];
                c1s[f] = mbase + c[1];
                c2s[f] = mbase + c[2];
                ++f;
            }
            mbase += packs[r].n_mass;
        }
    }
    // storage order: faces of one shape (corner offsets) together, by first
    // corner, so that consecutive threads of the face pass read consecutive
    // masses; the rows below keep every mass's faces in robot face order
    std::vector<uint32_t> order(nf), slot(nf);
    for (uint32_t f = 0; f < nf; ++f) order[f] = f;
    auto key = [&](uint32_t f) {
        return std::make_tuple((int32_t)c1s[f] - (int32_t)c0s[f], (int32_t)c2s[f] - (int32_t)c0s[f], c0s[f], f);
    };
    std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
    L.faces.resize(2 * (size_t)nf);
    for (uint32_t s = 0; s < nf; ++s) {
        const uint32_t f = order[s];
        slot[f] = s;
        L.faces[2 * s] = c0s[f] | (c1s[f] << 16);
        L.faces[2 * s + 1] = c2s[f];
    }
    std::vector<uint32_t> start(nm + 1, 0);
    for (uint32_t f = 0; f < nf; ++f) {
        start[c0s[f] + 1]++;
        start[c1s[f] + 1]++;
        start[c2s[f] + 1]++;
    }
    for (uint32_t i = 0; i < nm; ++i) start[i + 1] += start[i];
    L.face_inc.resize(start[nm]);
    L.face_row.resize(nm);
    std::vector<uint32_t> fill(start.begin(), start.end() - 1);
    for (uint32_t f = 0; f < nf; ++f) {
        L.face_inc[fill[c0s[f]]++] = (uint16_t)slot[f];
        L.face_inc[fill[c1s[f]]++] = (uint16_t)slot[f];
        L.face_inc[fill[c2s[f]]++] = (uint16_t)slot[f];
    }
    for (uint32_t i = 0; i < nm; ++i) L.face_row[i] = start[i] | ((start[i + 1] - start[i]) << 24);
    L.n_face = nf;
}

// rows_on_device: only the springs and masses; the rows get a region of
// generous capacity (twice the rank-layout estimate plus the alignment
// slack) for the device to build them in.
// Placement of a resident bin's springs (packed words a | b << 12 | ...)
// for the step kernel's endpoint loads: lanes 8q .. 8q + 7 of a warp form
// one shared-memory wavefront of 16-byte loads, conflict-free when their
// masses differ mod 8.  Greedy, in order: each group of 8 slots takes the
// earliest springs, within a window of the next kWindow unplaced ones, whose
// a and b are both new mod 8 in the group, then fills any slot left with the
// earliest unplaced spring.  Each chunk of kPlaceChunk springs is placed on
// its own (the device places the chunks of a bin in parallel).  Returns
// order[new position] = old position.
std::vector<uint32_t> bank_order(const std::vector<uint32_t>& words) {
    constexpr uint32_t kWindow = 64;
    const uint32_t n = (uint32_t)words.size();
    std::vector<uint32_t> order;
    order.reserve(n);
    for (uint32_t c0 = 0; c0 < n; c0 += kPlaceChunk) {
        const uint32_t c1 = std::min(n, c0 + kPlaceChunk);
        // the window: the earliest unplaced springs of the chunk, in order
        uint32_t win[kWindow], len = 0, next = c0;
        while (order.size() < c1) {
            while (len < kWindow && next < c1) win[len++] = next++;
            const uint32_t want = std::min<uint32_t>(8, c1 - (uint32_t)order.size());
            uint32_t used_a = 0, used_b = 0, got = 0;
            uint64_t picked = 0;  // bit k: win[k] placed in this group
            for (uint32_t k = 0; k < len && got < want; ++k) {
                const uint32_t w = words[win[k]];
                const uint32_t ba = 1u << (w & 7u), bb = 1u << ((w >> 12) & 7u);
                if ((used_a & ba) || (used_b & bb)) continue;
                used_a |= ba;
                used_b |= bb;
                picked |= 1ull << k;
                ++got;
            }
            for (uint32_t k = 0; k < len && got < want; ++k)
                if (!((picked >> k) & 1ull)) {
                    picked |= 1ull << k;
                    ++got;
                }
            // the group in window order (= spring order), then the window compacted
            uint32_t keep = 0;
            for (uint32_t k = 0; k < len; ++k)
                if ((picked >> k) & 1ull)
                    order.push_back(win[k]);
                else
                    win[keep++] = win[k];
            len = keep;
        }
    }
    return order;
}

void build_bin(const mb_batch_desc* b, const std::vector<RobotPack>& packs,
               const std::vector<uint32_t>& robots, const std::vector<int>& slot_of, bool streamed,
               bool rows_on_device, BinLocal& L) {
    uint32_t nm = 0, ns = 0;
    for (uint32_t r : robots) {
        nm += packs[r].n_mass;
        ns += (uint32_t)packs[r].springs.size();
    }
    L.mass_gidx.reserve(nm);
    L.spring_gidx.reserve(ns);
    L.pair.reserve(ns);
    L.lbar.reserve(ns);
    std::vector<uint32_t> row_start(nm + 1, 0);
    // the bin's springs robot by robot, each robot's in (b - a, a) order
    std::vector<uint32_t> words(ns), gids(ns);
    uint32_t mbase = 0, k = 0;
    for (uint32_t r : robots) {
        const int64_t m0 = b->mass_offsets[r], s0 = b->spring_offsets[r];
        for (uint32_t i = 0; i < packs[r].n_mass; ++i) L.mass_gidx.push_back((uint32_t)(m0 + i));
        for (uint32_t ls : packs[r].springs) {
            const int64_t g = s0 + ls;
            const uint32_t pa = mbase + b->pairs[2 * g], pc = mbase + b->pairs[2 * g + 1];
            gids[k] = (uint32_t)g;
            words[k++] = pa | (pc << 12) | ((uint32_t)slot_of[b->spring_material[g]] << 24);
            row_start[pa + 1]++;
            row_start[pc + 1]++;
        }
        mbase += packs[r].n_mass;
    }
    // resident bins: springs placed so that the 8 springs of every
    // quarter-warp read distinct 16-byte bank groups of the predicted
    // positions at both ends (newpos: old position -> packed position); with
    // the rows built on the device, the device places them too
    // (launch_bank_place, the same rule)
    std::vector<uint32_t> order = streamed || rows_on_device ? std::vector<uint32_t>{} : bank_order(words);
    std::vector<uint32_t> newpos(ns);
    for (uint32_t i = 0; i < ns; ++i) {
        const uint32_t o = order.empty() ? i : order[i];
        newpos[o] = i;
        L.spring_gidx.push_back(gids[o]);
        L.pair.push_back(words[o]);
        L.lbar.push_back(b->lbar[gids[o]]);
    }
    build_faces(b, packs, robots, nm, L);
    const uint32_t face_smem = streamed ? stream_face_smem_bytes(nm, L.n_face)
                                        : face_smem_bytes(nm, L.n_face, (uint32_t)L.face_inc.size());
    if (rows_on_device) {
        uint64_t est = 0;
        for (uint32_t r : robots) est += packs[r].inc_estimate;
        const uint32_t n_sl = (nm + kSliceWidth - 1) / kSliceWidth;
        const uint64_t cap = (2 * est + 4ull * kSliceWidth * n_sl + 31) / 32 * 32;
        L.n_mass = nm;
        L.n_spring = ns;
        L.n_inc = (uint32_t)std::min<uint64_t>(cap, 0xFFFFFFFFu);
        L.slice_off.assign(n_sl, 0);
        L.slice_width.assign(n_sl, 0);
        L.smem = bin_smem_bytes(nm, ns, (uint32_t)std::min<uint64_t>(est, 0xFFFFFFFFu)) + face_smem;
        return;
    }
    for (uint32_t i = 0; i < nm; ++i) row_start[i + 1] += row_start[i];
    raw_vector<Ent> ents(row_start[nm]);
    std::vector<uint32_t> fill(row_start.begin(), row_start.end() - 1);
    {
        uint32_t base = 0, sb = 0;
        for (uint32_t r : robots) {
            const int64_t s0 = b->spring_offsets[r];
            const auto& sp = packs[r].springs;
            // b ends in reverse spring order, then a ends in spring order:
            // with springs ordered by (b - a, a), every row of a lattice whose
            // springs point forward (b > a) arrives in summation order
            for (uint32_t k = (uint32_t)sp.size(); k-- > 0;) {
                const int64_t g = s0 + sp[k];
                const uint32_t a = b->pairs[2 * g], c = b->pairs[2 * g + 1];
                ents[fill[base + c]++] = {a, sp[k], 1u, newpos[sb + k], a};
            }
            for (uint32_t k = 0; k < sp.size(); ++k) {
                const int64_t g = s0 + sp[k];
                const uint32_t a = b->pairs[2 * g], c = b->pairs[2 * g + 1];
                ents[fill[base + a]++] = {c, sp[k], 0u, newpos[sb + k], c};
            }
            base += packs[r].n_mass;
            sb += (uint32_t)sp.size();
        }
    }
    sort_rows(nm, row_start, ents);
    L.n_mass = nm;
    L.n_spring = ns;
    slice_rows(nm, row_start, ents, streamed, L);
    L.smem = (streamed ? stream_smem_bytes(nm) : bin_smem_bytes(nm, ns, L.n_inc)) + face_smem;
}

// Offsets of every bin, then every bin copied in parallel into sized
// arrays; statistics.
void assemble(const std::vector<BinLocal>& locals, Packed& out, bool streamed, unsigned threads,
              bool rows_on_device = false) {
    const uint32_t nb = (uint32_t)locals.size();
    out.bins.assign(nb, BinDesc{});
    out.max_smem = 0;
    out.inc_entries = out.inc_padding = 0;
    out.aligned_slices = out.rank_slices = 0;
    uint64_t nm = 0, ns = 0, nsl = 0, ninc = 0, nf = 0, nfi = 0;
    for (uint32_t i = 0; i < nb; ++i) {
        const BinLocal& L = locals[i];
        BinDesc& d = out.bins[i];
        std::memset(&d, 0, sizeof(d));
        d.face_begin = (uint32_t)nf;
        d.n_face = L.n_face;
        d.face_inc_begin = (uint32_t)nfi;
        d.n_face_inc = (uint32_t)L.face_inc.size();
        nf += L.n_face;
        nfi += L.face_inc.size();
        d.mass_begin = (uint32_t)nm;
        d.n_mass = L.n_mass;
        d.spring_begin = (uint32_t)ns;
        d.n_spring = L.n_spring;
        d.inc_begin = (uint32_t)ninc;
        d.n_inc = L.n_inc;
        d.slice_begin = (uint32_t)nsl;
        d.row_cap = rows_on_device ? L.n_inc : 0u;
        nm += L.mass_gidx.size();
        ns += L.spring_gidx.size();
        nsl += L.slice_off.size();
        ninc += rows_on_device ? L.n_inc : streamed ? L.inc32.size() : L.inc.size();
        out.max_smem = std::max(out.max_smem, L.smem);
        out.inc_entries += L.n_inc;
        out.inc_padding += L.padding;
        out.aligned_slices += L.aligned;
        out.rank_slices += L.ranked;
    }
    out.mass_gidx.resize(nm);
    out.spring_gidx.resize(ns);
    out.pair.resize(ns);
    out.lbar.resize(ns);
    out.slice_off.resize(nsl);
    out.slice_width.resize(nsl);
    out.inc.resize(streamed || rows_on_device ? 0 : ninc);  // every entry is copied below
    out.inc32.resize(streamed ? ninc : 0);
    out.rows_on_device = rows_on_device;
    out.row_total = ninc;
    out.faces.resize(2 * nf);
    out.face_row.resize(nf ? nm : 0);
    out.face_inc.resize(nfi);
    parallel_for(nb, threads, [&](uint32_t i) {
        const BinLocal& L = locals[i];
        const BinDesc& d = out.bins[i];
        auto put = [](auto& dst, size_t at, const auto& src) {
            if (!src.empty()) std::memcpy(dst.data() + at, src.data(), src.size() * sizeof(src[0]));
        };
        put(out.mass_gidx, d.mass_begin, L.mass_gidx);
        put(out.spring_gidx, d.spring_begin, L.spring_gidx);
        put(out.pair, d.spring_begin, L.pair);
        put(out.lbar, d.spring_begin, L.lbar);
        put(out.slice_off, d.slice_begin, L.slice_off);
        put(out.slice_width, d.slice_begin, L.slice_width);
        if (streamed)
            put(out.inc32, d.inc_begin, L.inc32);
        else
            put(out.inc, d.inc_begin, L.inc);
        if (!out.face_row.empty()) {
            put(out.faces, 2 * (size_t)d.face_begin, L.faces);
            put(out.face_inc, d.face_inc_begin, L.face_inc);
            if (L.n_face)
                put(out.face_row, d.mass_begin, L.face_row);
            else
                std::memset(out.face_row.data() + d.mass_begin, 0, (size_t)d.n_mass * sizeof(uint32_t));
        }
    });
}

void build_all(const mb_batch_desc* b, const std::vector<RobotPack>& packs,
               const std::vector<std::vector<uint32_t>>& plan, const std::vector<int>& slot_of,
               bool streamed, unsigned threads, Packed& out, bool rows_on_device = false) {
    const uint32_t nb = (uint32_t)plan.size(), R = (uint32_t)packs.size();
    std::vector<BinLocal> locals(nb);
    parallel_for(nb, threads, [&](uint32_t i) {
        build_bin(b, packs, plan[i], slot_of, streamed, rows_on_device, locals[i]);
    });
    assemble(locals, out, streamed, threads, rows_on_device);
    out.robot_bin.assign(R, 0);
    out.robot_mass_base.assign(R, 0);
    for (uint32_t i = 0; i < nb; ++i) {
        uint32_t base = 0;
        for (uint32_t r : plan[i]) {
            out.robot_bin[r] = i;
            out.robot_mass_base[r] = base;
            base += packs[r].n_mass;
        }
    }
    out.exports.clear();
    out.cluster = out.cluster2 = out.split_bins0 = 0;
}

// ---- split bins: one robot simulated by a cluster of C CTAs ----
//
// A robot too large for one CTA's shared memory is cut into C = 2^levels
// parts by recursive coordinate bisection of its initial positions (each
// cut along the axis of largest extent, ties to the later axis, at the
// median; ties in position by mass index).  Part p is one bin: its own
// masses (ascending index), then a halo of the other parts' masses its
// springs reach; every active spring with an end in the part, so a spring
// across a cut is solved by both parts -- with the same operands, so with
// the same bits -- and only the part holding its a end writes its stress
// back (spring_gidx bit 31 marks the copies).  Rows exist for own masses
// only, in the usual summation order.  Every step each part writes its
// masses that others hold as halo into their predicted-position buffers
// (export entries: own mass | part << 12 | slot << 15).

// Part of every mass of robot r (positions: float4 per mass).
void partition_robot(const mb_batch_desc* b, uint32_t r, uint32_t levels, std::vector<uint8_t>& part_of) {
    const int64_t m0 = b->mass_offsets[r];
    const uint32_t n = (uint32_t)(b->mass_offsets[r + 1] - m0);
    std::vector<uint32_t> idx(n);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    part_of.assign(n, 0);
    // without positions (a topology-only description): index order
    auto coord = [&](uint32_t m, int axis) {
        if (!b->pos) return axis == 2 ? (float)m : 0.0f;
        const float v = b->pos[4 * (m0 + m) + axis];
        return std::isfinite(v) ? v : INFINITY;
    };
    struct Range {
        uint32_t lo, hi, level, part;
    };
    std::vector<Range> todo{{0, n, levels, 0}};
    while (!todo.empty()) {
        const Range q = todo.back();
        todo.pop_back();
        if (q.level == 0) {
            for (uint32_t i = q.lo; i < q.hi; ++i) part_of[idx[i]] = (uint8_t)q.part;
            continue;
        }
        int axis = 0;
        float best = -1.0f;
        for (int ax = 0; ax < 3; ++ax) {
            float lo = INFINITY, hi = -INFINITY;
            for (uint32_t i = q.lo; i < q.hi; ++i) {
                const float v = coord(idx[i], ax);
                if (v == INFINITY) continue;
                lo = std::min(lo, v);
                hi = std::max(hi, v);
            }
            const float ext = hi >= lo ? hi - lo : 0.0f;
            if (ext >= best) {
                best = ext;
                axis = ax;
            }
        }
        std::sort(idx.begin() + q.lo, idx.begin() + q.hi, [&](uint32_t x, uint32_t y) {
            const float cx = coord(x, axis), cy = coord(y, axis);
            return cx < cy || (cx == cy && x < y);
        });
        const uint32_t mid = q.lo + (q.hi - q.lo + 1) / 2;
        todo.push_back({mid, q.hi, q.level - 1, 2 * q.part + 1});
        todo.push_back({q.lo, mid, q.level - 1, 2 * q.part});
    }
}

struct PartMasses {
    std::vector<uint32_t> own, halo;  // robot-local indices, ascending
};

void build_part(const mb_batch_desc* b, uint32_t r, const RobotPack& pk, const std::vector<uint8_t>& part_of,
                uint32_t p, const std::vector<int>& slot_of, bool faces, std::vector<int32_t>& local_of,
                BinLocal& L, PartMasses& pm) {
    const int64_t m0 = b->mass_offsets[r], s0 = b->spring_offsets[r];
    const uint32_t n = pk.n_mass;
    pm.own.clear();
    pm.halo.clear();
    local_of.assign(n, -1);
    for (uint32_t m = 0; m < n; ++m)
        if (part_of[m] == p) {
            local_of[m] = (int32_t)pm.own.size();
            pm.own.push_back(m);
        }
    const uint32_t n_own = (uint32_t)pm.own.size();
    // halo masses are collected once each (local_of = -2 marks them)
    auto to_halo = [&](uint32_t m) {
        if (local_of[m] == -1) {
            local_of[m] = -2;
            pm.halo.push_back(m);
        }
    };
    std::vector<uint32_t> sp;
    sp.reserve(pk.springs.size());
    for (uint32_t ls : pk.springs) {
        const int64_t g = s0 + ls;
        const uint32_t a = b->pairs[2 * g], c = b->pairs[2 * g + 1];
        const bool ia = part_of[a] == p, ic = part_of[c] == p;
        if (!ia && !ic) continue;
        sp.push_back(ls);
        if (!ia) to_halo(a);
        if (!ic) to_halo(c);
    }
    // faces with a corner in the part (robot face order); their other
    // corners join the halo
    std::vector<uint32_t> fl;
    const int64_t f0 = faces && pk.n_face ? b->face_offsets[r] : 0;
    const int64_t f1 = faces && pk.n_face ? b->face_offsets[r + 1] : 0;
    for (int64_t f = f0; f < f1; ++f) {
        const uint16_t* c = b->faces + 3 * f;
        if (c[0] == c[1] || c[0] == c[2] || c[1] == c[2]) continue;
        if (part_of[c[0]] != p && part_of[c[1]] != p && part_of[c[2]] != p) continue;
        fl.push_back((uint32_t)f);
        for (int k = 0; k < 3; ++k)
            if (part_of[c[k]] != p) to_halo(c[k]);
    }
    std::sort(pm.halo.begin(), pm.halo.end());
    for (uint32_t j = 0; j < pm.halo.size(); ++j) local_of[pm.halo[j]] = (int32_t)(n_own + j);
    if (!fl.empty()) {
        // part-local corners; rows (ascending face order) for own masses
        std::vector<uint32_t> start(n_own + 1, 0);
        L.faces.reserve(2 * fl.size());
        for (uint32_t f : fl) {
            const uint16_t* c = b->faces + 3 * f;
            L.faces.push_back((uint32_t)local_of[c[0]] | ((uint32_t)local_of[c[1]] << 16));
            L.faces.push_back((uint32_t)local_of[c[2]]);
            for (int k = 0; k < 3; ++k)
                if (part_of[c[k]] == p) start[(uint32_t)local_of[c[k]] + 1]++;
        }
        for (uint32_t i = 0; i < n_own; ++i) start[i + 1] += start[i];
        L.face_inc.resize(start[n_own]);
        L.face_row.resize(n_own);
        std::vector<uint32_t> ffill(start.begin(), start.end() - 1);
        for (uint32_t q = 0; q < fl.size(); ++q) {
            const uint16_t* c = b->faces + 3 * fl[q];
            for (int k = 0; k < 3; ++k)
                if (part_of[c[k]] == p) L.face_inc[ffill[(uint32_t)local_of[c[k]]]++] = (uint16_t)q;
        }
        for (uint32_t i = 0; i < n_own; ++i) L.face_row[i] = start[i] | ((start[i + 1] - start[i]) << 24);
        L.n_face = (uint32_t)fl.size();
    }
    L.mass_gidx.reserve(n_own);
    for (uint32_t m : pm.own) L.mass_gidx.push_back((uint32_t)(m0 + m));
    const uint32_t ns = (uint32_t)sp.size();
    L.spring_gidx.reserve(ns);
    L.pair.reserve(ns);
    L.lbar.reserve(ns);
    std::vector<uint32_t> row_start(n_own + 1, 0);
    std::vector<uint32_t> words(ns);
    for (uint32_t k = 0; k < ns; ++k) {
        const int64_t g = s0 + sp[k];
        const uint32_t a = b->pairs[2 * g], c = b->pairs[2 * g + 1];
        const uint32_t la = (uint32_t)local_of[a], lc = (uint32_t)local_of[c];
        words[k] = la | (lc << 12) | ((uint32_t)slot_of[b->spring_material[g]] << 24);
        if (part_of[a] == p) row_start[la + 1]++;
        if (part_of[c] == p) row_start[lc + 1]++;
    }
    // placed for the endpoint loads as in resident bins (part-local indices:
    // own masses, then halo; newpos: spring order -> packed position)
    const std::vector<uint32_t> order = bank_order(words);
    std::vector<uint32_t> newpos(ns);
    for (uint32_t i = 0; i < ns; ++i) {
        const uint32_t k = order[i];
        const int64_t g = s0 + sp[k];
        newpos[k] = i;
        L.spring_gidx.push_back((uint32_t)g | (part_of[b->pairs[2 * g]] != p ? 0x80000000u : 0u));
        L.pair.push_back(words[k]);
        L.lbar.push_back(b->lbar[g]);
    }
    for (uint32_t i = 0; i < n_own; ++i) row_start[i + 1] += row_start[i];
    raw_vector<Ent> ents(row_start[n_own]);
    std::vector<uint32_t> fill(row_start.begin(), row_start.end() - 1);
    // b ends in reverse, then a ends in spring order (rows mostly arrive
    // sorted, as in build_bin).  Aligned by the robot-local index of the
    // other end: a row's column order must stay its summation order (halo
    // masses are numbered after the own ones, so part-local indices would
    // not keep it).
    for (uint32_t k = ns; k-- > 0;) {
        const int64_t g = s0 + sp[k];
        const uint32_t a = b->pairs[2 * g], c = b->pairs[2 * g + 1];
        if (part_of[c] == p) ents[fill[(uint32_t)local_of[c]]++] = {a, sp[k], 1u, newpos[k], a};
    }
    for (uint32_t k = 0; k < ns; ++k) {
        const int64_t g = s0 + sp[k];
        const uint32_t a = b->pairs[2 * g], c = b->pairs[2 * g + 1];
        if (part_of[a] == p) ents[fill[(uint32_t)local_of[a]]++] = {c, sp[k], 0u, newpos[k], c};
    }
    sort_rows(n_own, row_start, ents);
    L.n_mass = n_own;
    L.n_spring = ns;
    slice_rows(n_own, row_start, ents, false, L);
}

// Split robots placed in clusters of C CTAs: robot r has parts[r] parts in
// bins first[r] .. first[r] + parts[r] - 1, all inside one cluster (bins
// k*C .. k*C + C-1); slots no robot uses stay empty bins.  A part's
// predicted-position buffers hold its own and halo masses (n_all).
struct SplitParts {
    uint32_t C = 0;
    bool faces = false;  // the face layout (split_face_smem_bytes) in every part
    // second group (robots of at most two parts in two-CTA clusters, after
    // bin bins0), launched beside the first: 0 = one group
    uint32_t C2 = 0, bins0 = 0;
    std::vector<uint32_t> parts, first, slot0;   // per robot (slot0: rank of its first part)
    std::vector<BinLocal> locals;                // per bin
    std::vector<std::vector<uint32_t>> exports;  // per bin
    std::vector<uint32_t> n_all;                 // per bin
};

// Cuts robot r into P parts (part_of) and checks, from counts alone, that
// each could fit cap_s springs, cap_m own masses and the shared memory.
// Springs, halo and exports are counted exactly; a slice of rows is as wide
// as its longest row in the rank layout and at most 4 columns wider when
// aligned, so `upper` makes the check sufficient, otherwise necessary.
bool robot_parts_fit(const mb_batch_desc* b, const RobotPack& pk, uint32_t r, uint32_t P, uint64_t cap_s,
                     uint64_t cap_m, uint32_t smem_cap, bool upper, bool faces, std::vector<uint8_t>& part_of,
                     std::string* reason) {
    uint32_t levels = 0;
    while ((1u << levels) < P) ++levels;
    partition_robot(b, r, levels, part_of);
    const auto& po = part_of;
    const int64_t s0 = b->spring_offsets[r];
    const uint32_t n = pk.n_mass;
    std::vector<uint32_t> own(P, 0), ns(P, 0), halo(P, 0), exp(P, 0), mark(n, 0), deg(n, 0);
    for (uint32_t m = 0; m < n; ++m) own[po[m]]++;
    for (uint32_t ls : pk.springs) {
        const int64_t g = s0 + ls;
        const uint32_t a = b->pairs[2 * g], c = b->pairs[2 * g + 1];
        const uint32_t pa = po[a], pc = po[c];
        deg[a]++;
        deg[c]++;
        ns[pa]++;
        if (pc != pa) {
            ns[pc]++;
            // halo marks: bit p of mark[m] once m is counted in part p
            if (!(mark[c] & (1u << pa))) { mark[c] |= 1u << pa; halo[pa]++; }
            if (!(mark[a] & (1u << pc))) { mark[a] |= 1u << pc; halo[pc]++; }
        }
    }
    // faces (face layout): counted in every part owning a corner, their
    // other corners in its halo
    std::vector<uint32_t> nf(P, 0), nfi(P, 0);
    if (faces && pk.n_face)
        for (int64_t f = b->face_offsets[r]; f < b->face_offsets[r + 1]; ++f) {
            const uint16_t* c = b->faces + 3 * f;
            if (c[0] == c[1] || c[0] == c[2] || c[1] == c[2]) continue;
            const uint32_t in = (1u << po[c[0]]) | (1u << po[c[1]]) | (1u << po[c[2]]);
            for (uint32_t p = 0; p < P; ++p) {
                if (!(in & (1u << p))) continue;
                nf[p]++;
                for (int k = 0; k < 3; ++k) {
                    if (po[c[k]] == p)
                        nfi[p]++;
                    else if (!(mark[c[k]] & (1u << p))) {
                        mark[c[k]] |= 1u << p;
                        halo[p]++;
                    }
                }
            }
        }
    // rows: slices of 32 own masses (see above); exports: one per halo copy
    const uint32_t widen = upper ? 4u : 0u;
    std::vector<uint32_t> rows(P, 0), in_slice(P, 0), slice_max(P, 0);
    for (uint32_t m = 0; m < n; ++m) {
        const uint32_t p = po[m];
        exp[p] += (uint32_t)__builtin_popcount(mark[m]);
        slice_max[p] = std::max(slice_max[p], deg[m]);
        if (++in_slice[p] == kSliceWidth) {
            rows[p] += kSliceWidth * (slice_max[p] + widen);
            in_slice[p] = slice_max[p] = 0;
        }
    }
    for (uint32_t p = 0; p < P; ++p)
        if (in_slice[p]) rows[p] += kSliceWidth * (slice_max[p] + widen);
    for (uint32_t p = 0; p < P; ++p) {
        const uint64_t smem_lb = split_smem_bytes(own[p] + halo[p], ns[p], 0, exp[p]) + 2ull * rows[p] +
                                 (faces ? split_face_smem_bytes(own[p] + halo[p], own[p], nf[p], nfi[p]) : 0u);
        if (ns[p] > cap_s || own[p] > cap_m || own[p] + halo[p] > 4096 || smem_lb > smem_cap) {
            if (reason) {
                char buf[256];
                std::snprintf(buf, sizeof(buf),
                              "part %u of robot %u: %u springs, %u + %u masses, >= %llu B shared memory", p, r,
                              ns[p], own[p], halo[p], (unsigned long long)smem_lb);
                *reason = buf;
            }
            return false;
        }
    }
    return true;
}

// Capacity of the largest of `shapes`.
void split_caps(const std::vector<KernelShape>& shapes, uint64_t& cap_s, uint64_t& cap_m) {
    cap_s = cap_m = 0;
    for (const auto& sh : shapes) {
        cap_s = std::max<uint64_t>(cap_s, std::min<uint64_t>((uint64_t)sh.threads * sh.spt, kMaxBinSprings));
        cap_m = std::max<uint64_t>(cap_m, std::min<uint64_t>((uint64_t)sh.threads * sh.mpt, 4096));
    }
}

// Every robot cut into C parts (one cluster each), checked from counts
// before any rows are built; false with the reason otherwise.
bool split_partition(const mb_batch_desc* b, const std::vector<RobotPack>& packs, uint32_t C,
                     const std::vector<KernelShape>& shapes, uint32_t smem_cap, bool faces, unsigned threads,
                     std::vector<std::vector<uint8_t>>& part_of, std::string& why) {
    const uint32_t R = (uint32_t)packs.size();
    uint64_t cap_s, cap_m;
    split_caps(shapes, cap_s, cap_m);
    part_of.assign(R, {});
    std::atomic<bool> fits{true};
    std::vector<std::string> reason(R);
    parallel_for(R, threads, [&](uint32_t r) {
        if (!fits.load(std::memory_order_relaxed)) return;
        if (!robot_parts_fit(b, packs[r], r, C, cap_s, cap_m, smem_cap, false, faces, part_of[r], &reason[r]))
            fits = false;
    });
    if (!fits) {
        for (const auto& w : reason)
            if (!w.empty()) {
                why = w;
                break;
            }
        return false;
    }
    return true;
}

// Each robot at its fewest parts (1, 2, 4 or 8) that surely fit `shape`
// (the sufficient check); false if some robot needs more than 8.
bool split_partition_mixed(const mb_batch_desc* b, const std::vector<RobotPack>& packs, const KernelShape& shape,
                           uint32_t smem_cap, bool faces, unsigned threads,
                           std::vector<std::vector<uint8_t>>& part_of, std::vector<uint32_t>& parts) {
    const uint32_t R = (uint32_t)packs.size();
    uint64_t cap_s, cap_m;
    split_caps({shape}, cap_s, cap_m);
    part_of.assign(R, {});
    parts.assign(R, 0);
    std::atomic<bool> fits{true};
    parallel_for(R, threads, [&](uint32_t r) {
        if (!fits.load(std::memory_order_relaxed)) return;
        for (uint32_t P = 1; P <= 8; P *= 2)
            if (robot_parts_fit(b, packs[r], r, P, cap_s, cap_m, smem_cap, true, faces, part_of[r], nullptr)) {
                parts[r] = P;
                return;
            }
        fits = false;
    });
    return fits;
}

// Places `robots` in clusters of C slots from bin `base`, robots with more
// parts first (parts are powers of two, so the slots fill without gaps but
// in the last cluster); returns the number of bins used.
uint32_t place_parts(const std::vector<uint32_t>& robots, const std::vector<uint32_t>& parts, uint32_t C,
                     uint32_t base, std::vector<uint32_t>& first, std::vector<uint32_t>& slot0) {
    std::vector<uint32_t> order(robots);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return parts[x] > parts[y]; });
    uint32_t cluster = 0, slot = 0;
    for (uint32_t r : order) {
        if (slot + parts[r] > C) {
            ++cluster;
            slot = 0;
        }
        first[r] = base + cluster * C + slot;
        slot0[r] = slot;
        slot += parts[r];
    }
    return order.empty() ? 0 : (cluster + 1) * C;
}

// Placement of every robot: one group in clusters of C, or -- when some
// robots need more than two parts and others at most two -- the large ones
// in clusters of C and the others after them in clusters of two, which the
// device packs more densely (launched side by side).  Returns the bins.
uint32_t place_split(SplitParts& sp) {
    const uint32_t R = (uint32_t)sp.parts.size();
    sp.first.assign(R, 0);
    sp.slot0.assign(R, 0);
    std::vector<uint32_t> big, small;
    for (uint32_t r = 0; r < R; ++r) (sp.C > 2 && sp.parts[r] > 2 ? big : small).push_back(r);
    if (big.empty() || small.empty()) {
        sp.C2 = sp.bins0 = 0;
        std::vector<uint32_t> all(R);
        for (uint32_t r = 0; r < R; ++r) all[r] = r;
        return place_parts(all, sp.parts, sp.C, 0, sp.first, sp.slot0);
    }
    sp.bins0 = place_parts(big, sp.parts, sp.C, 0, sp.first, sp.slot0);
    sp.C2 = 2;
    return sp.bins0 + place_parts(small, sp.parts, 2, sp.bins0, sp.first, sp.slot0);
}

// Builds every part (rows, halos, export lists) from a partition and a
// placement (sp.parts, sp.first, sp.slot0 set) over `nb` bins.
void build_split_parts(const mb_batch_desc* b, const std::vector<RobotPack>& packs, uint32_t nb,
                       const std::vector<std::vector<uint8_t>>& part_of, const std::vector<int>& slot_of,
                       unsigned threads, SplitParts& sp) {
    const uint32_t R = (uint32_t)packs.size();
    sp.locals.assign(nb, BinLocal{});
    sp.exports.assign(nb, {});
    sp.n_all.assign(nb, 0);
    parallel_for(R, threads, [&](uint32_t r) {
        const uint32_t P = sp.parts[r], base = sp.first[r], slot0 = sp.slot0[r];
        std::vector<PartMasses> pm(P);
        std::vector<int32_t> local_of;
        for (uint32_t p = 0; p < P; ++p) {
            build_part(b, r, packs[r], part_of[r], p, slot_of, sp.faces, local_of, sp.locals[base + p], pm[p]);
            sp.n_all[base + p] = (uint32_t)(pm[p].own.size() + pm[p].halo.size());
        }
        // export entries name the destination by its rank in the cluster
        for (uint32_t q = 0; q < P; ++q)
            for (uint32_t j = 0; j < pm[q].halo.size(); ++j) {
                const uint32_t m = pm[q].halo[j], owner = part_of[r][m];
                const auto& own = pm[owner].own;
                const uint32_t li = (uint32_t)(std::lower_bound(own.begin(), own.end(), m) - own.begin());
                const uint32_t slot = (uint32_t)pm[q].own.size() + j;
                sp.exports[base + owner].push_back(li | ((slot0 + q) << 12) | (slot << 15));
            }
        for (uint32_t p = 0; p < P; ++p) std::sort(sp.exports[base + p].begin(), sp.exports[base + p].end());
    });
}

// Whether every part fits the shape and the shared memory; the reason if not.
// Shared memory of split bin i.
uint32_t split_bin_smem(const SplitParts& sp, uint32_t i) {
    const BinLocal& L = sp.locals[i];
    return split_smem_bytes(sp.n_all[i], L.n_spring, L.n_inc, (uint32_t)sp.exports[i].size()) +
           (sp.faces ? split_face_smem_bytes(sp.n_all[i], L.n_mass, L.n_face, (uint32_t)L.face_inc.size()) : 0u);
}

bool split_fits(const SplitParts& sp, const KernelShape& sh, uint32_t smem_cap, std::string& why) {
    const uint64_t cap_s = std::min<uint64_t>((uint64_t)sh.threads * sh.spt, kMaxBinSprings);
    const uint64_t cap_m = std::min<uint64_t>((uint64_t)sh.threads * sh.mpt, 4096);
    for (uint32_t i = 0; i < sp.locals.size(); ++i) {
        const BinLocal& L = sp.locals[i];
        const uint32_t smem = split_bin_smem(sp, i);
        if (L.n_spring > cap_s || L.n_mass > cap_m || sp.n_all[i] > 4096 || smem > smem_cap) {
            char buf[256];
            std::snprintf(buf, sizeof(buf), "part in bin %u: %u springs, %u + %u masses, %u B shared memory", i,
                          L.n_spring, L.n_mass, sp.n_all[i] - L.n_mass, smem);
            why = buf;
            return false;
        }
    }
    return true;
}

// The packed arrays of split parts.
void assemble_split(const SplitParts& sp, uint32_t R, unsigned threads, Packed& out) {
    const uint32_t nb = (uint32_t)sp.locals.size();
    assemble(sp.locals, out, false, threads);
    out.robot_bin.assign(R, 0);
    out.robot_mass_base.assign(R, 0);
    for (uint32_t r = 0; r < R; ++r) out.robot_bin[r] = sp.first[r];
    out.exports.clear();
    out.max_smem = 0;
    for (uint32_t i = 0; i < nb; ++i) {
        BinDesc& d = out.bins[i];
        d.x_stride = sp.n_all[i];
        d.export_begin = (uint32_t)out.exports.size();
        d.n_export = (uint32_t)sp.exports[i].size();
        d.n_all = sp.n_all[i];
        out.exports.insert(out.exports.end(), sp.exports[i].begin(), sp.exports[i].end());
        out.max_smem = std::max(out.max_smem, split_bin_smem(sp, i));
    }
}

}  // namespace

mb_status pack_population(const mb_batch_desc* b, const PackOptions& o, Packed& out, std::string& err) {
    const uint32_t R = b->n_robots;
    const unsigned threads = o.threads ? o.threads : std::max(1u, std::thread::hardware_concurrency());
    std::vector<RobotPack> packs(R);
    parallel_for(R, threads, [&](uint32_t r) { preprocess(b, r, packs[r]); });
    for (uint32_t r = 0; r < R; ++r)
        if (packs[r].status != MB_OK) {
            err = packs[r].error;
            return packs[r].status;
        }
    uint64_t tot_s = 0, tot_m = 0;
    uint32_t max_s = 0, max_m = 0;
    out.max_degree = 0;
    for (const auto& p : packs) {
        tot_s += p.springs.size();
        tot_m += p.n_mass;
        max_s = std::max<uint32_t>(max_s, (uint32_t)p.springs.size());
        max_m = std::max(max_m, p.n_mass);
        out.max_degree = std::max(out.max_degree, p.max_degree);
    }
    out.masses = tot_m;
    out.active_springs = tot_s;
    out.part_of.clear();
    out.robot_parts.clear();
    out.robot_slot0.clear();
    out.n_faces = 0;
    for (const auto& p : packs) out.n_faces += p.n_face;

    // material slots: the composite ids used by the whole population
    std::vector<int> slot_of(MB_COMPOSITE_COUNT, -1);
    {
        uint64_t used[4] = {0, 0, 0, 0};
        for (uint32_t r = 0; r < R; ++r)
            for (int w = 0; w < 4; ++w) used[w] |= packs[r].mats[w];
        for (int m = 0; m < MB_COMPOSITE_COUNT; ++m)
            if ((used[m >> 6] >> (m & 63)) & 1ull) slot_of[m] = 0;
    }
    out.mat_ids.clear();
    for (int m = 0; m < MB_COMPOSITE_COUNT; ++m)
        if (slot_of[m] == 0) {
            slot_of[m] = (int)out.mat_ids.size();
            out.mat_ids.push_back((uint8_t)m);
        }

    const uint32_t force_c = o.override.cluster;
    if (force_c != 0 && force_c != 1 && force_c != 2 && force_c != 4 && force_c != 8) {
        err = "cluster must be 0, 1, 2, 4 or 8";
        return MB_ERR_ARGUMENT;
    }
    std::vector<KernelShape> shapes;
    if (force_c > 1 || o.override.streamed)
        ;  // split or streamed: no resident bins
    else if (o.override.threads)
        shapes.push_back({o.override.threads, o.override.springs_per_thread, o.override.masses_per_thread});
    else
        for (const auto& s : kAuto) shapes.push_back(s);
    const uint32_t sms = std::max<uint32_t>(o.sms, 1);
    std::vector<std::vector<uint32_t>> plan;
    bool ok = false;
    // Automatic choice: a shape with a register-row variant is first planned
    // for it -- at most one mass per thread in every bin and room for its 8
    // bytes of shared memory per spring -- then, if that fails, as usual.
    std::vector<std::pair<KernelShape, bool>> attempts;
    for (const auto& sh : shapes) {
        if (!o.override.threads && out.n_faces == 0 && max_m <= sh.threads && row_reg_supported(sh) &&
            out.max_degree <= row_reg_width())
            attempts.push_back({sh, true});
        attempts.push_back({sh, false});
    }
    for (const auto& [sh, one_mass] : attempts) {
        if (!shape_supported(sh)) continue;
        const uint64_t cap_s = std::min<uint64_t>((uint64_t)sh.threads * sh.spt, kMaxBinSprings);
        const uint64_t cap_m = std::min<uint64_t>((uint64_t)sh.threads * (one_mass ? 1u : sh.mpt), 4096);
        if (max_s > cap_s || max_m > cap_m) continue;
        uint32_t nb = o.override.bins;
        const bool fixed = nb != 0;
        uint32_t wave = sms;
        if (R >= sms) {
            // One wave = SMs x resident CTAs per SM; shared memory is
            // estimated at the even share of the population.
            const uint32_t est_smem = std::min<uint32_t>(
                o.smem_cap, bin_smem_bytes((uint32_t)std::min<uint64_t>(cap_m, tot_m / sms + 1),
                                           (uint32_t)std::min<uint64_t>(cap_s, tot_s / sms + 1),
                                           (uint32_t)std::min<uint64_t>(3 * cap_s, 3 * (tot_s / sms + 1))));
            const int per_sm = o.ctas_per_sm ? std::max(1, o.ctas_per_sm(sh, est_smem)) : 1;
            wave = sms * (uint32_t)per_sm;
        }
        if (!nb) {
            const uint64_t need = std::max<uint64_t>((tot_s + cap_s - 1) / cap_s, (tot_m + cap_m - 1) / cap_m);
            nb = (uint32_t)std::max<uint64_t>(need, 1);
            if (R >= sms) {
                nb = std::max<uint32_t>(nb, wave);
                nb = (nb + wave - 1) / wave * wave;  // whole waves
            }
            nb = std::min<uint32_t>(nb, R);
        }
        uint32_t grid = 0;
        for (uint32_t tries = 0; tries < 16; ++tries) {
            // Several waves: one CTA per group of bins, groups balanced
            // (plan_bins_grouped); otherwise one CTA per bin.
            grid = 0;
            bool planned = false;
            const KernelShape psh{sh.threads, sh.spt, one_mass ? 1u : sh.mpt};
            const uint32_t extra = one_mass ? 8u : 0u;
            if (R >= sms && nb >= 2 * wave && nb % wave == 0 &&
                plan_bins_grouped(packs, nb, wave, psh, o.smem_cap, plan, extra)) {
                planned = true;
                grid = wave;
            }
            if (!planned) planned = plan_bins(packs, nb, psh, o.smem_cap, plan, extra);
            if (planned) {
                build_all(b, packs, plan, slot_of, false, threads, out, o.rows_on_device);
                uint64_t need = out.max_smem;
                if (one_mass)
                    for (const BinDesc& d : out.bins)
                        need = std::max<uint64_t>(need, bin_smem_bytes(d.n_mass, d.n_spring, 0) + 8ull +
                                                            8ull * d.n_spring);
                if (need <= o.smem_cap) {
                    ok = true;
                    break;
                }
            }
            if (fixed || nb >= R) break;
            nb = std::min<uint32_t>(R, nb + wave);
        }
        if (ok) {
            out.shape = sh;
            out.n_bins = nb;
            out.grid = grid;
            out.streamed = false;
            break;
        }
    }
    // Split over a cluster: when forced, or when no resident shape holds the
    // largest robot -- the fewest parts whose every part fits a shape.
    std::string why;
    const bool split_faces = o.split_faces && out.n_faces > 0;
    if (!ok && !o.override.streamed && force_c != 1) {
        std::vector<uint32_t> cs;
        if (force_c > 1)
            cs.push_back(force_c);
        else
            cs = {2u, 4u, 8u};
        std::vector<KernelShape> sshapes;
        if (o.override.threads)
            sshapes.push_back({o.override.threads, o.override.springs_per_thread, o.override.masses_per_thread});
        else
            for (const auto& sh : kSplit) sshapes.push_back(sh);
        std::vector<KernelShape> compiled;
        for (const auto& sh : sshapes)
            if (split_supported(sh)) compiled.push_back(sh);
        // the device must be able to hold one such cluster at a time
        auto schedulable = [&](const SplitParts& sp, const KernelShape& sh) {
            if (!o.cluster_fits) return true;
            uint32_t smem = 0;
            for (uint32_t i = 0; i < sp.locals.size(); ++i)
                smem = std::max(smem, split_bin_smem(sp, i));
            if (o.cluster_fits(sh, sp.C, smem)) return true;
            why = "clusters of " + std::to_string(sp.C) + " CTAs cannot be scheduled on this device";
            return false;
        };
        auto accept = [&](SplitParts& sp, const KernelShape& sh, uint32_t nb,
                          const std::vector<std::vector<uint8_t>>& part_of) {
            assemble_split(sp, R, threads, out);
            // the partition, for re-packing on the device after development
            out.part_of.resize((size_t)b->mass_offsets[R]);
            for (uint32_t r = 0; r < R; ++r)
                std::copy(part_of[r].begin(), part_of[r].end(), out.part_of.begin() + b->mass_offsets[r]);
            out.robot_parts = sp.parts;
            out.robot_slot0 = sp.slot0;
            ok = true;
            out.shape = sh;
            out.n_bins = nb;
            out.grid = 0;
            out.cluster = sp.C;
            out.cluster2 = sp.C2;
            out.split_bins0 = sp.bins0;
            out.streamed = false;
        };
        // automatic: every robot at its fewest parts, robots sharing clusters
        if (force_c == 0)
            for (const auto& sh : compiled) {
                std::vector<std::vector<uint8_t>> part_of;
                SplitParts sp;
                sp.faces = split_faces;
                if (!split_partition_mixed(b, packs, sh, o.smem_cap, split_faces, threads, part_of, sp.parts))
                    continue;
                sp.C = *std::max_element(sp.parts.begin(), sp.parts.end());
                if (sh.mpt == 1 && sp.C >= 2) {
                    // one own mass per thread only where it costs no CTAs: if two
                    // masses per thread place the robots in fewer bins, take that shape
                    const KernelShape sh2{sh.threads, sh.spt, 2};
                    std::vector<std::vector<uint8_t>> part_of2;
                    SplitParts sp2;
                    if (split_supported(sh2) &&
                        split_partition_mixed(b, packs, sh2, o.smem_cap, split_faces, threads, part_of2, sp2.parts)) {
                        sp2.C = *std::max_element(sp2.parts.begin(), sp2.parts.end());
                        SplitParts sp1;
                        sp1.parts = sp.parts;
                        sp1.C = sp.C;
                        if (place_split(sp2) < place_split(sp1)) continue;
                    }
                }
                if (sp.C < 2) continue;  // every robot fits a CTA alone: not a split population
                const uint32_t nb = place_split(sp);
                build_split_parts(b, packs, nb, part_of, slot_of, threads, sp);
                if (!split_fits(sp, sh, o.smem_cap, why) || !schedulable(sp, sh)) continue;
                accept(sp, sh, nb, part_of);
                break;
            }
        // forced (or when the mixed placement fails): every robot in C parts
        for (uint32_t C : cs) {
            if (ok || compiled.empty()) break;
            std::vector<std::vector<uint8_t>> part_of;
            if (!split_partition(b, packs, C, compiled, o.smem_cap, split_faces, threads, part_of, why)) continue;
            SplitParts sp;
            sp.C = C;
            sp.faces = split_faces;
            sp.parts.assign(R, C);
            sp.first.resize(R);
            sp.slot0.assign(R, 0);
            for (uint32_t r = 0; r < R; ++r) sp.first[r] = r * C;
            build_split_parts(b, packs, R * C, part_of, slot_of, threads, sp);
            for (const auto& sh : compiled) {
                if (!split_fits(sp, sh, o.smem_cap, why) || !schedulable(sp, sh)) continue;
                accept(sp, sh, R * C, part_of);
                break;
            }
        }
        if (!ok && force_c > 1) {
            err = "robots do not fit a split over " + std::to_string(force_c) + " CTAs: " + why;
            return MB_ERR_CAPACITY;
        }
    }
    // Streamed: when forced, or when neither a resident shape nor a split
    // holds the largest robot.  One robot per bin.
    if (o.override.streamed || !ok) {
        const uint32_t mpt = max_m <= 2048 ? 2u : 4u;
        if (max_m <= 4096 && stream_supported(1024, mpt)) {
            plan.assign(R, {});
            for (uint32_t r = 0; r < R; ++r) plan[r].push_back(r);
            build_all(b, packs, plan, slot_of, true, threads, out);
            if (out.max_smem <= o.smem_cap) {
                ok = true;
                out.streamed = true;
                out.shape = KernelShape{1024, 0, mpt};
                out.n_bins = R;
                out.grid = 0;
                out.cluster = out.cluster2 = out.split_bins0 = 0;
                out.exports.clear();
            }
        }
    }
    if (!ok) {
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "population does not fit any compiled kernel shape (largest robot: %u springs, %u masses)",
                      max_s, max_m);
        err = buf;
        return MB_ERR_CAPACITY;
    }
    return MB_OK;
}

}  // namespace mb
