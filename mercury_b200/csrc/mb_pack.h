// Host-side packing of a population into bins (no CUDA calls).
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <memory>
#include <utility>
#include <vector>

#include "../../include/mercury_b200.h"
#include "mb_internal.h"

namespace mb {

// std::vector whose resize leaves new elements uninitialised: the packed
// arrays are written in full after they are sized.
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U>&) {}
    template <class U>
    void construct(U* p) {
        ::new ((void*)p) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
};
template <class T>
using raw_vector = std::vector<T, NoInitAlloc<T>>;

struct PackOptions {
    uint32_t sms = 148;            // SMs of the device
    uint32_t smem_cap = 232448;    // dynamic shared memory per CTA, bytes
    uint32_t mode = 0;             // step mode (for occupancy queries)
    mb_launch_config override{};   // zero fields = automatic choice
    // resident CTAs per SM of a shape with a given dynamic shared memory;
    // empty = 1
    std::function<int(const KernelShape&, uint32_t)> ctas_per_sm;
    // whether clusters of that many CTAs of a split shape with that shared
    // memory can be scheduled at all; empty = yes
    std::function<bool(const KernelShape&, uint32_t, uint32_t)> cluster_fits;
    unsigned threads = 0;          // host threads (0 = hardware concurrency)
    // resident bins only: lay out springs and masses, leave the rows to the
    // device (bins[b].row_cap entries reserved per bin)
    bool rows_on_device = false;
    // split robots carry their faces (the face drag is on): velocities are
    // exchanged with the positions and each part computes the faces that
    // touch its own masses
    bool split_faces = false;
};

struct Packed {
    KernelShape shape{0, 0, 0};
    uint32_t n_bins = 0;
    uint32_t grid = 0;  // CTAs per launch, CTA g running bins g, g + grid, ...; 0 = one per bin
    uint32_t cluster = 0;  // split bins: CTAs per cluster (parts per robot); 0 = not split
    // split bins in two groups: bins [0, split_bins0) in clusters of `cluster`,
    // the rest in clusters of `cluster2`, launched side by side; 0 = one group
    uint32_t cluster2 = 0, split_bins0 = 0;
    bool rows_on_device = false;  // rows not built: row_total entries reserved (bins[b].row_cap each)
    uint64_t row_total = 0;
    bool streamed = false;
    uint32_t max_smem = 0;
    std::vector<BinDesc> bins;
    raw_vector<uint32_t> mass_gidx, spring_gidx, pair, slice_off, slice_width;
    std::vector<uint32_t> robot_bin;
    std::vector<uint32_t> robot_mass_base;  // bin-local index of each robot's first mass
    raw_vector<uint16_t> inc;    // resident rows
    raw_vector<uint32_t> inc32;  // streamed rows
    std::vector<uint32_t> exports;  // split bins: own mass | part << 12 | halo slot << 15
    // split populations: the part of every mass (upload order), and per robot
    // its part count and the cluster rank of its first part
    std::vector<uint8_t> part_of;
    std::vector<uint32_t> robot_parts, robot_slot0;
    // face drag (resident bins): corners {c0 | c1 << 16, c2} per face, row
    // per packed mass (first entry | count << 24), incidence entries; empty
    // when no bin has faces
    raw_vector<uint32_t> faces, face_row;
    raw_vector<uint16_t> face_inc;
    uint64_t n_faces = 0;  // faces of the population with three distinct corners
    uint32_t max_degree = 0;  // most non-air springs at one mass
    raw_vector<float> lbar;
    std::vector<uint8_t> mat_ids;
    // statistics
    uint64_t masses = 0, active_springs = 0, inc_entries = 0, inc_padding = 0;
    uint32_t aligned_slices = 0, rank_slices = 0;
};

// Runs f(i) for every i in [0, n) on up to `threads` host threads of a
// process-wide worker pool (the calling thread among them), in any order;
// returns when all are done.
void parallel_for(uint32_t n, unsigned threads, const std::function<void(uint32_t)>& f);

// Validates `b`, chooses the launch shape and bin count (or applies the
// override), and builds the packed arrays.  On failure returns the status
// and a message in `err`.
mb_status pack_population(const mb_batch_desc* b, const PackOptions& o, Packed& out, std::string& err);

}  // namespace mb
