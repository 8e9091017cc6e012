// Device development step (mb_devo.cu); internal to the library.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mb_internal.h"

namespace mb {

constexpr uint32_t kDevoMaxReplaced = 1024;   // springs replaced per robot and call
constexpr uint32_t kDevoReferenceRanks = 1u;  // rank window [r k, r k + k) of robot r

// One replaced spring: global spring index (0xFFFFFFFF = unused record),
// the new pair (a | b << 16, robot-local), composite material, mean length.
struct DevoRecord {
    uint32_t spring;
    uint32_t pair;
    uint32_t material;
    float lbar;
};

struct DevoParams {
    const float* stress;       // per spring, upload order
    const int64_t* mass_off;   // n_robots + 1
    const int64_t* spring_off; // n_robots + 1
    const float4* pos;         // upload order
    const uint8_t* mass_mat;   // upload order
    const float4* table;       // composite material table (k, dL0, omega, phi)
    float t;                   // clock of the mean lengths
    uint32_t k;                // springs replaced per robot (<= kDevoMaxReplaced)
    uint64_t seed;
    uint32_t flags;
    DevoRecord* out;           // n_robots * k records, rank order per robot
};

cudaError_t launch_devo(const DevoParams& p, uint32_t n_robots, cudaStream_t s);

// ---------------------------------------------------------------------------
// Re-packing on the device after development.  Springs keep their packed
// slot; a spring that becomes air turns its slot inert (spring_gidx = the
// population's spring count, a dummy stress element; no row references it)
// and frees it for a spring of its bin that stops being air.  The rows of
// every bin are then rebuilt: CSR by counting, each row sorted by (other
// end, spring index, a end before b end), SELL-32 slices aligned by
// neighbour offset when the host packer would align them.  Anything that
// does not fit (no free slot, no material slot, rows beyond the bin's
// capacity) is counted in status[0] and the host re-packs instead.

constexpr uint32_t kNoSlot = 0xFFFFFFFFu;
constexpr uint32_t kNoMatSlot = 0xFFu;

struct DevoApplyParams {
    const DevoRecord* rec;
    uint32_t n_rec;
    uint32_t k;                    // records per robot
    uint16_t* pairs;               // canonical topology, upload order
    uint8_t* spring_mat;
    float* lbar;
    uint32_t* pslot;               // canonical spring -> packed slot, or kNoSlot
    const uint32_t* robot_bin;
    const uint32_t* robot_mass_base;
    const uint8_t* slot_of;        // composite id -> material slot, or kNoMatSlot
    const BinDesc* bins;
    uint32_t* spring_pair;         // packed
    float* spring_lbar;
    uint32_t* spring_gidx;
    uint32_t inert;                // spring_gidx of an inert slot
    uint32_t* free_count;          // per bin
    uint32_t* free_taken;          // per bin
    uint32_t* free_slots;          // per packed slot region of each bin
    uint32_t* status;              // [0] problems, [1] max shared memory of a bin
};

struct RebuildParams {
    BinDesc* bins;
    uint32_t n_bins;
    const uint32_t* spring_pair;
    const uint32_t* spring_gidx;
    uint32_t inert;
    uint32_t* slice_off;
    uint32_t* slice_width;
    uint16_t* inc;                 // resident rows
    uint32_t* inc32;               // streamed rows
    uint32_t streamed;
    unsigned long long* rows;      // scratch: 2 per packed slot
    uint32_t* free_count;
    uint32_t* free_taken;
    uint32_t* status;
    // split parts: per bin the first entry of its key table (robot-local
    // index of every local mass); nullptr for resident and streamed bins
    const uint32_t* keys;
    const uint32_t* key_begin;
};

// Canonical spring -> packed slot map from spring_gidx (n_packed slots).
cudaError_t launch_build_pslot(const uint32_t* spring_gidx, uint32_t n_packed, uint32_t n_springs,
                               uint32_t* pslot, cudaStream_t s);
// Applies development records: pass 0 everything except air -> non-air,
// pass 1 air -> non-air (takes freed slots).
cudaError_t launch_devo_apply(const DevoApplyParams& p, int pass, cudaStream_t s);
// Moves each bin's rows to a region of `cap` entries (bins[b].row_cap =
// capacity); new_begin[b] is the new first entry.
cudaError_t launch_relayout(const BinDesc* old_bins, const uint32_t* new_begin, uint32_t n_bins,
                            const void* src, void* dst, uint32_t entry_bytes, cudaStream_t s);
// Rebuilds every bin's rows; status[1] gets the largest shared memory a
// bin needs.
cudaError_t launch_rebuild(const RebuildParams& p, cudaStream_t s);
// Places the springs of every resident bin for the step kernel's endpoint
// loads (the host packer's bank_order rule, same result): pair, gidx and
// lbar are permuted in place within each bin; scratch holds one u64 per
// packed slot; max_springs is the largest bin's spring count.
cudaError_t launch_bank_place(const BinDesc* bins, uint32_t n_bins, uint32_t max_springs, uint32_t* pair,
                              uint32_t* gidx, float* lbar, unsigned long long* scratch, cudaStream_t s);

// ---------------------------------------------------------------------------
// Development of robots split over thread-block clusters (one part per bin).
// The partition of each robot's masses into parts stays as packed; after the
// records are applied, every spring is in the parts that hold one of its
// ends, every part holds as halo the other parts' masses its springs reach,
// and every part exports those of its masses that other parts hold.
//
// Per bin, regions with spare capacity are set up once (first development
// of a split population): spring slots (spring_cap; unused ones on the free
// list), export entries (export_cap), local masses (x_stride: own, then halo),
// and the local index of every robot mass in the bin (map: kNoSlot when the
// bin does not hold it).  Springs keep their slots as long as they stay in a
// part; halo masses are appended (never renumbered); rows are rebuilt by
// rebuild_kernel keyed by robot-local index.  Anything that does not fit is
// counted in status[0] and the host re-packs instead.
struct SplitDevoParams {
    const DevoRecord* rec;
    uint32_t n_rec;
    uint32_t k;                    // records per robot
    uint32_t n_bins;
    uint16_t* pairs;               // canonical topology, upload order
    uint8_t* spring_mat;
    float* lbar;
    const int64_t* mass_off;       // n_robots + 1
    const uint8_t* part_of;        // per mass (upload order): its part
    const uint32_t* robot_bin;     // bin of each robot's part 0
    const uint32_t* robot_parts;
    const uint32_t* robot_slot0;   // cluster rank of each robot's part 0
    const uint32_t* bin_robot;     // robot of each bin (kNoSlot: empty bin)
    const uint32_t* mass_gidx;     // packed own mass -> upload index
    const uint8_t* slot_of;        // composite id -> material slot, or kNoMatSlot
    BinDesc* bins;
    uint32_t* spring_pair;         // packed
    float* spring_lbar;
    uint32_t* spring_gidx;
    uint32_t inert;                // spring_gidx of an inert slot
    uint32_t* slot_a;              // per spring: bin-relative slot in the part of its a end
    uint32_t* slot_b;              // ... of its b end (the same slot when both are in one part)
    const uint32_t* spring_cap;    // per bin
    const uint32_t* export_cap;    // per bin
    uint32_t* exports;
    uint32_t* map;                 // per bin, per robot mass: local index, kNoSlot, or kPending
    const uint32_t* map_begin;     // per bin
    uint32_t* keys;                // per bin, per local mass: robot-local index
    const uint32_t* key_begin;     // per bin
    uint32_t* free_count;          // per bin
    uint32_t* free_taken;          // per bin
    uint32_t* free_slots;          // per bin, spring_cap entries from spring_begin
    uint32_t* status;              // [0] problems
};

// One-time set-up of a split population's development state (maps, keys,
// slots, free lists) from its packed arrays.
cudaError_t launch_split_devo_setup(const SplitDevoParams& p, uint32_t n_bins, uint32_t n_springs, cudaStream_t s);
// Applies the records: frees slots of parts a spring leaves, takes slots in
// parts it joins, appends halo masses and exports, writes the packed springs
// and the canonical topology.
cudaError_t launch_split_devo_apply(const SplitDevoParams& p, uint32_t n_bins, cudaStream_t s);
// Moves per-bin ranges [old_begin, old_begin + count) to new_begin (entries
// of entry_bytes bytes).
cudaError_t launch_relayout_ranges(const uint32_t* old_begin, const uint32_t* count, const uint32_t* new_begin,
                                   uint32_t n_bins, const void* src, void* dst, uint32_t entry_bytes,
                                   cudaStream_t s);

}  // namespace mb
