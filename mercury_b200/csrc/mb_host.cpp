// Host side of the C ABI (include/mercury_b200.h): context, upload and
// packing of a population into bins, launch configuration, chunked step
// launches replayed from CUDA graphs, collection.
//
// Packing.  The reference gives every robot one CTA and pads every robot to
// the largest mass and spring count (Simulator.cu:231-239, 489-494).  Here
// robots keep their own sizes and are grouped into bins, each simulated by
// one CTA; bins are filled largest-robot-first onto the least loaded bin
// (LPT), and the bin count is a multiple of the SM count so that every SM
// gets the same work.  Inside a bin:
//   - masses keep robot order (robot r's masses, then robot r+1's ...);
//   - non-air springs of each robot are sorted by (b - a, a) (for a lattice:
//     one direction, consecutive a), then placed so that the 8 springs of a
//     quarter-warp read distinct shared-memory bank groups at both ends;
//   - every mass gets a row of incident springs sorted by (other end,
//     spring index, a end before b end) -- the fixed summation order -- and
//     rows are stored 32 masses per slice, column-major (SELL-32), so that a
//     warp's k-th entries are consecutive words.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/mercury_b200.h"
#include "mb_devo.h"
#include "mb_internal.h"
#include "mb_pack.h"
#include "mb_voxel.h"
#include "mb_voxel_dev.h"

namespace mb {

// Composite id of two base materials (material.h:192-213).
int composite_id(int m1, int m2) {
    if (m1 == 0 || m2 == 0) return 0;
    int i = std::min(m1, m2) - 1, j = std::max(m1, m2) - 1;
    if (i == j) return i + 1;
    // pairs (i < j) of 22 materials numbered from 23 in row-major order
    return 23 + i * 21 - i * (i - 1) / 2 + (j - i - 1);
}

// Composite id of a material encoding (material.h:275-322): the lowest set
// bit, and the next one if any; air (bit 0) as the lowest bit gives air.
int decode_id(uint32_t e) {
    int idx[2] = {0, 0}, count = 0;
    for (int i = 0; i < 32; ++i)
        if (e & (1u << i)) {
            idx[count++] = i;
            if (i == 0 || count == 2) break;
        }
    if (idx[0] == 0) return 0;
    if (idx[1] == 0) return idx[0];
    return composite_id(idx[0], idx[1]);
}

namespace {

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        if (count <= n && p) return cudaSuccess;
        release();
        size_t c = std::max<size_t>(count, 1);
        cudaError_t e = cudaMalloc(&p, c * sizeof(T));
        if (e == cudaSuccess) n = c;
        return e;
    }
};

struct GraphKey {
    uint32_t steps;
    uint32_t t0_bits;
    uint32_t track;
    bool operator<(const GraphKey& o) const {
        if (steps != o.steps) return steps < o.steps;
        if (t0_bits != o.t0_bits) return t0_bits < o.t0_bits;
        return track < o.track;
    }
};

}  // namespace
}  // namespace mb

struct mb_context {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    std::string err;

    float dt = 0.0001f;  // Simulator.h:55
    float total_time = 0.0f;
    mb_mode mode = MB_MODE_REF_XPBD;
    mb_environment env{9.81f, 1.0e6f, 1.0f, 0.8f, 0.05f, 0.999f, 0.0f};
    float table[4 * MB_COMPOSITE_COUNT] = {};
    bool have_table = false;

    // population
    bool loaded = false;
    uint32_t n_robots = 0;
    uint64_t n_mass = 0, n_spring = 0;
    std::vector<int64_t> mass_off, spring_off;

    // packing result
    mb::KernelShape shape{512, 8, 2};
    uint32_t n_bins = 0;
    uint32_t max_bin_mass = 0;  // most (own) masses in one bin
    uint32_t rr_smem = 0;       // shared memory of the register-row kernel over every bin
    uint32_t max_degree = 0;    // most springs at one mass when uploaded
    uint32_t smem_optin = 0;    // the device's shared memory per CTA (opt-in)
    uint32_t grid = 0;  // CTAs per step launch (0 = one per bin)
    uint32_t chunk = 1000;
    bool use_graph = true;
    uint32_t smem_bytes = 0;
    mb_launch_config override_cfg{};

    // device buffers
    mb::DevBuf<float4> pos, vel;
    mb::DevBuf<float> stress;
    mb::DevBuf<uint8_t> mass_mat;
    mb::DevBuf<int64_t> d_mass_off;
    mb::DevBuf<float4> d_table;
    mb::DevBuf<mb::BinDesc> bins;
    mb::DevBuf<uint32_t> mass_gidx, spring_gidx, spring_pair, slice_off, slice_width;
    mb::DevBuf<uint16_t> inc;
    // streamed path: one robot per CTA, rows with u32 entries, per-spring scratch
    bool streamed = false;
    uint32_t stream_mpt = 2;
    mb::DevBuf<uint32_t> inc32;
    mb::DevBuf<uint32_t> exports;          // split bins: halo positions each part writes into the others
    // face drag (resident bins): corners, rows per packed mass, incidence
    mb::DevBuf<uint2> faces;
    mb::DevBuf<uint32_t> face_row;
    mb::DevBuf<uint16_t> face_inc;
    uint64_t n_faces = 0;          // faces of the population (three distinct corners)
    bool faces_packed = false;     // the packed bins hold them
    mb::DevBuf<float4> fd_scratch;  // streamed bins: face forces of a step
    mb::Packed upload_pack;                // host packing of the last mb_set_elements (reused)
    uint32_t cluster = 0;                  // split bins: CTAs per robot (0 = not split)
    // split bins in two groups: bins from split_bins0 in clusters of
    // cluster2, launched on stream2 beside the first group (fork and join
    // through the two events)
    uint32_t cluster2 = 0, split_bins0 = 0;
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    mb::DevBuf<float4> dp_scratch;
    mb::DevBuf<float> st_scratch;
    mb::DevBuf<float> spring_lbar;
    mb::DevBuf<uint8_t> mat_ids;           // composite ids used by the population
    mb::DevBuf<uint32_t> n_mat;            // their count (device scalar)
    mb::DevBuf<float> rates, invk;         // actuation table of one launch; 1/K per material
    uint32_t n_mat_host = 0;
    mb::DevBuf<uint32_t> bin_flags, robot_bin, robot_flags;
    mb::DevBuf<float> com;

    // topology in upload order, kept on the host for re-packing after
    // development (mb_devo) and for mb_collect_springs
    std::vector<uint16_t> h_pairs;
    std::vector<uint8_t> h_spring_mat, h_mass_mat;
    std::vector<float> h_lbar;
    std::vector<int64_t> h_face_off;  // empty: no faces
    std::vector<uint16_t> h_faces;
    // the next upload's copies are taken into these and swapped in when the
    // population is accepted: both sets keep their capacity, so a repeated
    // upload writes to memory that is already mapped
    std::vector<uint16_t> nx_pairs;
    std::vector<uint8_t> nx_spring_mat, nx_mass_mat;
    std::vector<float> nx_lbar;
    std::vector<int64_t> nx_face_off;
    std::vector<uint16_t> nx_faces;
    mb::DevBuf<int64_t> d_spring_off;
    mb::DevBuf<mb::DevoRecord> devo_out;
    std::vector<mb::DevoRecord> h_devo;
    double devo_ms[3] = {0.0, 0.0, 0.0};  // last mb_devo: select+read-back, re-pack, upload
    uint32_t devo_host_repacks = 0;       // mb_devo calls that fell back to the host packer

    // re-packing on the device after development, set up by the first
    // mb_devo after an upload: canonical topology on the device, packed slot
    // of every spring, free inert slots per bin, rows with spare capacity
    bool devo_ready = false;
    uint32_t n_packed = 0;                // packed spring slots
    std::vector<mb::BinDesc> h_bins;
    std::vector<uint32_t> h_robot_mass_base;
    std::vector<uint8_t> h_mat_ids;
    mb::DevBuf<uint16_t> d_pairs;
    mb::DevBuf<uint8_t> d_spring_mat, slot_of;
    mb::DevBuf<float> d_lbar;
    mb::DevBuf<uint32_t> pslot, robot_mass_base, free_count, free_taken, free_slots, devo_status, new_begin;
    mb::DevBuf<unsigned long long> rows_scratch;
    // development of split populations on the device (the partition of the
    // last packing; regions with spare capacity per bin, set up by the first
    // mb_devo after an upload)
    std::vector<uint8_t> h_part_of;
    std::vector<uint32_t> h_robot_parts, h_robot_slot0, h_robot_bin_first;
    bool split_devo = false;  // devo_ready holds the split state
    mb::DevBuf<uint8_t> d_part_of;
    mb::DevBuf<uint32_t> d_robot_parts, d_robot_slot0, d_bin_robot, sp_spring_cap, sp_export_cap, sp_map,
        sp_map_begin, sp_keys, sp_key_begin, slot_a, slot_b;

    // voxel populations built on the device (mb_set_voxel_population): the
    // template packing of one grid, reused while the key matches
    struct Voxel {
        bool valid = false;      // template packing uploaded
        uint32_t n_robots = 0;
        int sx = 0, sy = 0, sz = 0;
        uint32_t h_bits = 0, mass_bits = 0, mode = 0;
        uint32_t n_points = 0, n_springs = 0;  // per robot
        uint32_t max_bin_springs = 0;          // the template's largest bin (active springs bound)
        mb::DevBuf<float> pos;
        mb::DevBuf<uint16_t> src;
        mb::DevBuf<uint8_t> dir, cells;
        mb::DevBuf<uint32_t> n_spring, word, gidx;
        mb::DevBuf<float> lbar;
    } vox;
    bool vox_live = false;             // the population on the device came from the voxel builder
    bool host_topology_stale = false;  // h_mass_mat / h_spring_mat / h_bins behind the device

    std::map<mb::GraphKey, cudaGraphExec_t> graphs;
    // pinned staging of the packed arrays an upload copies to the device
    // (grown on demand, kept across uploads)
    void* stage = nullptr;
    size_t stage_bytes = 0;

    void clear_graphs() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }
    ~mb_context() {
        clear_graphs();
        if (stage) cudaFreeHost(stage);
        if (stream2) cudaStreamDestroy(stream2);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

mb_status fail(mb_context* c, mb_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return s;
}

mb_status cuda_fail(mb_context* c, cudaError_t e, const char* what) {
    return fail(c, MB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define MB_CUDA(ctx, call)                                  \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
    } while (0)

}  // namespace

namespace mb_detail {

uint32_t row_reg_smem(const mb_context* c);

// Whether the step applies the face drag (water mode, rho != 0): split
// robots are then packed with their faces (velocities exchanged with the
// positions).
bool face_drag_on(const mb_context* c) { return c->mode == MB_MODE_FORCE_WATER && c->env.face_drag != 0.0f; }

// Packs a population (caller's arrays or the context's host copy) with the
// context's device limits and launch override.  With `fallback_auto`, a
// population that no longer fits the override (after development) is
// re-planned automatically.
mb_status pack(mb_context* ctx, const mb_batch_desc* b, bool fallback_auto, mb::Packed& out,
               bool allow_split, bool rows_on_device = false) {
    mb::PackOptions po;
    po.rows_on_device = rows_on_device;
    po.sms = (uint32_t)std::max(ctx->num_sms, 1);
    po.smem_cap = mb::max_step_smem(ctx->device);
    po.mode = (uint32_t)ctx->mode;
    po.override = ctx->override_cfg;
    po.split_faces = face_drag_on(ctx);
    if (!allow_split) po.override.cluster = 1;
    po.ctas_per_sm = [ctx](const mb::KernelShape& sh, uint32_t smem) {
        return mb::ctas_per_sm(sh, (uint32_t)ctx->mode, false, smem);
    };
    po.cluster_fits = [ctx](const mb::KernelShape& sh, uint32_t cluster, uint32_t smem) {
        return mb::max_active_clusters(sh, (uint32_t)ctx->mode, cluster, smem) > 0;
    };
    std::string err;
    mb_status pst = mb::pack_population(b, po, out, err);
    const mb_launch_config none{};
    if (pst == MB_ERR_CAPACITY && fallback_auto && std::memcmp(&po.override, &none, sizeof(none)) != 0) {
        po.override = none;
        po.override.chunk = ctx->override_cfg.chunk;
        po.override.use_graph = ctx->override_cfg.use_graph;
        if (!allow_split) po.override.cluster = 1;
        pst = mb::pack_population(b, po, out, err);
    }
    if (pst != MB_OK) return fail(ctx, pst, "%s", err.c_str());
    return MB_OK;
}

// Uploads the packed arrays of `out` and the per-launch buffers sized by
// them; positions, velocities and stresses are not touched.  Rows the host
// did not build are built on the device (the development re-pack kernel);
// if they do not fit their regions or the shared memory, *rows_failed is
// set and the caller packs again with host-built rows.
mb_status upload_packed(mb_context* ctx, const mb::Packed& out, bool* rows_failed = nullptr) {
    ctx->clear_graphs();
    ctx->shape = out.shape;
    ctx->n_bins = out.n_bins;
    ctx->grid = out.grid;
    // the register-row kernel's layout: the usual one without the rows, 8
    // bytes of alignment, 8 bytes per spring (mb::row_reg_supported)
    ctx->max_bin_mass = ctx->rr_smem = 0;
    ctx->max_degree = out.max_degree;
    for (const mb::BinDesc& d : out.bins) {
        ctx->max_bin_mass = std::max(ctx->max_bin_mass, d.n_mass);
        ctx->rr_smem = std::max(ctx->rr_smem, mb::bin_smem_bytes(d.n_mass, d.n_spring, 0) + 8u + 8u * d.n_spring);
    }
    if (!ctx->smem_optin) ctx->smem_optin = mb::max_step_smem(ctx->device);
    ctx->smem_bytes = out.max_smem;
    ctx->streamed = out.streamed;
    ctx->cluster = out.cluster;
    ctx->cluster2 = out.cluster2;
    ctx->split_bins0 = out.split_bins0;
    if (ctx->cluster2 && !ctx->stream2) {  // created once, outside any capture
        MB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking));
        MB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
        MB_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
    }
    ctx->stream_mpt = out.shape.mpt;
    const uint32_t nb = out.n_bins;
    cudaStream_t st = ctx->stream;
    auto up = [&](auto& buf, const auto* src, size_t n) -> cudaError_t {
        cudaError_t e = buf.alloc(n);
        if (e != cudaSuccess || n == 0) return e;
        return cudaMemcpyAsync(buf.p, src, n * sizeof(*src), cudaMemcpyHostToDevice, st);
    };
    // the large packed arrays go through the pinned stage: copied into it by
    // host threads, then one DMA copy each
    {
        struct Item {
            void* dst;
            const void* src;
            size_t bytes, off;
        };
        std::vector<Item> items;
        size_t total = 0;
        auto add = [&](auto& buf, const auto& vec) -> cudaError_t {
            cudaError_t e = buf.alloc(vec.size());
            if (e != cudaSuccess || vec.empty()) return e;
            const size_t bytes = vec.size() * sizeof(vec[0]);
            items.push_back({buf.p, vec.data(), bytes, total});
            total += (bytes + 255) & ~size_t(255);
            return cudaSuccess;
        };
        MB_CUDA(ctx, add(ctx->mass_gidx, out.mass_gidx));
        MB_CUDA(ctx, add(ctx->spring_gidx, out.spring_gidx));
        MB_CUDA(ctx, add(ctx->spring_pair, out.pair));
        MB_CUDA(ctx, add(ctx->spring_lbar, out.lbar));
        MB_CUDA(ctx, add(ctx->inc, out.inc));
        if (total > ctx->stage_bytes) {
            if (ctx->stage) cudaFreeHost(ctx->stage);
            ctx->stage = nullptr;
            ctx->stage_bytes = 0;
            MB_CUDA(ctx, cudaHostAlloc(&ctx->stage, total + total / 4, cudaHostAllocDefault));
            ctx->stage_bytes = total + total / 4;
        }
        // nothing may still read the stage (or the buffers being replaced)
        MB_CUDA(ctx, cudaStreamSynchronize(st));
        // in four rounds, so that the DMA of one round overlaps the host copy
        // of the next (each round fills its own range of the stage)
        const unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
        constexpr size_t kRounds = 4;
        const size_t round = std::max<size_t>(4 << 20, (total + kRounds - 1) / kRounds);
        for (size_t r0 = 0; r0 < total; r0 += round) {
            const size_t r1 = std::min(total, r0 + round);
            const size_t piece = (r1 - r0 + nt - 1) / nt;
            mb::parallel_for(nt, nt, [&](uint32_t t) {
                const size_t lo = r0 + t * piece, hi = std::min(r1, lo + piece);
                for (const Item& it : items) {
                    const size_t a = std::max(lo, it.off), z = std::min(hi, it.off + it.bytes);
                    if (a < z)
                        std::memcpy(static_cast<char*>(ctx->stage) + a,
                                    static_cast<const char*>(it.src) + (a - it.off), z - a);
                }
            });
            for (const Item& it : items) {
                const size_t a = std::max(r0, it.off), z = std::min(r1, it.off + it.bytes);
                if (a < z)
                    MB_CUDA(ctx, cudaMemcpyAsync(static_cast<char*>(it.dst) + (a - it.off),
                                                 static_cast<char*>(ctx->stage) + a, z - a,
                                                 cudaMemcpyHostToDevice, st));
            }
        }
    }
    MB_CUDA(ctx, up(ctx->bins, out.bins.data(), out.bins.size()));
    MB_CUDA(ctx, up(ctx->slice_off, out.slice_off.data(), out.slice_off.size()));
    MB_CUDA(ctx, up(ctx->slice_width, out.slice_width.data(), out.slice_width.size()));
    MB_CUDA(ctx, up(ctx->exports, out.exports.data(), out.exports.size()));
    MB_CUDA(ctx, up(ctx->faces, reinterpret_cast<const uint2*>(out.faces.data()), out.faces.size() / 2));
    MB_CUDA(ctx, up(ctx->face_row, out.face_row.data(), out.face_row.size()));
    MB_CUDA(ctx, up(ctx->face_inc, out.face_inc.data(), out.face_inc.size()));
    ctx->n_faces = out.n_faces;
    ctx->faces_packed = !out.face_row.empty();
    if (out.streamed && ctx->faces_packed) MB_CUDA(ctx, ctx->fd_scratch.alloc(out.faces.size() / 2));
    if (out.streamed) {
        MB_CUDA(ctx, up(ctx->inc32, out.inc32.data(), out.inc32.size()));
        MB_CUDA(ctx, ctx->dp_scratch.alloc(std::max<size_t>(out.pair.size(), 1)));
        MB_CUDA(ctx, ctx->st_scratch.alloc(std::max<size_t>(out.pair.size(), 1)));
    }
    MB_CUDA(ctx, up(ctx->mat_ids, out.mat_ids.data(), out.mat_ids.size()));
    ctx->n_mat_host = (uint32_t)out.mat_ids.size();
    MB_CUDA(ctx, up(ctx->n_mat, &ctx->n_mat_host, 1));
    MB_CUDA(ctx, ctx->invk.alloc(std::max<uint32_t>(ctx->n_mat_host, 1)));
    MB_CUDA(ctx, ctx->rates.alloc((size_t)std::max<uint32_t>(ctx->n_mat_host, 1) * ctx->chunk));
    MB_CUDA(ctx, up(ctx->robot_bin, out.robot_bin.data(), out.robot_bin.size()));
    ctx->h_bins = out.bins;
    ctx->h_robot_mass_base = out.robot_mass_base;
    ctx->h_part_of = out.part_of;
    ctx->h_robot_parts = out.robot_parts;
    ctx->h_robot_slot0 = out.robot_slot0;
    ctx->h_robot_bin_first = out.robot_bin;
    ctx->split_devo = false;
    ctx->h_mat_ids = out.mat_ids;
    ctx->n_packed = (uint32_t)out.pair.size();
    ctx->devo_ready = false;
    MB_CUDA(ctx, ctx->bin_flags.alloc(nb));
    MB_CUDA(ctx, cudaMemsetAsync(ctx->bin_flags.p, 0, nb * sizeof(uint32_t), st));
    if (out.rows_on_device) {
        MB_CUDA(ctx, ctx->inc.alloc(std::max<uint64_t>(out.row_total, 1)));
        MB_CUDA(ctx, ctx->rows_scratch.alloc(2 * std::max<size_t>(out.pair.size(), 1)));
        MB_CUDA(ctx, ctx->free_count.alloc(nb));
        MB_CUDA(ctx, ctx->free_taken.alloc(nb));
        MB_CUDA(ctx, ctx->devo_status.alloc(2));
        MB_CUDA(ctx, cudaMemsetAsync(ctx->free_count.p, 0, nb * sizeof(uint32_t), st));
        MB_CUDA(ctx, cudaMemsetAsync(ctx->free_taken.p, 0, nb * sizeof(uint32_t), st));
        MB_CUDA(ctx, cudaMemsetAsync(ctx->devo_status.p, 0, 2 * sizeof(uint32_t), st));
        // the springs of every bin placed for the endpoint loads (the host
        // packer left them in upload order), then the rows built
        uint32_t max_springs = 0;
        for (const mb::BinDesc& d : out.bins) max_springs = std::max(max_springs, d.n_spring);
        MB_CUDA(ctx, mb::launch_bank_place(ctx->bins.p, nb, max_springs, ctx->spring_pair.p, ctx->spring_gidx.p,
                                           ctx->spring_lbar.p, ctx->rows_scratch.p, st));
        // no packed slot is inert here: spring_gidx < n_spring everywhere
        const mb::RebuildParams rp{ctx->bins.p,        nb,                   ctx->spring_pair.p,
                                   ctx->spring_gidx.p, (uint32_t)ctx->n_spring, ctx->slice_off.p,
                                   ctx->slice_width.p, ctx->inc.p,           ctx->inc32.p,
                                   0u,                 ctx->rows_scratch.p,  ctx->free_count.p,
                                   ctx->free_taken.p,  ctx->devo_status.p};
        MB_CUDA(ctx, mb::launch_rebuild(rp, st));
        uint32_t status[2] = {0, 0};
        MB_CUDA(ctx, cudaMemcpyAsync(status, ctx->devo_status.p, sizeof(status), cudaMemcpyDeviceToHost, st));
        MB_CUDA(ctx, cudaMemcpyAsync(ctx->h_bins.data(), ctx->bins.p, nb * sizeof(mb::BinDesc),
                                     cudaMemcpyDeviceToHost, st));
        MB_CUDA(ctx, cudaStreamSynchronize(st));
        if (status[0] || status[1] > mb::max_step_smem(ctx->device)) {
            if (rows_failed) *rows_failed = true;
            return MB_OK;
        }
        ctx->smem_bytes = status[1];  // the largest bin's need, exactly
    }
    // the host vectors of `out` may die after this call: wait for the copies
    MB_CUDA(ctx, cudaStreamSynchronize(st));
    return MB_OK;
}


// Material slots for every composite development can create: pairs of the
// base materials the masses carry.  Extra slots only widen the per-launch
// actuation table.
mb_status devo_material_slots(mb_context* c) {
    cudaStream_t st = c->stream;
    auto up = [&](auto& buf, const auto* src, size_t n) -> cudaError_t {
        cudaError_t e = buf.alloc(n);
        if (e != cudaSuccess || n == 0) return e;
        return cudaMemcpyAsync(buf.p, src, n * sizeof(*src), cudaMemcpyHostToDevice, st);
    };
    bool base[23] = {};
    for (uint8_t m : c->h_mass_mat) base[m] = true;
    std::vector<uint8_t> slot(256, mb::kNoMatSlot);
    for (size_t i = 0; i < c->h_mat_ids.size(); ++i) slot[c->h_mat_ids[i]] = (uint8_t)i;
    for (int i = 1; i < 23; ++i)
        for (int j = i; j < 23; ++j) {
            if (!base[i] || !base[j]) continue;
            const int id = mb::composite_id(i, j);
            if (slot[id] != mb::kNoMatSlot) continue;
            slot[id] = (uint8_t)c->h_mat_ids.size();
            c->h_mat_ids.push_back((uint8_t)id);
        }
    c->n_mat_host = (uint32_t)c->h_mat_ids.size();
    MB_CUDA(c, up(c->mat_ids, c->h_mat_ids.data(), c->h_mat_ids.size()));
    MB_CUDA(c, up(c->n_mat, &c->n_mat_host, 1));
    MB_CUDA(c, c->invk.alloc(c->n_mat_host));
    MB_CUDA(c, c->rates.alloc((size_t)c->n_mat_host * c->chunk));
    MB_CUDA(c, up(c->slot_of, slot.data(), 256));
    return MB_OK;
}

// Whether the split launch groups can still be scheduled with `smem` bytes
// of shared memory per CTA.
bool split_schedulable(const mb_context* c, uint32_t smem) {
    if (mb::max_active_clusters(c->shape, (uint32_t)c->mode, c->cluster, smem) <= 0) return false;
    return !c->cluster2 || mb::max_active_clusters(c->shape, (uint32_t)c->mode, c->cluster2, smem) > 0;
}

// Device pointers of the split development state.
mb::SplitDevoParams split_params(mb_context* c, const mb::DevoRecord* rec, uint32_t n_rec, uint32_t k) {
    mb::SplitDevoParams p{};
    p.rec = rec;
    p.n_rec = n_rec;
    p.k = k;
    p.n_bins = c->n_bins;
    p.pairs = c->d_pairs.p;
    p.spring_mat = c->d_spring_mat.p;
    p.lbar = c->d_lbar.p;
    p.mass_off = c->d_mass_off.p;
    p.part_of = c->d_part_of.p;
    p.robot_bin = c->robot_bin.p;
    p.robot_parts = c->d_robot_parts.p;
    p.robot_slot0 = c->d_robot_slot0.p;
    p.bin_robot = c->d_bin_robot.p;
    p.mass_gidx = c->mass_gidx.p;
    p.slot_of = c->slot_of.p;
    p.bins = c->bins.p;
    p.spring_pair = c->spring_pair.p;
    p.spring_lbar = c->spring_lbar.p;
    p.spring_gidx = c->spring_gidx.p;
    p.inert = (uint32_t)c->n_spring;
    p.slot_a = c->slot_a.p;
    p.slot_b = c->slot_b.p;
    p.spring_cap = c->sp_spring_cap.p;
    p.export_cap = c->sp_export_cap.p;
    p.exports = c->exports.p;
    p.map = c->sp_map.p;
    p.map_begin = c->sp_map_begin.p;
    p.keys = c->sp_keys.p;
    p.key_begin = c->sp_key_begin.p;
    p.free_count = c->free_count.p;
    p.free_taken = c->free_taken.p;
    p.free_slots = c->free_slots.p;
    p.status = c->devo_status.p;
    return p;
}

// One-time state of development on the device for a split population
// (first mb_devo after an upload): every bin's springs, exports and rows
// move to regions with spare capacity, its predicted-position buffers get
// room for more halo masses, and the maps from robot masses to local
// indices, the key tables and the slots of every spring are built.
// MB_ERR_CAPACITY: not possible here (faces, limits); the caller re-packs on
// the host instead.
mb_status split_devo_setup(mb_context* c) {
    if (c->faces_packed || c->h_part_of.size() != c->n_mass) return MB_ERR_CAPACITY;
    cudaStream_t st = c->stream;
    const uint64_t S = c->n_spring;
    const uint32_t nb = c->n_bins, R = c->n_robots;
    auto up = [&](auto& buf, const auto* src, size_t n) -> cudaError_t {
        cudaError_t e = buf.alloc(std::max<size_t>(n, 1));
        if (e != cudaSuccess || n == 0) return e;
        return cudaMemcpyAsync(buf.p, src, n * sizeof(*src), cudaMemcpyHostToDevice, st);
    };
    for (uint32_t r = 0; r < R; ++r)
        if (c->mass_off[r + 1] - c->mass_off[r] >= 65536) return MB_ERR_CAPACITY;
    MB_CUDA(c, up(c->d_pairs, c->h_pairs.data(), 2 * S));
    MB_CUDA(c, up(c->d_spring_mat, c->h_spring_mat.data(), S));
    MB_CUDA(c, up(c->d_lbar, c->h_lbar.data(), S));
    {
        const mb_status ms = devo_material_slots(c);
        if (ms != MB_OK) return ms;
    }
    // capacities and new regions
    const uint32_t smem_max = mb::max_step_smem(c->device);
    const uint32_t shape_cap = std::min<uint32_t>(c->shape.threads * c->shape.spt, mb::kMaxBinSprings);
    std::vector<uint32_t> bin_robot(nb, mb::kNoSlot), scap(nb), ecap(nb), kbeg(nb), mbeg(nb);
    std::vector<uint32_t> old_s(nb), cnt_s(nb), new_s(nb), old_e(nb), cnt_e(nb), new_e(nb);
    std::vector<uint32_t> new_i(nb);
    for (uint32_t r = 0; r < R; ++r)
        for (uint32_t q = 0; q < c->h_robot_parts[r]; ++q) bin_robot[c->h_robot_bin_first[r] + q] = r;
    std::vector<mb::BinDesc> nbins = c->h_bins;
    uint64_t ts = 0, te = 0, ti = 0, tk = 0, tm = 0;
    uint32_t smem = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        mb::BinDesc& d = nbins[b];
        const uint32_t ns = d.n_spring;
        if (ns > shape_cap) return MB_ERR_CAPACITY;
        scap[b] = std::max(ns, std::min(shape_cap, ns + std::max(256u, ns / 4)));
        ecap[b] = d.n_export + 256 + d.n_export / 4;
        uint32_t xc = bin_robot[b] == mb::kNoSlot ? d.n_all : std::max(d.n_all, std::min(4096u, d.n_all + 128 + d.n_all / 8));
        while (xc > d.n_all && mb::split_smem_bytes(xc, ns, d.n_inc, d.n_export) > smem_max) --xc;
        const uint32_t rc = (d.n_inc + d.n_inc / 2 + 8 * mb::kSliceWidth + 31) / 32 * 32;
        old_s[b] = d.spring_begin;
        cnt_s[b] = ns;
        new_s[b] = (uint32_t)ts;
        old_e[b] = d.export_begin;
        cnt_e[b] = d.n_export;
        new_e[b] = (uint32_t)te;
        new_i[b] = (uint32_t)ti;
        kbeg[b] = (uint32_t)tk;
        mbeg[b] = (uint32_t)tm;
        d.spring_begin = (uint32_t)ts;
        d.export_begin = (uint32_t)te;
        d.inc_begin = (uint32_t)ti;
        d.row_cap = rc;
        d.x_stride = xc;
        ts += scap[b];
        te += ecap[b];
        ti += rc;
        tk += xc;
        if (bin_robot[b] != mb::kNoSlot)
            tm += (uint64_t)(c->mass_off[bin_robot[b] + 1] - c->mass_off[bin_robot[b]]);
        smem = std::max(smem, mb::split_smem_bytes(xc, ns, d.n_inc, d.n_export));
    }
    if (ts >= (1ull << 31) || te >= (1ull << 31) || ti >= (1ull << 31) || tk >= (1ull << 31) ||
        tm >= (1ull << 31))
        return MB_ERR_CAPACITY;
    if (smem > smem_max || !split_schedulable(c, smem)) return MB_ERR_CAPACITY;
    // move the packed arrays into the new regions
    mb::DevBuf<uint32_t> d_old, d_cnt, d_new;
    auto relayout = [&](auto& buf, const std::vector<uint32_t>& ob, const std::vector<uint32_t>& cn,
                        const std::vector<uint32_t>& nbg, uint64_t total) -> cudaError_t {
        using T = std::remove_reference_t<decltype(*buf.p)>;
        cudaError_t e = up(d_old, ob.data(), nb);
        if (e == cudaSuccess) e = up(d_cnt, cn.data(), nb);
        if (e == cudaSuccess) e = up(d_new, nbg.data(), nb);
        mb::DevBuf<T> fresh;
        if (e == cudaSuccess) e = fresh.alloc(std::max<uint64_t>(total, 1));
        if (e == cudaSuccess)
            e = mb::launch_relayout_ranges(d_old.p, d_cnt.p, d_new.p, nb, buf.p, fresh.p, sizeof(T), st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) {
            std::swap(buf.p, fresh.p);
            std::swap(buf.n, fresh.n);
        }
        return e;
    };
    MB_CUDA(c, relayout(c->spring_pair, old_s, cnt_s, new_s, ts));
    MB_CUDA(c, relayout(c->spring_lbar, old_s, cnt_s, new_s, ts));
    MB_CUDA(c, relayout(c->spring_gidx, old_s, cnt_s, new_s, ts));
    MB_CUDA(c, relayout(c->exports, old_e, cnt_e, new_e, te));
    {
        std::vector<uint32_t> old_i(nb), cnt_i(nb);
        for (uint32_t b = 0; b < nb; ++b) {
            old_i[b] = c->h_bins[b].inc_begin;
            cnt_i[b] = c->h_bins[b].n_inc;
        }
        MB_CUDA(c, relayout(c->inc, old_i, cnt_i, new_i, ti));
    }
    c->h_bins = nbins;
    MB_CUDA(c, up(c->bins, c->h_bins.data(), nb));
    MB_CUDA(c, up(c->d_part_of, c->h_part_of.data(), c->h_part_of.size()));
    MB_CUDA(c, up(c->d_robot_parts, c->h_robot_parts.data(), R));
    MB_CUDA(c, up(c->d_robot_slot0, c->h_robot_slot0.data(), R));
    MB_CUDA(c, up(c->d_bin_robot, bin_robot.data(), nb));
    MB_CUDA(c, up(c->sp_spring_cap, scap.data(), nb));
    MB_CUDA(c, up(c->sp_export_cap, ecap.data(), nb));
    MB_CUDA(c, up(c->sp_map_begin, mbeg.data(), nb));
    MB_CUDA(c, up(c->sp_key_begin, kbeg.data(), nb));
    MB_CUDA(c, c->sp_map.alloc(std::max<uint64_t>(tm, 1)));
    MB_CUDA(c, cudaMemsetAsync(c->sp_map.p, 0xFF, std::max<uint64_t>(tm, 1) * sizeof(uint32_t), st));
    MB_CUDA(c, c->sp_keys.alloc(std::max<uint64_t>(tk, 1)));
    MB_CUDA(c, cudaMemsetAsync(c->sp_keys.p, 0, std::max<uint64_t>(tk, 1) * sizeof(uint32_t), st));
    MB_CUDA(c, c->slot_a.alloc(std::max<uint64_t>(S, 1)));
    MB_CUDA(c, c->slot_b.alloc(std::max<uint64_t>(S, 1)));
    MB_CUDA(c, c->free_count.alloc(nb));
    MB_CUDA(c, c->free_taken.alloc(nb));
    MB_CUDA(c, c->free_slots.alloc(std::max<uint64_t>(ts, 1)));
    MB_CUDA(c, c->rows_scratch.alloc(2 * std::max<uint64_t>(ts, 1)));
    MB_CUDA(c, c->devo_status.alloc(2));
    MB_CUDA(c, mb::launch_split_devo_setup(split_params(c, nullptr, 0, 0), nb, (uint32_t)S, st));
    MB_CUDA(c, cudaStreamSynchronize(st));
    c->n_packed = (uint32_t)ts;
    c->smem_bytes = smem;
    c->clear_graphs();
    c->devo_ready = true;
    c->split_devo = true;
    return MB_OK;
}

// One-time state of device re-packing (first mb_devo after an upload).
mb_status devo_setup(mb_context* c) {
    cudaStream_t st = c->stream;
    const uint64_t S = c->n_spring;
    const uint32_t nb = c->n_bins, R = c->n_robots;
    auto up = [&](auto& buf, const auto* src, size_t n) -> cudaError_t {
        cudaError_t e = buf.alloc(n);
        if (e != cudaSuccess || n == 0) return e;
        return cudaMemcpyAsync(buf.p, src, n * sizeof(*src), cudaMemcpyHostToDevice, st);
    };
    MB_CUDA(c, up(c->d_pairs, c->h_pairs.data(), 2 * S));
    MB_CUDA(c, up(c->d_spring_mat, c->h_spring_mat.data(), S));
    MB_CUDA(c, up(c->d_lbar, c->h_lbar.data(), S));
    MB_CUDA(c, c->pslot.alloc(S));
    MB_CUDA(c, mb::launch_build_pslot(c->spring_gidx.p, c->n_packed, (uint32_t)S, c->pslot.p, st));
    MB_CUDA(c, up(c->robot_mass_base, c->h_robot_mass_base.data(), R));
    {
        const mb_status ms = devo_material_slots(c);
        if (ms != MB_OK) return ms;
    }
    MB_CUDA(c, c->free_count.alloc(nb));
    MB_CUDA(c, c->free_taken.alloc(nb));
    MB_CUDA(c, cudaMemsetAsync(c->free_count.p, 0, nb * sizeof(uint32_t), st));
    MB_CUDA(c, cudaMemsetAsync(c->free_taken.p, 0, nb * sizeof(uint32_t), st));
    MB_CUDA(c, c->free_slots.alloc(c->n_packed));
    MB_CUDA(c, c->rows_scratch.alloc(2 * (size_t)c->n_packed));
    MB_CUDA(c, c->devo_status.alloc(2));
    // rows get spare capacity: half their size plus 8 slice columns
    std::vector<uint32_t> begin(nb);
    std::vector<mb::BinDesc> nbins = c->h_bins;
    uint64_t total = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t n = c->h_bins[b].n_inc;
        const uint32_t cap = (n + n / 2 + 8 * mb::kSliceWidth + 31) / 32 * 32;
        begin[b] = (uint32_t)total;
        nbins[b].inc_begin = (uint32_t)total;
        nbins[b].row_cap = cap;
        total += cap;
    }
    if (total >= (1ull << 32)) return fail(c, MB_ERR_CAPACITY, "rows too large for development");
    MB_CUDA(c, up(c->new_begin, begin.data(), nb));
    const uint32_t eb = c->streamed ? 4u : 2u;
    if (c->streamed) {
        mb::DevBuf<uint32_t> fresh;
        MB_CUDA(c, fresh.alloc(total));
        MB_CUDA(c, mb::launch_relayout(c->bins.p, c->new_begin.p, nb, c->inc32.p, fresh.p, eb, st));
        MB_CUDA(c, cudaStreamSynchronize(st));
        std::swap(c->inc32.p, fresh.p);
        std::swap(c->inc32.n, fresh.n);
    } else {
        mb::DevBuf<uint16_t> fresh;
        MB_CUDA(c, fresh.alloc(total));
        MB_CUDA(c, mb::launch_relayout(c->bins.p, c->new_begin.p, nb, c->inc.p, fresh.p, eb, st));
        MB_CUDA(c, cudaStreamSynchronize(st));
        std::swap(c->inc.p, fresh.p);
        std::swap(c->inc.n, fresh.n);
    }
    c->h_bins = nbins;
    MB_CUDA(c, up(c->bins, c->h_bins.data(), nb));
    MB_CUDA(c, cudaStreamSynchronize(st));
    c->clear_graphs();
    c->devo_ready = true;
    return MB_OK;
}

// Host re-packing of the context's topology copy: the fallback of
// development (`devo`), or a re-plan with the faces in the split parts when
// the face drag is switched on for a split population.
mb_status host_repack(mb_context* c, bool devo = true) {
    // split robots are cut by their current positions
    std::vector<float> pos;
    if (c->cluster) {
        pos.resize(4 * (size_t)c->n_mass);
        MB_CUDA(c, cudaMemcpyAsync(pos.data(), c->pos.p, pos.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                   c->stream));
        MB_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    const bool faces = !c->h_face_off.empty();
    const mb_batch_desc d{c->n_robots,
                          c->mass_off.data(),
                          pos.empty() ? nullptr : pos.data(),
                          nullptr,
                          c->h_mass_mat.data(),
                          c->spring_off.data(),
                          c->h_pairs.data(),
                          c->h_spring_mat.data(),
                          c->h_lbar.data(),
                          faces ? c->h_face_off.data() : nullptr,
                          faces ? c->h_faces.data() : nullptr};
    mb::Packed out;
    mb_status st = pack(c, &d, true, out, true);
    if (st == MB_OK) st = upload_packed(c, out);
    if (st != MB_OK) c->loaded = false;  // topology and packed arrays disagree now
    c->vox.valid = false;
    c->vox_live = false;
    if (devo) ++c->devo_host_repacks;
    return st;
}

// Brings the host copies of materials and bins up to date after a device
// build.
mb_status ensure_host_topology(mb_context* c) {
    if (!c->host_topology_stale) return MB_OK;
    cudaStream_t st = c->stream;
    c->h_mass_mat.resize(c->n_mass);
    c->h_spring_mat.resize(c->n_spring);
    MB_CUDA(c, cudaMemcpyAsync(c->h_mass_mat.data(), c->mass_mat.p, c->n_mass, cudaMemcpyDeviceToHost, st));
    MB_CUDA(c, cudaMemcpyAsync(c->h_spring_mat.data(), c->d_spring_mat.p, c->n_spring, cudaMemcpyDeviceToHost, st));
    MB_CUDA(c, cudaMemcpyAsync(c->h_bins.data(), c->bins.p, c->h_bins.size() * sizeof(mb::BinDesc),
                               cudaMemcpyDeviceToHost, st));
    MB_CUDA(c, cudaStreamSynchronize(st));
    c->host_topology_stale = false;
    return MB_OK;
}

// Template packing of a voxel population: every robot is the full lattice
// of the grid with every spring active; rows get the template's size as
// capacity (a robot's rows never need more than with every spring active).
mb_status voxel_setup(mb_context* c, uint32_t R, int sx, int sy, int sz, float h, float mass) {
    mb::VoxelTemplate T;
    mb::voxel_template(sx + 1, sy + 1, sz + 1, h, T);
    const uint32_t P = (uint32_t)((sx + 1) * (sy + 1) * (sz + 1)), Sr = (uint32_t)T.lbar.size();
    const uint64_t M = (uint64_t)R * P, S = (uint64_t)R * Sr;
    if (M >= (1ull << 31) || S >= (1ull << 31)) return fail(c, MB_ERR_CAPACITY, "population too large");
    std::vector<int64_t> mo(R + 1), so(R + 1);
    for (uint32_t r = 0; r <= R; ++r) {
        mo[r] = (int64_t)r * P;
        so[r] = (int64_t)r * Sr;
    }
    std::vector<uint16_t> pairs(2 * S);
    std::vector<float> lbar(S);
    for (uint32_t r = 0; r < R; ++r) {
        std::memcpy(pairs.data() + 2 * (size_t)r * Sr, T.pairs.data(), 2 * Sr * sizeof(uint16_t));
        std::memcpy(lbar.data() + (size_t)r * Sr, T.lbar.data(), Sr * sizeof(float));
    }
    std::vector<uint8_t> mm(M, 1), sm(S, 1);
    const mb_batch_desc d{R, mo.data(), nullptr, nullptr, mm.data(), so.data(), pairs.data(), sm.data(), lbar.data()};
    mb::Packed out;
    mb_status st = pack(c, &d, false, out, false);  // the device builder handles no split robots
    if (st != MB_OK) return st;
    // rows with their template size as capacity, plus spare slice columns
    {
        const bool streamed = out.streamed;
        mb::raw_vector<uint16_t> inc;
        mb::raw_vector<uint32_t> inc32;
        uint64_t total = 0;
        for (auto& bd : out.bins) {
            const uint32_t cap = (bd.n_inc + 8 * mb::kSliceWidth + 31) / 32 * 32;
            if (streamed)
                inc32.insert(inc32.end(), out.inc32.begin() + bd.inc_begin,
                             out.inc32.begin() + bd.inc_begin + bd.n_inc);
            else
                inc.insert(inc.end(), out.inc.begin() + bd.inc_begin, out.inc.begin() + bd.inc_begin + bd.n_inc);
            bd.inc_begin = (uint32_t)total;
            bd.row_cap = cap;
            total += cap;
            if (streamed)
                inc32.resize(total, mb::kPadEntry32);
            else
                inc.resize(total, mb::kPadEntry);
        }
        if (total >= (1ull << 32)) return fail(c, MB_ERR_CAPACITY, "rows too large");
        out.inc.swap(inc);
        out.inc32.swap(inc32);
    }
    c->clear_graphs();
    c->loaded = false;
    c->n_robots = R;
    c->n_mass = M;
    c->n_spring = S;
    c->mass_off = mo;
    c->spring_off = so;
    c->h_pairs.swap(pairs);
    c->h_lbar.swap(lbar);
    c->h_mass_mat.assign(M, 0);
    c->h_spring_mat.assign(S, 0);
    c->h_face_off.clear();  // voxel robots carry no faces
    c->h_faces.clear();
    st = upload_packed(c, out);
    if (st != MB_OK) return st;
    cudaStream_t cs = c->stream;
    auto up = [&](auto& buf, const auto* src, size_t n) -> cudaError_t {
        cudaError_t e = buf.alloc(n);
        if (e != cudaSuccess || n == 0) return e;
        return cudaMemcpyAsync(buf.p, src, n * sizeof(*src), cudaMemcpyHostToDevice, cs);
    };
    // every non-air composite gets a material slot
    std::vector<uint8_t> ids, slot(256, mb::kNoMatSlot);
    for (int id = 1; id < MB_COMPOSITE_COUNT; ++id) {
        slot[id] = (uint8_t)ids.size();
        ids.push_back((uint8_t)id);
    }
    c->h_mat_ids = ids;
    c->n_mat_host = (uint32_t)ids.size();
    MB_CUDA(c, up(c->mat_ids, ids.data(), ids.size()));
    MB_CUDA(c, up(c->n_mat, &c->n_mat_host, 1));
    MB_CUDA(c, c->invk.alloc(c->n_mat_host));
    MB_CUDA(c, c->rates.alloc((size_t)c->n_mat_host * c->chunk));
    MB_CUDA(c, up(c->slot_of, slot.data(), 256));
    // template arrays
    std::vector<uint32_t> word(out.pair.size()), nsp(out.bins.size());
    for (size_t i = 0; i < word.size(); ++i) word[i] = out.pair[i] & 0xFFFFFFu;
    for (size_t b = 0; b < out.bins.size(); ++b) nsp[b] = out.bins[b].n_spring;
    auto& v = c->vox;
    v.max_bin_springs = nsp.empty() ? 0u : *std::max_element(nsp.begin(), nsp.end());
    MB_CUDA(c, up(v.word, word.data(), word.size()));
    MB_CUDA(c, up(v.lbar, out.lbar.data(), out.lbar.size()));
    MB_CUDA(c, up(v.gidx, out.spring_gidx.data(), out.spring_gidx.size()));
    MB_CUDA(c, up(v.n_spring, nsp.data(), nsp.size()));
    MB_CUDA(c, up(v.pos, T.pos.data(), T.pos.size()));
    std::vector<uint16_t> src(Sr);
    for (uint32_t s = 0; s < Sr; ++s) src[s] = T.pairs[2 * s];
    MB_CUDA(c, up(v.src, src.data(), Sr));
    MB_CUDA(c, up(v.dir, T.dir.data(), Sr));
    // population arrays
    MB_CUDA(c, up(c->d_mass_off, mo.data(), R + 1));
    MB_CUDA(c, up(c->d_spring_off, so.data(), R + 1));
    MB_CUDA(c, c->pos.alloc(M));
    MB_CUDA(c, c->vel.alloc(M));
    MB_CUDA(c, c->mass_mat.alloc(M));
    MB_CUDA(c, c->d_spring_mat.alloc(S));
    MB_CUDA(c, c->stress.alloc(S + 1));
    MB_CUDA(c, cudaMemsetAsync(c->stress.p, 0, (S + 1) * sizeof(float), cs));
    MB_CUDA(c, c->robot_flags.alloc(R));
    MB_CUDA(c, c->com.alloc(3 * (size_t)R));
    const uint32_t nb = c->n_bins;
    MB_CUDA(c, c->free_count.alloc(nb));
    MB_CUDA(c, c->free_taken.alloc(nb));
    MB_CUDA(c, c->rows_scratch.alloc(2 * (size_t)c->n_packed));
    MB_CUDA(c, c->devo_status.alloc(2));
    MB_CUDA(c, v.cells.alloc((size_t)R * sx * sy * sz));
    MB_CUDA(c, cudaStreamSynchronize(cs));
    v.valid = true;
    v.n_robots = R;
    v.sx = sx;
    v.sy = sy;
    v.sz = sz;
    std::memcpy(&v.h_bits, &h, 4);
    std::memcpy(&v.mass_bits, &mass, 4);
    v.mode = (uint32_t)c->mode;
    v.n_points = P;
    v.n_springs = Sr;
    return MB_OK;
}

}  // namespace mb_detail

extern "C" {

const char* mb_version(void) { return "mercury_b200 0.1"; }

mb_status mb_context_create(int device, mb_context** out) {
    if (!out) return MB_ERR_ARGUMENT;
    *out = nullptr;
    std::unique_ptr<mb_context> c(new mb_context());
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return MB_ERR_CUDA;
    e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return MB_ERR_CUDA;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return MB_ERR_CUDA;
    *out = c.release();
    return MB_OK;
}

void mb_context_destroy(mb_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete ctx;
}

const char* mb_last_error(const mb_context* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

mb_status mb_set_materials(mb_context* ctx, const float* table) {
    if (!ctx || !table) return fail(ctx, MB_ERR_ARGUMENT, "null argument");
    for (int i = 0; i < 4 * MB_COMPOSITE_COUNT; ++i)
        if (!std::isfinite(table[i])) return fail(ctx, MB_ERR_ARGUMENT, "non-finite material entry %d", i);
    std::memcpy(ctx->table, table, sizeof(ctx->table));
    ctx->have_table = true;
    cudaSetDevice(ctx->device);
    MB_CUDA(ctx, ctx->d_table.alloc(MB_COMPOSITE_COUNT));
    MB_CUDA(ctx, cudaMemcpyAsync(ctx->d_table.p, ctx->table, sizeof(ctx->table),
                                 cudaMemcpyHostToDevice, ctx->stream));
    MB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->clear_graphs();
    return MB_OK;
}

mb_status mb_set_time_step(mb_context* ctx, float dt) {
    if (!ctx) return MB_ERR_ARGUMENT;
    if (!(dt > 0.0f) || !std::isfinite(dt)) return fail(ctx, MB_ERR_ARGUMENT, "time step must be > 0");
    if (dt != ctx->dt) ctx->clear_graphs();
    ctx->dt = dt;
    return MB_OK;
}
float mb_get_time_step(const mb_context* ctx) { return ctx ? ctx->dt : 0.0f; }
mb_status mb_set_total_time(mb_context* ctx, float t) {
    if (!ctx) return MB_ERR_ARGUMENT;
    ctx->total_time = t;
    return MB_OK;
}
float mb_get_total_time(const mb_context* ctx) { return ctx ? ctx->total_time : 0.0f; }

mb_status mb_set_mode(mb_context* ctx, mb_mode mode) {
    if (!ctx) return MB_ERR_ARGUMENT;
    if (mode != MB_MODE_REF_XPBD && mode != MB_MODE_FORCE_LAND && mode != MB_MODE_FORCE_WATER)
        return fail(ctx, MB_ERR_ARGUMENT, "unknown mode %d", (int)mode);
    if (mode != ctx->mode) ctx->clear_graphs();
    ctx->mode = mode;
    return MB_OK;
}

mb_status mb_get_mode(const mb_context* ctx, mb_mode* mode) {
    if (!ctx || !mode) return MB_ERR_ARGUMENT;
    *mode = ctx->mode;
    return MB_OK;
}

mb_status mb_set_environment(mb_context* ctx, const mb_environment* env) {
    if (!ctx || !env) return fail(ctx, MB_ERR_ARGUMENT, "null argument");
    const float v[7] = {env->g,    env->floor_stiffness, env->friction_static, env->friction_kinetic,
                        env->drag, env->damping,         env->face_drag};
    for (float f : v)
        if (!std::isfinite(f) || f < 0.0f) return fail(ctx, MB_ERR_ARGUMENT, "environment values must be finite and >= 0");
    ctx->env = *env;
    ctx->clear_graphs();
    return MB_OK;
}

mb_status mb_get_environment(const mb_context* ctx, mb_environment* env) {
    if (!ctx || !env) return MB_ERR_ARGUMENT;
    *env = ctx->env;
    return MB_OK;
}

void* mb_get_stream(const mb_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

mb_status mb_get_launch_config(const mb_context* ctx, mb_launch_config* cfg) {
    if (!ctx || !cfg) return MB_ERR_ARGUMENT;
    cfg->threads = ctx->shape.threads;
    cfg->springs_per_thread = ctx->shape.spt;
    cfg->masses_per_thread = ctx->shape.mpt;
    cfg->bins = ctx->n_bins;
    cfg->chunk = ctx->chunk;
    cfg->use_graph = ctx->use_graph ? 1 : 0;
    cfg->streamed = ctx->streamed ? 1 : 0;
    cfg->cluster = ctx->cluster;
    return MB_OK;
}

mb_status mb_get_step_variant(const mb_context* ctx, uint32_t* register_rows, uint32_t* smem_bytes) {
    if (!ctx) return MB_ERR_ARGUMENT;
    if (!ctx->loaded) return MB_ERR_STATE;
    const uint32_t rr = mb_detail::row_reg_smem(ctx);
    if (register_rows) *register_rows = rr ? 1u : 0u;
    if (smem_bytes) *smem_bytes = rr ? rr : ctx->smem_bytes;
    return MB_OK;
}

mb_status mb_get_packed_springs(const mb_context* ctx, uint32_t* words, uint64_t capacity, uint64_t* count) {
    if (!ctx || !count) return MB_ERR_ARGUMENT;
    if (!ctx->loaded) return MB_ERR_STATE;
    *count = ctx->n_packed;
    if (!words) return MB_OK;
    if (capacity < ctx->n_packed) return MB_ERR_CAPACITY;
    cudaSetDevice(ctx->device);
    if (ctx->n_packed &&
        cudaMemcpyAsync(words, ctx->spring_pair.p, ctx->n_packed * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                        ctx->stream) != cudaSuccess)
        return MB_ERR_CUDA;
    return cudaStreamSynchronize(ctx->stream) == cudaSuccess ? MB_OK : MB_ERR_CUDA;
}

mb_status mb_plan_population(const mb_batch_desc* batch, const mb_launch_config* cfg, uint32_t num_sms,
                             uint32_t smem_bytes, mb_plan_stats* stats) {
    if (!batch || !stats || batch->n_robots == 0 || !batch->mass_offsets || !batch->spring_offsets ||
        !batch->mass_material || (batch->spring_offsets[batch->n_robots] &&
                                  (!batch->pairs || !batch->spring_material || !batch->lbar)))
        return MB_ERR_ARGUMENT;
    mb::PackOptions po;
    po.sms = num_sms ? num_sms : 148;
    po.smem_cap = smem_bytes ? smem_bytes : 232448;
    if (cfg) po.override = *cfg;
    mb::Packed out;
    std::string err;
    const mb_status st = mb::pack_population(batch, po, out, err);
    if (st != MB_OK) return st;
    std::memset(stats, 0, sizeof(*stats));
    stats->threads = out.shape.threads;
    stats->springs_per_thread = out.shape.spt;
    stats->masses_per_thread = out.shape.mpt;
    stats->bins = out.n_bins;
    stats->streamed = out.streamed ? 1u : 0u;
    stats->cluster = out.cluster;
    stats->cluster2 = out.cluster2;
    stats->split_bins0 = out.split_bins0;
    stats->max_smem_bytes = out.max_smem;
    stats->masses = out.masses;
    stats->active_springs = out.active_springs;
    stats->incidence_entries = out.inc_entries;
    stats->incidence_padding = out.inc_padding;
    stats->aligned_slices = out.aligned_slices;
    stats->rank_slices = out.rank_slices;
    stats->material_slots = (uint32_t)out.mat_ids.size();
    uint32_t mx = 0, mn = 0xFFFFFFFFu;
    for (const auto& d : out.bins) {
        mx = std::max(mx, d.n_spring);
        mn = std::min(mn, d.n_spring);
    }
    stats->max_bin_springs = mx;
    stats->min_bin_springs = out.bins.empty() ? 0 : mn;
    const uint32_t ctas = out.grid ? std::min(out.grid, out.n_bins) : out.n_bins;
    std::vector<uint64_t> per(ctas, 0);
    for (size_t b = 0; b < out.bins.size(); ++b) per[b % ctas] += out.bins[b].n_spring;
    stats->ctas = ctas;
    stats->max_cta_springs = per.empty() ? 0 : (uint32_t)*std::max_element(per.begin(), per.end());
    stats->min_cta_springs = per.empty() ? 0 : (uint32_t)*std::min_element(per.begin(), per.end());
    return MB_OK;
}

uint32_t mb_kernel_shapes(mb_launch_config* out, uint32_t capacity) {
    mb::KernelShape tmp[64];
    const uint32_t nr = mb::list_shapes(tmp, 64, false);
    const uint32_t ns = mb::list_shapes(tmp + std::min<uint32_t>(nr, 64), 64 - std::min<uint32_t>(nr, 64), true);
    const uint32_t n = std::min<uint32_t>(nr + ns, 64);
    for (uint32_t i = 0; i < n && out && i < capacity; ++i) {
        mb_launch_config c{};
        c.threads = tmp[i].threads;
        c.springs_per_thread = tmp[i].spt;
        c.masses_per_thread = tmp[i].mpt;
        c.streamed = i >= nr ? 1u : 0u;
        c.use_graph = 1;
        out[i] = c;
    }
    return n;
}

mb_status mb_set_launch_config(mb_context* ctx, const mb_launch_config* cfg) {
    if (!ctx || !cfg) return MB_ERR_ARGUMENT;
    const uint32_t cl = cfg->cluster;
    if (cl != 0 && cl != 1 && cl != 2 && cl != 4 && cl != 8)
        return fail(ctx, MB_ERR_ARGUMENT, "cluster must be 0, 1, 2, 4 or 8");
    if (cfg->threads && !cfg->streamed) {
        mb::KernelShape s{cfg->threads, cfg->springs_per_thread, cfg->masses_per_thread};
        if (cl > 1 ? !mb::split_supported(s) : !mb::shape_supported(s))
            return fail(ctx, MB_ERR_ARGUMENT, "kernel shape %u/%u/%u not compiled%s", s.threads,
                        s.spt, s.mpt, cl > 1 ? " for split robots" : "");
    }
    ctx->override_cfg = *cfg;
    if (cfg->chunk) {
        ctx->chunk = cfg->chunk;
        if (ctx->loaded) {
            cudaSetDevice(ctx->device);
            MB_CUDA(ctx, ctx->rates.alloc((size_t)std::max<uint32_t>(ctx->n_mat_host, 1) * ctx->chunk));
        }
    }
    ctx->use_graph = cfg->use_graph != 0;
    ctx->clear_graphs();
    ctx->vox.valid = false;  // the next voxel upload re-plans its template
    return MB_OK;
}

mb_status mb_set_elements(mb_context* ctx, const mb_batch_desc* b) {
    if (!ctx || !b) return fail(ctx, MB_ERR_ARGUMENT, "null argument");
    if (!ctx->have_table) return fail(ctx, MB_ERR_STATE, "material table not set");
    const uint32_t R = b->n_robots;
    if (R == 0) return fail(ctx, MB_ERR_ARGUMENT, "empty population");
    if (!b->mass_offsets || !b->spring_offsets || !b->pos || !b->vel || !b->mass_material)
        return fail(ctx, MB_ERR_ARGUMENT, "null array");
    if (b->mass_offsets[0] != 0 || b->spring_offsets[0] != 0)
        return fail(ctx, MB_ERR_ARGUMENT, "offsets must start at 0");
    const uint64_t M = (uint64_t)b->mass_offsets[R], S = (uint64_t)b->spring_offsets[R];
    if (S && (!b->pairs || !b->spring_material || !b->lbar))
        return fail(ctx, MB_ERR_ARGUMENT, "null spring array");
    if (M >= (1ull << 31) || S >= (1ull << 31)) return fail(ctx, MB_ERR_CAPACITY, "population too large");
    const bool faces = b->face_offsets && b->faces;
    if ((b->face_offsets != nullptr) != (b->faces != nullptr))
        return fail(ctx, MB_ERR_ARGUMENT, "face_offsets and faces must both be given or both be NULL");
    if (faces && b->face_offsets[0] != 0) return fail(ctx, MB_ERR_ARGUMENT, "offsets must start at 0");
    const uint64_t F = faces ? (uint64_t)b->face_offsets[R] : 0;
    if (F >= (1ull << 31)) return fail(ctx, MB_ERR_CAPACITY, "population too large");

    cudaSetDevice(ctx->device);
    // the host copy of the topology is taken while the population is
    // packed, by three copier threads (the pairs alone are the largest array)
    std::thread copier([&] {
        ctx->nx_face_off.clear();
        ctx->nx_faces.clear();
        if (F) {
            ctx->nx_face_off.assign(b->face_offsets, b->face_offsets + R + 1);
            ctx->nx_faces.assign(b->faces, b->faces + 3 * F);
        }
        ctx->nx_mass_mat.assign(b->mass_material, b->mass_material + M);
        ctx->nx_spring_mat.assign(b->spring_material, b->spring_material + S);
    });
    std::thread copier_pairs([&] { ctx->nx_pairs.assign(b->pairs, b->pairs + 2 * S); });
    std::thread copier_lbar([&] { ctx->nx_lbar.assign(b->lbar, b->lbar + S); });
    // kept in the context: its arrays keep their capacity across uploads.
    // Resident rows are built on the device unless MB_HOST_ROWS=1.
    mb::Packed& out = ctx->upload_pack;
    const char* host_rows = std::getenv("MB_HOST_ROWS");
    const bool device_rows = !(host_rows && host_rows[0] == '1');
    const mb_status pst = mb_detail::pack(ctx, b, false, out, true, device_rows);
    copier.join();
    copier_pairs.join();
    copier_lbar.join();
    if (pst != MB_OK) return pst;

    // the population is accepted: keep its topology on the host (for
    // re-packing after development) and upload state and packed arrays
    ctx->clear_graphs();
    ctx->loaded = false;
    ctx->vox.valid = false;
    ctx->vox_live = false;
    ctx->host_topology_stale = false;
    ctx->n_robots = R;
    ctx->n_mass = M;
    ctx->n_spring = S;
    ctx->mass_off.assign(b->mass_offsets, b->mass_offsets + R + 1);
    ctx->spring_off.assign(b->spring_offsets, b->spring_offsets + R + 1);
    ctx->h_mass_mat.swap(ctx->nx_mass_mat);
    ctx->h_pairs.swap(ctx->nx_pairs);
    ctx->h_spring_mat.swap(ctx->nx_spring_mat);
    ctx->h_lbar.swap(ctx->nx_lbar);
    ctx->h_face_off.swap(ctx->nx_face_off);
    ctx->h_faces.swap(ctx->nx_faces);
    cudaStream_t st = ctx->stream;
    auto up = [&](auto& buf, const auto* src, size_t n) -> cudaError_t {
        cudaError_t e = buf.alloc(n);
        if (e != cudaSuccess || n == 0) return e;
        return cudaMemcpyAsync(buf.p, src, n * sizeof(*src), cudaMemcpyHostToDevice, st);
    };
    MB_CUDA(ctx, up(ctx->pos, reinterpret_cast<const float4*>(b->pos), M));
    MB_CUDA(ctx, up(ctx->vel, reinterpret_cast<const float4*>(b->vel), M));
    MB_CUDA(ctx, up(ctx->mass_mat, b->mass_material, M));
    MB_CUDA(ctx, up(ctx->d_mass_off, b->mass_offsets, R + 1));
    MB_CUDA(ctx, up(ctx->d_spring_off, b->spring_offsets, R + 1));
    // one element more: the stress of inert packed slots (development)
    MB_CUDA(ctx, ctx->stress.alloc(S + 1));
    MB_CUDA(ctx, cudaMemsetAsync(ctx->stress.p, 0, (S + 1) * sizeof(float), st));
    MB_CUDA(ctx, ctx->robot_flags.alloc(R));
    MB_CUDA(ctx, ctx->com.alloc(3 * (size_t)R));
    bool rows_failed = false;
    mb_status ust = mb_detail::upload_packed(ctx, out, &rows_failed);
    if (ust == MB_OK && rows_failed) {  // rare: the host builds the rows
        ust = mb_detail::pack(ctx, b, false, out, true, false);
        if (ust == MB_OK) ust = mb_detail::upload_packed(ctx, out);
    }
    if (ust != MB_OK) return ust;
    ctx->loaded = true;
    return MB_OK;
}

mb_status mb_set_state(mb_context* ctx, const float* pos, const float* vel) {
    if (!ctx || !pos || !vel) return fail(ctx, MB_ERR_ARGUMENT, "null argument");
    if (!ctx->loaded) return fail(ctx, MB_ERR_STATE, "no population uploaded");
    cudaSetDevice(ctx->device);
    const size_t bytes = ctx->n_mass * sizeof(float4);
    MB_CUDA(ctx, cudaMemcpyAsync(ctx->pos.p, pos, bytes, cudaMemcpyHostToDevice, ctx->stream));
    MB_CUDA(ctx, cudaMemcpyAsync(ctx->vel.p, vel, bytes, cudaMemcpyHostToDevice, ctx->stream));
    MB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MB_OK;
}

}  // extern "C"

// Internal helpers: C++ linkage, internal to this file.
namespace mb_detail {

// Shared memory of the register-row step kernel, or 0 when it does not
// apply: streamed or split bins, a bin of more than one mass per thread, a
// mass with more springs than the registers hold rows for (at upload: the
// kernel stays correct when development adds springs, reading longer rows
// from global memory), face drag, a shape without the variant, or too little
// shared memory.  Device development of resident bins keeps every bin's
// spring count, and the device voxel builder only removes springs, so the
// planned bins bound the need.
uint32_t row_reg_smem(const mb_context* c) {
    const bool faces = face_drag_on(c) && c->faces_packed;
    if (c->streamed || c->cluster || faces || !mb::row_reg_supported(c->shape) ||
        c->max_bin_mass > c->shape.threads || c->max_degree > mb::row_reg_width())
        return 0;
    return c->rr_smem <= c->smem_optin ? c->rr_smem : 0u;
}

mb::StepParams make_params(mb_context* c, float t0, uint32_t steps, bool track) {
    mb::StepParams p{};
    p.bins = c->bins.p;
    p.n_bins = c->n_bins;
    p.grid = c->grid;
    p.pos = c->pos.p;
    p.vel = c->vel.p;
    p.stress = c->stress.p;
    p.mass_gidx = c->mass_gidx.p;
    p.spring_gidx = c->spring_gidx.p;
    p.spring_pair = c->spring_pair.p;
    p.spring_lbar = c->spring_lbar.p;
    p.slice_off = c->slice_off.p;
    p.slice_width = c->slice_width.p;
    p.inc = c->inc.p;
    p.n_mat = c->n_mat.p;
    p.rates = c->rates.p;
    p.invk = c->invk.p;
    p.bin_flags = c->bin_flags.p;
    p.dt = c->dt;
    p.t0 = t0;
    p.steps = steps;
    p.track = track ? 1u : 0u;
    p.smem_bytes = c->smem_bytes;
    p.mode = (uint32_t)c->mode;
    p.inc32 = c->inc32.p;
    p.exports = c->exports.p;
    p.dp = c->dp_scratch.p;
    p.st = c->st_scratch.p;
    p.g = c->env.g;
    p.floor_stiffness = c->env.floor_stiffness;
    p.mu_s = c->env.friction_static;
    p.mu_k = c->env.friction_kinetic;
    p.drag = c->env.drag;
    p.damping = c->env.damping;
    p.faces = c->faces.p;
    p.face_row = c->face_row.p;
    p.face_inc = c->face_inc.p;
    p.fd = c->fd_scratch.p;
    p.face_coef = (float)(-(double)c->env.face_drag / 6.0);
    p.face_on = c->mode == MB_MODE_FORCE_WATER && c->env.face_drag != 0.0f && c->faces_packed ? 1u : 0u;
    if (const uint32_t rr = row_reg_smem(c)) {
        p.one_mass_per_thread = 1u;
        p.smem_bytes = rr;
    }
    return p;
}

// Float clock after `n` steps from t (Simulator.cu:447).
float advance(float t, float dt, uint32_t n) {
    volatile float v = t;
    for (uint32_t i = 0; i < n; ++i) v = v + dt;
    return v;
}

// Split bins: one launch, or the two groups side by side (the second on
// stream2, forked from the main stream and joined back before the next
// launch).  Once forked, stream2 is joined back even when a launch failed,
// so that a stream capture never ends with an unjoined fork.
cudaError_t launch_split_groups(mb_context* c, const mb::StepParams& p) {
    if (!c->cluster2) return mb::launch_split(p, c->shape, c->cluster, c->stream);
    cudaError_t e = cudaEventRecord(c->ev_fork, c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream2, c->ev_fork, 0);
    if (e != cudaSuccess) return e;
    mb::StepParams p0 = p, p1 = p;
    p0.n_bins = c->split_bins0;
    p1.bins = p.bins + c->split_bins0;
    p1.bin_flags = p.bin_flags + c->split_bins0;
    p1.n_bins = p.n_bins - c->split_bins0;
    e = mb::launch_split(p0, c->shape, c->cluster, c->stream);
    const cudaError_t e1 = mb::launch_split(p1, c->shape, c->cluster2, c->stream2);
    cudaError_t j = cudaEventRecord(c->ev_join, c->stream2);
    if (j == cudaSuccess) j = cudaStreamWaitEvent(c->stream, c->ev_join, 0);
    return e != cudaSuccess ? e : e1 != cudaSuccess ? e1 : j;
}

// Issues the chunk launches for `steps` steps from clock t0 on the stream.
cudaError_t issue_chunks(mb_context* c, float t0, uint32_t steps, bool track) {
    float t = t0;
    uint32_t done = 0;
    while (done < steps) {
        const uint32_t n = std::min(c->chunk, steps - done);
        cudaError_t ea = mb::launch_actuation(c->d_table.p, c->mat_ids.p, c->n_mat.p, t, c->dt, n,
                                              (uint32_t)c->mode, c->rates.p, c->invk.p, c->stream);
        if (ea != cudaSuccess) return ea;
        mb::StepParams p = make_params(c, t, n, track);
        cudaError_t e = c->streamed  ? mb::launch_stream(p, 1024, c->stream_mpt, c->stream)
                        : c->cluster ? launch_split_groups(c, p)
                                     : mb::launch_step(p, c->shape, c->stream);
        if (e != cudaSuccess) return e;
        t = advance(t, c->dt, n);
        done += n;
    }
    return cudaSuccess;
}

mb_status run(mb_context* c, uint32_t steps, bool track) {
    if (!c->loaded) return fail(c, MB_ERR_STATE, "no population uploaded");
    if (steps == 0) return MB_OK;
    if (face_drag_on(c) && c->n_faces && !c->faces_packed) {
        // split robots packed without their faces: re-plan them with (once)
        const mb_status rs = host_repack(c, false);
        if (rs != MB_OK) return rs;
        if (!c->faces_packed) return fail(c, MB_ERR_CAPACITY, "face drag: the faces do not fit the step kernels");
    }
    cudaSetDevice(c->device);
    const float t0 = c->total_time;
    if (c->use_graph) {
        uint32_t bits;
        std::memcpy(&bits, &t0, 4);
        const mb::GraphKey key{steps, bits, track ? 1u : 0u};
        auto it = c->graphs.find(key);
        if (it == c->graphs.end()) {
            if (c->graphs.size() >= 16) c->clear_graphs();
            // kernel attributes cannot change inside a capture
            MB_CUDA(c, c->streamed ? mb::prepare_stream(1024, c->stream_mpt, (uint32_t)c->mode, track, c->smem_bytes)
                                    : c->cluster ? mb::prepare_split(c->shape, (uint32_t)c->mode, track, c->smem_bytes)
                                    : mb::prepare_step(c->shape, (uint32_t)c->mode, track,
                                                       std::max(c->smem_bytes, row_reg_smem(c))));
            cudaGraph_t g;
            MB_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = issue_chunks(c, t0, steps, track);
            cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
            if (e != cudaSuccess) {
                if (e2 == cudaSuccess) cudaGraphDestroy(g);
                return cuda_fail(c, e, "capture of step launches");
            }
            if (e2 != cudaSuccess) return cuda_fail(c, e2, "cudaStreamEndCapture");
            cudaGraphExec_t ex;
            cudaError_t e3 = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            if (e3 != cudaSuccess) return cuda_fail(c, e3, "cudaGraphInstantiate");
            it = c->graphs.emplace(key, ex).first;
        }
        MB_CUDA(c, cudaGraphLaunch(it->second, c->stream));
    } else {
        MB_CUDA(c, c->streamed ? mb::prepare_stream(1024, c->stream_mpt, (uint32_t)c->mode, track, c->smem_bytes)
                                    : c->cluster ? mb::prepare_split(c->shape, (uint32_t)c->mode, track, c->smem_bytes)
                                    : mb::prepare_step(c->shape, (uint32_t)c->mode, track,
                                                       std::max(c->smem_bytes, row_reg_smem(c))));
        cudaError_t e = issue_chunks(c, t0, steps, track);
        if (e != cudaSuccess) return cuda_fail(c, e, "step launch");
    }
    c->total_time = advance(t0, c->dt, steps);
    return MB_OK;
}

}  // namespace mb_detail

extern "C" {

mb_status mb_run_steps(mb_context* ctx, uint32_t steps, int track_stresses) {
    if (!ctx) return MB_ERR_ARGUMENT;
    return mb_detail::run(ctx, steps, track_stresses != 0);
}

mb_status mb_simulate(mb_context* ctx, float duration, int track_stresses, uint32_t* steps_taken) {
    if (!ctx) return MB_ERR_ARGUMENT;
    if (!std::isfinite(duration)) return fail(ctx, MB_ERR_ARGUMENT, "non-finite duration");
    // step count of the reference loop (Simulator.cu:428-449)
    uint32_t n = 0;
    volatile float rem = duration;
    while (rem > 0.0f) {
        rem = rem - ctx->dt;
        ++n;
        if (n == 0xFFFFFFFFu) return fail(ctx, MB_ERR_ARGUMENT, "too many steps");
    }
    if (steps_taken) *steps_taken = n;
    return mb_detail::run(ctx, n, track_stresses != 0);
}

mb_status mb_collect(mb_context* ctx, float* pos, float* vel, float* stress) {
    if (!ctx) return MB_ERR_ARGUMENT;
    if (!ctx->loaded) return fail(ctx, MB_ERR_STATE, "no population uploaded");
    cudaSetDevice(ctx->device);
    const size_t mb4 = ctx->n_mass * sizeof(float4);
    if (pos) MB_CUDA(ctx, cudaMemcpyAsync(pos, ctx->pos.p, mb4, cudaMemcpyDeviceToHost, ctx->stream));
    if (vel) MB_CUDA(ctx, cudaMemcpyAsync(vel, ctx->vel.p, mb4, cudaMemcpyDeviceToHost, ctx->stream));
    if (stress && ctx->n_spring)
        MB_CUDA(ctx, cudaMemcpyAsync(stress, ctx->stress.p, ctx->n_spring * sizeof(float),
                                     cudaMemcpyDeviceToHost, ctx->stream));
    MB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MB_OK;
}

mb_status mb_centre_of_mass(mb_context* ctx, float* com) {
    if (!ctx || !com) return fail(ctx, MB_ERR_ARGUMENT, "null argument");
    if (!ctx->loaded) return fail(ctx, MB_ERR_STATE, "no population uploaded");
    cudaSetDevice(ctx->device);
    MB_CUDA(ctx, mb::launch_com(ctx->pos.p, ctx->mass_mat.p, ctx->d_mass_off.p, ctx->n_robots,
                                ctx->com.p, ctx->stream));
    MB_CUDA(ctx, cudaMemcpyAsync(com, ctx->com.p, 3 * sizeof(float) * ctx->n_robots,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    MB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MB_OK;
}

mb_status mb_robot_flags(mb_context* ctx, uint32_t* flags) {
    if (!ctx || !flags) return fail(ctx, MB_ERR_ARGUMENT, "null argument");
    if (!ctx->loaded) return fail(ctx, MB_ERR_STATE, "no population uploaded");
    cudaSetDevice(ctx->device);
    MB_CUDA(ctx, mb::launch_flags(ctx->pos.p, ctx->d_mass_off.p, ctx->n_robots,
                                  ctx->robot_flags.p, ctx->stream));
    if (!ctx->streamed && !ctx->cluster)
        MB_CUDA(ctx, mb::launch_bin_flags(ctx->bin_flags.p, ctx->robot_bin.p, ctx->n_robots, ctx->robot_flags.p,
                                          ctx->stream));
    MB_CUDA(ctx, cudaMemcpyAsync(flags, ctx->robot_flags.p, sizeof(uint32_t) * ctx->n_robots,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    MB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MB_OK;
}

mb_status mb_synchronize(mb_context* ctx) {
    if (!ctx) return MB_ERR_ARGUMENT;
    cudaSetDevice(ctx->device);
    MB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return MB_OK;
}

mb_status mb_device_state(mb_context* ctx, void** pos, void** vel, void** stress) {
    if (!ctx) return MB_ERR_ARGUMENT;
    if (!ctx->loaded) return fail(ctx, MB_ERR_STATE, "no population uploaded");
    if (pos) *pos = ctx->pos.p;
    if (vel) *vel = ctx->vel.p;
    if (stress) *stress = ctx->stress.p;
    return MB_OK;
}

static_assert(MB_DEVO_MAX_REPLACED == mb::kDevoMaxReplaced, "devo limit");
static_assert(MB_DEVO_REFERENCE_RANKS == mb::kDevoReferenceRanks, "devo flag");
static_assert(sizeof(mb::DevoRecord) == 16, "devo record");

mb_status mb_devo(mb_context* ctx, uint32_t replaced_per_robot, uint64_t seed, uint32_t flags,
                  uint32_t* n_replaced) {
    if (!ctx) return MB_ERR_ARGUMENT;
    if (n_replaced) *n_replaced = 0;
    if (!ctx->loaded) return fail(ctx, MB_ERR_STATE, "no population uploaded");
    if (replaced_per_robot > MB_DEVO_MAX_REPLACED)
        return fail(ctx, MB_ERR_ARGUMENT, "at most %u springs per robot and call", MB_DEVO_MAX_REPLACED);
    if (flags & ~(uint32_t)MB_DEVO_REFERENCE_RANKS) return fail(ctx, MB_ERR_ARGUMENT, "unknown devo flags");
    if (replaced_per_robot == 0 || ctx->n_spring == 0) return MB_OK;
    cudaSetDevice(ctx->device);
    using clock = std::chrono::steady_clock;
    const auto t0 = clock::now();
    cudaStream_t st = ctx->stream;
    {
        mb_status s = mb_detail::ensure_host_topology(ctx);
        // a population from the voxel builder becomes a regular packing first
        if (s == MB_OK && ctx->vox_live) s = mb_detail::host_repack(ctx);
        if (s != MB_OK) return s;
    }
    const char* force_host = std::getenv("MB_DEVO_HOST_REPACK");
    bool on_device = !(force_host && force_host[0] == '1');
    // split robots keep their partition; their parts are re-derived on the
    // device (split_devo_setup prepares it once; MB_ERR_CAPACITY there, for
    // split populations with faces or beyond its limits: host re-pack)
    const bool split = ctx->cluster != 0;
    if (on_device && !ctx->devo_ready) {
        const mb_status s = split ? mb_detail::split_devo_setup(ctx) : mb_detail::devo_setup(ctx);
        if (s == MB_ERR_CAPACITY && split)
            on_device = false;
        else if (s != MB_OK)
            return s;
    }
    const size_t nrec = (size_t)ctx->n_robots * replaced_per_robot;
    MB_CUDA(ctx, ctx->devo_out.alloc(nrec));
    mb::DevoParams p{ctx->stress.p, ctx->d_mass_off.p, ctx->d_spring_off.p, ctx->pos.p, ctx->mass_mat.p,
                     ctx->d_table.p, ctx->total_time, replaced_per_robot, seed, flags, ctx->devo_out.p};
    MB_CUDA(ctx, mb::launch_devo(p, ctx->n_robots, st));
    uint32_t status[2] = {0, 0};
    if (on_device && split) {
        MB_CUDA(ctx, cudaMemsetAsync(ctx->devo_status.p, 0, 2 * sizeof(uint32_t), st));
        MB_CUDA(ctx, mb::launch_split_devo_apply(
                         mb_detail::split_params(ctx, ctx->devo_out.p, (uint32_t)nrec, replaced_per_robot),
                         ctx->n_bins, st));
        mb::RebuildParams rp{ctx->bins.p,        ctx->n_bins,          ctx->spring_pair.p,
                             ctx->spring_gidx.p, (uint32_t)ctx->n_spring, ctx->slice_off.p,
                             ctx->slice_width.p, ctx->inc.p,           ctx->inc32.p,
                             0u,                 ctx->rows_scratch.p,  ctx->free_count.p,
                             ctx->free_taken.p,  ctx->devo_status.p,   ctx->sp_keys.p,
                             ctx->sp_key_begin.p};
        MB_CUDA(ctx, mb::launch_rebuild(rp, st));
        MB_CUDA(ctx, cudaMemcpyAsync(status, ctx->devo_status.p, sizeof(status), cudaMemcpyDeviceToHost, st));
        MB_CUDA(ctx, cudaMemcpyAsync(ctx->h_bins.data(), ctx->bins.p, ctx->h_bins.size() * sizeof(mb::BinDesc),
                                     cudaMemcpyDeviceToHost, st));
    } else if (on_device) {
        MB_CUDA(ctx, cudaMemsetAsync(ctx->devo_status.p, 0, 2 * sizeof(uint32_t), st));
        mb::DevoApplyParams ap{ctx->devo_out.p,      (uint32_t)nrec,        replaced_per_robot,
                               ctx->d_pairs.p,       ctx->d_spring_mat.p,   ctx->d_lbar.p,
                               ctx->pslot.p,         ctx->robot_bin.p,      ctx->robot_mass_base.p,
                               ctx->slot_of.p,       ctx->bins.p,           ctx->spring_pair.p,
                               ctx->spring_lbar.p,   ctx->spring_gidx.p,    (uint32_t)ctx->n_spring,
                               ctx->free_count.p,    ctx->free_taken.p,     ctx->free_slots.p,
                               ctx->devo_status.p};
        MB_CUDA(ctx, mb::launch_devo_apply(ap, 0, st));
        MB_CUDA(ctx, mb::launch_devo_apply(ap, 1, st));
        mb::RebuildParams rp{ctx->bins.p,        ctx->n_bins,          ctx->spring_pair.p,
                             ctx->spring_gidx.p, (uint32_t)ctx->n_spring, ctx->slice_off.p,
                             ctx->slice_width.p, ctx->inc.p,           ctx->inc32.p,
                             ctx->streamed ? 1u : 0u, ctx->rows_scratch.p, ctx->free_count.p,
                             ctx->free_taken.p,  ctx->devo_status.p};
        MB_CUDA(ctx, mb::launch_rebuild(rp, st));
        MB_CUDA(ctx, cudaMemcpyAsync(status, ctx->devo_status.p, sizeof(status), cudaMemcpyDeviceToHost, st));
    }
    ctx->h_devo.resize(nrec);
    MB_CUDA(ctx, cudaMemcpyAsync(ctx->h_devo.data(), ctx->devo_out.p, nrec * sizeof(mb::DevoRecord),
                                 cudaMemcpyDeviceToHost, st));
    MB_CUDA(ctx, cudaStreamSynchronize(st));
    uint32_t count = 0;
    for (const mb::DevoRecord& rec : ctx->h_devo) {
        if (rec.spring == 0xFFFFFFFFu) continue;
        if (rec.spring >= ctx->n_spring || rec.material >= MB_COMPOSITE_COUNT)
            return fail(ctx, MB_ERR_STATE, "development record out of range");
        ctx->h_pairs[2 * (size_t)rec.spring] = (uint16_t)(rec.pair & 0xFFFFu);
        ctx->h_pairs[2 * (size_t)rec.spring + 1] = (uint16_t)(rec.pair >> 16);
        ctx->h_spring_mat[rec.spring] = (uint8_t)rec.material;
        ctx->h_lbar[rec.spring] = rec.lbar;
        ++count;
    }
    const auto t1 = clock::now();
    bool repack = !on_device || status[0] != 0;
    if (!repack && !ctx->streamed && status[1] > ctx->smem_bytes) {
        if (status[1] > mb::max_step_smem(ctx->device) || (split && !mb_detail::split_schedulable(ctx, status[1]))) {
            repack = true;
        } else {
            ctx->smem_bytes = status[1];
            ctx->clear_graphs();  // the graphs hold the old shared memory size
        }
    }
    if (repack) {
        const mb_status s = mb_detail::host_repack(ctx);
        if (s != MB_OK) return s;
    }
    const auto t2 = clock::now();
    ctx->devo_ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    ctx->devo_ms[1] = repack ? std::chrono::duration<double, std::milli>(t2 - t1).count() : 0.0;
    ctx->devo_ms[2] = (double)ctx->devo_host_repacks;
    if (n_replaced) *n_replaced = count;
    return MB_OK;
}

mb_status mb_devo_profile(const mb_context* ctx, double* ms) {
    if (!ctx || !ms) return MB_ERR_ARGUMENT;
    for (int i = 0; i < 3; ++i) ms[i] = ctx->devo_ms[i];
    return MB_OK;
}

mb_status mb_set_voxel_population(mb_context* ctx, uint32_t n_robots, int sx, int sy, int sz,
                                  const uint8_t* cells, float h, float mass) {
    if (!ctx || !cells) return fail(ctx, MB_ERR_ARGUMENT, "null argument");
    if (!ctx->have_table) return fail(ctx, MB_ERR_STATE, "material table not set");
    if (n_robots == 0 || sx <= 0 || sy <= 0 || sz <= 0) return fail(ctx, MB_ERR_ARGUMENT, "empty population");
    if ((int64_t)(sx + 1) * (sy + 1) * (sz + 1) > (int64_t)mb::kVoxelMaxPoints)
        return fail(ctx, MB_ERR_CAPACITY, "at most %u grid points per robot", mb::kVoxelMaxPoints);
    if (!std::isfinite(h) || !(h > 0.0f) || !std::isfinite(mass))
        return fail(ctx, MB_ERR_ARGUMENT, "cell size and mass must be finite, cell size positive");
    cudaSetDevice(ctx->device);
    auto& v = ctx->vox;
    uint32_t hb, mbits;
    std::memcpy(&hb, &h, 4);
    std::memcpy(&mbits, &mass, 4);
    if (!v.valid || v.n_robots != n_robots || v.sx != sx || v.sy != sy || v.sz != sz || v.h_bits != hb ||
        v.mass_bits != mbits || v.mode != (uint32_t)ctx->mode) {
        const mb_status s = mb_detail::voxel_setup(ctx, n_robots, sx, sy, sz, h, mass);
        if (s != MB_OK) {
            ctx->loaded = false;
            v.valid = false;
            return s;
        }
    }
    cudaStream_t st = ctx->stream;
    const size_t nc = (size_t)n_robots * sx * sy * sz;
    MB_CUDA(ctx, cudaMemcpyAsync(v.cells.p, cells, nc, cudaMemcpyHostToDevice, st));
    MB_CUDA(ctx, cudaMemsetAsync(ctx->devo_status.p, 0, 2 * sizeof(uint32_t), st));
    MB_CUDA(ctx, cudaMemsetAsync(ctx->free_count.p, 0, ctx->n_bins * sizeof(uint32_t), st));
    MB_CUDA(ctx, cudaMemsetAsync(ctx->free_taken.p, 0, ctx->n_bins * sizeof(uint32_t), st));
    const mb::VoxelBuildParams bp{n_robots, sx, sy, sz, v.cells.p, v.pos.p, v.src.p, v.dir.p, v.n_springs, mass,
                                  ctx->pos.p, ctx->vel.p, ctx->mass_mat.p, ctx->d_spring_mat.p, ctx->stress.p,
                                  ctx->devo_status.p};
    MB_CUDA(ctx, mb::launch_voxel_build(bp, st));
    const mb::CompactParams cp{ctx->bins.p, ctx->n_bins, v.n_spring.p, v.word.p, v.lbar.p, v.gidx.p,
                               ctx->d_spring_mat.p, ctx->slot_of.p, ctx->spring_pair.p, ctx->spring_lbar.p,
                               ctx->spring_gidx.p, ctx->devo_status.p};
    MB_CUDA(ctx, mb::launch_compact(cp, st));
    if (!ctx->streamed) {
        // the compaction keeps the template's placement minus the air
        // springs, which breaks its groups: the active springs are placed
        // again for the endpoint loads (the template's counts bound the bins)
        MB_CUDA(ctx, mb::launch_bank_place(ctx->bins.p, ctx->n_bins, v.max_bin_springs, ctx->spring_pair.p,
                                           ctx->spring_gidx.p, ctx->spring_lbar.p, ctx->rows_scratch.p, st));
    }
    const mb::RebuildParams rp{ctx->bins.p,        ctx->n_bins,          ctx->spring_pair.p,
                               ctx->spring_gidx.p, (uint32_t)ctx->n_spring, ctx->slice_off.p,
                               ctx->slice_width.p, ctx->inc.p,           ctx->inc32.p,
                               ctx->streamed ? 1u : 0u, ctx->rows_scratch.p, ctx->free_count.p,
                               ctx->free_taken.p,  ctx->devo_status.p};
    MB_CUDA(ctx, mb::launch_rebuild(rp, st));
    uint32_t status[2] = {0, 0};
    MB_CUDA(ctx, cudaMemcpyAsync(status, ctx->devo_status.p, sizeof(status), cudaMemcpyDeviceToHost, st));
    MB_CUDA(ctx, cudaStreamSynchronize(st));
    ctx->host_topology_stale = true;
    ctx->vox_live = true;
    ctx->devo_ready = false;
    if (status[0]) {
        ctx->loaded = false;
        return fail(ctx, MB_ERR_ARGUMENT, "cell materials must be base material ids 0..22");
    }
    if (!ctx->streamed && status[1] > ctx->smem_bytes) {
        if (status[1] > mb::max_step_smem(ctx->device)) {
            ctx->loaded = false;
            return fail(ctx, MB_ERR_CAPACITY, "rows exceed shared memory");
        }
        ctx->smem_bytes = status[1];
        ctx->clear_graphs();
    }
    ctx->loaded = true;
    return MB_OK;
}

mb_status mb_collect_mass_materials(mb_context* ctx, uint8_t* material) {
    if (!ctx || !material) return fail(ctx, MB_ERR_ARGUMENT, "null argument");
    if (!ctx->loaded) return fail(ctx, MB_ERR_STATE, "no population uploaded");
    const mb_status s = mb_detail::ensure_host_topology(ctx);
    if (s != MB_OK) return s;
    if (!ctx->h_mass_mat.empty()) std::memcpy(material, ctx->h_mass_mat.data(), ctx->h_mass_mat.size());
    return MB_OK;
}

mb_status mb_collect_springs(mb_context* ctx, uint16_t* pairs, uint8_t* material, float* lbar) {
    if (!ctx) return MB_ERR_ARGUMENT;
    if (!ctx->loaded) return fail(ctx, MB_ERR_STATE, "no population uploaded");
    {
        const mb_status s = mb_detail::ensure_host_topology(ctx);
        if (s != MB_OK) return s;
    }
    if (pairs && !ctx->h_pairs.empty()) std::memcpy(pairs, ctx->h_pairs.data(), ctx->h_pairs.size() * sizeof(uint16_t));
    if (material && !ctx->h_spring_mat.empty())
        std::memcpy(material, ctx->h_spring_mat.data(), ctx->h_spring_mat.size());
    if (lbar && !ctx->h_lbar.empty()) std::memcpy(lbar, ctx->h_lbar.data(), ctx->h_lbar.size() * sizeof(float));
    return MB_OK;
}

}  // extern "C"
