// Internal types shared by the host library (mb_host.cpp) and the CUDA
// kernels (mb_kernels.cu).  Not part of the C ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mb {

// Sentinel in the incidence lists: a padding entry that points at the zero
// correction slot kept after the last spring of a bin.
constexpr uint32_t kMaxMaterialSlots = 256;
constexpr uint32_t kSliceWidth = 32;  // masses per SELL slice (one warp)

// One bin: a group of whole robots that one CTA simulates together.  Masses
// and springs of the bin are numbered 0..n-1 in "packed" order; packed
// arrays hold them contiguously from *_begin.
struct BinDesc {
    uint32_t mass_begin;   // first packed mass
    uint32_t n_mass;
    uint32_t spring_begin; // first packed spring
    uint32_t n_spring;
    uint32_t inc_begin;    // first incidence entry (SELL-32 layout)
    uint32_t n_inc;        // incidence entries incl. padding
    uint32_t slice_begin;  // first slice descriptor
    uint32_t mat_begin;    // first material slot
    uint32_t n_mat;        // material slots used by the bin
    uint32_t pad[3];
};

// Everything one step launch needs.  Pointers are device addresses.
struct StepParams {
    const BinDesc* bins;
    uint32_t n_bins;
    float4* pos;                  // upload layout, w = mass
    float4* vel;                  // upload layout
    float* stress;                // upload layout, one per spring
    const uint32_t* mass_gidx;    // packed mass -> upload index
    const uint32_t* spring_gidx;  // packed spring -> upload index
    const uint32_t* spring_pair;  // packed spring: a | b << 16 (bin-local)
    const float* spring_lbar;     // packed spring mean length
    const uint8_t* spring_slot;   // packed spring material slot (bin-local)
    const uint32_t* slice_off;    // per slice: first entry relative to bin inc_begin
    const uint32_t* slice_width;  // per slice: entries per mass (row length)
    const uint32_t* inc;          // incidence entries: spring << 1 | (b end)
    const uint8_t* mat_ids;       // per material slot: composite id
    const float4* table;          // composite table {k, dL0, omega, phi}
    uint32_t* bin_flags;          // per bin: bit 0 = non-finite position
    float dt;
    float t0;
    uint32_t steps;
    uint32_t track;
    uint32_t smem_bytes;
};

struct KernelShape {
    uint32_t threads;
    uint32_t spt;  // springs per thread
    uint32_t mpt;  // masses per thread
};

// Sets the dynamic shared memory limit of a kernel variant; call before
// launching (and outside stream capture).
cudaError_t prepare_step(const KernelShape& shape, bool track, uint32_t smem_bytes);

// Launches the step kernel for `p.steps` steps.  Returns a CUDA error.
cudaError_t launch_step(const StepParams& p, const KernelShape& shape, cudaStream_t s);

// Resident CTAs per SM of a kernel variant with `smem_bytes` of dynamic
// shared memory (0 if the shape is not compiled or does not fit).
int ctas_per_sm(const KernelShape& shape, bool track, uint32_t smem_bytes);

// Shared memory a bin needs, in bytes.
uint32_t bin_smem_bytes(uint32_t n_mass, uint32_t n_spring, uint32_t n_inc);

// Largest dynamic shared memory the step kernel may use on this device.
uint32_t max_step_smem(int device);

// Whether a kernel shape is compiled in.
bool shape_supported(const KernelShape& shape);

// Centre of mass of the non-air masses of each robot: one warp per robot.
cudaError_t launch_com(const float4* pos, const uint8_t* mass_mat,
                       const int64_t* mass_off, uint32_t n_robots, float* com,
                       cudaStream_t s);

// Per-robot flags: bit 0 = a position is NaN or Inf.  One warp per robot.
cudaError_t launch_flags(const float4* pos, const int64_t* mass_off, uint32_t n_robots,
                         uint32_t* robot_flags, cudaStream_t s);

}  // namespace mb
