// Internal types shared by the host library (mb_host.cpp) and the CUDA
// kernels (mb_kernels.cu).  Not part of the C ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mb {

// Incidence entries are uint16: packed spring index << 1 | (1 at the b end);
// kPadEntry pads rows to the slice width and is skipped by the gather.
constexpr uint32_t kMaxMaterialSlots = 256;
constexpr uint16_t kPadEntry = 0xFFFFu;
constexpr uint32_t kPadEntry32 = 0xFFFFFFFFu;
constexpr uint32_t kMaxBinSprings = 32767;  // 15-bit spring index in an entry
constexpr uint32_t kSliceWidth = 32;  // masses per SELL slice (one warp)
// springs of a resident bin placed independently for the endpoint loads
// (a multiple of 8: whole groups of a quarter-warp)
constexpr uint32_t kPlaceChunk = 1024;

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
    uint32_t row_cap;      // incidence entries the bin's row region holds (device re-pack)
    // split bins (one part of a robot simulated by a cluster of CTAs):
    uint32_t x_stride;     // float4 slots of one predicted-position buffer (own + halo masses)
    uint32_t export_begin; // first export entry (own mass | rank << 12 | slot << 15)
    uint32_t n_export;
    uint32_t n_all;        // own + halo masses
    // surface triangles of the bin's robots (face drag of the water mode;
    // resident bins only): bin-local corners, and per mass the faces it is
    // a corner of, in face order
    uint32_t face_begin;   // first packed face
    uint32_t n_face;
    uint32_t face_inc_begin;  // first face incidence entry
    uint32_t n_face_inc;
};

// Everything one step launch needs.  Pointers are device addresses.
struct StepParams {
    const BinDesc* bins;
    uint32_t n_bins;
    uint32_t grid;                // CTAs of the launch (bins g, g + grid, ... on CTA g); 0 = n_bins
    float4* pos;                  // upload layout, w = mass
    float4* vel;                  // upload layout
    float* stress;                // upload layout, one per spring
    const uint32_t* mass_gidx;    // packed mass -> upload index
    const uint32_t* spring_gidx;  // packed spring -> upload index
    const uint32_t* spring_pair;  // packed spring: a | b << 12 | material slot << 24 (bin-local)
    const float* spring_lbar;     // packed spring mean length
    const uint32_t* slice_off;    // per slice: first entry relative to bin inc_begin
    const uint32_t* slice_width;  // per slice: entries per mass (row length)
    const uint16_t* inc;          // incidence entries: spring << 1 | (b end), or kPadEntry
    const uint32_t* exports;      // split bins: own mass | part << 12 | halo slot << 15
    const uint32_t* n_mat;        // material slots used by the population (device scalar)
    const float* rates;           // [steps][n_mat]: dL0 * sin(omega t_n + phi) of this launch
    const float* invk;            // [n_mat]: 1 / (2 + 1/(k dt^2))
    uint32_t* bin_flags;          // per bin: bit 0 = non-finite position
    float dt;
    float t0;
    uint32_t steps;
    uint32_t track;
    uint32_t smem_bytes;
    uint32_t mode;                // 0 reference XPBD, 1 force + land, 2 force + water
    // streamed kernel only: rows with 32-bit entries (spring << 1 | b end, or
    // kPadEntry32) and per-spring scratch in packed order
    const uint32_t* inc32;
    float4* dp;                   // corrections / forces of the current step
    float* st;                    // stresses during a launch
    // environment of the force modes
    float g;                      // gravity along -z (land)
    float floor_stiffness;        // penalty stiffness of the ground z = 0 (land)
    float mu_s, mu_k;             // static / kinetic friction coefficients (land)
    float drag;                   // 0.5 rho Cd A of the quadratic drag per mass (water)
    float damping;                // velocity factor per step
    // face drag (water, resident bins)
    const uint2* faces;           // packed face: {c0 | c1 << 16, c2}, bin-local corners
    const uint32_t* face_row;     // packed mass: first entry (bin-relative) | count << 24
    const uint16_t* face_inc;     // face incidence entries: bin-local face index
    float4* fd;                   // streamed kernel: face forces of the current step
    float face_coef;              // -rho/6: -rho/2 of the face law and the 1/3 per corner
    uint32_t face_on;             // face drag active (water mode, rho != 0)
    uint32_t one_mass_per_thread; // every bin has at most 1,024 masses (0 = unknown)
};

enum StepMode : uint32_t { kModeXpbd = 0, kModeForceLand = 1, kModeForceWater = 2 };
// Kernel variant of the water mode with the face drag compiled in (chosen
// by launch_step when StepParams::face_on is set; never a StepParams mode).
constexpr uint32_t kModeForceWaterFaces = 3;

struct KernelShape {
    uint32_t threads;
    uint32_t spt;  // springs per thread
    uint32_t mpt;  // masses per thread
};

// Mode-dependent launch helpers take the mode of the step as well.

// Sets the dynamic shared memory limit of a kernel variant; call before
// launching (and outside stream capture).
cudaError_t prepare_step(const KernelShape& shape, uint32_t mode, bool track, uint32_t smem_bytes);

// Actuation factors of one launch: rates[n][i] = dL0 * sin(omega t_n + phi)
// for steps n < steps of the float clock t_0 = t0, t_{n+1} = t_n + dt, and
// the materials mat_ids[i], i < *n_mat; coef[i] = 1/(2 + 1/k/dt/dt) for the
// reference step, k for the force modes.
cudaError_t launch_actuation(const float4* table, const uint8_t* mat_ids, const uint32_t* n_mat,
                             float t0, float dt, uint32_t steps, uint32_t mode, float* rates,
                             float* coef, cudaStream_t s);

// Launches the step kernel for `p.steps` steps.  Returns a CUDA error.
cudaError_t launch_step(const StepParams& p, const KernelShape& shape, cudaStream_t s);

// Resident CTAs per SM of a kernel variant with `smem_bytes` of dynamic
// shared memory (0 if the shape is not compiled or does not fit).
int ctas_per_sm(const KernelShape& shape, uint32_t mode, bool track, uint32_t smem_bytes);
// Clusters of `cluster` split-kernel CTAs that can be resident at once on
// the current device (0: such a cluster cannot be scheduled).
int max_active_clusters(const KernelShape& shape, uint32_t mode, uint32_t cluster, uint32_t smem_bytes);

// Streamed variant for bins whose springs do not fit in shared memory:
// only predicted positions live in shared memory; springs, rows and the
// per-spring scratch stream through global memory (L2).
cudaError_t prepare_stream(uint32_t threads, uint32_t mpt, uint32_t mode, bool track,
                           uint32_t smem_bytes);
cudaError_t launch_stream(const StepParams& p, uint32_t threads, uint32_t mpt, cudaStream_t s);
uint32_t stream_smem_bytes(uint32_t n_mass);
bool stream_supported(uint32_t threads, uint32_t mpt);
// Whether the split (cluster) step kernel is compiled for a shape.
bool split_supported(const KernelShape& shape);
cudaError_t prepare_split(const KernelShape& shape, uint32_t mode, bool track, uint32_t smem_bytes);
cudaError_t launch_split(const StepParams& p, const KernelShape& shape, uint32_t cluster, cudaStream_t s);

// Compiled shapes of the resident (streamed = false) or streamed kernel;
// writes up to cap entries, returns the count.
uint32_t list_shapes(KernelShape* out, uint32_t cap, bool streamed);

// Shared memory a bin needs, in bytes.
uint32_t bin_smem_bytes(uint32_t n_mass, uint32_t n_spring, uint32_t n_inc);
// The same on the device: x~ and dp as float4 per mass and spring, the
// material factors of every slot, the rows as uint16 entries.
__host__ __device__ constexpr uint32_t bin_smem_bytes_dev(uint32_t n_mass, uint32_t n_spring, uint32_t n_inc) {
    return 16u * n_mass + 16u * n_spring + 8u * kMaxMaterialSlots + 2u * n_inc;
}

// Face drag of a resident bin, after its rows (16-byte aligned): the
// velocities of its masses, the forces and corners of its faces, the face
// row of each mass and the incidence entries.
__host__ __device__ inline uint32_t face_smem_bytes(uint32_t n_mass, uint32_t n_face, uint32_t n_face_inc) {
    return n_face ? 16u + 20u * n_mass + 24u * n_face + 2u * n_face_inc : 0u;
}
constexpr uint32_t kMaxFacesPerMass = 255;  // 8-bit count in face_row
constexpr uint32_t kMaxRobotFaces = 65535;   // 16-bit face index in an entry
// Streamed bins: the velocities after the material factors (face forces
// go through global memory).
__host__ __device__ inline uint32_t stream_face_smem_bytes(uint32_t n_mass, uint32_t n_face) {
    return n_face ? 16u * n_mass : 0u;
}

// Split bins: two predicted-position buffers of x_stride slots, the
// corrections, the material factors, the buffer strides of the cluster's
// parts, the export list and the rows.
constexpr uint32_t kMaxClusterParts = 8;
__host__ __device__ inline uint32_t split_smem_bytes(uint32_t x_stride, uint32_t n_spring, uint32_t n_inc,
                                                     uint32_t n_export) {
    return 32u * x_stride + 16u * n_spring + 8u * kMaxMaterialSlots + 4u * kMaxClusterParts + 4u * n_export +
           2u * n_inc;
}

// Split bins with the face layout (the face drag on a split population):
// two velocity buffers of x_stride slots after the position buffers, and
// after the rows (16-byte aligned) the face forces and corners, the face
// rows of the own masses and the incidence entries.
__host__ __device__ inline uint32_t split_face_smem_bytes(uint32_t x_stride, uint32_t n_own, uint32_t n_face,
                                                          uint32_t n_face_inc) {
    return 32u * x_stride + 16u + 24u * n_face + 4u * n_own + 2u * n_face_inc;
}

// Largest dynamic shared memory the step kernel may use on this device.
uint32_t max_step_smem(int device);

// Whether a kernel shape is compiled in.
bool shape_supported(const KernelShape& shape);
// Whether the shape of resident bins has a register-row twin (one mass per
// thread, rows of incident springs in registers), which launch_step uses
// when StepParams::one_mass_per_thread is set.  Its shared memory per bin:
// the usual layout without the rows, 8 bytes of alignment, then 8 bytes per
// spring.  Rows longer than row_reg_width() entries are read from global
// memory, so the host uses it only when no mass has more incident springs.
bool row_reg_supported(const KernelShape& shape);
uint32_t row_reg_width();

// Centre of mass of the non-air masses of each robot: one warp per robot.
cudaError_t launch_com(const float4* pos, const uint8_t* mass_mat,
                       const int64_t* mass_off, uint32_t n_robots, float* com,
                       cudaStream_t s);

// Per-robot flags: bit 0 = a position is NaN or Inf.  One warp per robot.
// ORs bit 1 of each robot's first bin's step flags into out[robot].
cudaError_t launch_bin_flags(const uint32_t* bin_flags, const uint32_t* robot_bin, uint32_t n_robots,
                             uint32_t* out, cudaStream_t s);
cudaError_t launch_flags(const float4* pos, const int64_t* mass_off, uint32_t n_robots,
                         uint32_t* robot_flags, cudaStream_t s);

}  // namespace mb
