/*
 * mercury_b200 -- C ABI of the B200 batched soft-body simulation step.
 *
 * Plain C types only; every call returns an mb_status and never exits the
 * process.  One mb_context owns one population ("batch") of robots resident
 * on one GPU, the launch configuration chosen for it and one CUDA stream.
 * A context is not thread-safe; use one per host thread.
 *
 * The entry points replace the reference's internal kernel ABI
 * (common/simulator/softbodysystem.h:63-75) and the device-facing half of
 * class Simulator (common/simulator/Simulator.h:19-149, Simulator.cu).  Each
 * declaration names the reference interface it stands in for.
 *
 * Units and layouts follow the reference:
 *   - positions and velocities are float4 per mass: x, y, z and w, where w of
 *     a position is the mass (Simulator.cu:256-259) and w of a velocity is
 *     carried unchanged;
 *   - springs join two robot-local mass indices (uint16, spring.h:9-10) and
 *     carry a composite material id (0..253, 0 = air, material.h:79-107)
 *     and a mean length (spring.h:12);
 *   - masses carry their base material id (0..22, 0 = air), used by the
 *     centre-of-mass reduction (SoftBody.cpp:112-121).
 */
#ifndef MERCURY_B200_H
#define MERCURY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Only the entry points below are exported; the library is built with
 * hidden default visibility. */
#if defined(__GNUC__)
#define MB_API __attribute__((visibility("default")))
#else
#define MB_API
#endif

#define MB_COMPOSITE_COUNT 254 /* material.h:106 COMPOSITE_COUNT = 22*23/2 + 1 */

typedef struct mb_context mb_context;

typedef enum mb_status {
    MB_OK = 0,
    MB_ERR_ARGUMENT = 1,  /* bad pointer, size or index; nothing changed   */
    MB_ERR_CUDA = 2,      /* a CUDA call failed; see mb_last_error          */
    MB_ERR_CAPACITY = 3,  /* a robot or batch exceeds what a launch holds   */
    MB_ERR_STATE = 4,     /* call out of order (e.g. simulate before upload) */
    MB_ERR_NONFINITE = 5  /* a mass position became NaN or Inf              */
} mb_status;

typedef enum mb_mode {
    MB_MODE_REF_XPBD = 0,    /* the reference step: sim_kernel.cu:141-269 */
    MB_MODE_FORCE_LAND = 1,  /* Hooke springs, gravity, ground with friction */
    MB_MODE_FORCE_WATER = 2  /* Hooke springs, quadratic drag, no net gravity */
} mb_mode;

/* Environment of the force modes (the fields of the reference's
 * Environment, environment.h:6-32, with both friction coefficients and a
 * drag coefficient that acts):
 *   g                gravity along -z (land), m/s^2
 *   floor_stiffness  penalty stiffness of the ground plane z = 0, N/m
 *   friction_static, friction_kinetic   Coulomb coefficients (land)
 *   drag             0.5 * rho * Cd * A of the quadratic drag per mass (water)
 *   damping          velocity factor per step
 *   face_drag        fluid density rho of the drag on the robots' surface
 *                    triangles (water; 0 = faces exert no drag).  Each face
 *                    (i0, i1, i2) with mean vertex velocity v, N = (x1 - x0)
 *                    x (x2 - x0), A = |N| and unit normal n = N/(A + 1e-12)
 *                    turned so that v.n > 0, pushes
 *                    -rho/2 A ((v.n) v + 0.2 |v|^2 n) / 3 on each vertex: the
 *                    face law of the reference's surfaceDragForce
 *                    (sim_kernel.cu:96-121), whose result never reaches the
 *                    reference's integrator, added here to the spring forces.
 * Force modes integrate x' = x + v dt + (F/m) dt^2, v' = damping (x' - x)/dt
 * with m the w component of the position. */
typedef struct mb_environment {
    float g;
    float floor_stiffness;
    float friction_static;
    float friction_kinetic;
    float drag;
    float damping;
    float face_drag;
} mb_environment;

/* One population on the host.  Offsets have n_robots + 1 entries and index
 * the flat arrays; pairs and faces are local to their robot.  Faces are the
 * robots' surface triangles (Face m0, m1, m2, face.h:6-10; Element::faces,
 * element.h:12), used only by the face drag of the water mode; both face
 * pointers NULL = no faces.  A face with two equal corners is skipped, as
 * the reference skips it (sim_kernel.cu:99). */
typedef struct mb_batch_desc {
    uint32_t n_robots;
    const int64_t* mass_offsets;
    const float* pos;               /* 4 per mass */
    const float* vel;               /* 4 per mass */
    const uint8_t* mass_material;   /* base material id per mass */
    const int64_t* spring_offsets;
    const uint16_t* pairs;          /* 2 per spring */
    const uint8_t* spring_material; /* composite material id per spring */
    const float* lbar;              /* mean length per spring */
    const int64_t* face_offsets;    /* n_robots + 1, or NULL */
    const uint16_t* faces;          /* 3 per face, or NULL */
} mb_batch_desc;

/* Launch configuration of the step kernel.  threads: CTA size; bins: number
 * of robot groups, each simulated by one CTA; chunk: steps per launch;
 * streamed: 1 = keep only positions in shared memory and stream springs,
 * rows and per-spring scratch through global memory (one robot per CTA);
 * cluster: 2, 4 or 8 = split every robot into that many parts, one CTA
 * each, the parts of a robot forming a thread-block cluster that exchanges
 * boundary positions through distributed shared memory; 1 = never split;
 * 0 = automatic (split when a robot does not fit a resident bin: each
 * robot into the fewest parts that fit, at most 8, robots with fewer parts
 * sharing a cluster; streamed when no split fits).  Reading the
 * configuration reports the cluster size in use (0 = not split). */
typedef struct mb_launch_config {
    uint32_t threads;
    uint32_t springs_per_thread;
    uint32_t masses_per_thread;
    uint32_t bins;
    uint32_t chunk;
    uint32_t use_graph;
    uint32_t streamed;
    uint32_t cluster;
} mb_launch_config;

/* Creates a context on CUDA device `device` with its own stream.
 * Replaces Simulator::Simulator / Initialize (Simulator.cu:103-109). */
MB_API mb_status mb_context_create(int device, mb_context** out);

/* Frees every device and host buffer of the context.
 * Replaces Simulator::~Simulator / freeMemory (Simulator.cu:45-101). */
MB_API void mb_context_destroy(mb_context* ctx);

/* Message of the last failed call on this context (never NULL). */
MB_API const char* mb_last_error(const mb_context* ctx);

/* Composite material table, MB_COMPOSITE_COUNT float4 {k, dL0, omega, phi}
 * indexed by composite id.  Replaces setCompositeMats_id
 * (softbodysystem.h:65, sim_kernel.cu:58-60). */
MB_API mb_status mb_set_materials(mb_context* ctx, const float* table);

/* Time step and accumulated clock.  Replace Simulator::setTimeStep,
 * getDeltaT, getTotalTime and Reset (Simulator.h:42-48). */
MB_API mb_status mb_set_time_step(mb_context* ctx, float dt);
MB_API float mb_get_time_step(const mb_context* ctx);
MB_API mb_status mb_set_total_time(mb_context* ctx, float t);
MB_API float mb_get_total_time(const mb_context* ctx);

/* Step semantics.  Replaces the fixed kernel set of integrateBodies
 * (sim_kernel.cu:271-325). */
MB_API mb_status mb_set_mode(mb_context* ctx, mb_mode mode);
MB_API mb_status mb_get_mode(const mb_context* ctx, mb_mode* mode);

/* Environment of the force modes; the default is land with g = 9.81,
 * floor_stiffness = 1e6 (environment.h:15-22), friction 1.0 / 0.8, drag 0.05,
 * damping 0.999, face_drag 0.  A population whose robots carry faces is
 * packed with them when the face drag is on (water, face_drag != 0); one
 * packed while it was off is re-packed at the next mb_simulate after it is
 * switched on.  Replaces Simulator::_initialize's environment choice
 * (Simulator.cu:191-196). */
MB_API mb_status mb_set_environment(mb_context* ctx, const mb_environment* env);
MB_API mb_status mb_get_environment(const mb_context* ctx, mb_environment* env);

/* Uploads a population: packs it into bins, builds the per-mass incidence
 * lists, copies everything to the device and zeroes the spring stresses.
 * Robots may differ in mass and spring count.  Replaces
 * Simulator::SetElements / AllocateElement (Simulator.cu:206-367, 460-529)
 * and the kernel-side part of setSimOpts (sim_kernel.cu:62-64). */
MB_API mb_status mb_set_elements(mb_context* ctx, const mb_batch_desc* batch);

/* Replaces the uploaded positions and velocities (same robots, same
 * layout) without repacking the topology.  Stresses are kept. */
MB_API mb_status mb_set_state(mb_context* ctx, const float* pos, const float* vel);

/* Runs the step loop for `duration` seconds of simulated time: the number of
 * steps and the clock follow the reference's float accumulation
 * (Simulator.cu:428-449).  Replaces Simulator::Simulate (Simulator.cu:369-458)
 * and integrateBodies (sim_kernel.cu:271-325).  Asynchronous on the
 * context's stream; *steps_taken may be NULL. */
MB_API mb_status mb_simulate(mb_context* ctx, float duration, int track_stresses,
                      uint32_t* steps_taken);

/* Runs exactly `steps` steps from the current clock. */
MB_API mb_status mb_run_steps(mb_context* ctx, uint32_t steps, int track_stresses);

/* Copies the state back to host arrays in the upload layout (pos, vel: 4
 * floats per mass; stress: 1 per spring; any may be NULL).  Synchronous.
 * Replaces Simulator::Collect (Simulator.cu:537-580). */
MB_API mb_status mb_collect(mb_context* ctx, float* pos, float* vel, float* stress);

/* Centre of mass of the non-air masses of every robot (3 floats per robot),
 * reduced on the device.  Synchronous.  Replaces the host-side
 * SoftBody::updateCOM after Collect (SoftBody.cpp:112-121). */
MB_API mb_status mb_centre_of_mass(mb_context* ctx, float* com);

/* Per-robot status after the last run: bit 0 = a position became NaN/Inf;
 * bit 1 = the robot's bin did not fit the shared memory the launch was
 * sized for and was not stepped (a safeguard of the register-row kernel;
 * the host sizes every launch so that it does not happen).  Synchronous.
 * The reference asserts on NaN in Collect (Simulator.cu:550). */
MB_API mb_status mb_robot_flags(mb_context* ctx, uint32_t* flags);

/* Waits for all work on the context's stream. */
MB_API mb_status mb_synchronize(mb_context* ctx);

/* The stream the context launches on (a cudaStream_t). */
MB_API void* mb_get_stream(const mb_context* ctx);

/* Device addresses of the state arrays in the upload layout, for callers
 * that keep inputs resident on the device. */
MB_API mb_status mb_device_state(mb_context* ctx, void** pos, void** vel, void** stress);

/* Development (Simulator::Devo, Simulator.cu:640-668, with the kernels of
 * devo_kernel.cu:56-184 and the stress sort of Simulator.cu:597-631).  For
 * every robot with at least two masses, the springs of stress ranks [0, k)
 * -- stress accumulated by runs with stress tracking, descending, ties by
 * ascending spring index -- get a random pair of distinct masses, the
 * composite material of the two masses and the mean length
 * |x_a - x_b| / (1 + dL0 sin(omega t + phi)) at the current clock.  With
 * MB_DEVO_REFERENCE_RANKS, robot r replaces ranks [r k, r k + k) instead, the
 * window the reference's indexing selects (devo_kernel.cu:112-116), clipped
 * to the robot's own springs.  The pairs come from a counter-based
 * generator over (seed, robot, rank), not cuRAND: same seed, same result on
 * any device.  Stresses are kept (as in the reference); positions and
 * velocities are untouched.  The packed layout is updated on the device:
 * springs keep their slots and the rows of every bin are rebuilt; only when
 * that does not fit (rows beyond their spare capacity, no free slot for a
 * spring that stops being air) is the population re-packed on the host
 * (the launch override stays if the population still fits it).
 * Synchronous.  k <= MB_DEVO_MAX_REPLACED; *n_replaced (may be NULL) gets
 * the number of springs replaced. */
#define MB_DEVO_MAX_REPLACED 1024
#define MB_DEVO_REFERENCE_RANKS 1u
MB_API mb_status mb_devo(mb_context* ctx, uint32_t replaced_per_robot, uint64_t seed, uint32_t flags,
                         uint32_t* n_replaced);

/* Phases of the last mb_devo: ms[0] host wall time (ms) of the device part
 * -- selection, rewiring of the packed springs, rebuild of the rows, read-back
 * of the new springs; ms[1] wall time of a host re-pack and upload (0 when
 * the device re-pack sufficed); ms[2] the number of mb_devo calls on this
 * context that needed the host re-pack.  No reference counterpart. */
MB_API mb_status mb_devo_profile(const mb_context* ctx, double* ms);

/* Population of voxel robots built on the device from cell grids -- the
 * equivalent of VoxelRobot::Build (VoxelRobot.cpp:310-331, as mb_voxel_build
 * restates it) for every robot followed by mb_set_elements, without the host
 * build and packing.  cells: n_robots grids of sx*sy*sz base material ids
 * (0 = air .. 22), x fastest, robot after robot (host memory); robot r is the
 * lattice of (sx+1)(sy+1)(sz+1) points whose point (x, y, z) carries cell
 * (x, y, z) and whose upper faces are air; spacing h, every mass `mass`,
 * zero velocity.  Grids of one shape share one packing, planned on the
 * first call and reused while n_robots, the shape, h, mass, the mode and
 * the launch override stay the same; each call then costs one copy of the
 * cells and three kernels.  At most 4,096 points per robot.  Synchronous.
 * The topology read-back functions and mb_devo work on the result as on an
 * uploaded batch. */
MB_API mb_status mb_set_voxel_population(mb_context* ctx, uint32_t n_robots, int sx, int sy, int sz,
                                         const uint8_t* cells, float h, float mass);

/* k-nearest-neighbour springs of point-cloud robots, built on `device`
 * (the springs of the reference's NNRobot, common/evolvables/knn.cu:62-145
 * and knn_kernel.cu:34-60): every mass is joined to its k nearest masses of
 * the same robot -- squared distances the float32 sum (dx*dx + dy*dy) +
 * dz*dz, ties by lower index -- and each unordered pair appears once, the
 * lower index first, pairs in lexicographic order, with the float32
 * distance as mean length and the composite material of the two masses.
 * pos: 3 floats per mass (host); at most 4,096 masses per robot, k <= 32.
 * spring_offsets (n_robots + 1) is always written; with pairs == NULL the
 * call only counts.  Synchronous.  Its device scratch and stream are kept
 * per device for later calls (grown when a call needs more, held until the
 * process exits); calls on one device are serialised.  No context needed. */
MB_API mb_status mb_knn_springs(int device, uint32_t n_robots, const int64_t* mass_offsets, const float* pos,
                                const uint8_t* mass_material, uint32_t k, int64_t* spring_offsets,
                                uint16_t* pairs, uint8_t* spring_material, float* lbar, uint64_t capacity);

/* Mass materials in the upload layout (after the strip of a device build). */
MB_API mb_status mb_collect_mass_materials(mb_context* ctx, uint8_t* material);

/* Topology in the upload layout (2 pair entries, 1 material, 1 mean length
 * per spring; any pointer may be NULL), as changed by mb_devo.  The
 * reference copies pairs, materials and mean lengths back in Collect
 * (Simulator.cu:542-561). */
MB_API mb_status mb_collect_springs(mb_context* ctx, uint16_t* pairs, uint8_t* material, float* lbar);

/* Launch configuration: read, override (0 fields keep the automatic
 * choice), and the automatic choice for the uploaded batch. */
MB_API mb_status mb_get_launch_config(const mb_context* ctx, mb_launch_config* cfg);
MB_API mb_status mb_set_launch_config(mb_context* ctx, const mb_launch_config* cfg);

/* The step kernel the next launches of the uploaded batch use:
 * *register_rows = 1 when each mass's row of incident springs is held in
 * registers (resident bins of a 1,024-thread shape with at most one mass per
 * thread, no face drag, and room for 8 more bytes of shared memory per
 * spring), else 0; *smem_bytes = the dynamic shared memory per CTA of those
 * launches.  Either pointer may be NULL.  No reference counterpart. */
MB_API mb_status mb_get_step_variant(const mb_context* ctx, uint32_t* register_rows, uint32_t* smem_bytes);

/* The packed spring slots of the uploaded batch, in device order: *count =
 * the number of slots; when `words` is not NULL and capacity >= *count, the
 * packed word of every slot (a | b << 12 | material slot << 24, bin-local
 * mass indices) is copied into it, else MB_ERR_CAPACITY.  For tests and
 * tools that check how springs are placed.  No reference counterpart. */
MB_API mb_status mb_get_packed_springs(const mb_context* ctx, uint32_t* words, uint64_t capacity,
                                       uint64_t* count);

/* Launch plan of a population, computed on the host without a device:
 * the shape, bin count and path the automatic choice (or `cfg`, may be
 * NULL) would use on a GPU with `num_sms` SMs and `smem_bytes` of dynamic
 * shared memory per CTA (0 = B200: 148, 232,448), and statistics of the
 * packed layout.  No reference counterpart. */
typedef struct mb_plan_stats {
    uint32_t threads, springs_per_thread, masses_per_thread, bins, streamed;
    uint32_t max_smem_bytes;
    uint64_t masses, active_springs, incidence_entries, incidence_padding;
    uint32_t aligned_slices, rank_slices, material_slots;
    uint32_t max_bin_springs, min_bin_springs;
    /* CTAs of a step launch (CTA g runs bins g, g + ctas, ...) and the
     * largest / smallest number of springs one CTA runs per step */
    uint32_t ctas, max_cta_springs, min_cta_springs;
    /* robots split over clusters of this many CTAs (0 = not split); with
     * cluster2 = 2, the robots of at most two parts run in two-CTA clusters
     * from bin split_bins0 on, launched beside the first group */
    uint32_t cluster, cluster2, split_bins0;
} mb_plan_stats;
MB_API mb_status mb_plan_population(const mb_batch_desc* batch, const mb_launch_config* cfg,
                                    uint32_t num_sms, uint32_t smem_bytes, mb_plan_stats* stats);

/* Compiled kernel shapes, for autotuners: writes up to `capacity` entries
 * (threads, springs_per_thread, masses_per_thread; streamed = 1 for the
 * streamed kernel, whose springs_per_thread is 0) and returns the count.  No
 * reference counterpart (the reference launches fixed shapes,
 * sim_kernel.cu:277-304). */
MB_API uint32_t mb_kernel_shapes(mb_launch_config* out, uint32_t capacity);

/* Builds a voxel-lattice robot (one mass per grid point, 13 forward lattice
 * springs per point, largest 6-connected component kept, shifted so that
 * max x = 0 and min y = 0).  Grid point i = x + y*nx + z*nx*ny carries base
 * material mats[i].  Output buffers hold nx*ny*nz masses (pos: 3 floats) and
 * 13*nx*ny*nz springs.  Replaces VoxelRobot::Build (VoxelRobot.cpp:310-331).
 * Host only. */
MB_API mb_status mb_voxel_build(int nx, int ny, int nz, float h, const uint8_t* mats,
                         int* n_masses, int* n_springs, float* pos,
                         uint8_t* mass_material, uint16_t* pairs, float* lbar,
                         uint8_t* spring_material);

/* ----------------------------------------------------------------------
 * Entry point that allocates nothing.  It has no counterpart in the
 * reference; it exists for callers that cannot call cudaMalloc -- an engine
 * that owns every device allocation through its own pool, or a plugin host
 * with a fixed memory budget.
 *
 * Runs `steps` steps of the reference step on ONE robot whose arrays are
 * already on the current device (device pointers; layouts as in
 * mb_batch_desc: pos/vel 4 floats per mass, pairs 2 per spring, stress 1
 * per spring, table MB_COMPOSITE_COUNT float4), starting from clock t0, on
 * `stream` (a cudaStream_t; NULL = the legacy default stream).  pos, vel and
 * stress (when track_stresses != 0) are updated in place; *t_end (may be
 * NULL) receives the float clock after the last step.  Results are bit for
 * bit those of mb_set_elements + mb_run_steps on the same robot.
 *
 * Limits: n_masses <= MB_NOALLOC_MAX_MASSES, n_springs <=
 * MB_NOALLOC_MAX_SPRINGS, and at most MB_NOALLOC_MAX_INCIDENCE incidence
 * entries (32 x the longest per-mass row of each group of 32 masses);
 * larger robots return MB_ERR_CAPACITY.  The packed topology is built on the
 * device in one scratch array of about 300 KB that is part of the library
 * image: every GPU that loads the library holds it until the process exits.
 * The call calls no cudaMalloc, cudaFree or other allocating routine.
 *
 * The first call on a device looks up the scratch array's device address
 * and keeps it for the life of the process: make that first call before any
 * stream capture, and do not reset the device (cudaDeviceReset) after it.  Every call shares the
 * scratch array and keeps the last call's contents, so calls that overlap on
 * the GPU (different streams or host threads) race: serialise them.  The
 * call synchronises `stream` to read its status. */
#define MB_NOALLOC_MAX_MASSES 2048
#define MB_NOALLOC_MAX_SPRINGS 8192
#define MB_NOALLOC_MAX_INCIDENCE 26624
MB_API mb_status mb_simulate_robot_noalloc(void* stream, const float* table,
                                           uint32_t n_masses, float* pos, float* vel,
                                           uint32_t n_springs, const uint16_t* pairs,
                                           const uint8_t* spring_material,
                                           const float* lbar, float* stress, float dt,
                                           float t0, uint32_t steps, int track_stresses,
                                           float* t_end);

/* ----------------------------------------------------------------------
 * Fitness surrogate (no reference counterpart): a 3-D convolutional network
 * over 6x6x6 voxel genomes of 5 classes (0 air, 1 bone, 2 tissue, 3 muscle
 * a, 4 muscle b; any other value reads as no class) that predicts the
 * simulated fitness.  Three 3x3x3 convolutions of 32 channels with ReLU, a
 * 6,912 -> 128 -> 128 MLP with ReLU, a linear output; BF16 tensor-core
 * GEMMs with FP32 accumulation, FP32 master weights, Adam.  Genome and
 * target pointers are host memory; every call is synchronous. */
typedef struct mb_surrogate mb_surrogate;
MB_API mb_status mb_surrogate_create(int device, uint32_t max_batch, uint64_t seed, mb_surrogate** out);
MB_API void mb_surrogate_destroy(mb_surrogate* s);
MB_API const char* mb_surrogate_last_error(const mb_surrogate* s);
/* Parameters as one FP32 array: W1 [32][27*8] (k = offset*8 + channel,
 * offset = (dx+1) + 3(dy+1) + 9(dz+1)), b1 [32], W2 [32][27*32], b2, W3
 * [32][27*32], b3, W4 [128][6912] (input index voxel*32 + channel, voxel =
 * x + 6y + 36z), b4 [128], W5 [128][128], b5, W6 [128], b6 [1]; each tensor
 * starts at offsets[i] (13 entries, the last the total count). */
MB_API uint32_t mb_surrogate_param_count(void);
MB_API void mb_surrogate_layout(uint32_t* offsets);
MB_API mb_status mb_surrogate_get_params(mb_surrogate* s, float* params);
/* Sets the weights and resets the optimiser state. */
MB_API mb_status mb_surrogate_set_params(mb_surrogate* s, const float* params);
/* Predictions for n genomes (216 bytes each, voxel x + 6y + 36z). */
MB_API mb_status mb_surrogate_predict(mb_surrogate* s, const uint8_t* genomes, uint32_t n, float* out);
/* Mean-squared-error loss and its gradient (layout of the parameters) for
 * one batch of n <= max_batch genomes, without an update. */
MB_API mb_status mb_surrogate_gradients(mb_surrogate* s, const uint8_t* genomes, const float* targets, uint32_t n,
                                        float* grads, float* loss);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) at learning rate lr, with
 * decoupled weight decay (AdamW) when set. */
MB_API mb_status mb_surrogate_set_weight_decay(mb_surrogate* s, float weight_decay);
/* Forward products on tcgen05 (5th-generation tensor cores, TMEM
 * accumulators; the default) or, with on = 0, on the mma.sync kernel that
 * also does the backward products. */
MB_API mb_status mb_surrogate_use_tcgen05(mb_surrogate* s, int on);
MB_API mb_status mb_surrogate_train_step(mb_surrogate* s, const uint8_t* genomes, const float* targets, uint32_t n,
                                         float lr, float* loss);

/* ----------------------------------------------------------------------
 * Measurement (no reference counterpart).
 *
 * Shared-memory read bandwidth of `device`: one 1,024-thread CTA per SM
 * streams conflict-free 128-bit shared loads; bytes_per_s from CUDA events
 * (best of 5 launches), bytes_per_clk_sm (may be NULL) from the SMs' own
 * clock counters.  The roofline denominator of the resident step kernel,
 * which keeps robots in shared memory for a whole launch.  Allocates a few
 * bytes of device memory and synchronises.
 * -------------------------------------------------------------------- */
MB_API mb_status mb_measure_smem_bandwidth(int device, double* bytes_per_s, double* bytes_per_clk_sm);

/* Library version string. */
MB_API const char* mb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MERCURY_B200_H */
