// Test infrastructure only: a C-ABI harness over the reference implementation
// (DawsonCohen/Mercury), compiled from the reference's own sources by
// oracle/Makefile into oracle/_ref/.  Nothing in the product links this file.
//
// Two services:
//   ref_voxel_build  - runs the reference's VoxelRobot::Build
//                      (common/evolvables/VoxelRobot.cpp:310-331) on a given
//                      grid of materials and returns the Element it produces
//                      (masses, springs, baseline COM and length).
//   ref_simulate     - runs the reference's Simulator
//                      (common/simulator/Simulator.cu:206-458, 537-580) on a
//                      batch of robots given as flat arrays and returns the
//                      collected state and spring stresses.  Needs a GPU.
//   ref_simulate_timed - the same, timing Simulate alone as the reference's
//                      benchmark does (optimize/benchmark.cpp:96-99).
//   ref_devo_time    - times the reference's Simulator::Devo
//                      (Simulator.cu:597-668) after a stress-tracked run.
//                      Needs a GPU.
//
// Material arguments are reference material ids: for masses and voxels a base
// id (0..22, materials::matLookup), for springs a composite id (0..253,
// materials::id_lookup).
#include "Simulator.h"
#include "VoxelRobot.h"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// Exposes the protected members of the reference Simulator that the harness
// needs (stress buffer and per-element spring padding).
struct HarnessSimulator : public Simulator {
    const float* stresses() const { return m_hSpringStresses; }
    unsigned springs_per_element() const { return springsPerElement; }
    unsigned masses_per_element() const { return massesPerElement; }
};

// Exposes SoftBody::mLength (protected), set by updateBaseline.
struct HarnessVoxelRobot : public VoxelRobot {
    using VoxelRobot::VoxelRobot;
    float length() const { return mLength; }
};

// Elements of a batch given as flat arrays; masses are padded per robot to
// the largest mass count with isolated air masses (the reference requires an
// equal mass count per element, Simulator.cu:231).
std::vector<Element> make_elements(int n_robots, const int* mass_off, const float* pos, const float* vel,
                                   const uint8_t* mass_mat, const int* spring_off, const uint16_t* pairs,
                                   const float* lbar, const uint8_t* spring_mat) {
    int max_m = 0;
    for (int r = 0; r < n_robots; ++r)
        max_m = std::max(max_m, mass_off[r + 1] - mass_off[r]);
    std::vector<Element> elements(n_robots);
    for (int r = 0; r < n_robots; ++r) {
        Element& e = elements[r];
        for (int i = mass_off[r]; i < mass_off[r + 1]; ++i) {
            Mass m(i - mass_off[r], pos[3 * i], pos[3 * i + 1], pos[3 * i + 2],
                   1.0f, materials::matLookup(mass_mat[i]));
            m.vel = Eigen::Vector3f(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
            e.masses.push_back(m);
        }
        for (int i = mass_off[r + 1] - mass_off[r]; i < max_m; ++i)
            e.masses.push_back(Mass(i, 0.0f, 0.0f, 0.0f, 1.0f, materials::air));
        for (int s = spring_off[r]; s < spring_off[r + 1]; ++s) {
            Spring sp{pairs[2 * s], pairs[2 * s + 1], lbar[s], lbar[s],
                      materials::id_lookup(spring_mat[s])};
            e.springs.push_back(sp);
        }
    }
    return elements;
}

HarnessSimulator* harness_sim() {
    static HarnessSimulator* sim = nullptr;
    if (!sim) sim = new HarnessSimulator();
    return sim;
}

}  // namespace

extern "C" {

// Builds a VoxelRobot on an nx*ny*nz grid of points with spacing h.
// mats[i] is the base material of grid point i (index x + y*nx + z*nx*ny).
// Output buffers must hold nx*ny*nz masses and 13*nx*ny*nz springs.
// Returns 0 on success.
int ref_voxel_build(int nx, int ny, int nz, float h, const uint8_t* mats,
                    int* n_masses, int* n_springs,
                    float* pos, uint8_t* mass_mat,
                    uint16_t* pairs, float* lbar, uint8_t* spring_mat,
                    float* com0, float* length) {
    const int n = nx * ny * nz;
    std::vector<Voxel> voxels(n);
    for (int i = 0; i < n; ++i) {
        int ix = i % nx, iy = (i / nx) % ny, iz = i / (nx * ny);
        Eigen::Vector3f base(h * (float)ix, h * (float)iy, h * (float)iz);
        Eigen::Vector3f center = base + Eigen::Vector3f(0.5f * h, 0.5f * h, 0.5f * h);
        voxels[i] = {(uint)i, {ix, iy, iz}, center, base, materials::matLookup(mats[i])};
    }
    HarnessVoxelRobot R((float)nx, (float)ny, (float)nz, 1.0f, voxels);
    const auto& ms = R.getMasses();
    const auto& ss = R.getSprings();
    *n_masses = (int)ms.size();
    *n_springs = (int)ss.size();
    for (size_t i = 0; i < ms.size(); ++i) {
        pos[3 * i + 0] = ms[i].pos.x();
        pos[3 * i + 1] = ms[i].pos.y();
        pos[3 * i + 2] = ms[i].pos.z();
        mass_mat[i] = ms[i].material.id;
    }
    for (size_t i = 0; i < ss.size(); ++i) {
        pairs[2 * i + 0] = ss[i].m0;
        pairs[2 * i + 1] = ss[i].m1;
        lbar[i] = ss[i].mean_length;
        spring_mat[i] = ss[i].material.id;
    }
    Eigen::Vector3f c = R.getCOM();
    com0[0] = c.x(); com0[1] = c.y(); com0[2] = c.z();
    *length = R.length();
    return 0;
}

// Runs the reference simulator on a batch.  Masses are padded per robot to
// the largest mass count with isolated air masses (the reference requires an
// equal mass count per element, Simulator.cu:231).  Per-robot offsets are
// into the flat arrays.  pos/vel are xyz triples; mass is 1.0 per mass as in
// the reference Mass default.  Outputs have the input (unpadded) layout.
// Returns the number of steps taken, or -1 on error.
int ref_simulate(int n_robots,
                 const int* mass_off, const float* pos, const float* vel,
                 const uint8_t* mass_mat,
                 const int* spring_off, const uint16_t* pairs,
                 const float* lbar, const uint8_t* spring_mat,
                 float dt, float duration, int track_stresses,
                 float* pos_out, float* vel_out, float* stress_out,
                 float* total_time_out) {
    std::vector<Element> elements =
        make_elements(n_robots, mass_off, pos, vel, mass_mat, spring_off, pairs, lbar, spring_mat);
    HarnessSimulator* sim = harness_sim();
    sim->setTimeStep(dt);
    std::vector<ElementTracker> trackers = sim->SetElements(elements);
    sim->Reset();
    sim->Simulate(duration, track_stresses != 0);
    std::vector<Element> out = sim->Collect(trackers);
    int steps = 0;
    {
        float rem = duration;
        while (rem > 0.0f) { rem -= dt; ++steps; }
    }
    *total_time_out = sim->getTotalTime();
    const float* st = sim->stresses();
    unsigned spe = sim->springs_per_element();
    for (int r = 0; r < n_robots; ++r) {
        for (int i = mass_off[r]; i < mass_off[r + 1]; ++i) {
            const Mass& m = out[r].masses[i - mass_off[r]];
            pos_out[3 * i] = m.pos.x(); pos_out[3 * i + 1] = m.pos.y(); pos_out[3 * i + 2] = m.pos.z();
            vel_out[3 * i] = m.vel.x(); vel_out[3 * i + 1] = m.vel.y(); vel_out[3 * i + 2] = m.vel.z();
        }
        if (stress_out)
            for (int s = spring_off[r]; s < spring_off[r + 1]; ++s)
                stress_out[s] = st[(size_t)r * spe + (s - spring_off[r])];
    }
    return steps;
}

// ref_simulate with timings: seconds[0] = Simulate(duration) alone on the
// host clock, as the reference's own benchmark times it
// (optimize/benchmark.cpp:96-99; Simulate synchronises the device after
// every launch, Simulator.cu:428-449 with sim_kernel.cu:271-325);
// seconds[1] = SetElements + Reset + Simulate + Collect.
int ref_simulate_timed(int n_robots,
                       const int* mass_off, const float* pos, const float* vel,
                       const uint8_t* mass_mat,
                       const int* spring_off, const uint16_t* pairs,
                       const float* lbar, const uint8_t* spring_mat,
                       float dt, float duration, int track_stresses,
                       float* pos_out, float* vel_out, double* seconds) {
    std::vector<Element> elements =
        make_elements(n_robots, mass_off, pos, vel, mass_mat, spring_off, pairs, lbar, spring_mat);
    HarnessSimulator* sim = harness_sim();
    sim->setTimeStep(dt);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<ElementTracker> trackers = sim->SetElements(elements);
    sim->Reset();
    auto t1 = std::chrono::steady_clock::now();
    sim->Simulate(duration, track_stresses != 0);
    auto t2 = std::chrono::steady_clock::now();
    std::vector<Element> out = sim->Collect(trackers);
    auto t3 = std::chrono::steady_clock::now();
    seconds[0] = std::chrono::duration<double>(t2 - t1).count();
    seconds[1] = std::chrono::duration<double>(t3 - t0).count();
    int steps = 0;
    {
        float rem = duration;
        while (rem > 0.0f) { rem -= dt; ++steps; }
    }
    for (int r = 0; r < n_robots; ++r)
        for (int i = mass_off[r]; i < mass_off[r + 1]; ++i) {
            const Mass& m = out[r].masses[i - mass_off[r]];
            pos_out[3 * i] = m.pos.x(); pos_out[3 * i + 1] = m.pos.y(); pos_out[3 * i + 2] = m.pos.z();
            vel_out[3 * i] = m.vel.x(); vel_out[3 * i + 1] = m.vel.y(); vel_out[3 * i + 2] = m.vel.z();
        }
    return steps;
}

// Times Simulator::Devo (Simulator.cu:640-668) the way the reference's
// DevoBenchmark calls it (optimize/benchmark.cpp:171-217), after a
// stress-tracked Simulate(duration) so that the sort has stresses to rank:
// Initialize with replaced_springs_per_element = `replaced`, SetElements,
// Simulate, then `calls` Devo() calls, each timed on the host clock (Devo
// synchronises the device itself).  Robots should be identical, as in the
// benchmark: the reference indexes springs as if every robot had the
// largest spring count.  Returns 0.
int ref_devo_time(int n_robots,
                  const int* mass_off, const float* pos, const float* vel,
                  const uint8_t* mass_mat,
                  const int* spring_off, const uint16_t* pairs,
                  const float* lbar, const uint8_t* spring_mat,
                  unsigned replaced, float dt, float duration, int calls, double* seconds) {
    std::vector<Element> elements =
        make_elements(n_robots, mass_off, pos, vel, mass_mat, spring_off, pairs, lbar, spring_mat);
    HarnessSimulator* sim = harness_sim();
    Config::Simulator config;
    config.replaced_springs_per_element = replaced;
    config.time_step = dt;
    sim->Initialize(config);
    sim->SetElements(elements);
    sim->Reset();
    sim->Simulate(duration, true);
    for (int i = 0; i < calls; ++i) {
        auto t0 = std::chrono::steady_clock::now();
        sim->Devo();
        auto t1 = std::chrono::steady_clock::now();
        seconds[i] = std::chrono::duration<double>(t1 - t0).count();
    }
    return 0;
}

// Composite material table exactly as Simulator::SetElements uploads it
// (Simulator.cu:286-292): float4 {k, dL0, omega, phi} per composite id.
void ref_material_table(float* out /* 4*COMPOSITE_COUNT */) {
    for (unsigned i = 0; i < COMPOSITE_COUNT; ++i) {
        Material m = materials::id_lookup(i);
        out[4 * i] = m.k; out[4 * i + 1] = m.dL0; out[4 * i + 2] = m.omega; out[4 * i + 3] = m.phi;
    }
}

// materials::decode(encoding).id and encoding of the decoded material.
int ref_decode_id(uint32_t encoding) { return materials::decode(encoding).id; }

int ref_composite_count() { return COMPOSITE_COUNT; }

}  // extern "C"
