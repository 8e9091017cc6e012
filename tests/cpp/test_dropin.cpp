// C++ test of the drop-in Simulator (mercury_b200/compat) used the way the
// reference's TestSimulator uses its own (common/tests/test_simulator.cpp:
// 19-63): reference VoxelRobots, Initialize with dt = 1e-3, SetElements,
// Simulate, Collect, SoftBody::Update (fitness), run twice -> identical
// fitness.  Then one Devo() (Simulator.cu:640-668) and a second Collect.
// Writes the robots, the collected state and the rewired springs to a binary
// file for the GPU pytest to compare with the oracle.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "Simulator.h"
#include "VoxelRobot.h"

namespace {

VoxelRobot make_robot(int cells, unsigned seed) {
    const int n = cells + 1;
    std::mt19937 rng(seed);
    const uint8_t choices[5] = {0, 22, 21, 1, 11};  // air, bone, tissue, adductor0, abductor0
    std::discrete_distribution<int> pick({0.3, 0.175, 0.175, 0.175, 0.175});
    std::vector<Voxel> voxels(n * n * n);
    for (int i = 0; i < n * n * n; ++i) {
        int ix = i % n, iy = (i / n) % n, iz = i / (n * n);
        uint8_t m = (ix == n - 1 || iy == n - 1 || iz == n - 1) ? 0 : choices[pick(rng)];
        Eigen::Vector3f base(0.1f * ix, 0.1f * iy, 0.1f * iz);
        voxels[i] = {(uint)i, {ix, iy, iz}, base + Eigen::Vector3f(0.05f, 0.05f, 0.05f), base,
                     materials::matLookup(m)};
    }
    return VoxelRobot((float)n, (float)n, (float)n, 1.0f, voxels);
}

std::vector<float> run(Simulator& sim, std::vector<SoftBody>& robots, float t) {
    sim.Reset();
    std::vector<Element> elements;
    for (auto& R : robots) {
        R.Reset();
        elements.push_back(R);
    }
    std::vector<ElementTracker> trackers = sim.SetElements(elements);
    sim.Simulate(t, true);
    std::vector<Element> results = sim.Collect(trackers);
    std::vector<float> fit;
    for (size_t i = 0; i < robots.size(); ++i) {
        robots[i].Update(results[i]);
        fit.push_back(robots[i].fitness());
    }
    return fit;
}

}  // namespace

int main(int argc, char** argv) {
    const char* out_path = argc > 1 ? argv[1] : "dropin.bin";
    std::vector<SoftBody> robots;
    for (int r = 0; r < 10; ++r) robots.push_back(make_robot(3 + r % 5, 1000u + r));
    Config config;
    config.simulator.time_step = 1e-3f;
    Simulator sim;
    sim.Initialize(config.simulator);
    std::vector<float> a = run(sim, robots, 0.5f);
    std::vector<float> b = run(sim, robots, 0.5f);
    int failures = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        std::printf("robot %zu fitness %.9g rerun %.9g\n", i, a[i], b[i]);
        if (a[i] != b[i]) ++failures;
    }
    // one more run, collected with the inputs, for the comparison with the oracle
    for (auto& R : robots) R.Reset();
    std::vector<Element> elements(robots.begin(), robots.end());
    std::vector<ElementTracker> trackers = sim.SetElements(elements);
    sim.Reset();
    sim.Simulate(0.25f, true);
    std::vector<Element> results = sim.Collect(trackers);
    std::vector<std::vector<float>> stresses;
    for (const auto& t : trackers) stresses.push_back(sim.Stresses(t));
    sim.Devo();
    std::vector<Element> devo = sim.Collect(trackers);
    FILE* f = std::fopen(out_path, "wb");
    if (!f) return 2;
    uint32_t R = (uint32_t)robots.size();
    std::fwrite(&R, 4, 1, f);
    for (uint32_t r = 0; r < R; ++r) {
        const Element& in = elements[r];
        const Element& o = results[r];
        uint32_t nm = (uint32_t)in.masses.size(), ns = (uint32_t)in.springs.size();
        std::fwrite(&nm, 4, 1, f);
        std::fwrite(&ns, 4, 1, f);
        for (const Mass& m : in.masses) {
            float v[4] = {m.pos.x(), m.pos.y(), m.pos.z(), m.mass};
            uint8_t id = m.material.id;
            std::fwrite(v, 4, 4, f);
            std::fwrite(&id, 1, 1, f);
        }
        for (const Spring& s : in.springs) {
            uint16_t p[2] = {s.m0, s.m1};
            uint8_t id = s.material.id;
            float l = s.mean_length;
            std::fwrite(p, 2, 2, f);
            std::fwrite(&id, 1, 1, f);
            std::fwrite(&l, 4, 1, f);
        }
        for (const Mass& m : o.masses) {
            float v[6] = {m.pos.x(), m.pos.y(), m.pos.z(), m.vel.x(), m.vel.y(), m.vel.z()};
            std::fwrite(v, 4, 6, f);
        }
        std::fwrite(stresses[r].data(), 4, stresses[r].size(), f);
        for (const Spring& s : devo[r].springs) {
            uint16_t p[2] = {s.m0, s.m1};
            uint8_t id = s.material.id;
            float l = s.mean_length;
            std::fwrite(p, 2, 2, f);
            std::fwrite(&id, 1, 1, f);
            std::fwrite(&l, 4, 1, f);
        }
    }
    float tt = sim.getTotalTime();
    std::fwrite(&tt, 4, 1, f);
    std::fclose(f);
    std::printf("%s: %d fitness mismatches\n", failures ? "FAIL" : "OK", failures);
    return failures ? 1 : 0;
}
