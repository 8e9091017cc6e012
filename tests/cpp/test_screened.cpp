// C++ test of ScreenedEvaluator (mercury_b200/compat/ScreenedEvaluator.h) in
// the reference's evaluation loop: reference VoxelRobots of 6x6x6 five-class
// cells, children made by the reference's own VoxelRobot::Crossover (two-
// point, VoxelRobot.cpp:428-445), evaluated by the reference's
// Evaluator<VoxelRobot>::BatchEvaluate (Evaluator_impl.h:38-107) on the
// drop-in Simulator -- once in full, once through the screen.
//
// Prints one line of key=value pairs for the GPU pytest; exit status 0 when
// every check below holds:
//   - while warming up, every child is evaluated, with the full fitness;
//   - once screening, the evaluated count is round(0.35 n) + round(0.05 of
//     the rest), each evaluated child has the fitness the full evaluation
//     gives it (bit for bit), every other child has fitness 0;
//   - a child the surrogate cannot represent (a material outside the five)
//     is always evaluated;
//   - the screen finds more of the truly best 10 % than its share of the
//     children would by chance.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "Evaluator.h"
#include "ScreenedEvaluator.h"
#include "VoxelRobot.h"

namespace {

VoxelRobot make_robot(std::mt19937& rng) {
    const int n = 7;  // 6x6x6 cells on 7x7x7 points, outer layer air
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

std::vector<VoxelRobot> children_of(const std::vector<VoxelRobot>& parents, size_t n, std::mt19937& rng) {
    std::uniform_int_distribution<size_t> any(0, parents.size() - 1);
    std::vector<VoxelRobot> kids;
    while (kids.size() < n) {
        CandidatePair<VoxelRobot> c = VoxelRobot::Crossover({parents[any(rng)], parents[any(rng)]});
        kids.push_back(c.first);
        if (kids.size() < n) kids.push_back(c.second);
    }
    return kids;
}

}  // namespace

int main() {
    VoxelRobot::repr = VoxelRobot::ENCODE_DIRECT;  // two-point crossover of the voxels
    OptimizerConfig config;
    config.simulator.time_step = 0.005f;
    config.evaluator.base_time = 0.0f;
    config.evaluator.eval_time = 1.0f;
    config.devo.devo_cycles = 0;
    Evaluator<VoxelRobot>::Initialize(config);

    ScreenedEvaluator<VoxelRobot>::Options opt;
    opt.warmup = 2048;
    opt.warmup_epochs = 20;
    opt.steps = 40;
    ScreenedEvaluator<VoxelRobot> screen(0, mercury_screen::voxel_genome<VoxelRobot>, opt);

    std::mt19937 rng(7);
    const size_t n = 1024;
    bool ok = true;
    // warm-up: random robots, then children of the best so far
    std::vector<VoxelRobot> elite;
    for (int gen = 0; gen < 2; ++gen) {
        std::vector<VoxelRobot> batch;
        if (elite.empty())
            for (size_t i = 0; i < n; ++i) batch.push_back(make_robot(rng));
        else
            batch = children_of(elite, n, rng);
        std::vector<VoxelRobot> full = batch;
        Evaluator<VoxelRobot>::BatchEvaluate(full);
        screen.BatchEvaluate(batch);
        ok &= !screen.last().screening && screen.last().evaluated == n;
        for (size_t i = 0; i < n; ++i) ok &= batch[i].fitness() == full[i].fitness();
        std::vector<size_t> idx(n);
        for (size_t i = 0; i < n; ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return full[a].fitness() > full[b].fitness(); });
        elite.clear();
        for (size_t k = 0; k < 64; ++k) elite.push_back(full[idx[k]]);
    }
    ok &= screen.screening();
    // a screened generation, with one child outside the surrogate's classes
    std::vector<VoxelRobot> kids = children_of(elite, n, rng);
    {
        auto& vox = kids[5].getVoxels();  // another material: not representable
        vox[0].mat = materials::matLookup(2);
        kids[5].Build();
    }
    std::vector<VoxelRobot> full = kids;
    Evaluator<VoxelRobot>::BatchEvaluate(full);
    screen.BatchEvaluate(kids);
    const auto st = screen.last();
    const size_t rep = n - st.unrepresentable;
    const size_t top = (size_t)std::lround(0.35 * rep), aud = (size_t)std::lround(0.05 * rep);
    ok &= st.screening && st.unrepresentable == 1 && st.evaluated == top + aud + 1;
    std::vector<char> chosen(n, 0);
    for (size_t i : screen.chosen()) chosen[i] = 1;
    size_t zeros = 0;
    for (size_t i = 0; i < n; ++i) {
        if (chosen[i]) {
            ok &= kids[i].fitness() == full[i].fitness();  // the reference's evaluation, bit for bit
        } else {
            ok &= kids[i].fitness() == 0.0f;  // never evaluated: reset, fitness 0
            ++zeros;
        }
    }
    ok &= chosen[5] == 1 && zeros == st.screened_out;
    // recall of the best 10 % of the children
    std::vector<size_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return full[a].fitness() > full[b].fitness(); });
    size_t hit = 0;
    for (size_t k = 0; k < n / 10; ++k) hit += chosen[idx[k]];
    const double recall = (double)hit / (n / 10), chance = (double)st.evaluated / n;
    ok &= recall > chance + 0.1;
    std::printf("ok=%d evaluated=%zu screened_out=%zu zeros=%zu unrepresentable=%zu recall=%.4f chance=%.4f\n",
                ok ? 1 : 0, st.evaluated, st.screened_out, zeros, st.unrepresentable, recall, chance);
    return ok ? 0 : 1;
}
