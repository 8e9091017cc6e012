// Surrogate-screened evaluation for the reference's optimizer.
//
// The reference's child step (optimize/optimizer/optimizer_impl.h:113-276,
// Optimizer<T>::ChildStep) builds every child and evaluates all of them with
// Evaluator<T>::BatchEvaluate (optimize/optimizer/Evaluator_impl.h:38-107).
// ScreenedEvaluator<T>::BatchEvaluate takes the same vector and stands in for
// that one call: a fitness surrogate (libmercury_b200's BF16 network,
// include/mercury_b200.h, mb_surrogate_*) ranks the children, and only its
// top `screen` fraction plus a random `audit` fraction is evaluated -- by the
// reference's own Evaluator<T>::BatchEvaluate, on the drop-in Simulator.
// The others are reset to their initial state with fitness 0 (never
// evaluated), so that ChildStep's replacement keeps none of them.  The
// surrogate trains online on every evaluated child; until `warmup` children
// have been evaluated every child is evaluated.
//
// Children are represented to the surrogate by a genome function: for the
// reference's VoxelRobot, voxel_genome() below (6x6x6 cells of air, bone,
// tissue, adductor_muscle0, abductor_muscle0).  Children it cannot
// represent (other sizes or materials) are always evaluated.
//
// Ranking: the prediction averaged over the 8 horizontal orientations of the
// genome (mirror x, mirror y, swap x and y: the fitness is the same), plus
// `kappa` times its spread over them in fitness units.  Training: minibatches
// of `batch` genomes in random orientations, half from the newest
// evaluations, targets standardised by the warm-up's mean and deviation.
//
// Not re-entrant (one surrogate, one stream); the reference's Evaluator is
// a static singleton as well.
#ifndef MERCURY_B200_COMPAT_SCREENED_EVALUATOR_H
#define MERCURY_B200_COMPAT_SCREENED_EVALUATOR_H

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <functional>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "Evaluator.h"
#include "mercury_b200.h"

namespace mercury_screen {

constexpr int kVox = 216;  // 6 x 6 x 6 cells, index x + 6y + 36z

// The 8 symmetries of the horizontal square as voxel permutations:
// oriented[v] = genome[perm[o][v]].
inline const std::vector<std::vector<int>>& orientations() {
    static const std::vector<std::vector<int>> perms = [] {
        std::vector<std::vector<int>> out;
        for (int mx = 0; mx < 2; ++mx)
            for (int my = 0; my < 2; ++my)
                for (int sw = 0; sw < 2; ++sw) {
                    std::vector<int> p(kVox);
                    for (int v = 0; v < kVox; ++v) {
                        int x = v % 6, y = (v / 6) % 6, z = v / 36;
                        int xx = mx ? 5 - x : x, yy = my ? 5 - y : y;
                        if (sw) std::swap(xx, yy);
                        p[v] = xx + 6 * yy + 36 * z;
                    }
                    out.push_back(p);
                }
        return out;
    }();
    return perms;
}

// Genome of a reference VoxelRobot built on 7 x 7 x 7 grid points whose
// outer layer (any index 6) is air: the class of the material at point
// (x, y, z) of cell x + 6y + 36z -- 0 air, 1 bone, 2 tissue, 3
// adductor_muscle0, 4 abductor_muscle0 (material ids 0, 22, 21, 1, 11).
// False for any other size or material.
template <typename R>
bool voxel_genome(R& robot, uint8_t* out) {
    const auto& voxels = robot.getVoxels();
    if (voxels.size() != 343) return false;
    for (const auto& v : voxels) {
        const int x = v.indices.x, y = v.indices.y, z = v.indices.z;
        if (x < 0 || y < 0 || z < 0 || x > 6 || y > 6 || z > 6) return false;
        int cls;
        switch (v.mat.id) {
            case 0: cls = 0; break;
            case 22: cls = 1; break;
            case 21: cls = 2; break;
            case 1: cls = 3; break;
            case 11: cls = 4; break;
            default: return false;
        }
        if (x == 6 || y == 6 || z == 6) {
            if (cls != 0) return false;
            continue;
        }
        out[x + 6 * y + 36 * z] = (uint8_t)cls;
    }
    return true;
}

}  // namespace mercury_screen

template <typename T>
class ScreenedEvaluator {
public:
    using GenomeFn = std::function<bool(T&, uint8_t*)>;

    struct Options {
        float screen = 0.35f;      // top fraction of the ranked children evaluated
        float audit = 0.05f;       // random fraction of the rest evaluated as well
        size_t warmup = 4096;      // evaluations before the first screen
        float warmup_epochs = 30;  // passes over the warm-up set before screening
        uint32_t steps = 60;       // training steps after every screened batch
        uint32_t batch = 256;      // training minibatch
        float lr = 1e-3f;          // warm-up learning rate (cosine)
        float finetune_lr = 3e-4f; // online learning rate
        float kappa = 1.0f;        // bonus per unit of spread over the orientations
        uint64_t seed = 0;
    };

    struct Stats {
        size_t children = 0, evaluated = 0, screened_out = 0, unrepresentable = 0;
        bool screening = false;  // false while warming up
    };

    ScreenedEvaluator(int device, GenomeFn genome, Options opt) : genome_(std::move(genome)), o_(opt), rng_(opt.seed) {
        if (mb_surrogate_create(device, std::max<uint32_t>(opt.batch, 1024u), opt.seed, &sg_) != MB_OK)
            throw std::runtime_error(std::string("mb_surrogate_create: ") + mb_surrogate_last_error(sg_));
    }
    ScreenedEvaluator(int device, GenomeFn genome) : ScreenedEvaluator(device, std::move(genome), Options()) {}
    ~ScreenedEvaluator() { mb_surrogate_destroy(sg_); }
    ScreenedEvaluator(const ScreenedEvaluator&) = delete;
    ScreenedEvaluator& operator=(const ScreenedEvaluator&) = delete;

    // Drop-in for Evaluator<T>::BatchEvaluate(solutions).
    void BatchEvaluate(std::vector<T>& solutions) {
        const size_t n = solutions.size();
        last_ = Stats();
        last_.children = n;
        if (n == 0) return;
        std::vector<uint8_t> g(n * mercury_screen::kVox);
        std::vector<char> ok(n);
        for (size_t i = 0; i < n; ++i) {
            ok[i] = genome_(solutions[i], g.data() + i * mercury_screen::kVox) ? 1 : 0;
            last_.unrepresentable += ok[i] ? 0 : 1;
        }
        std::vector<size_t> chosen;  // evaluated
        const bool screening = trained_;
        last_.screening = screening;
        if (!screening) {
            chosen.resize(n);
            std::iota(chosen.begin(), chosen.end(), 0);
        } else {
            std::vector<size_t> rep;
            for (size_t i = 0; i < n; ++i) (ok[i] ? rep : chosen).push_back(i);
            std::vector<uint8_t> gr(rep.size() * mercury_screen::kVox);
            for (size_t k = 0; k < rep.size(); ++k)
                std::copy_n(g.data() + rep[k] * mercury_screen::kVox, mercury_screen::kVox,
                            gr.data() + k * mercury_screen::kVox);
            const std::vector<float> score = rank_score(gr);
            std::vector<size_t> order(rep.size());
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return score[a] > score[b]; });
            const size_t top = (size_t)std::lround(o_.screen * rep.size());
            const size_t aud = std::min(rep.size() - top, (size_t)std::lround(o_.audit * rep.size()));
            for (size_t k = 0; k < top; ++k) chosen.push_back(rep[order[k]]);
            std::vector<size_t> rest(order.begin() + top, order.end());
            std::shuffle(rest.begin(), rest.end(), rng_);
            for (size_t k = 0; k < aud; ++k) chosen.push_back(rep[rest[k]]);
            std::sort(chosen.begin(), chosen.end());
        }
        // the reference's evaluation of the chosen children
        std::vector<T> sub;
        sub.reserve(chosen.size());
        for (size_t i : chosen) sub.push_back(solutions[i]);
        Evaluator<T>::BatchEvaluate(sub);
        std::vector<char> done(n, 0);
        for (size_t k = 0; k < chosen.size(); ++k) {
            solutions[chosen[k]] = sub[k];
            done[chosen[k]] = 1;
        }
        for (size_t i = 0; i < n; ++i)
            if (!done[i]) {  // never evaluated: initial state, fitness 0
                solutions[i].Reset();
                solutions[i].updateFitness();
                ++last_.screened_out;
            }
        last_.evaluated = chosen.size();
        chosen_ = chosen;
        // training set: every evaluated child the surrogate can represent
        std::vector<uint8_t> ng;
        std::vector<float> nf;
        for (size_t i : chosen)
            if (ok[i]) {
                ng.insert(ng.end(), g.begin() + i * mercury_screen::kVox, g.begin() + (i + 1) * mercury_screen::kVox);
                nf.push_back(solutions[i].fitness());
            }
        data_g_.insert(data_g_.end(), ng.begin(), ng.end());
        data_f_.insert(data_f_.end(), nf.begin(), nf.end());
        if (!trained_) {
            if (data_f_.size() >= o_.warmup) warm_up();
        } else if (!nf.empty()) {
            train(o_.steps, o_.finetune_lr, false, &ng, &nf);
        }
    }

    const Stats& last() const { return last_; }
    // indices of the children the last call evaluated, ascending
    const std::vector<size_t>& chosen() const { return chosen_; }
    bool screening() const { return trained_; }
    mb_surrogate* surrogate() { return sg_; }

    // Mean prediction over the orientations plus kappa times their spread,
    // in fitness units (for tests and callers that rank themselves).
    std::vector<float> rank_score(const std::vector<uint8_t>& genomes) {
        const size_t m = genomes.size() / mercury_screen::kVox;
        const auto& P = mercury_screen::orientations();
        std::vector<double> s1(m, 0.0), s2(m, 0.0);
        std::vector<uint8_t> view(genomes.size());
        std::vector<float> out(m);
        for (const auto& p : P) {
            for (size_t i = 0; i < m; ++i)
                for (int v = 0; v < mercury_screen::kVox; ++v)
                    view[i * mercury_screen::kVox + v] = genomes[i * mercury_screen::kVox + p[v]];
            check(mb_surrogate_predict(sg_, view.data(), (uint32_t)m, out.data()), "mb_surrogate_predict");
            for (size_t i = 0; i < m; ++i) {
                s1[i] += out[i];
                s2[i] += (double)out[i] * out[i];
            }
        }
        std::vector<float> score(m);
        const double k = (double)P.size();
        for (size_t i = 0; i < m; ++i) {
            const double mean = s1[i] / k, var = std::max(0.0, s2[i] / k - mean * mean);
            score[i] = (float)((mean + o_.kappa * std::sqrt(var)) * sd_ + mu_);
        }
        return score;
    }

private:
    void check(mb_status s, const char* what) {
        if (s != MB_OK) throw std::runtime_error(std::string(what) + ": " + mb_surrogate_last_error(sg_));
    }

    void warm_up() {
        const size_t m = data_f_.size();
        double s = 0.0, s2 = 0.0;
        for (float f : data_f_) {
            s += f;
            s2 += (double)f * f;
        }
        mu_ = s / m;
        sd_ = std::sqrt(std::max(1e-18, s2 / m - mu_ * mu_)) + 1e-9;
        train((uint32_t)std::ceil(o_.warmup_epochs * m / o_.batch), o_.lr, true, nullptr, nullptr);
        trained_ = true;
    }

    // `steps` Adam steps on minibatches in random orientations; with a
    // newest set, half of every batch from it.
    void train(uint32_t steps, float lr, bool cosine, const std::vector<uint8_t>* ng, const std::vector<float>* nf) {
        const size_t m = data_f_.size();
        if (m == 0) return;
        const auto& P = mercury_screen::orientations();
        std::uniform_int_distribution<size_t> any(0, m - 1);
        std::uniform_int_distribution<int> orient(0, (int)P.size() - 1);
        const size_t nn = nf ? nf->size() : 0;
        std::vector<uint8_t> bg((size_t)o_.batch * mercury_screen::kVox);
        std::vector<float> bt(o_.batch);
        for (uint32_t it = 0; it < steps; ++it) {
            const float step_lr = cosine ? lr * 0.5f * (1.0f + std::cos(3.14159265f * it / steps)) : lr;
            for (uint32_t j = 0; j < o_.batch; ++j) {
                const uint8_t* src;
                float f;
                if (nn && j >= o_.batch / 2) {
                    const size_t r = std::uniform_int_distribution<size_t>(0, nn - 1)(rng_);
                    src = ng->data() + r * mercury_screen::kVox;
                    f = (*nf)[r];
                } else {
                    const size_t r = any(rng_);
                    src = data_g_.data() + r * mercury_screen::kVox;
                    f = data_f_[r];
                }
                const auto& p = P[orient(rng_)];
                for (int v = 0; v < mercury_screen::kVox; ++v) bg[j * mercury_screen::kVox + v] = src[p[v]];
                bt[j] = (float)((f - mu_) / sd_);
            }
            float loss = 0.0f;
            check(mb_surrogate_train_step(sg_, bg.data(), bt.data(), o_.batch, step_lr, &loss),
                  "mb_surrogate_train_step");
        }
    }

    mb_surrogate* sg_ = nullptr;
    GenomeFn genome_;
    Options o_;
    std::mt19937_64 rng_;
    std::vector<uint8_t> data_g_;
    std::vector<float> data_f_;
    double mu_ = 0.0, sd_ = 1.0;
    bool trained_ = false;
    Stats last_;
    std::vector<size_t> chosen_;
};

#endif  // MERCURY_B200_COMPAT_SCREENED_EVALUATOR_H
