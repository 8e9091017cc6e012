// Adapter of the reference's Simulator API (Simulator.h) over the C ABI of
// libmercury_b200.  Packing follows the reference's SetElements
// (Simulator.cu:249-308) without its per-robot padding; the composite
// material table is the reference's own id_lookup table
// (Simulator.cu:286-292).
#include "Simulator.h"

#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>

#include "../../include/mercury_b200.h"

namespace {

void check(mb_context* ctx, mb_status s, const char* what) {
    if (s == MB_OK) return;
    std::string msg = std::string(what) + " failed (status " + std::to_string((int)s) + ")";
    if (ctx) msg += ": " + std::string(mb_last_error(ctx));
    throw std::runtime_error(msg);
}

}  // namespace

Simulator::Simulator() {
    check(nullptr, mb_context_create(0, &ctx_), "mb_context_create");
    float table[4 * MB_COMPOSITE_COUNT];
    for (unsigned i = 0; i < MB_COMPOSITE_COUNT; ++i) {
        Material m = materials::id_lookup((uint8_t)i);
        table[4 * i] = m.k;
        table[4 * i + 1] = m.dL0;
        table[4 * i + 2] = m.omega;
        table[4 * i + 3] = m.phi;
    }
    check(ctx_, mb_set_materials(ctx_, table), "mb_set_materials");
    check(ctx_, mb_set_time_step(ctx_, m_deltaT), "mb_set_time_step");
}

Simulator::~Simulator() { mb_context_destroy(ctx_); }

void Simulator::Initialize(Config::Simulator config) {
    m_config = config;
    setTimeStep(config.time_step);
    Reset();
}

void Simulator::setTimeStep(float dt) {
    check(ctx_, mb_set_time_step(ctx_, dt), "mb_set_time_step");
    m_deltaT = dt;
}

float Simulator::getTotalTime() const { return mb_get_total_time(ctx_); }

void Simulator::Reset() { check(ctx_, mb_set_total_time(ctx_, 0.0f), "mb_set_total_time"); }

void Simulator::setMode(int mode) { check(ctx_, mb_set_mode(ctx_, (mb_mode)mode), "mb_set_mode"); }

void Simulator::setEnvironment(const Environment& env) {
    mb_environment e;
    check(ctx_, mb_get_environment(ctx_, &e), "mb_get_environment");
    e.g = env.g;
    e.floor_stiffness = env.floor_stiffness;
    e.friction_kinetic = env.friction;
    if (env.type == ENVIRONMENT_WATER) {
        // the reference's water drag is the density of its face law
        // (EnvironmentWater.drag = 1000 reaches surfaceDragForce as rho)
        e.drag = 0.0f;
        e.face_drag = env.drag;
    } else {
        e.face_drag = 0.0f;
    }
    check(ctx_, mb_set_environment(ctx_, &e), "mb_set_environment");
}

ElementTracker Simulator::SetElement(const Element& element) {
    return SetElements(std::vector<Element>{element})[0];
}

std::vector<ElementTracker> Simulator::SetElements(const std::vector<Element>& elements) {
    elements_ = elements;
    upload();
    std::vector<ElementTracker> trackers;
    for (size_t r = 0; r < elements_.size(); ++r) {
        ElementTracker t;
        t.ID = (uint)r;
        t.mass_begin = massBuf_.data() + massOff_[r];
        t.mass_end = massBuf_.data() + massOff_[r + 1];
        t.spring_begin = springBuf_.data() + springOff_[r];
        t.spring_end = springBuf_.data() + springOff_[r + 1];
        trackers.push_back(t);
    }
    return trackers;
}

ElementTracker Simulator::AllocateElement(const Element& e) {
    std::vector<Element> all = elements_;
    all.push_back(e);
    return SetElements(all).back();
}

void Simulator::upload() {
    const size_t R = elements_.size();
    massOff_.assign(1, 0);
    springOff_.assign(1, 0);
    faceOff_.assign(1, 0);
    massBuf_.clear();
    springBuf_.clear();
    faces_.clear();
    for (const Element& e : elements_) {
        massBuf_.insert(massBuf_.end(), e.masses.begin(), e.masses.end());
        springBuf_.insert(springBuf_.end(), e.springs.begin(), e.springs.end());
        for (const Face& f : e.faces) {  // Simulator.cu:310-317
            faces_.push_back(f.m0);
            faces_.push_back(f.m1);
            faces_.push_back(f.m2);
        }
        massOff_.push_back((int64_t)massBuf_.size());
        springOff_.push_back((int64_t)springBuf_.size());
        faceOff_.push_back((int64_t)(faces_.size() / 3));
    }
    const size_t M = massBuf_.size(), S = springBuf_.size();
    pos_.assign(4 * M, 0.0f);
    vel_.assign(4 * M, 0.0f);
    massMat_.assign(M, 0);
    for (size_t i = 0; i < M; ++i) {
        const Mass& m = massBuf_[i];
        pos_[4 * i] = m.pos.x();
        pos_[4 * i + 1] = m.pos.y();
        pos_[4 * i + 2] = m.pos.z();
        pos_[4 * i + 3] = m.mass;
        vel_[4 * i] = m.vel.x();
        vel_[4 * i + 1] = m.vel.y();
        vel_[4 * i + 2] = m.vel.z();
        massMat_[i] = m.material.id;
    }
    pairs_.assign(2 * S, 0);
    springMat_.assign(S, 0);
    lbar_.assign(S, 0.0f);
    stress_.assign(S, 0.0f);
    for (size_t s = 0; s < S; ++s) {
        const Spring& sp = springBuf_[s];
        pairs_[2 * s] = sp.m0;
        pairs_[2 * s + 1] = sp.m1;
        springMat_[s] = sp.material.id;
        lbar_[s] = sp.mean_length;
    }
    const bool faces = !faces_.empty();
    mb_batch_desc d{(uint32_t)R,
                    massOff_.data(),
                    pos_.data(),
                    vel_.data(),
                    massMat_.data(),
                    springOff_.data(),
                    pairs_.data(),
                    springMat_.data(),
                    lbar_.data(),
                    faces ? faceOff_.data() : nullptr,
                    faces ? faces_.data() : nullptr};
    check(ctx_, mb_set_elements(ctx_, &d), "mb_set_elements");
}

void Simulator::Simulate(float sim_duration, bool trackStresses, bool trace, std::string tracefile) {
    if (!trace) {
        check(ctx_, mb_simulate(ctx_, sim_duration, trackStresses ? 1 : 0, nullptr), "mb_simulate");
        return;
    }
    // Trace: the state every 20 steps (Simulator.cu:432-444), as CSV rows
    // "id, time, x, y, z, vx, vy, vz" appended to `tracefile`.
    uint32_t steps = 0;
    {
        volatile float rem = sim_duration;
        while (rem > 0.0f) {
            rem = rem - m_deltaT;
            ++steps;
        }
    }
    std::ofstream out(tracefile, std::ios::app);
    uint32_t done = 0;
    while (done < steps) {
        const float t = getTotalTime();
        check(ctx_, mb_collect(ctx_, pos_.data(), vel_.data(), nullptr), "mb_collect");
        for (size_t i = 0; i < massBuf_.size(); ++i)
            out << i << "," << t << "," << pos_[4 * i] << "," << pos_[4 * i + 1] << "," << pos_[4 * i + 2]
                << "," << vel_[4 * i] << "," << vel_[4 * i + 1] << "," << vel_[4 * i + 2] << "\n";
        const uint32_t n = steps - done < 20u ? steps - done : 20u;
        check(ctx_, mb_run_steps(ctx_, n, trackStresses ? 1 : 0), "mb_run_steps");
        done += n;
    }
}

void Simulator::Devo() {
    // Simulator.cu:640-668: the seed counts Devo calls from 0 (per simulator
    // here; the reference's counter is a function-local static).
    check(ctx_, mb_devo(ctx_, m_config.replaced_springs_per_element, (uint64_t)devoSeed_, 0, nullptr),
          "mb_devo");
    ++devoSeed_;
}

void Simulator::download() {
    check(ctx_, mb_collect(ctx_, pos_.data(), vel_.data(), stress_.data()), "mb_collect");
    // pairs, materials and mean lengths as Devo left them (Simulator.cu:542-561)
    check(ctx_, mb_collect_springs(ctx_, pairs_.data(), springMat_.data(), lbar_.data()), "mb_collect_springs");
    for (size_t s = 0; s < springBuf_.size(); ++s) {
        springBuf_[s].m0 = pairs_[2 * s];
        springBuf_[s].m1 = pairs_[2 * s + 1];
        springBuf_[s].mean_length = lbar_[s];
        springBuf_[s].material = materials::id_lookup(springMat_[s]);
    }
    std::vector<uint32_t> flags(elements_.size(), 0);
    check(ctx_, mb_robot_flags(ctx_, flags.data()), "mb_robot_flags");
    for (size_t r = 0; r < flags.size(); ++r)
        if (flags[r] & 1u) std::fprintf(stderr, "mercury_b200: robot %zu has non-finite positions\n", r);
    for (size_t i = 0; i < massBuf_.size(); ++i) {
        massBuf_[i].pos = Eigen::Vector3f(pos_[4 * i], pos_[4 * i + 1], pos_[4 * i + 2]);
        massBuf_[i].vel = Eigen::Vector3f(vel_[4 * i], vel_[4 * i + 1], vel_[4 * i + 2]);
    }
}

Element Simulator::Collect(const ElementTracker& tracker) {
    return Collect(std::vector<ElementTracker>{tracker})[0];
}

std::vector<Element> Simulator::Collect(const std::vector<ElementTracker>& trackers) {
    download();
    std::vector<Element> out;
    for (const ElementTracker& t : trackers) out.push_back(CollectElement(t));
    return out;
}

Element Simulator::CollectElement(const ElementTracker& tracker) {
    Element e;
    e.masses.assign(tracker.mass_begin, tracker.mass_end);
    e.springs.assign(tracker.spring_begin, tracker.spring_end);
    return e;
}

std::vector<float> Simulator::Stresses(const ElementTracker& tracker) const {
    const size_t b = (size_t)(tracker.spring_begin - springBuf_.data());
    const size_t e = (size_t)(tracker.spring_end - springBuf_.data());
    return std::vector<float>(stress_.begin() + b, stress_.begin() + e);
}
