// Drop-in replacement for the reference's common/simulator/Simulator.h.
//
// Same class name, public methods, defaults and ElementTracker as the
// reference (Simulator.h:11-48), so the reference's callers -- the
// optimizer's Evaluator, the benchmark, the visualizer, the tests -- compile
// and link against it unchanged.  The data model (Element, Mass, Spring,
// Material, Environment, Config) is the reference's own headers, which this
// header includes; the implementation (Simulator.cpp) is a thin adapter over
// the C ABI of libmercury_b200 (include/mercury_b200.h).
//
// Differences, by design: robots may have different mass counts; errors
// throw std::runtime_error instead of exiting the process; the stresses the
// reference copies back but drops are available through Stresses(); the
// trace CSV is written to `tracefile` itself.
#ifndef MERCURY_B200_COMPAT_SIMULATOR_H
#define MERCURY_B200_COMPAT_SIMULATOR_H

#include <cstdint>
#include <string>
#include <vector>

#include "config.h"
#include "element.h"
#include "environment.h"

struct mb_context;

struct ElementTracker {
    uint ID;
    Mass* mass_begin;
    Mass* mass_end;
    Spring* spring_begin;
    Spring* spring_end;
};

class Simulator {
public:
    Simulator();
    ~Simulator();
    Simulator(const Simulator&) = delete;
    Simulator& operator=(const Simulator&) = delete;

    void Initialize(Config::Simulator = Config::Simulator());

    ElementTracker SetElement(const Element& element);
    std::vector<ElementTracker> SetElements(const std::vector<Element>& elements);
    ElementTracker AllocateElement(const Element& e);
    void Simulate(float sim_duration, bool trackStresses = false, bool trace = false,
                  std::string tracefile = "trace.csv");
    void Devo();
    Element Collect(const ElementTracker& tracker);
    std::vector<Element> Collect(const std::vector<ElementTracker>& trackers);
    Element CollectElement(const ElementTracker& tracker);

    float getDeltaT() const { return m_deltaT; }
    void setTimeStep(float dt);
    float getTotalTime() const;
    void Reset();

    // Not in the reference: stresses of a robot's springs after Collect, the
    // step semantics (0 = the reference's XPBD step, 1 = force + land,
    // 2 = force + water; see include/mercury_b200.h), and the environment of
    // the force modes from the reference's Environment (g, floor stiffness,
    // friction as the kinetic coefficient; water: drag is the density of
    // the face drag on the elements' faces).
    std::vector<float> Stresses(const ElementTracker& tracker) const;
    void setMode(int mode);
    void setEnvironment(const Environment& env);

private:
    void upload();
    void download();

    mb_context* ctx_ = nullptr;
    float m_deltaT = 0.0001f;  // the reference's default before Initialize (Simulator.h:55)
    Config::Simulator m_config;
    std::vector<Element> elements_;
    std::vector<Mass> massBuf_;
    std::vector<Spring> springBuf_;
    std::vector<int64_t> massOff_, springOff_, faceOff_;
    std::vector<float> pos_, vel_, stress_, lbar_;
    std::vector<uint8_t> massMat_, springMat_;
    std::vector<uint16_t> pairs_, faces_;
    uint64_t devoSeed_ = 0;
};

#endif
