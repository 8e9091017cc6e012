// Device development step (mb_devo.cu); internal to the library.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mb {

constexpr uint32_t kDevoMaxReplaced = 1024;   // springs replaced per robot and call
constexpr uint32_t kDevoReferenceRanks = 1u;  // rank window [r k, r k + k) of robot r

// One replaced spring: global spring index (0xFFFFFFFF = unused record),
// the new pair (a | b << 16, robot-local), composite material, mean length.
struct DevoRecord {
    uint32_t spring;
    uint32_t pair;
    uint32_t material;
    float lbar;
};

struct DevoParams {
    const float* stress;       // per spring, upload order
    const int64_t* mass_off;   // n_robots + 1
    const int64_t* spring_off; // n_robots + 1
    const float4* pos;         // upload order
    const uint8_t* mass_mat;   // upload order
    const float4* table;       // composite material table (k, dL0, omega, phi)
    float t;                   // clock of the mean lengths
    uint32_t k;                // springs replaced per robot (<= kDevoMaxReplaced)
    uint64_t seed;
    uint32_t flags;
    DevoRecord* out;           // n_robots * k records, rank order per robot
};

cudaError_t launch_devo(const DevoParams& p, uint32_t n_robots, cudaStream_t s);

}  // namespace mb
