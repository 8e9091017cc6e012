// Device builder of voxel robot populations (mb_voxel_dev.cu); internal.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mb_devo.h"
#include "mb_internal.h"

namespace mb {

constexpr uint32_t kVoxelMaxPoints = 4096;  // grid points per robot (12-bit bin-local indices)

struct VoxelBuildParams {
    uint32_t n_robots;
    int sx, sy, sz;               // cells per axis; points are cells + 1 per axis
    const uint8_t* cells;         // n_robots * sx*sy*sz base material ids, x fastest
    const float* tmpl_pos;        // 3 per grid point
    const uint16_t* tmpl_src;     // per template spring: source grid point
    const uint8_t* tmpl_dir;      // per template spring: walk direction (0..12)
    uint32_t n_tmpl_springs;
    float mass;                   // per mass
    float4* pos;                  // upload layout: robot r's points from r * points
    float4* vel;
    uint8_t* mass_mat;
    uint8_t* spring_mat;          // robot r's springs from r * n_tmpl_springs
    float* stress;
    uint32_t* status;             // [0] problems (material ids above 22)
};

struct CompactParams {
    BinDesc* bins;
    uint32_t n_bins;
    const uint32_t* tmpl_n_spring;  // per bin: packed springs of the template (all active)
    const uint32_t* tmpl_word;      // template packed words a | b << 12 (no material slot)
    const float* tmpl_lbar;
    const uint32_t* tmpl_gidx;
    const uint8_t* spring_mat;      // upload layout
    const uint8_t* slot_of;         // composite id -> material slot
    uint32_t* spring_pair;          // packed arrays written
    float* spring_lbar;
    uint32_t* spring_gidx;
    uint32_t* status;               // [0] problems (no material slot)
};

cudaError_t launch_voxel_build(const VoxelBuildParams& p, cudaStream_t s);
cudaError_t launch_compact(const CompactParams& p, cudaStream_t s);

}  // namespace mb
