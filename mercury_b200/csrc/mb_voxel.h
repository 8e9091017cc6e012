// Voxel-lattice robots (mb_voxel.cpp host builder, mb_voxel_dev.cu device
// builder); internal to the library.
#pragma once
#include <cstdint>
#include <vector>

namespace mb {

// The material-independent part of a VoxelRobot on an nx x ny x nz point
// grid: masses at h * index shifted as ShiftX/ShiftY do, and the springs of
// the depth-first walk (VoxelRobot.cpp:60-193) with their mean lengths and
// the walk direction (index into the 13 forward directions) of each.
struct VoxelTemplate {
    int nx = 0, ny = 0, nz = 0;
    std::vector<float> pos;        // 3 per grid point
    std::vector<uint16_t> pairs;   // 2 per spring: source point, target point
    std::vector<float> lbar;
    std::vector<uint8_t> dir;
};

void voxel_template(int nx, int ny, int nz, float h, VoxelTemplate& t);

}  // namespace mb
