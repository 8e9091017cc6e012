// Voxel-lattice robot builder: the topology the reference's VoxelRobot
// produces (common/evolvables/VoxelRobot.cpp:60-193, 195-283, 310-331),
// written over flat arrays.
//
// Grid point i = x + y*nx + z*nx*ny carries a base material (0 = air); the
// material of grid point p is the material of the cell whose lowest corner
// is p.  Build:
//   1. keep the largest 6-connected component of non-air points (the first in
//      index order among equals), all other points become air (Strip);
//   2. one mass per grid point at h*(x, y, z);
//   3. a depth-first walk from point 0 emits one spring per point and valid
//      forward direction, in the walk's order, with the composite material of
//      the cells that share the edge and the initial length as mean length;
//   4. shift so that max x = 0 and min y = 0 (ShiftX, ShiftY).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/mercury_b200.h"
#include "mb_voxel.h"

namespace mb {

int composite_id(int m1, int m2);
int decode_id(uint32_t enc);

namespace {

struct Idx {
    int x, y, z;
};

struct Lattice {
    int nx, ny, nz;
    bool valid(Idx i) const {
        return i.x >= 0 && i.x < nx && i.y >= 0 && i.y < ny && i.z >= 0 && i.z < nz;
    }
    int id(Idx i) const { return i.x + i.y * nx + i.z * nx * ny; }
    Idx at(int v) const { return {v % nx, (v / nx) % ny, (v / nx / ny) % nz}; }
};

// The 13 forward directions in walk order (VoxelRobot.cpp:160-192).
const Idx kDirs[13] = {
    {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1},
    {1, -1, 0}, {0, 1, -1}, {-1, 0, 1},
    {-1, 1, 1}, {1, -1, 1}, {1, 1, -1},
};

inline Idx sub(Idx a, Idx b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Idx add(Idx a, Idx b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }

inline uint32_t enc(uint8_t m) { return 1u << m; }

// Material of the spring from src along path (VoxelRobot.cpp:72-147).
int edge_material(const Lattice& L, const std::vector<uint8_t>& mat, Idx src, Idx path) {
    const int man = std::abs(path.x) + std::abs(path.y) + std::abs(path.z);
    const uint8_t msrc = mat[L.id(src)];
    if (man == 1) {
        uint32_t e = 0;
        for (int i = 0; i < 4; ++i) {
            const int p = (i / 2) % 2, q = i % 2;
            Idx nprox = std::abs(path.x) == 1 ? Idx{0, p, q}
                      : std::abs(path.y) == 1 ? Idx{p, 0, q}
                                              : Idx{p, q, 0};
            Idx n = sub(src, nprox);
            if (!L.valid(n)) continue;
            const uint8_t mn = mat[L.id(n)];
            if (mn != 0) e |= enc(mn);
        }
        return decode_id(e);
    }
    if (man == 2) {
        const Idx nprox = {path.x == 0, path.y == 0, path.z == 0};
        Idx msrc_idx = src;
        if (!(path.x >= 0 && path.y >= 0 && path.z >= 0))
            msrc_idx = sub(src, Idx{path.x == -1, path.y == -1, path.z == -1});
        const uint8_t mm = mat[L.id(msrc_idx)];
        const Idx n = sub(msrc_idx, nprox);
        if (!L.valid(n)) return mm;
        uint32_t e = 0;
        const uint8_t mn = mat[L.id(n)];
        if (mn != 0) e |= enc(mn);
        if (mm != 0) e |= enc(mm);
        return decode_id(e);
    }
    // body diagonal
    if (path.x >= 0 && path.y >= 0 && path.z >= 0) return msrc;
    return mat[L.id(sub(src, Idx{path.x == -1, path.y == -1, path.z == -1}))];
}

// Largest 6-connected component of non-air points (VoxelRobot.cpp:195-283).
void strip(const Lattice& L, std::vector<uint8_t>& mat) {
    const int n = L.nx * L.ny * L.nz;
    std::vector<int> label(n, -1);
    std::vector<int> sizes;
    std::vector<int> stack;
    const Idx six[6] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    int best = -1, best_size = 0;
    for (int v = 0; v < n; ++v) {
        if (label[v] >= 0 || mat[v] == 0) continue;
        const int c = (int)sizes.size();
        int size = 0;
        stack.assign(1, v);
        label[v] = c;
        while (!stack.empty()) {
            const int u = stack.back();
            stack.pop_back();
            ++size;
            const Idx iu = L.at(u);
            for (const Idx& d : six) {
                const Idx w = add(iu, d);
                if (!L.valid(w)) continue;
                const int wi = L.id(w);
                if (label[wi] >= 0 || mat[wi] == 0) continue;
                label[wi] = c;
                stack.push_back(wi);
            }
        }
        sizes.push_back(size);
        if (size > best_size) {
            best_size = size;
            best = c;
        }
    }
    for (int v = 0; v < n; ++v)
        if (label[v] != best) mat[v] = 0;
}

}  // namespace

void voxel_template(int nx, int ny, int nz, float h, VoxelTemplate& t) {
    const Lattice L{nx, ny, nz};
    const int n = nx * ny * nz;
    t.nx = nx;
    t.ny = ny;
    t.nz = nz;
    // masses at h * index
    std::vector<float> px(n), py(n), pz(n);
    for (int v = 0; v < n; ++v) {
        const Idx i = L.at(v);
        px[v] = h * (float)i.x;
        py[v] = h * (float)i.y;
        pz[v] = h * (float)i.z;
    }
    // depth-first walk from point 0 (VoxelRobot.cpp:60-193), iterative; it
    // visits every grid point whatever the materials, so the springs, their
    // order and mean lengths depend on the grid size only
    t.pairs.clear();
    t.lbar.clear();
    t.dir.clear();
    std::vector<uint8_t> visited(n, 0);
    struct Frame {
        int v, k;
    };
    std::vector<Frame> stack;
    visited[0] = 1;
    stack.push_back({0, 0});
    while (!stack.empty()) {
        Frame& f = stack.back();
        if (f.k == 13) {
            stack.pop_back();
            continue;
        }
        const int k = f.k++;
        const int src = f.v;
        const Idx it = add(L.at(src), kDirs[k]);
        if (!L.valid(it)) continue;
        const int v = L.id(it);
        // mean length |base_src - base_v| as Eigen's norm(): d0^2 + (d1^2 + d2^2)
        const float d0 = px[src] - px[v], d1 = py[src] - py[v], d2 = pz[src] - pz[v];
        const float q12 = d1 * d1 + d2 * d2;
        const float len = std::sqrt(d0 * d0 + q12);
        t.pairs.push_back((uint16_t)src);
        t.pairs.push_back((uint16_t)v);
        t.lbar.push_back(len);
        t.dir.push_back((uint8_t)k);
        if (visited[v]) continue;
        visited[v] = 1;
        stack.push_back({v, 0});
    }
    // ShiftX then ShiftY (VoxelRobot.cpp:30-56): translate by -max x, then by
    // -min y, over all masses.
    float max_x = px[0];
    for (int v = 1; v < n; ++v)
        if (px[v] > max_x) max_x = px[v];
    const float tx = -max_x;
    for (int v = 0; v < n; ++v) px[v] = px[v] + tx;
    float min_y = py[0];
    for (int v = 1; v < n; ++v)
        if (py[v] < min_y) min_y = py[v];
    const float ty = -min_y;
    for (int v = 0; v < n; ++v) py[v] = py[v] + ty;
    t.pos.resize(3 * (size_t)n);
    for (int v = 0; v < n; ++v) {
        t.pos[3 * v] = px[v];
        t.pos[3 * v + 1] = py[v];
        t.pos[3 * v + 2] = pz[v];
    }
}

}  // namespace mb

extern "C" mb_status mb_voxel_build(int nx, int ny, int nz, float h, const uint8_t* mats,
                                    int* n_masses, int* n_springs, float* pos,
                                    uint8_t* mass_material, uint16_t* pairs, float* lbar,
                                    uint8_t* spring_material) {
    using namespace mb;
    if (nx <= 0 || ny <= 0 || nz <= 0 || !mats || !n_masses || !n_springs || !pos ||
        !mass_material || !pairs || !lbar || !spring_material)
        return MB_ERR_ARGUMENT;
    const long long n = (long long)nx * ny * nz;
    if (n > 65536) return MB_ERR_CAPACITY;  // uint16 mass indices (spring.h:9-10)
    for (long long i = 0; i < n; ++i)
        if (mats[i] > 22) return MB_ERR_ARGUMENT;
    const Lattice L{nx, ny, nz};
    std::vector<uint8_t> mat(mats, mats + n);
    strip(L, mat);
    VoxelTemplate t;
    voxel_template(nx, ny, nz, h, t);
    const int ns = (int)t.lbar.size();
    for (int s = 0; s < ns; ++s) {
        pairs[2 * s] = t.pairs[2 * s];
        pairs[2 * s + 1] = t.pairs[2 * s + 1];
        lbar[s] = t.lbar[s];
        spring_material[s] = (uint8_t)edge_material(L, mat, L.at(t.pairs[2 * s]), kDirs[t.dir[s]]);
    }
    for (long long v = 0; v < n; ++v) {
        pos[3 * v] = t.pos[3 * v];
        pos[3 * v + 1] = t.pos[3 * v + 1];
        pos[3 * v + 2] = t.pos[3 * v + 2];
        mass_material[v] = mat[v];
    }
    *n_masses = (int)n;
    *n_springs = ns;
    return MB_OK;
}
