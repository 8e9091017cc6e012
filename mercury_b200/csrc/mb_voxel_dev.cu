// Voxel robots built on the device from cell grids (mb_set_voxel_population).
//
// A VoxelRobot on a fixed point grid has the same masses, springs, spring
// order and mean lengths whatever its materials (VoxelRobot.cpp:60-193: the
// depth-first walk visits every grid point); materials decide only
//   - which points stay non-air: the largest 6-connected component of
//     non-air points, the first in index order among equals
//     (VoxelRobot.cpp:195-283), the rest become air, and
//   - each spring's material, from the cells that share its edge
//     (VoxelRobot.cpp:72-147).
// So a population of genomes on one grid is packed once (every spring
// active); per upload, build_kernel computes the materials of every robot
// (one CTA each), and compact_kernel drops the springs that are air from
// each bin's packed list (one CTA per bin, order kept), after which the rows
// are rebuilt by the development re-pack kernel.
#include "mb_voxel_dev.h"

namespace mb {
namespace {

constexpr uint32_t kBuildThreads = 256;
constexpr uint32_t kCompactThreads = 1024;

__device__ const int8_t kDir[13][3] = {
    {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1},
    {1, -1, 0}, {0, 1, -1}, {-1, 0, 1},
    {-1, 1, 1}, {1, -1, 1}, {1, 1, -1},
};

__device__ __forceinline__ int composite_dev(int m1, int m2) {
    if (m1 == 0 || m2 == 0) return 0;
    const int i = min(m1, m2) - 1, j = max(m1, m2) - 1;
    if (i == j) return i + 1;
    return 23 + i * 21 - i * (i - 1) / 2 + (j - i - 1);
}

// materials::decode(encoding).id (material.h:275-322)
__device__ __forceinline__ int decode_dev(uint32_t e) {
    if (e == 0 || (e & 1u)) return 0;
    const int i0 = __ffs(e) - 1;
    const uint32_t rest = e & (e - 1);
    if (!rest) return i0;
    return composite_dev(i0, __ffs(rest) - 1);
}

struct Grid {
    int nx, ny, nz;
    __device__ bool valid(int x, int y, int z) const {
        return x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz;
    }
    __device__ int id(int x, int y, int z) const { return x + y * nx + z * nx * ny; }
};

// Material of the spring from point (x, y, z) along direction k
// (VoxelRobot.cpp:72-147).
__device__ int edge_material_dev(const Grid& g, const uint8_t* pm, int x, int y, int z, int k) {
    const int px = kDir[k][0], py = kDir[k][1], pz = kDir[k][2];
    const int man = abs(px) + abs(py) + abs(pz);
    if (man == 1) {
        uint32_t e = 0;
        for (int i = 0; i < 4; ++i) {
            const int p = (i / 2) % 2, q = i % 2;
            int ox, oy, oz;
            if (abs(px) == 1) {
                ox = 0; oy = p; oz = q;
            } else if (abs(py) == 1) {
                ox = p; oy = 0; oz = q;
            } else {
                ox = p; oy = q; oz = 0;
            }
            const int nx = x - ox, ny = y - oy, nz = z - oz;
            if (!g.valid(nx, ny, nz)) continue;
            const uint8_t mn = pm[g.id(nx, ny, nz)];
            if (mn) e |= 1u << mn;
        }
        return decode_dev(e);
    }
    if (man == 2) {
        const int ox = px == 0, oy = py == 0, oz = pz == 0;
        int sx = x, sy = y, sz = z;
        if (!(px >= 0 && py >= 0 && pz >= 0)) {
            sx -= px == -1;
            sy -= py == -1;
            sz -= pz == -1;
        }
        const uint8_t mm = pm[g.id(sx, sy, sz)];
        const int nx = sx - ox, ny = sy - oy, nz = sz - oz;
        if (!g.valid(nx, ny, nz)) return mm;
        uint32_t e = 0;
        const uint8_t mn = pm[g.id(nx, ny, nz)];
        if (mn) e |= 1u << mn;
        if (mm) e |= 1u << mm;
        return decode_dev(e);
    }
    if (px >= 0 && py >= 0 && pz >= 0) return pm[g.id(x, y, z)];
    return pm[g.id(x - (px == -1), y - (py == -1), z - (pz == -1))];
}

__global__ void __launch_bounds__(kBuildThreads) build_kernel(const VoxelBuildParams p) {
    __shared__ uint8_t pm[kVoxelMaxPoints];
    __shared__ uint32_t label[kVoxelMaxPoints];
    __shared__ uint32_t cnt[kVoxelMaxPoints];
    __shared__ uint32_t best_key;
    const uint32_t r = blockIdx.x, tid = threadIdx.x;
    const Grid g{p.sx + 1, p.sy + 1, p.sz + 1};
    const uint32_t n = (uint32_t)(g.nx * g.ny * g.nz);
    const uint8_t* cells = p.cells + (size_t)r * p.sx * p.sy * p.sz;
    // point materials: point (x, y, z) carries cell (x, y, z); the upper
    // faces are air
    for (uint32_t v = tid; v < n; v += kBuildThreads) {
        const int x = v % g.nx, y = (v / g.nx) % g.ny, z = v / (g.nx * g.ny);
        uint8_t m = 0;
        if (x < p.sx && y < p.sy && z < p.sz) m = cells[x + y * p.sx + z * p.sx * p.sy];
        if (m > 22) {
            atomicAdd(&p.status[0], 1u);
            m = 0;
        }
        pm[v] = m;
        label[v] = m ? v : 0xFFFFFFFFu;
        cnt[v] = 0;
    }
    if (tid == 0) best_key = 0;
    __syncthreads();
    // components: labels fall to the smallest index of the component
    for (uint32_t it = 0; it <= n; ++it) {
        int mine = 0;
        for (uint32_t v = tid; v < n; v += kBuildThreads) {
            if (!pm[v]) continue;
            const int x = v % g.nx, y = (v / g.nx) % g.ny, z = v / (g.nx * g.ny);
            uint32_t m = label[v];
            const int nb[6][3] = {{x + 1, y, z}, {x - 1, y, z}, {x, y + 1, z},
                                  {x, y - 1, z}, {x, y, z + 1}, {x, y, z - 1}};
            for (int d = 0; d < 6; ++d) {
                if (!g.valid(nb[d][0], nb[d][1], nb[d][2])) continue;
                const uint32_t q = (uint32_t)g.id(nb[d][0], nb[d][1], nb[d][2]);
                if (pm[q]) m = min(m, label[q]);
            }
            m = min(m, label[m]);  // pointer jump
            if (m < label[v]) {
                label[v] = m;
                mine = 1;
            }
        }
        if (!__syncthreads_or(mine)) break;
    }
    // largest component, the smallest label among equals
    for (uint32_t v = tid; v < n; v += kBuildThreads)
        if (pm[v]) atomicAdd(&cnt[label[v]], 1u);
    __syncthreads();
    for (uint32_t v = tid; v < n; v += kBuildThreads)
        if (cnt[v]) atomicMax(&best_key, (cnt[v] << 12) | (kVoxelMaxPoints - 1 - v));
    __syncthreads();
    const uint32_t best = best_key ? kVoxelMaxPoints - 1 - (best_key & (kVoxelMaxPoints - 1)) : 0xFFFFFFFFu;
    for (uint32_t v = tid; v < n; v += kBuildThreads)
        if (pm[v] && label[v] != best) pm[v] = 0;
    __syncthreads();
    // masses
    const size_t m0 = (size_t)r * n;
    for (uint32_t v = tid; v < n; v += kBuildThreads) {
        p.mass_mat[m0 + v] = pm[v];
        p.pos[m0 + v] = make_float4(p.tmpl_pos[3 * v], p.tmpl_pos[3 * v + 1], p.tmpl_pos[3 * v + 2], p.mass);
        p.vel[m0 + v] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    // springs
    const size_t s0 = (size_t)r * p.n_tmpl_springs;
    for (uint32_t s = tid; s < p.n_tmpl_springs; s += kBuildThreads) {
        const int v = p.tmpl_src[s];
        const int x = v % g.nx, y = (v / g.nx) % g.ny, z = v / (g.nx * g.ny);
        p.spring_mat[s0 + s] = (uint8_t)edge_material_dev(g, pm, x, y, z, p.tmpl_dir[s]);
        p.stress[s0 + s] = 0.0f;
    }
}

__global__ void __launch_bounds__(kCompactThreads) compact_kernel(const CompactParams p) {
    __shared__ uint32_t warp_cnt[kCompactThreads / 32];
    __shared__ uint32_t s_base;
    const uint32_t b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t first = p.bins[b].spring_begin, nt = p.tmpl_n_spring[b];
    if (tid == 0) s_base = 0;
    __syncthreads();
    for (uint32_t c = 0; c < nt; c += kCompactThreads) {
        const uint32_t j = c + tid;
        uint32_t word = 0, g = 0, mat = 0;
        float lb = 0.0f;
        if (j < nt) {
            g = p.tmpl_gidx[first + j];
            mat = p.spring_mat[g];
            word = p.tmpl_word[first + j];
            lb = p.tmpl_lbar[first + j];
        }
        const bool active = j < nt && mat != 0;
        const uint32_t bal = __ballot_sync(0xffffffffu, active);
        if (lane == 0) warp_cnt[warp] = __popc(bal);
        __syncthreads();
        uint32_t before = s_base;
        for (uint32_t w = 0; w < warp; ++w) before += warp_cnt[w];
        before += __popc(bal & ((1u << lane) - 1u));
        if (active) {
            const uint32_t slot = p.slot_of[mat];
            if (slot == kNoMatSlot) atomicAdd(&p.status[0], 1u);
            p.spring_pair[first + before] = word | ((slot & 0xFFu) << 24);
            p.spring_lbar[first + before] = lb;
            p.spring_gidx[first + before] = g;
        }
        __syncthreads();
        if (tid == 0) {
            uint32_t t = 0;
            for (uint32_t w = 0; w < kCompactThreads / 32; ++w) t += warp_cnt[w];
            s_base += t;
        }
        __syncthreads();
    }
    if (tid == 0) p.bins[b].n_spring = s_base;
}

}  // namespace

cudaError_t launch_voxel_build(const VoxelBuildParams& p, cudaStream_t s) {
    if (p.n_robots == 0) return cudaSuccess;
    build_kernel<<<p.n_robots, kBuildThreads, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_compact(const CompactParams& p, cudaStream_t s) {
    if (p.n_bins == 0) return cudaSuccess;
    compact_kernel<<<p.n_bins, kCompactThreads, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace mb
