// Step kernels of the batched soft-body simulator (sm_100a).
//
// The reference step (common/simulator/sim_kernel.cu:141-269) launches four
// kernels per step and re-stages every robot through shared memory each
// time, accumulating the spring corrections with shared-memory float
// atomics.  Here one CTA simulates one "bin" (a group of whole robots) for a
// whole chunk of steps without leaving the SM:
//
//   registers : each thread's springs (packed pair + material slot, mean
//               length, optional 1/length and stress) and masses (x, v);
//   shared    : predicted positions x~ (SoA), per-spring corrections dp
//               (SoA), the bin's incidence lists (SELL-32), and the per-step
//               actuation factors and 1/K of the bin's materials.
//
// Per step: (1) warp 0 evaluates the actuation factor dL0*sin(omega*t+phi)
// of each material of the bin; every thread predicts x~ = x + v*dt for its
// masses; barrier.  (2) every thread solves its springs (XPBD distance
// constraint, sim_kernel.cu:209-243) and stores dp per spring; barrier.
// (3) every thread gathers, for each of its masses, the corrections of the
// incident springs in a fixed order from its SELL row (no atomics), then
// integrates x and v (sim_kernel.cu:246-252, 261-268).
//
// All arithmetic uses explicit round-to-nearest intrinsics so that the
// result is bit-identical to the CPU restatement in the oracle.
#include <cooperative_groups.h>

#include "mb_internal.h"
#include "mb_sin.cuh"

namespace mb {

namespace cg = cooperative_groups;

namespace {

constexpr float kEps = 1e-12f;  // sim_kernel.cu:6

// Packed spring word: a (12 bits) | b << 12 (12 bits) | slot << 24 (8 bits).
__device__ __forceinline__ uint32_t pk_a(uint32_t w) { return w & 0xFFFu; }
__device__ __forceinline__ uint32_t pk_b(uint32_t w) { return (w >> 12) & 0xFFFu; }
__device__ __forceinline__ uint32_t pk_slot(uint32_t w) { return w >> 24; }

// Force modes, per mass, after the spring forces (fx, fy, fz) are gathered:
// environment forces, then x' = x + v dt + (F/m) dt^2, v' = damping (x' - x)/dt.
//   land : gravity -m g along z; below z = 0 a penalty normal force
//          fn = k_floor (-z) and Coulomb friction on the horizontal velocity
//          h = v + (F_h/m) dt the step would reach: static (the friction force
//          cancels the horizontal motion, F_h = -m v_h/dt) when |h| <= mu_s fn
//          dt/m, else kinetic, mu_k fn against h.
//   water: gravity balanced by buoyancy; quadratic drag -drag |v| v.
// Divisions by m and dt are multiplications by the correctly rounded
// reciprocals (inv_dt = RN(1/dt) per launch, RN(1/m) per mass and step);
// only the kinetic friction divides.
template <int MODE>
__device__ __forceinline__ void force_integrate(const StepParams& p, float3& x, float3& v, float m,
                                                float inv_dt, float fx, float fy, float fz) {
    const float dt = p.dt;
    const float inv_m = __frcp_rn(m);
    if (MODE == kModeForceLand) {
        fz = __fsub_rn(fz, __fmul_rn(m, p.g));
        if (x.z < 0.0f) {
            const float fn = __fmul_rn(p.floor_stiffness, -x.z);
            fz = __fadd_rn(fz, fn);
            const float hx = __fadd_rn(v.x, __fmul_rn(__fmul_rn(fx, inv_m), dt));
            const float hy = __fadd_rn(v.y, __fmul_rn(__fmul_rn(fy, inv_m), dt));
            const float hs = __fsqrt_rn(__fmaf_rn(hx, hx, __fmul_rn(hy, hy)));
            const float budget = __fmul_rn(__fmul_rn(fn, inv_m), dt);
            if (hs <= __fmul_rn(p.mu_s, budget)) {
                fx = __fmul_rn(__fmul_rn(-m, v.x), inv_dt);
                fy = __fmul_rn(__fmul_rn(-m, v.y), inv_dt);
            } else {
                const float s = __fdiv_rn(__fmul_rn(p.mu_k, fn), hs);
                fx = __fsub_rn(fx, __fmul_rn(s, hx));
                fy = __fsub_rn(fy, __fmul_rn(s, hy));
            }
        }
    } else {
        const float sp = __fsqrt_rn(__fmaf_rn(v.x, v.x, __fmaf_rn(v.y, v.y, __fmul_rn(v.z, v.z))));
        const float c = __fmul_rn(p.drag, sp);
        fx = __fsub_rn(fx, __fmul_rn(c, v.x));
        fy = __fsub_rn(fy, __fmul_rn(c, v.y));
        fz = __fsub_rn(fz, __fmul_rn(c, v.z));
    }
    const float dt2 = __fmul_rn(dt, dt);
    const float nx = __fadd_rn(__fadd_rn(x.x, __fmul_rn(v.x, dt)), __fmul_rn(__fmul_rn(fx, inv_m), dt2));
    const float ny = __fadd_rn(__fadd_rn(x.y, __fmul_rn(v.y, dt)), __fmul_rn(__fmul_rn(fy, inv_m), dt2));
    const float nz = __fadd_rn(__fadd_rn(x.z, __fmul_rn(v.z, dt)), __fmul_rn(__fmul_rn(fz, inv_m), dt2));
    v.x = __fmul_rn(p.damping, __fmul_rn(__fsub_rn(nx, x.x), inv_dt));
    v.y = __fmul_rn(p.damping, __fmul_rn(__fsub_rn(ny, x.y), inv_dt));
    v.z = __fmul_rn(p.damping, __fmul_rn(__fsub_rn(nz, x.z), inv_dt));
    x = make_float3(nx, ny, nz);
}

// Velocity of the reference step, v = (float)(0.99 * (double)delta / (double)dt)
// (sim_kernel.cu:265-267): the double product, the correctly rounded double
// quotient, then rounding to float -- without a double division in the
// common case.  q = RN(a * inv_dt), with inv_dt = RN(1/dt), differs from
// the exact a/dt by at most 2u + u^2 relative (u = 2^-53), so from the
// correctly rounded quotient by less than 3.01 units in the last place of
// q.  Rounding to float can only differ between q and that quotient if a
// float rounding boundary -- the midpoint between two floats, whose low 29
// significand bits are 1 << 28 in double -- lies between them.  So when
// q's low 29 bits are more than 4 units from 1 << 28 and q lies in the
// normal float range, (float)q is the result (Ziv's rounding test: Ziv,
// "Fast evaluation of elementary mathematical functions with correctly
// rounded last bit", ACM TOMS 17(3), 1991); otherwise -- about 9 inputs in
// 2^29, zeros excepted -- the division itself is done.
__device__ __forceinline__ float velocity_of(float delta, double dt, double inv_dt) {
    const double a = __dmul_rn(0.99, (double)delta);
    const double q = __dmul_rn(a, inv_dt);
    const unsigned long long bits = (unsigned long long)__double_as_longlong(q);
    const uint32_t e = (uint32_t)(bits >> 52) & 0x7FFu;
    const uint32_t low29 = (uint32_t)bits & 0x1FFFFFFFu;
    // normal float range 2^-126 <= |q| < 2^127 (biased double exponents 897..1149)
    const bool clear = (e - 897u) < 253u && (low29 - (0x10000000u - 4u)) > 8u;
    if (clear || (bits << 1) == 0) return __double2float_rn(q);
    return __double2float_rn(__ddiv_rn(a, dt));
}

// Face drag of one surface triangle (water), the share of each corner:
// mean corner velocity v = (v0 + v1 + v2) * RN(1/3), N = (x1 - x0) x (x2 - x0), A = |N|, unit normal
// n = N * RN(1/(A + eps)) turned so that v.n > 0 (sim_kernel.cu:106-109),
// force coef * A * ((v.n) v + 0.2 |v|^2 n) with coef = -rho/6, i.e.
// -rho/2 A (...) / 3 (sim_kernel.cu:110-111).  Every operation rounds once,
// in this order.
__device__ __forceinline__ float4 face_force(const float4 x0, const float4 x1, const float4 x2, const float4 v0,
                                             const float4 v1, const float4 v2, const float coef) {
    constexpr float kThird = 0x1.555556p-2f;  // 1/3 rounded to nearest
    const float vx = __fmul_rn(__fadd_rn(__fadd_rn(v0.x, v1.x), v2.x), kThird);
    const float vy = __fmul_rn(__fadd_rn(__fadd_rn(v0.y, v1.y), v2.y), kThird);
    const float vz = __fmul_rn(__fadd_rn(__fadd_rn(v0.z, v1.z), v2.z), kThird);
    const float ax = __fsub_rn(x1.x, x0.x), ay = __fsub_rn(x1.y, x0.y), az = __fsub_rn(x1.z, x0.z);
    const float bx = __fsub_rn(x2.x, x0.x), by = __fsub_rn(x2.y, x0.y), bz = __fsub_rn(x2.z, x0.z);
    const float nx = __fsub_rn(__fmul_rn(ay, bz), __fmul_rn(az, by));
    const float ny = __fsub_rn(__fmul_rn(az, bx), __fmul_rn(ax, bz));
    const float nz = __fsub_rn(__fmul_rn(ax, by), __fmul_rn(ay, bx));
    const float area = __fsqrt_rn(__fmaf_rn(nx, nx, __fmaf_rn(ny, ny, __fmul_rn(nz, nz))));
    const float r = __frcp_rn(__fadd_rn(area, kEps));
    float ux = __fmul_rn(nx, r), uy = __fmul_rn(ny, r), uz = __fmul_rn(nz, r);
    float vn = __fmaf_rn(ux, vx, __fmaf_rn(uy, vy, __fmul_rn(uz, vz)));
    if (!(vn > 0.0f)) {  // negating n negates the rounded dot product exactly
        ux = -ux;
        uy = -uy;
        uz = -uz;
        vn = -vn;
    }
    const float lift = __fmul_rn(0.2f, __fmaf_rn(vx, vx, __fmaf_rn(vy, vy, __fmul_rn(vz, vz))));
    const float c = __fmul_rn(coef, area);
    return make_float4(__fmul_rn(c, __fmaf_rn(lift, ux, __fmul_rn(vn, vx))),
                       __fmul_rn(c, __fmaf_rn(lift, uy, __fmul_rn(vn, vy))),
                       __fmul_rn(c, __fmaf_rn(lift, uz, __fmul_rn(vn, vz))), 0.0f);
}

// RW > 0 (register rows): each thread's row of up to RW entries is kept in
// registers (two 16-bit entries per register, loaded once per bin), so that
// the gather's correction loads no longer wait on a row-entry load and
// issue RG at a time; a slice wider than RW reads its row from global
// memory.  The rows are not staged in shared memory; to make room, the
// springs leave the registers for {packed word, mean length} pairs in
// shared memory where the rows would start (8 bytes per spring in place of
// 2 per row entry).  One mass per thread (MPT = 1), no face drag.  Same
// operations in the same order: same bits.  Resident bins only: on the
// parts of split robots it measured slower.
template <int T, int SPT, int MPT, int MODE, bool TRACK, bool SPLIT, int RW = 0>
__global__ void __launch_bounds__(T, 1024 / T) step_kernel(const StepParams p) {
    constexpr bool XPBD = MODE == kModeXpbd;
    constexpr bool FACES = MODE == kModeForceWaterFaces;  // face drag compiled in
    constexpr int RG = 2;  // correction loads in flight per group
    static_assert(RW == 0 || (MPT == 1 && !SPLIT && !FACES && RW % RG == 0), "register rows: one mass per thread");
    extern __shared__ float4 smem4[];
    const int tid = threadIdx.x;
    const float dt = p.dt;
    const double ddt = (double)dt;
    const double inv_dt = __drcp_rn(ddt);
    const float inv_dt_f = __frcp_rn(dt);

    for (uint32_t b = blockIdx.x; b < p.n_bins; b += gridDim.x) {
        const BinDesc bd = p.bins[b];
        // predicted positions x~, one float4 per mass (split bins: two
        // buffers, own masses then halo, alternating by step; with faces,
        // two velocity buffers of the same shape follow)
        float4* sxt = smem4;
        float4* sdp = sxt + (SPLIT ? (FACES ? 4u : 2u) * bd.x_stride : bd.n_mass);  // corrections dp, one float4 per spring
        float2* smat = reinterpret_cast<float2*>(sdp + bd.n_spring);  // {dL0 sin(..), 1/K} per slot
        // split bins: the buffer stride of every part of the cluster, then
        // the export list
        uint32_t* sstride = reinterpret_cast<uint32_t*>(smat + kMaxMaterialSlots);
        uint32_t* sexp = sstride + (SPLIT ? kMaxClusterParts : 0u);
        uint16_t* sinc = reinterpret_cast<uint16_t*>(sexp + (SPLIT ? bd.n_export : 0u));
        // face drag (water, bins with faces), after the rows at a 16-byte
        // boundary: velocities (resident bins; split bins keep them after
        // the positions), face forces, corners, face rows (first entry |
        // count << 24), incidence
        const uint32_t n_face = FACES && p.face_on ? bd.n_face : 0u;
        float4* sv = reinterpret_cast<float4*>((reinterpret_cast<uintptr_t>(sinc + bd.n_inc) + 15u) & ~uintptr_t(15));
        float4* sfd = SPLIT ? sv : sv + bd.n_mass;
        if (SPLIT) sv = sxt + 2u * bd.x_stride;
        uint2* sface = reinterpret_cast<uint2*>(sfd + n_face);
        uint32_t* sfrow = reinterpret_cast<uint32_t*>(sface + n_face);
        uint16_t* sfinc = reinterpret_cast<uint16_t*>(sfrow + bd.n_mass);

        const uint32_t n_mat = *p.n_mat;
        // register rows: the rows are not staged in shared memory; the springs
        // leave the registers to make room, into {packed word, mean length}
        // pairs where the rows would start (8-byte aligned)
        uint2* ssl = reinterpret_cast<uint2*>((reinterpret_cast<uintptr_t>(sinc) + 7u) & ~uintptr_t(7));
        if (RW > 0) {
            // the host sizes the launch for every bin; a bin that would still
            // not fit is skipped and flagged (bit 1) rather than overrun
            uint32_t dyn;
            asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
            if (reinterpret_cast<const char*>(ssl + bd.n_spring) - reinterpret_cast<const char*>(smem4) > dyn) {
                if (tid == 0) atomicOr(&p.bin_flags[b], 2u);
                continue;
            }
        }
        if (RW > 0)
            for (uint32_t i = tid; i < bd.n_spring; i += T)
                ssl[i] = make_uint2(__ldg(&p.spring_pair[bd.spring_begin + i]),
                                    __float_as_uint(__ldg(&p.spring_lbar[bd.spring_begin + i])));
        else
            for (uint32_t i = tid; i < bd.n_inc; i += T) sinc[i] = __ldg(&p.inc[bd.inc_begin + i]);
        if (n_face) {
            for (uint32_t i = tid; i < n_face; i += T) sface[i] = __ldg(&p.faces[bd.face_begin + i]);
            for (uint32_t i = tid; i < bd.n_mass; i += T) sfrow[i] = __ldg(&p.face_row[bd.mass_begin + i]);
            for (uint32_t i = tid; i < bd.n_face_inc; i += T) sfinc[i] = __ldg(&p.face_inc[bd.face_inc_begin + i]);
        }
        if (SPLIT) {
            for (uint32_t i = tid; i < bd.n_export; i += T) sexp[i] = __ldg(&p.exports[bd.export_begin + i]);
            const cg::cluster_group cl = cg::this_cluster();
            if (tid < cl.num_blocks()) sstride[tid] = p.bins[b - cl.block_rank() + tid].x_stride;
        }
        float next_rate = 0.0f;  // actuation factor of material tid for the coming step
        if (tid < n_mat) {
            smat[tid].y = __ldg(&p.invk[tid]);  // 1/K (reference step) or k (force modes)
            next_rate = __ldg(&p.rates[tid]);
        }

        // Springs of this thread: packed word and mean length (+ stress).
        uint32_t sw[SPT];
        float lb[SPT], st[SPT];
#pragma unroll
        for (int j = 0; j < SPT; ++j) {
            const uint32_t s = tid + j * T;
            sw[j] = 0;
            lb[j] = 0.0f;
            st[j] = 0.0f;
            if (s < bd.n_spring) {
                const uint32_t g = bd.spring_begin + s;
                if (RW == 0) {
                    sw[j] = __ldg(&p.spring_pair[g]);
                    lb[j] = __ldg(&p.spring_lbar[g]);
                }
                if (TRACK) st[j] = p.stress[__ldg(&p.spring_gidx[g]) & 0x7FFFFFFFu];
            }
        }
        // Masses of this thread: x, v, mass and the SELL row (offset | width << 20).
        float3 x[MPT], v[MPT];
        float mass[MPT];
        uint32_t row[MPT];
#pragma unroll
        for (int j = 0; j < MPT; ++j) {
            const uint32_t m = tid + j * T;
            x[j] = make_float3(0.f, 0.f, 0.f);
            v[j] = make_float3(0.f, 0.f, 0.f);
            row[j] = 0;
            mass[j] = 1.0f;
            if (m < bd.n_mass) {
                const uint32_t g = __ldg(&p.mass_gidx[bd.mass_begin + m]);
                const float4 P = p.pos[g], V = p.vel[g];
                x[j] = make_float3(P.x, P.y, P.z);
                mass[j] = P.w;
                v[j] = make_float3(V.x, V.y, V.z);
                const uint32_t sl = bd.slice_begin + m / kSliceWidth;
                row[j] = (__ldg(&p.slice_off[sl]) + (m % kSliceWidth)) | (__ldg(&p.slice_width[sl]) << 20);
            }
        }
        // register rows: entry k of this thread's mass in half k & 1 of rr[k / 2]
        uint32_t rr[RW > 0 ? RW / 2 : 1];
        if constexpr (RW > 0) {
            const uint32_t w = row[0] >> 20;
            const uint16_t* gp = p.inc + bd.inc_begin + (row[0] & 0xFFFFFu);
#pragma unroll
            for (int k = 0; k < RW; k += 2) {
                const uint32_t lo = (uint32_t)k < w ? (uint32_t)__ldg(gp + k * kSliceWidth) : kPadEntry;
                const uint32_t hi = (uint32_t)k + 1u < w ? (uint32_t)__ldg(gp + (k + 1) * kSliceWidth) : kPadEntry;
                rr[k / 2] = lo | hi << 16;
            }
        }
        if (SPLIT)
            cg::this_cluster().sync();  // every part of the robot has started
        else
            __syncthreads();

        for (uint32_t step = 0; step < p.steps; ++step) {
            float4* X = SPLIT ? sxt + (step & 1u) * bd.x_stride : sxt;
            float4* V = SPLIT ? sv + (step & 1u) * bd.x_stride : sv;  // velocities (face drag)
            // (1) actuation factors of this step (sim_kernel.cu:222), loaded one
            // step ahead from the launch's table
            if (tid < n_mat) {
                smat[tid].x = next_rate;
                if (step + 1 < p.steps) next_rate = __ldg(&p.rates[(step + 1) * n_mat + tid]);
            }
            // (1) reference step: predict x~ = x + v*dt (sim_kernel.cu:147-152);
            //     force modes: publish the current positions
#pragma unroll
            for (int j = 0; j < MPT; ++j) {
                const uint32_t m = tid + j * T;
                if (m >= bd.n_mass) break;
                if (XPBD)
                    X[m] = make_float4(__fadd_rn(x[j].x, __fmul_rn(v[j].x, dt)),
                                       __fadd_rn(x[j].y, __fmul_rn(v[j].y, dt)),
                                       __fadd_rn(x[j].z, __fmul_rn(v[j].z, dt)), 0.0f);
                else
                    X[m] = make_float4(x[j].x, x[j].y, x[j].z, 0.0f);
                // split bins publish every velocity: other parts' faces may
                // have corners here
                if (FACES && (SPLIT || n_face)) V[m] = make_float4(v[j].x, v[j].y, v[j].z, 0.0f);
            }
            __syncthreads();
            if (SPLIT) {
                // masses the other parts hold as halo, into their buffer of
                // this step (at the part's own stride); the cluster barrier
                // makes them visible.  A part is at most one step ahead of
                // another, so the other buffer is never read meanwhile.
                cg::cluster_group cl = cg::this_cluster();
                for (uint32_t i = tid; i < bd.n_export; i += T) {
                    const uint32_t ex = sexp[i], q = (ex >> 12) & 7u;
                    float4* dst = cl.map_shared_rank(sxt, q) + (step & 1u) * sstride[q];
                    dst[ex >> 15] = X[ex & 0xFFFu];
                    if (FACES) dst[2u * sstride[q] + (ex >> 15)] = V[ex & 0xFFFu];  // the velocity buffer
                }
                cl.sync();
            }
            // (2) distance constraints (sim_kernel.cu:209-243)
#pragma unroll
            for (int j = 0; j < SPT; ++j) {
                const uint32_t s = tid + j * T;
                if (s >= bd.n_spring) break;
                const uint2 q = RW > 0 ? ssl[s] : make_uint2(sw[j], __float_as_uint(lb[j]));
                const uint32_t wj = q.x;
                const float4 pa = X[pk_a(wj)], pb = X[pk_b(wj)];
                const float2 mt = smat[pk_slot(wj)];
                const float lbj = __uint_as_float(q.y);
                const float L = __fmaf_rn(lbj, mt.x, lbj);
                const float dx = __fsub_rn(pa.x, pb.x);
                const float dy = __fsub_rn(pa.y, pb.y);
                const float dz = __fsub_rn(pa.z, pb.z);
                const float d = __fsqrt_rn(__fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz))));
                const float r = __frcp_rn(__fadd_rn(d, kEps));
                // reference step: lambda = -C/K, dp = lambda n (sim_kernel.cu:230-232);
                // force modes: Hooke force on the a end, -k (d - L) n
                const float lam = __fmul_rn(-__fsub_rn(d, L), mt.y);
                const float coef = __fmul_rn(lam, r);
                sdp[s] = make_float4(__fmul_rn(coef, dx), __fmul_rn(coef, dy), __fmul_rn(coef, dz), 0.0f);
                // stress: lambda/Lbar (reference, sim_kernel.cu:234); k (d - L)/Lbar (force)
                if (TRACK) st[j] = __fadd_rn(st[j], __fmul_rn(XPBD ? lam : -lam, __frcp_rn(lbj)));
            }
            // face drag: the share of each corner, per face
            for (uint32_t f = tid; f < n_face; f += T) {
                const uint2 c = sface[f];
                const uint32_t i0 = c.x & 0xFFFFu, i1 = c.x >> 16, i2 = c.y;
                sfd[f] = face_force(X[i0], X[i1], X[i2], V[i0], V[i1], V[i2], p.face_coef);
            }
            __syncthreads();
            // (3) gather in summation order and integrate (sim_kernel.cu:246-268).
            // acc + (+-c) is computed as fma(c, +-1, acc): c*(+-1) is exact, so
            // the single rounding equals that of the addition.
#pragma unroll
            for (int j = 0; j < MPT; ++j) {
                const uint32_t m = tid + j * T;
                if (m >= bd.n_mass) break;
                float ax = 0.0f, ay = 0.0f, az = 0.0f;
                const uint16_t* rp = sinc + (row[j] & 0xFFFFFu);
                const uint32_t w = row[j] >> 20;  // the same for the warp (one slice)
                if (RW > 0 && w <= (uint32_t)RW) {
                    // entries in [w, RW) are padding; a padding entry adds a
                    // zero (acc + -0 == acc: a sum that starts at +0 is never -0)
#pragma unroll
                    for (int k0 = 0; k0 < RW; k0 += RG) {
                        if ((uint32_t)k0 >= w) break;
                        float4 c[RG];
                        float sg[RG];
#pragma unroll
                        for (int u = 0; u < RG; ++u) {
                            const int k = k0 + u;
                            const uint32_t e = (k & 1) ? rr[k / 2] >> 16 : rr[k / 2] & 0xFFFFu;
                            c[u] = e != kPadEntry ? sdp[e >> 1] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                            sg[u] = __uint_as_float(0x3f800000u | ((e & 1u) << 31));
                        }
#pragma unroll
                        for (int u = 0; u < RG; ++u) {
                            ax = __fmaf_rn(c[u].x, sg[u], ax);
                            ay = __fmaf_rn(c[u].y, sg[u], ay);
                            az = __fmaf_rn(c[u].z, sg[u], az);
                        }
                    }
                } else
                for (uint32_t k = 0; k < w; ++k) {
                    // (register rows: a slice wider than RW reads its row from global memory)
                    const uint32_t e = RW > 0 ? __ldg(p.inc + bd.inc_begin + (row[j] & 0xFFFFFu) + k * kSliceWidth)
                                              : rp[k * kSliceWidth];
                    if (e != kPadEntry) {
                        const float4 c = sdp[e >> 1];
                        const float sg = __uint_as_float(0x3f800000u | ((e & 1u) << 31));
                        ax = __fmaf_rn(c.x, sg, ax);
                        ay = __fmaf_rn(c.y, sg, ay);
                        az = __fmaf_rn(c.z, sg, az);
                    }
                }
                if (XPBD) {
                    const float4 xt = X[m];
                    const float nx = __fadd_rn(xt.x, ax);
                    const float ny = __fadd_rn(xt.y, ay);
                    const float nz = __fadd_rn(xt.z, az);
                    // v = 0.99*(x~ - x)/dt in double (sim_kernel.cu:265-267)
                    v[j].x = velocity_of(__fsub_rn(nx, x[j].x), ddt, inv_dt);
                    v[j].y = velocity_of(__fsub_rn(ny, x[j].y), ddt, inv_dt);
                    v[j].z = velocity_of(__fsub_rn(nz, x[j].z), ddt, inv_dt);
                    x[j] = make_float3(nx, ny, nz);
                } else {
                    // face drag after the springs, faces in ascending order
                    // (the face row: first entry | count << 24)
                    const uint32_t fr = n_face ? sfrow[m] : 0u;
                    const uint16_t* fp = sfinc + (fr & 0xFFFFFFu);
                    for (uint32_t k = 0; k < (fr >> 24); ++k) {
                        const float4 c = sfd[fp[k]];
                        ax = __fadd_rn(ax, c.x);
                        ay = __fadd_rn(ay, c.y);
                        az = __fadd_rn(az, c.z);
                    }
                    force_integrate<MODE>(p, x[j], v[j], mass[j], inv_dt_f, ax, ay, az);
                }
            }
        }

        // Write back in the upload layout (w components unchanged); flag
        // non-finite positions.
        bool bad = false;
#pragma unroll
        for (int j = 0; j < MPT; ++j) {
            const uint32_t m = tid + j * T;
            if (m < bd.n_mass) {
                const uint32_t g = __ldg(&p.mass_gidx[bd.mass_begin + m]);
                p.pos[g] = make_float4(x[j].x, x[j].y, x[j].z, p.pos[g].w);
                p.vel[g] = make_float4(v[j].x, v[j].y, v[j].z, p.vel[g].w);
                bad |= !(isfinite(x[j].x) && isfinite(x[j].y) && isfinite(x[j].z));
            }
        }
        if (TRACK) {
#pragma unroll
            for (int j = 0; j < SPT; ++j) {
                const uint32_t s = tid + j * T;
                if (s < bd.n_spring) {
                    const uint32_t g = __ldg(&p.spring_gidx[bd.spring_begin + s]);
                    if (!(g >> 31)) p.stress[g] = st[j];  // bit 31: a copy in a split part
                }
            }
        }
        if (__syncthreads_or(bad) && tid == 0) atomicOr(&p.bin_flags[b], 1u);
        if (SPLIT) cg::this_cluster().sync();
    }
}


// Streamed step: one CTA per bin (typically one large robot).  Shared memory
// holds the predicted positions and the material factors; every step reads
// the bin's springs and rows from global memory and exchanges the per-spring
// corrections through a global scratch array (L2-resident), with the same
// arithmetic and summation order as step_kernel.
template <int T, int MPT, int MODE, bool TRACK>
__global__ void __launch_bounds__(T, 1024 / T) stream_kernel(const StepParams p) {
    constexpr bool XPBD = MODE == kModeXpbd;
    constexpr bool FACES = MODE == kModeForceWaterFaces;  // face drag compiled in
    extern __shared__ float4 smem4[];
    const int tid = threadIdx.x;
    const float dt = p.dt;
    const double ddt = (double)dt;
    const double inv_dt = __drcp_rn(ddt);
    const float inv_dt_f = __frcp_rn(dt);

    for (uint32_t b = blockIdx.x; b < p.n_bins; b += gridDim.x) {
        const BinDesc bd = p.bins[b];
        float4* sxt = smem4;
        float2* smat = reinterpret_cast<float2*>(sxt + bd.n_mass);
        float4* dp = p.dp + bd.spring_begin;
        float* stp = p.st + bd.spring_begin;
        const uint32_t* pair = p.spring_pair + bd.spring_begin;
        const float* lbar = p.spring_lbar + bd.spring_begin;
        const uint32_t* inc = p.inc32 + bd.inc_begin;
        // face drag: velocities in shared memory after the material factors,
        // face forces through the global scratch like the corrections
        const uint32_t n_face = FACES && p.face_on ? bd.n_face : 0u;
        float4* sv = reinterpret_cast<float4*>(smat + kMaxMaterialSlots);
        float4* fd = p.fd + bd.face_begin;
        const uint2* fcorner = p.faces + bd.face_begin;
        const uint16_t* finc = p.face_inc + bd.face_inc_begin;
        const uint32_t n_mat = *p.n_mat;
        float next_rate = 0.0f;
        if (tid < n_mat) {
            smat[tid].y = __ldg(&p.invk[tid]);
            next_rate = __ldg(&p.rates[tid]);
        }
        if (TRACK)
            for (uint32_t s = tid; s < bd.n_spring; s += T)
                stp[s] = p.stress[__ldg(&p.spring_gidx[bd.spring_begin + s])];

        float3 x[MPT], v[MPT];
        float mass[MPT];
        uint32_t roff[MPT], rwid[MPT], frow[MPT];
#pragma unroll
        for (int j = 0; j < MPT; ++j) {
            const uint32_t m = tid + j * T;
            x[j] = make_float3(0.f, 0.f, 0.f);
            v[j] = make_float3(0.f, 0.f, 0.f);
            mass[j] = 1.0f;
            roff[j] = 0;
            rwid[j] = 0;
            frow[j] = 0;
            if (n_face && m < bd.n_mass) frow[j] = __ldg(&p.face_row[bd.mass_begin + m]);
            if (m < bd.n_mass) {
                const uint32_t g = __ldg(&p.mass_gidx[bd.mass_begin + m]);
                const float4 P = p.pos[g], V = p.vel[g];
                x[j] = make_float3(P.x, P.y, P.z);
                v[j] = make_float3(V.x, V.y, V.z);
                mass[j] = P.w;
                const uint32_t sl = bd.slice_begin + m / kSliceWidth;
                roff[j] = __ldg(&p.slice_off[sl]) + (m % kSliceWidth);
                rwid[j] = __ldg(&p.slice_width[sl]);
            }
        }
        __syncthreads();

        for (uint32_t step = 0; step < p.steps; ++step) {
            if (tid < n_mat) {
                smat[tid].x = next_rate;
                if (step + 1 < p.steps) next_rate = __ldg(&p.rates[(step + 1) * n_mat + tid]);
            }
#pragma unroll
            for (int j = 0; j < MPT; ++j) {
                const uint32_t m = tid + j * T;
                if (m >= bd.n_mass) break;
                if (XPBD)
                    sxt[m] = make_float4(__fadd_rn(x[j].x, __fmul_rn(v[j].x, dt)),
                                         __fadd_rn(x[j].y, __fmul_rn(v[j].y, dt)),
                                         __fadd_rn(x[j].z, __fmul_rn(v[j].z, dt)), 0.0f);
                else
                    sxt[m] = make_float4(x[j].x, x[j].y, x[j].z, 0.0f);
                if (n_face) sv[m] = make_float4(v[j].x, v[j].y, v[j].z, 0.0f);
            }
            __syncthreads();
            for (uint32_t s = tid; s < bd.n_spring; s += T) {
                const uint32_t w = __ldg(&pair[s]);
                const float lb = __ldg(&lbar[s]);
                const float4 pa = sxt[pk_a(w)], pb = sxt[pk_b(w)];
                const float2 mt = smat[pk_slot(w)];
                const float L = __fmaf_rn(lb, mt.x, lb);
                const float dx = __fsub_rn(pa.x, pb.x);
                const float dy = __fsub_rn(pa.y, pb.y);
                const float dz = __fsub_rn(pa.z, pb.z);
                const float d = __fsqrt_rn(__fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz))));
                const float r = __frcp_rn(__fadd_rn(d, kEps));
                const float lam = __fmul_rn(-__fsub_rn(d, L), mt.y);
                const float coef = __fmul_rn(lam, r);
                __stcg(&dp[s], make_float4(__fmul_rn(coef, dx), __fmul_rn(coef, dy), __fmul_rn(coef, dz), 0.0f));
                if (TRACK) stp[s] = __fadd_rn(stp[s], __fmul_rn(XPBD ? lam : -lam, __frcp_rn(lb)));
            }
            for (uint32_t f = tid; f < n_face; f += T) {
                const uint2 c = __ldg(&fcorner[f]);
                const uint32_t i0 = c.x & 0xFFFFu, i1 = c.x >> 16, i2 = c.y;
                __stcg(&fd[f], face_force(sxt[i0], sxt[i1], sxt[i2], sv[i0], sv[i1], sv[i2], p.face_coef));
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < MPT; ++j) {
                const uint32_t m = tid + j * T;
                if (m >= bd.n_mass) break;
                float ax = 0.0f, ay = 0.0f, az = 0.0f;
                for (uint32_t k = 0; k < rwid[j]; ++k) {
                    const uint32_t e = __ldg(&inc[roff[j] + k * kSliceWidth]);
                    if (e != kPadEntry32) {
                        const float4 c = __ldcg(&dp[e >> 1]);
                        const float sg = __uint_as_float(0x3f800000u | ((e & 1u) << 31));
                        ax = __fmaf_rn(c.x, sg, ax);
                        ay = __fmaf_rn(c.y, sg, ay);
                        az = __fmaf_rn(c.z, sg, az);
                    }
                }
                // face drag after the springs, faces in ascending order
                for (uint32_t k = 0; k < (frow[j] >> 24); ++k) {
                    const float4 c = __ldcg(&fd[__ldg(&finc[(frow[j] & 0xFFFFFFu) + k])]);
                    ax = __fadd_rn(ax, c.x);
                    ay = __fadd_rn(ay, c.y);
                    az = __fadd_rn(az, c.z);
                }
                if (XPBD) {
                    const float4 xt = sxt[m];
                    const float nx = __fadd_rn(xt.x, ax);
                    const float ny = __fadd_rn(xt.y, ay);
                    const float nz = __fadd_rn(xt.z, az);
                    v[j].x = velocity_of(__fsub_rn(nx, x[j].x), ddt, inv_dt);
                    v[j].y = velocity_of(__fsub_rn(ny, x[j].y), ddt, inv_dt);
                    v[j].z = velocity_of(__fsub_rn(nz, x[j].z), ddt, inv_dt);
                    x[j] = make_float3(nx, ny, nz);
                } else {
                    force_integrate<MODE>(p, x[j], v[j], mass[j], inv_dt_f, ax, ay, az);
                }
            }
        }

        bool bad = false;
#pragma unroll
        for (int j = 0; j < MPT; ++j) {
            const uint32_t m = tid + j * T;
            if (m < bd.n_mass) {
                const uint32_t g = __ldg(&p.mass_gidx[bd.mass_begin + m]);
                p.pos[g] = make_float4(x[j].x, x[j].y, x[j].z, p.pos[g].w);
                p.vel[g] = make_float4(v[j].x, v[j].y, v[j].z, p.vel[g].w);
                bad |= !(isfinite(x[j].x) && isfinite(x[j].y) && isfinite(x[j].z));
            }
        }
        if (TRACK) {
            __syncthreads();
            for (uint32_t s = tid; s < bd.n_spring; s += T)
                p.stress[__ldg(&p.spring_gidx[bd.spring_begin + s])] = stp[s];
        }
        if (__syncthreads_or(bad) && tid == 0) atomicOr(&p.bin_flags[b], 1u);
    }
}

// Actuation factors of one launch.  Block b covers steps [256 b, 256 b + 256):
// thread 0 accumulates the float clock from t0 (the clock is a sequential
// float sum, Simulator.cu:447, so it is not reassociated), then every thread
// evaluates its step for every material.
__global__ void __launch_bounds__(256) actuation_kernel(const float4* __restrict__ table,
                                                        const uint8_t* __restrict__ mat_ids,
                                                        const uint32_t* __restrict__ n_mat_ptr,
                                                        float t0, float dt, uint32_t steps,
                                                        uint32_t mode, float* __restrict__ rates,
                                                        float* __restrict__ invk) {
    __shared__ float s_t[256];
    const uint32_t n_mat = *n_mat_ptr;
    const uint32_t base = blockIdx.x * 256u;
    if (threadIdx.x == 0) {
        float t = t0;
        for (uint32_t i = 0; i < base; ++i) t = __fadd_rn(t, dt);
        for (uint32_t i = 0; i < 256u; ++i) {
            s_t[i] = t;
            t = __fadd_rn(t, dt);
        }
    }
    if (blockIdx.x == 0) {
        for (uint32_t i = threadIdx.x; i < n_mat; i += 256u) {
            const float4 mt = table[mat_ids[i]];
            if (mode == kModeXpbd) {
                // alpha = 1/k/dt/dt, K = 2 + alpha (sim_kernel.cu:220, 225)
                const float alpha = __fdiv_rn(__fdiv_rn(__fdiv_rn(1.0f, mt.x), dt), dt);
                invk[i] = __frcp_rn(__fadd_rn(2.0f, alpha));
            } else {
                invk[i] = mt.x;
            }
        }
    }
    __syncthreads();
    const uint32_t n = base + threadIdx.x;
    if (n >= steps) return;
    const float t = s_t[threadIdx.x];
    for (uint32_t i = 0; i < n_mat; ++i) {
        const float4 mt = table[mat_ids[i]];
        const float arg = __fmaf_rn(mt.z, t, mt.w);
        rates[(size_t)n * n_mat + i] = __fmul_rn(mt.y, __double2float_rn(sin_cw((double)arg)));
    }
}

// Centre of mass of non-air masses, one warp per robot: lane l sums masses
// l, l+32, ... in double, then an xor butterfly; mean rounded to float.
__global__ void com_kernel(const float4* __restrict__ pos, const uint8_t* __restrict__ mat,
                           const int64_t* __restrict__ off, uint32_t n_robots,
                           float* __restrict__ com) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const uint32_t lane = threadIdx.x % 32;
    if (warp >= n_robots) return;
    const int64_t b = off[warp], n = off[warp + 1] - b;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    long long cnt = 0;
    for (int64_t i = lane; i < n; i += 32) {
        if (!mat[b + i]) continue;
        const float4 q = pos[b + i];
        sx = __dadd_rn(sx, (double)q.x);
        sy = __dadd_rn(sy, (double)q.y);
        sz = __dadd_rn(sz, (double)q.z);
        ++cnt;
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        sx = __dadd_rn(sx, __shfl_xor_sync(0xffffffffu, sx, o));
        sy = __dadd_rn(sy, __shfl_xor_sync(0xffffffffu, sy, o));
        sz = __dadd_rn(sz, __shfl_xor_sync(0xffffffffu, sz, o));
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    if (lane == 0) {
        const double dc = (double)cnt;
        com[3 * warp + 0] = cnt ? __double2float_rn(__ddiv_rn(sx, dc)) : 0.0f;
        com[3 * warp + 1] = cnt ? __double2float_rn(__ddiv_rn(sy, dc)) : 0.0f;
        com[3 * warp + 2] = cnt ? __double2float_rn(__ddiv_rn(sz, dc)) : 0.0f;
    }
}

// Per-robot status: bit 0 set when any position of the robot is NaN/Inf.
// One warp per robot.
__global__ void flags_kernel(const float4* __restrict__ pos, const int64_t* __restrict__ off,
                             uint32_t n_robots, uint32_t* __restrict__ out) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const uint32_t lane = threadIdx.x % 32;
    if (warp >= n_robots) return;
    bool bad = false;
    for (int64_t i = off[warp] + lane; i < off[warp + 1]; i += 32) {
        const float4 q = pos[i];
        bad |= !(isfinite(q.x) && isfinite(q.y) && isfinite(q.z));
    }
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) out[warp] = bad ? 1u : 0u;
}

// Bit 1 of a robot's status: its (first) bin was skipped by the step kernel.
__global__ void bin_flags_kernel(const uint32_t* __restrict__ bin_flags, const uint32_t* __restrict__ robot_bin,
                                 uint32_t n_robots, uint32_t* __restrict__ out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n_robots) out[r] |= bin_flags[robot_bin[r]] & 2u;
}

using StepFn = void (*)(const StepParams);

struct ShapeEntry {
    uint32_t threads, spt, mpt;
    StepFn fn[4][2];  // [mode][track]; mode 3: water with face drag
};

#define MB_SHAPE(T, S, M, SPLIT)                                                               \
    {                                                                                          \
        T, S, M, {                                                                             \
            {step_kernel<T, S, M, kModeXpbd, false, SPLIT>,                                    \
             step_kernel<T, S, M, kModeXpbd, true, SPLIT>},                                    \
                {step_kernel<T, S, M, kModeForceLand, false, SPLIT>,                           \
                 step_kernel<T, S, M, kModeForceLand, true, SPLIT>},                           \
                {step_kernel<T, S, M, kModeForceWater, false, SPLIT>,                          \
                 step_kernel<T, S, M, kModeForceWater, true, SPLIT>},                          \
                {step_kernel<T, S, M, kModeForceWaterFaces, false, SPLIT>,                     \
                 step_kernel<T, S, M, kModeForceWaterFaces, true, SPLIT>},                     \
        }                                                                                      \
    }
const ShapeEntry kShapes[] = {
    MB_SHAPE(256, 8, 2, false),   MB_SHAPE(512, 4, 1, false),   MB_SHAPE(512, 8, 2, false),
    MB_SHAPE(512, 16, 4, false),  MB_SHAPE(1024, 4, 1, false),  MB_SHAPE(1024, 6, 2, false),
    MB_SHAPE(1024, 8, 2, false),  MB_SHAPE(1024, 10, 2, false), MB_SHAPE(1024, 12, 2, false),
};
// register-row twins of the 1,024-thread shapes (one mass per thread; no
// face drag): launch_step uses one when the host marks the launch eligible
// (StepParams::one_mass_per_thread)
#define MB_RR(T, S, RW)                                                                          \
    {                                                                                            \
        T, S, 1, {                                                                               \
            {step_kernel<T, S, 1, kModeXpbd, false, false, RW>,                                  \
             step_kernel<T, S, 1, kModeXpbd, true, false, RW>},                                  \
                {step_kernel<T, S, 1, kModeForceLand, false, false, RW>,                         \
                 step_kernel<T, S, 1, kModeForceLand, true, false, RW>},                         \
                {step_kernel<T, S, 1, kModeForceWater, false, false, RW>,                        \
                 step_kernel<T, S, 1, kModeForceWater, true, false, RW>},                        \
                {nullptr, nullptr},                                                              \
        }                                                                                        \
    }
constexpr int kRowRegWidth = 26;  // register rows: entries per mass (lattice robots: at most 26)
const ShapeEntry kRowRegShapes[] = {MB_RR(1024, 8, kRowRegWidth), MB_RR(1024, 10, kRowRegWidth),
                                    MB_RR(1024, 12, kRowRegWidth)};
#undef MB_RR
// the parts of split robots (thread-block clusters)
const ShapeEntry kSplitShapes[] = {
    MB_SHAPE(1024, 8, 1, true),
    MB_SHAPE(1024, 10, 1, true),
    MB_SHAPE(1024, 8, 2, true),
    MB_SHAPE(1024, 10, 2, true),
    MB_SHAPE(1024, 12, 2, true),
};
#undef MB_SHAPE


struct StreamEntry {
    uint32_t threads, mpt;
    StepFn fn[4][2];  // [mode][track]; mode 3: water with face drag
};
#define MB_STREAM(T, M)                                                                          \
    {                                                                                            \
        T, M, {                                                                                  \
            {stream_kernel<T, M, kModeXpbd, false>, stream_kernel<T, M, kModeXpbd, true>},       \
                {stream_kernel<T, M, kModeForceLand, false>,                                     \
                 stream_kernel<T, M, kModeForceLand, true>},                                     \
                {stream_kernel<T, M, kModeForceWater, false>,                                    \
                 stream_kernel<T, M, kModeForceWater, true>},                                    \
                {stream_kernel<T, M, kModeForceWaterFaces, false>,                               \
                 stream_kernel<T, M, kModeForceWaterFaces, true>},                               \
        }                                                                                        \
    }
// up to threads * MPT masses per bin (2,048 or 4,096 with 1,024 threads)
const StreamEntry kStream[] = {MB_STREAM(1024, 2), MB_STREAM(1024, 4)};
#undef MB_STREAM

const StreamEntry* find_stream(uint32_t threads, uint32_t mpt) {
    for (const auto& e : kStream)
        if (e.threads == threads && e.mpt == mpt) return &e;
    return nullptr;
}

const ShapeEntry* find_shape(const KernelShape& s) {
    for (const auto& e : kShapes)
        if (e.threads == s.threads && e.spt == s.spt && e.mpt == s.mpt) return &e;
    return nullptr;
}

// The register-row twin of a 1,024-thread shape, for the launches the host
// marks eligible (no face drag).
const ShapeEntry* find_row_reg(const KernelShape& s, const StepParams& p) {
    if (s.threads != 1024 || !p.one_mass_per_thread || p.face_on) return nullptr;
    for (const auto& e : kRowRegShapes)
        if (e.spt == s.spt) return &e;
    return nullptr;
}

const ShapeEntry* find_split(const KernelShape& s) {
    for (const auto& e : kSplitShapes)
        if (e.threads == s.threads && e.spt == s.spt && e.mpt == s.mpt) return &e;
    return nullptr;
}

}  // namespace

uint32_t bin_smem_bytes(uint32_t n_mass, uint32_t n_spring, uint32_t n_inc) {
    return bin_smem_bytes_dev(n_mass, n_spring, n_inc);
}

uint32_t max_step_smem(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    return (uint32_t)v;
}

bool shape_supported(const KernelShape& shape) { return find_shape(shape) != nullptr; }

bool row_reg_supported(const KernelShape& shape) {
    if (shape.threads != 1024) return false;
    for (const auto& e : kRowRegShapes)
        if (e.spt == shape.spt) return true;
    return false;
}

uint32_t row_reg_width() { return kRowRegWidth; }

bool split_supported(const KernelShape& shape) { return find_split(shape) != nullptr; }

cudaError_t prepare_split(const KernelShape& shape, uint32_t mode, bool track, uint32_t smem_bytes) {
    const ShapeEntry* e = find_split(shape);
    if (!e || mode > kModeForceWater) return cudaErrorInvalidValue;
    cudaError_t r = cudaFuncSetAttribute(e->fn[mode][track ? 1 : 0], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_bytes);
    if (r == cudaSuccess && mode == kModeForceWater)  // and the face-drag variant
        r = cudaFuncSetAttribute(e->fn[kModeForceWaterFaces][track ? 1 : 0],
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    return r;
}

// One CTA per part, the parts of a robot (bins r*C .. r*C + C-1) forming a
// cluster of C CTAs.
cudaError_t launch_split(const StepParams& p, const KernelShape& shape, uint32_t cluster, cudaStream_t s) {
    const ShapeEntry* e = find_split(shape);
    if (!e || p.mode > kModeForceWater || cluster < 2 || cluster > 8 || p.n_bins % cluster)
        return cudaErrorInvalidValue;
    if (p.n_bins == 0) return cudaSuccess;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(p.n_bins, 1, 1);
    cfg.blockDim = dim3(shape.threads, 1, 1);
    cfg.dynamicSmemBytes = p.smem_bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const uint32_t variant = p.mode == kModeForceWater && p.face_on ? kModeForceWaterFaces : p.mode;
    return cudaLaunchKernelEx(&cfg, e->fn[variant][p.track ? 1 : 0], p);
}

cudaError_t prepare_step(const KernelShape& shape, uint32_t mode, bool track, uint32_t smem_bytes) {
    const ShapeEntry* e = find_shape(shape);
    if (!e || mode > kModeForceWater) return cudaErrorInvalidValue;
    cudaError_t r = cudaFuncSetAttribute(e->fn[mode][track ? 1 : 0], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_bytes);
    if (shape.threads == 1024)  // the register-row twin, when there is one
        for (const auto& t : kRowRegShapes)
            if (r == cudaSuccess && t.spt == shape.spt)
                r = cudaFuncSetAttribute(t.fn[mode][track ? 1 : 0], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_bytes);
    if (r == cudaSuccess && mode == kModeForceWater)  // and the face-drag variant
        r = cudaFuncSetAttribute(e->fn[kModeForceWaterFaces][track ? 1 : 0],
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    return r;
}

int ctas_per_sm(const KernelShape& shape, uint32_t mode, bool track, uint32_t smem_bytes) {
    const ShapeEntry* e = find_shape(shape);
    if (!e || mode > kModeForceWater) return 0;
    StepFn fn = e->fn[mode][track ? 1 : 0];
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, (int)shape.threads, smem_bytes) != cudaSuccess)
        return 0;
    return n;
}

int max_active_clusters(const KernelShape& shape, uint32_t mode, uint32_t cluster, uint32_t smem_bytes) {
    const ShapeEntry* e = find_split(shape);
    if (!e || mode > kModeForceWater || cluster < 1 || cluster > kMaxClusterParts) return 0;
    StepFn fn = e->fn[mode][0];
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes) != cudaSuccess)
        return 0;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(cluster, 1, 1);
    cfg.blockDim = dim3(shape.threads, 1, 1);
    cfg.dynamicSmemBytes = smem_bytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return n;
}

uint32_t list_shapes(KernelShape* out, uint32_t cap, bool streamed) {
    uint32_t n = 0;
    if (streamed) {
        for (const auto& e : kStream) {
            if (n < cap) out[n] = KernelShape{e.threads, 0, e.mpt};
            ++n;
        }
    } else {
        for (const auto& e : kShapes) {
            if (n < cap) out[n] = KernelShape{e.threads, e.spt, e.mpt};
            ++n;
        }
    }
    return n;
}

uint32_t stream_smem_bytes(uint32_t n_mass) { return 16u * n_mass + 8u * kMaxMaterialSlots; }

bool stream_supported(uint32_t threads, uint32_t mpt) { return find_stream(threads, mpt) != nullptr; }

cudaError_t prepare_stream(uint32_t threads, uint32_t mpt, uint32_t mode, bool track,
                           uint32_t smem_bytes) {
    const StreamEntry* e = find_stream(threads, mpt);
    if (!e || mode > kModeForceWater) return cudaErrorInvalidValue;
    cudaError_t r = cudaFuncSetAttribute(e->fn[mode][track ? 1 : 0],
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    if (r == cudaSuccess && mode == kModeForceWater)  // and the face-drag variant
        r = cudaFuncSetAttribute(e->fn[kModeForceWaterFaces][track ? 1 : 0],
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    return r;
}

cudaError_t launch_stream(const StepParams& p, uint32_t threads, uint32_t mpt, cudaStream_t s) {
    const StreamEntry* e = find_stream(threads, mpt);
    if (!e || p.mode > kModeForceWater) return cudaErrorInvalidValue;
    if (p.n_bins == 0) return cudaSuccess;
    const uint32_t variant = p.mode == kModeForceWater && p.face_on ? kModeForceWaterFaces : p.mode;
    e->fn[variant][p.track ? 1 : 0]<<<p.n_bins, threads, p.smem_bytes, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_step(const StepParams& p, const KernelShape& shape, cudaStream_t s) {
    const ShapeEntry* e = find_shape(shape);
    if (!e) return cudaErrorInvalidValue;
    if (p.n_bins == 0) return cudaSuccess;
    if (p.mode > kModeForceWater) return cudaErrorInvalidValue;
    const uint32_t grid = p.grid ? std::min(p.grid, p.n_bins) : p.n_bins;
    const uint32_t variant = p.mode == kModeForceWater && p.face_on ? kModeForceWaterFaces : p.mode;
    if (const ShapeEntry* rr = find_row_reg(shape, p)) e = rr;
    e->fn[variant][p.track ? 1 : 0]<<<grid, shape.threads, p.smem_bytes, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_actuation(const float4* table, const uint8_t* mat_ids, const uint32_t* n_mat,
                             float t0, float dt, uint32_t steps, uint32_t mode, float* rates,
                             float* coef, cudaStream_t s) {
    if (steps == 0) return cudaSuccess;
    actuation_kernel<<<(steps + 255) / 256, 256, 0, s>>>(table, mat_ids, n_mat, t0, dt, steps, mode,
                                                         rates, coef);
    return cudaGetLastError();
}

cudaError_t launch_com(const float4* pos, const uint8_t* mass_mat, const int64_t* mass_off,
                       uint32_t n_robots, float* com, cudaStream_t s) {
    if (n_robots == 0) return cudaSuccess;
    const uint32_t threads = 256, warps = threads / 32;
    com_kernel<<<(n_robots + warps - 1) / warps, threads, 0, s>>>(pos, mass_mat, mass_off,
                                                                   n_robots, com);
    return cudaGetLastError();
}

cudaError_t launch_bin_flags(const uint32_t* bin_flags, const uint32_t* robot_bin, uint32_t n_robots,
                             uint32_t* out, cudaStream_t s) {
    if (n_robots == 0) return cudaSuccess;
    bin_flags_kernel<<<(n_robots + 255) / 256, 256, 0, s>>>(bin_flags, robot_bin, n_robots, out);
    return cudaGetLastError();
}

cudaError_t launch_flags(const float4* pos, const int64_t* mass_off, uint32_t n_robots,
                         uint32_t* out, cudaStream_t s) {
    if (n_robots == 0) return cudaSuccess;
    const uint32_t threads = 256, warps = threads / 32;
    flags_kernel<<<(n_robots + warps - 1) / warps, threads, 0, s>>>(pos, mass_off, n_robots, out);
    return cudaGetLastError();
}

}  // namespace mb
