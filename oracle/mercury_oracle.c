/*
 * CPU ORACLE -- test infrastructure, never shipped.
 *
 * A restatement of the reference's (DawsonCohen/Mercury) batched soft-body
 * step, used by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py as the checker.  The product (mercury_b200/) never links it.
 *
 * Pinned by: the reference's own code run through oracle/ref_harness.cpp
 * (material table, composite decode, lattice topology on the CPU; the CUDA
 * step on the GPU), see tests/golden/.
 *
 * What follows the reference, and where:
 *   material table .......... common/simulator/material.h:9-10, 111-133,
 *                             192-227 (avg), 253-273 (id_lookup)
 *   composite decode ........ material.h:275-322
 *   step count / clock ...... common/simulator/Simulator.cu:428-449
 *   XPBD step ............... common/simulator/sim_kernel.cu:141-153 (predict),
 *                             166-253 (distance constraint), 255-269 (update)
 *   centre of mass .......... common/evolvables/SoftBody.cpp:112-121
 *   development (Devo) ...... common/simulator/Simulator.cu:597-668,
 *                             devo_kernel.cu:56-168 (see or_devo)
 *   face drag ............... sim_kernel.cu:96-121 (the face law of
 *                             surfaceDragForce; see face_force_f32), added
 *                             to the forces of the water mode
 *
 * The reference accumulates the per-mass corrections with shared-memory
 * atomics, so its own summation order is unspecified and run-to-run
 * non-deterministic.  This restatement fixes one order: for every mass, the
 * corrections of its incident non-air springs are summed by the spring's
 * other end (ascending), then spring index, the "a" end (+dp) of a spring
 * before its "b" end (-dp).  The CUDA kernels use the same order, so kernel
 * and oracle agree to the bit.
 *
 * Arithmetic choices (all IEEE-754 round-to-nearest, no contraction; build
 * with -ffp-contract=off):
 *   - sin of the actuation phase: the float phase fmaf(omega, t, phi) (nvcc
 *     contracts the reference's omega*t+phi into one fma) is widened to
 *     double, and sin is evaluated by Cody-Waite reduction by pi/2 and Taylor
 *     polynomials (or_sin), then rounded to float.  The reference calls sinf
 *     (or __sinf under -use_fast_math).
 *   - |x| is sqrtf(fmaf(dx,dx, fmaf(dy,dy, dz*dz))); the reference calls
 *     norm3df.
 *   - the three divisions by (d + EPS) become one correctly rounded
 *     reciprocal and multiplications; -C/K becomes -C * (1/K); lambda/Lbar
 *     becomes lambda * (1/Lbar).
 *   - the velocity update keeps the reference's double-precision expression
 *     0.99*(x~ - x)/dt (sim_kernel.cu:265-267: 0.99 is a double literal).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_COMPOSITE_COUNT 254
#define OR_BASE_COUNT 23
#define OR_EPS 1e-12f

/* ------------------------------------------------------------------ */
/* Materials (material.h:111-133).  Each base material: k, dL0, omega, phi
 * as the reference's constexpr initialisers evaluate them (double
 * expressions narrowed to float). */
static void base_material(int id, float* k, float* dl0, float* om, float* ph) {
    const double PI = 3.14159265358979323846;
    const double OMEGA = (double)(float)1.0f * (2.0f * PI); /* (float)1.0f*(2.0f*M_PI) */
    const float AMP = .14f;
    if (id == 0) { *k = 0; *dl0 = 0; *om = 0; *ph = 0; return; }
    if (id >= 1 && id <= 20) {
        int j = (id - 1) % 10; /* 0..9 */
        int abductor = id >= 11;
        *k = 50.0f; *dl0 = AMP;
        if (j <= 7) {
            /* phi = n*M_PI/8 with n = j (adductor) or 8 + j (abductor);
             * 5*M_PI/4 etc. in the reference are the same doubles. */
            *om = (float)OMEGA;
            *ph = (float)((double)((abductor ? 8 : 0) + j) * PI / 8.0);
        } else if (j == 8) {
            *om = (float)(OMEGA * 2);
            *ph = (float)(abductor ? PI : 0.0);
        } else {
            *om = (float)(OMEGA / 2);
            *ph = (float)(abductor ? PI : 0.0);
        }
        return;
    }
    if (id == 21) { *k = 40.0f; *dl0 = 0.0f; *om = (float)OMEGA; *ph = 0.0f; return; }
    /* id == 22 */
    *k = 100.0f; *dl0 = 0.0f; *om = (float)OMEGA; *ph = 0.0f;
}

/* Composite id of a pair of base materials (material.h:192-213): ids 1..22
 * for a base material with itself, then pairs (i<j) numbered from 23 in
 * row-major order. */
int or_composite_id(int m1, int m2) {
    if (m1 == 0 || m2 == 0) return 0;
    int i = m1 < m2 ? m1 - 1 : m2 - 1, j = m1 < m2 ? m2 - 1 : m1 - 1;
    if (i == j) return i + 1;
    int count = 23;
    for (int a = 0; a < 22; ++a)
        for (int b = a + 1; b < 22; ++b) {
            if (a == i && b == j) return count;
            ++count;
        }
    return -1;
}

/* id_lookup table (material.h:253-273): base materials at their ids, pair
 * composites at or_composite_id with every field the double-precision mean
 * of the two (material.h:215-227). */
void or_material_table(float* out) {
    memset(out, 0, sizeof(float) * 4 * OR_COMPOSITE_COUNT);
    for (int i = 0; i < OR_BASE_COUNT; ++i)
        base_material(i, &out[4 * i], &out[4 * i + 1], &out[4 * i + 2], &out[4 * i + 3]);
    for (int i = 1; i < OR_BASE_COUNT; ++i)
        for (int j = i + 1; j < OR_BASE_COUNT; ++j) {
            float a[4], b[4];
            base_material(i, &a[0], &a[1], &a[2], &a[3]);
            base_material(j, &b[0], &b[1], &b[2], &b[3]);
            int id = or_composite_id(i, j);
            for (int c = 0; c < 4; ++c) out[4 * id + c] = (float)(((double)a[c] + (double)b[c]) / 2.0);
        }
}

/* materials::decode(encoding).id (material.h:275-322): the lowest set bit
 * selects the first material; bit 0 (air) anywhere below the second set bit
 * gives air; otherwise the two lowest set bits form the composite. */
int or_decode_id(uint32_t enc) {
    int idx[2] = {0, 0}, count = 0;
    for (int i = 0; i < 32; ++i)
        if (enc & (1u << i)) {
            idx[count++] = i;
            if (i == 0 || count == 2) break;
        }
    if (idx[0] == 0) return 0;
    if (idx[1] == 0) return idx[0];
    return or_composite_id(idx[0], idx[1]);
}

/* ------------------------------------------------------------------ */
/* Clock (Simulator.cu:428-449): steps taken by Simulate(duration) and the
 * float clock after them. */
uint32_t or_step_count(float duration, float dt) {
    volatile float rem = duration;
    uint32_t n = 0;
    while (rem > 0.0f) { rem = rem - dt; ++n; }
    return n;
}

float or_advance_clock(float t0, float dt, uint32_t steps) {
    volatile float t = t0;
    for (uint32_t i = 0; i < steps; ++i) t = t + dt;
    return t;
}

/* ------------------------------------------------------------------ */
/* sin(x) for |x| < 2^20: Cody & Waite (1980) reduction by pi/2 with a
 * three-part constant, then the Taylor series of sin / cos on |r| <= pi/4
 * evaluated by Horner's rule with fused multiply-adds.  The coefficients are
 * (-1)^k/(2k+1)! and (-1)^k/(2k)!, rounded to double. */
/* Values printed by oracle/sin_constants.py. */
static const double OR_2_OVER_PI = 0.6366197723675814;
static const double OR_PIO2_1 = 1.5707963267341256;  /* 33 bits of pi/2 */
static const double OR_PIO2_2 = 6.077100506303966e-11;  /* next 33 bits   */
static const double OR_PIO2_3 = 2.0222662487959506e-21;  /* remainder      */
static const double OR_SIN_C[10] = {
    1.0, -0.16666666666666666, 0.008333333333333333, -0.0001984126984126984, 2.7557319223985893e-06, -2.505210838544172e-08, 1.6059043836821613e-10, -7.647163731819816e-13, 2.8114572543455206e-15, -8.22063524662433e-18};
static const double OR_COS_C[11] = {
    1.0, -0.5, 0.041666666666666664, -0.001388888888888889, 2.48015873015873e-05, -2.755731922398589e-07, 2.08767569878681e-09, -1.1470745597729725e-11, 4.779477332387385e-14, -1.5619206968586225e-16, 4.110317623312165e-19};

double or_sin(double x) {
    double k = nearbyint(x * OR_2_OVER_PI);
    double r = fma(-k, OR_PIO2_1, x);
    r = fma(-k, OR_PIO2_2, r);
    r = fma(-k, OR_PIO2_3, r);
    long q = (long)k & 3;
    double r2 = r * r, p;
    if (q == 0 || q == 2) {
        p = OR_SIN_C[9];
        for (int i = 8; i >= 0; --i) p = fma(p, r2, OR_SIN_C[i]);
        p = p * r;
    } else {
        p = OR_COS_C[10];
        for (int i = 9; i >= 0; --i) p = fma(p, r2, OR_COS_C[i]);
    }
    return (q >= 2) ? -p : p;
}

/* ------------------------------------------------------------------ */
/* Incidence entry h = 2*spring + (1 if this mass is the b end).  Returns 1
 * if entry x sorts after entry y: key (other end, spring, end). */
static int inc_after(int x, int y, const uint16_t* pairs) {
    int sx = x >> 1, sy = y >> 1;
    int ox = (x & 1) ? pairs[2 * sx] : pairs[2 * sx + 1];
    int oy = (y & 1) ? pairs[2 * sy] : pairs[2 * sy + 1];
    if (ox != oy) return ox > oy;
    if (sx != sy) return sx > sy;
    return (x & 1) > (y & 1);
}

/* ------------------------------------------------------------------ */
/* One robot, FP32 reference semantics, `steps` steps from clock t0.
 * pos/vel: float4 per mass (x, y, z, w); w of pos is the mass and is
 * carried unchanged, w of vel is untouched.  stress: one float per spring,
 * accumulated when track != 0.  Springs with material 0 (air) are skipped
 * (sim_kernel.cu:211). */
static void xpbd_robot_f32(int nm, float* pos, float* vel, int ns,
                           const uint16_t* pairs, const uint8_t* mat,
                           const float* lbar, float* stress,
                           const float* table, float dt, float t0,
                           uint32_t steps, int track) {
    /* Incidence lists in ascending spring order: +dp at a, then -dp at b. */
    int* deg = (int*)calloc((size_t)nm + 1, sizeof(int));
    for (int s = 0; s < ns; ++s) {
        if (!mat[s]) continue;
        deg[pairs[2 * s] + 1]++;
        deg[pairs[2 * s + 1] + 1]++;
    }
    for (int i = 0; i < nm; ++i) deg[i + 1] += deg[i];
    int* inc = (int*)malloc(sizeof(int) * (size_t)(deg[nm] + 1));
    int* fill = (int*)malloc(sizeof(int) * (size_t)(nm + 1));
    memcpy(fill, deg, sizeof(int) * (size_t)nm);
    for (int s = 0; s < ns; ++s) {
        if (!mat[s]) continue;
        inc[fill[pairs[2 * s]]++] = 2 * s;          /* even: +dp */
        inc[fill[pairs[2 * s + 1]]++] = 2 * s + 1;  /* odd:  -dp */
    }
    /* Summation order of a mass: by the spring's other end, then spring
     * index, then the a end before the b end (insertion sort per row). */
    for (int i = 0; i < nm; ++i)
        for (int e = deg[i] + 1; e < deg[i + 1]; ++e) {
            int h = inc[e], k = e - 1;
            while (k >= deg[i] && inc_after(inc[k], h, pairs)) { inc[k + 1] = inc[k]; --k; }
            inc[k + 1] = h;
        }
    float* xt = (float*)malloc(sizeof(float) * 3 * (size_t)(nm + 1));
    float* dp = (float*)malloc(sizeof(float) * 3 * (size_t)(ns + 1));
    float rc[OR_COMPOSITE_COUNT], invK[OR_COMPOSITE_COUNT];
    for (int m = 0; m < OR_COMPOSITE_COUNT; ++m) {
        float k = table[4 * m];
        float alpha = ((1.0f / k) / dt) / dt;
        float K = 2.0f + alpha;
        invK[m] = 1.0f / K;
    }
    volatile float t = t0;
    for (uint32_t step = 0; step < steps; ++step) {
        float tn = t;
        for (int m = 0; m < OR_COMPOSITE_COUNT; ++m) {
            float arg = fmaf(table[4 * m + 2], tn, table[4 * m + 3]);
            float sn = (float)or_sin((double)arg);
            rc[m] = table[4 * m + 1] * sn;
        }
        /* predict (sim_kernel.cu:147-152) */
        for (int i = 0; i < nm; ++i)
            for (int c = 0; c < 3; ++c) {
                float dv = vel[4 * i + c] * dt;
                xt[3 * i + c] = pos[4 * i + c] + dv;
            }
        /* distance constraints (sim_kernel.cu:209-243) */
        for (int s = 0; s < ns; ++s) {
            int m = mat[s];
            if (!m) continue;
            int a = pairs[2 * s], b = pairs[2 * s + 1];
            float L = fmaf(lbar[s], rc[m], lbar[s]);
            float dx = xt[3 * a] - xt[3 * b];
            float dy = xt[3 * a + 1] - xt[3 * b + 1];
            float dz = xt[3 * a + 2] - xt[3 * b + 2];
            float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            float d = sqrtf(d2);
            float r = 1.0f / (d + OR_EPS);
            float C = d - L;
            float lam = (-C) * invK[m];
            float coef = lam * r;
            dp[3 * s] = coef * dx;
            dp[3 * s + 1] = coef * dy;
            dp[3 * s + 2] = coef * dz;
            if (track) {
                float il = 1.0f / lbar[s];
                stress[s] = stress[s] + lam * il;
            }
        }
        /* gather + update (sim_kernel.cu:246-252, 261-268) */
        for (int i = 0; i < nm; ++i) {
            float acc[3] = {0.0f, 0.0f, 0.0f};
            for (int e = deg[i]; e < deg[i + 1]; ++e) {
                int h = inc[e], s = h >> 1;
                for (int c = 0; c < 3; ++c)
                    acc[c] = (h & 1) ? acc[c] - dp[3 * s + c] : acc[c] + dp[3 * s + c];
            }
            for (int c = 0; c < 3; ++c) {
                float xn = xt[3 * i + c] + acc[c];
                float diff = xn - pos[4 * i + c];
                vel[4 * i + c] = (float)((0.99 * (double)diff) / (double)dt);
                pos[4 * i + c] = xn;
            }
        }
        t = t + dt;
    }
    free(deg); free(inc); free(fill); free(xt); free(dp);
}

/* Batch driver.  mass_off / spring_off: n_robots+1 offsets into the flat
 * arrays; pairs are robot-local mass indices.  Robots are independent and
 * are spread over `threads` OpenMP threads (0 = library default). */
int or_xpbd_run(int n_robots, const int64_t* mass_off, float* pos, float* vel,
                const int64_t* spring_off, const uint16_t* pairs,
                const uint8_t* mat, const float* lbar, float* stress,
                const float* table, float dt, float t0, uint32_t steps,
                int track, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int r = 0; r < n_robots; ++r) {
        int64_t m0 = mass_off[r], s0 = spring_off[r];
        xpbd_robot_f32((int)(mass_off[r + 1] - m0), pos + 4 * m0, vel + 4 * m0,
                       (int)(spring_off[r + 1] - s0), pairs + 2 * s0, mat + s0,
                       lbar + s0, stress ? stress + s0 : NULL, table, dt, t0,
                       steps, track && stress);
    }
    return 0;
}

int or_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* FP64 transcription of the same step (libm sin and sqrt, true divisions),
 * used to measure FP32 drift.  State in double, same layout as above. */
static void xpbd_robot_f64(int nm, double* pos, double* vel, int ns,
                           const uint16_t* pairs, const uint8_t* mat,
                           const double* lbar, double* stress,
                           const float* table, double dt, double t0,
                           uint32_t steps, int track) {
    double* xt = (double*)malloc(sizeof(double) * 3 * (size_t)(nm + 1));
    double* acc = (double*)malloc(sizeof(double) * 3 * (size_t)(nm + 1));
    for (uint32_t step = 0; step < steps; ++step) {
        double tn = t0 + dt * (double)step;
        for (int i = 0; i < nm; ++i)
            for (int c = 0; c < 3; ++c) {
                xt[3 * i + c] = pos[4 * i + c] + vel[4 * i + c] * dt;
                acc[3 * i + c] = 0.0;
            }
        for (int s = 0; s < ns; ++s) {
            int m = mat[s];
            if (!m) continue;
            int a = pairs[2 * s], b = pairs[2 * s + 1];
            double k = table[4 * m], dl0 = table[4 * m + 1], om = table[4 * m + 2], ph = table[4 * m + 3];
            double L = lbar[s] * (1.0 + dl0 * sin(om * tn + ph));
            double dx = xt[3 * a] - xt[3 * b], dy = xt[3 * a + 1] - xt[3 * b + 1], dz = xt[3 * a + 2] - xt[3 * b + 2];
            double d = sqrt(dx * dx + dy * dy + dz * dz);
            double K = 2.0 + 1.0 / (k * dt * dt);
            double lam = -(d - L) / K;
            double inv = 1.0 / (d + 1e-12);
            acc[3 * a] += lam * dx * inv; acc[3 * a + 1] += lam * dy * inv; acc[3 * a + 2] += lam * dz * inv;
            acc[3 * b] -= lam * dx * inv; acc[3 * b + 1] -= lam * dy * inv; acc[3 * b + 2] -= lam * dz * inv;
            if (track) stress[s] += lam / lbar[s];
        }
        for (int i = 0; i < nm; ++i)
            for (int c = 0; c < 3; ++c) {
                double xn = xt[3 * i + c] + acc[3 * i + c];
                vel[4 * i + c] = 0.99 * (xn - pos[4 * i + c]) / dt;
                pos[4 * i + c] = xn;
            }
    }
    free(xt); free(acc);
}

int or_xpbd_run_f64(int n_robots, const int64_t* mass_off, double* pos, double* vel,
                    const int64_t* spring_off, const uint16_t* pairs,
                    const uint8_t* mat, const double* lbar, double* stress,
                    const float* table, double dt, double t0, uint32_t steps,
                    int track) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int r = 0; r < n_robots; ++r) {
        int64_t m0 = mass_off[r], s0 = spring_off[r];
        xpbd_robot_f64((int)(mass_off[r + 1] - m0), pos + 4 * m0, vel + 4 * m0,
                       (int)(spring_off[r + 1] - s0), pairs + 2 * s0, mat + s0,
                       lbar + s0, stress ? stress + s0 : NULL, table, dt, t0,
                       steps, track && stress);
    }
    return 0;
}


/* ------------------------------------------------------------------ */
/* Face drag of one surface triangle (water mode), the share of each corner
 * (this library's law after sim_kernel.cu:96-121): mean corner velocity
 * v = (v0 + v1 + v2) * RN(1/3),
 * N = (x1 - x0) x (x2 - x0), A = |N|, n = N * (1/(A + eps)) turned so that
 * v.n > 0, out = coef * A * ((v.n) v + 0.2 |v|^2 n), coef = -rho/6.  Each
 * operation rounds once, in this order. */
static void face_force_f32(const float* x0, const float* x1, const float* x2, const float* v0,
                           const float* v1, const float* v2, float coef, float* out) {
    float v[3], a[3], b[3], u[3];
    for (int q = 0; q < 3; ++q) {
        v[q] = ((v0[q] + v1[q]) + v2[q]) * 0x1.555556p-2f; /* RN(1/3) */
        a[q] = x1[q] - x0[q];
        b[q] = x2[q] - x0[q];
    }
    const float nx = a[1] * b[2] - a[2] * b[1];
    const float ny = a[2] * b[0] - a[0] * b[2];
    const float nz = a[0] * b[1] - a[1] * b[0];
    const float area = sqrtf(fmaf(nx, nx, fmaf(ny, ny, nz * nz)));
    const float r = 1.0f / (area + OR_EPS);
    u[0] = nx * r;
    u[1] = ny * r;
    u[2] = nz * r;
    float vn = fmaf(u[0], v[0], fmaf(u[1], v[1], u[2] * v[2]));
    if (!(vn > 0.0f)) {
        for (int q = 0; q < 3; ++q) u[q] = -u[q];
        vn = -vn;
    }
    const float lift = 0.2f * fmaf(v[0], v[0], fmaf(v[1], v[1], v[2] * v[2]));
    const float c = coef * area;
    for (int q = 0; q < 3; ++q) out[q] = c * fmaf(lift, u[q], vn * v[q]);
}

/* Force modes (no reference code: restated from the paper's Algorithm 1,
 * mercury_fall_2023.pdf section II.B, and the benchmark configurations):
 * Hooke springs F_a = -k (d - L) n, n = (x_a - x_b)/d, L = Lbar (1 + dL0
 * sin(omega t + phi)); per mass, mode 1 (land): gravity -m g along z, a
 * penalty ground below z = 0 with normal force fn = k_floor (-z) and
 * Coulomb friction on the horizontal velocity h = v + (F_h/m) dt the step
 * would reach -- static (F_h = -m v_h / dt) when |h| <= mu_s fn dt / m,
 * else kinetic mu_k fn against h; mode 2 (water): drag -c |v| v.  Then
 * x' = x + v dt + (F/m) dt^2, v' = damping (x' - x)/dt.  Stress accumulates
 * k (d - L)/Lbar.  The same fixed gather order as the reference step.
 * In FP32 the divisions by m and dt are multiplications by the correctly
 * rounded reciprocals 1/m and 1/dt (the law is this library's own, so its
 * rounding is too); only the kinetic friction divides, by |h|.
 * env = {g, floor_stiffness, mu_s, mu_k, drag, damping[, face_drag]}; m = pos.w.
 * Faces (nf triangles, robot-local corners; water only, when face_drag is
 * given): each face with three distinct corners adds face_force_f32 to the
 * force of each corner, after the springs, faces in ascending order. */
static void force_robot_f32(int mode, int nm, float* pos, float* vel, int ns,
                            const uint16_t* pairs, const uint8_t* mat,
                            const float* lbar, float* stress,
                            const float* table, const float* env, float dt, float t0,
                            uint32_t steps, int track, int nf, const uint16_t* faces) {
    int* deg = (int*)calloc((size_t)nm + 1, sizeof(int));
    for (int s = 0; s < ns; ++s) {
        if (!mat[s]) continue;
        deg[pairs[2 * s] + 1]++;
        deg[pairs[2 * s + 1] + 1]++;
    }
    for (int i = 0; i < nm; ++i) deg[i + 1] += deg[i];
    int* inc = (int*)malloc(sizeof(int) * (size_t)(deg[nm] + 1));
    int* fill = (int*)malloc(sizeof(int) * (size_t)(nm + 1));
    memcpy(fill, deg, sizeof(int) * (size_t)nm);
    for (int s = 0; s < ns; ++s) {
        if (!mat[s]) continue;
        inc[fill[pairs[2 * s]]++] = 2 * s;
        inc[fill[pairs[2 * s + 1]]++] = 2 * s + 1;
    }
    for (int i = 0; i < nm; ++i)
        for (int e = deg[i] + 1; e < deg[i + 1]; ++e) {
            int h = inc[e], k = e - 1;
            while (k >= deg[i] && inc_after(inc[k], h, pairs)) { inc[k + 1] = inc[k]; --k; }
            inc[k + 1] = h;
        }
    float* f = (float*)malloc(sizeof(float) * 3 * (size_t)(ns + 1));
    /* per mass: the faces it is a corner of, ascending */
    if (mode != 2 || !faces || env[6] == 0.0f) nf = 0;
    int* fdeg = (int*)calloc((size_t)nm + 1, sizeof(int));
    int* finc = (int*)malloc(sizeof(int) * (3 * (size_t)nf + 1));
    float* ff = (float*)malloc(sizeof(float) * (3 * (size_t)nf + 1));
    for (int q = 0; q < nf; ++q) {
        const uint16_t* c = faces + 3 * q;
        if (c[0] == c[1] || c[0] == c[2] || c[1] == c[2]) continue;
        for (int k = 0; k < 3; ++k) fdeg[c[k] + 1]++;
    }
    for (int i = 0; i < nm; ++i) fdeg[i + 1] += fdeg[i];
    {
        int* ffill = (int*)malloc(sizeof(int) * ((size_t)nm + 1));
        memcpy(ffill, fdeg, sizeof(int) * (size_t)nm);
        for (int q = 0; q < nf; ++q) {
            const uint16_t* c = faces + 3 * q;
            if (c[0] == c[1] || c[0] == c[2] || c[1] == c[2]) continue;
            for (int k = 0; k < 3; ++k) finc[ffill[c[k]]++] = q;
        }
        free(ffill);
    }
    const float fcoef = nf ? (float)(-(double)env[6] / 6.0) : 0.0f;
    float rc[OR_COMPOSITE_COUNT];
    const float g = env[0], kfl = env[1], mus = env[2], muk = env[3], cdrag = env[4], damp = env[5];
    const float inv_dt = 1.0f / dt;
    volatile float t = t0;
    for (uint32_t step = 0; step < steps; ++step) {
        float tn = t;
        for (int m = 0; m < OR_COMPOSITE_COUNT; ++m) {
            float arg = fmaf(table[4 * m + 2], tn, table[4 * m + 3]);
            rc[m] = table[4 * m + 1] * (float)or_sin((double)arg);
        }
        for (int s = 0; s < ns; ++s) {
            int m = mat[s];
            if (!m) continue;
            int a = pairs[2 * s], b = pairs[2 * s + 1];
            float L = fmaf(lbar[s], rc[m], lbar[s]);
            float dx = pos[4 * a] - pos[4 * b];
            float dy = pos[4 * a + 1] - pos[4 * b + 1];
            float dz = pos[4 * a + 2] - pos[4 * b + 2];
            float d = sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
            float r = 1.0f / (d + OR_EPS);
            float lam = (-(d - L)) * table[4 * m];
            float coef = lam * r;
            f[3 * s] = coef * dx;
            f[3 * s + 1] = coef * dy;
            f[3 * s + 2] = coef * dz;
            if (track) stress[s] = stress[s] + (-lam) * (1.0f / lbar[s]);
        }
        for (int q = 0; q < nf; ++q) {
            const uint16_t* c = faces + 3 * q;
            if (c[0] == c[1] || c[0] == c[2] || c[1] == c[2]) continue;
            face_force_f32(pos + 4 * c[0], pos + 4 * c[1], pos + 4 * c[2], vel + 4 * c[0], vel + 4 * c[1],
                           vel + 4 * c[2], fcoef, ff + 3 * q);
        }
        for (int i = 0; i < nm; ++i) {
            float F[3] = {0.0f, 0.0f, 0.0f};
            for (int e = deg[i]; e < deg[i + 1]; ++e) {
                int h = inc[e], s = h >> 1;
                for (int c = 0; c < 3; ++c) F[c] = (h & 1) ? F[c] - f[3 * s + c] : F[c] + f[3 * s + c];
            }
            for (int e = fdeg[i]; e < fdeg[i + 1]; ++e)
                for (int c = 0; c < 3; ++c) F[c] = F[c] + ff[3 * finc[e] + c];
            float* x = pos + 4 * i;
            float* v = vel + 4 * i;
            float mass = x[3];
            float inv_m = 1.0f / mass;
            if (mode == 1) {
                F[2] = F[2] - mass * g;
                if (x[2] < 0.0f) {
                    float fn = kfl * (-x[2]);
                    F[2] = F[2] + fn;
                    float hx = v[0] + (F[0] * inv_m) * dt;
                    float hy = v[1] + (F[1] * inv_m) * dt;
                    float hs = sqrtf(fmaf(hx, hx, hy * hy));
                    float budget = (fn * inv_m) * dt;
                    if (hs <= mus * budget) {
                        F[0] = ((-mass) * v[0]) * inv_dt;
                        F[1] = ((-mass) * v[1]) * inv_dt;
                    } else {
                        float sc = (muk * fn) / hs;
                        F[0] = F[0] - sc * hx;
                        F[1] = F[1] - sc * hy;
                    }
                }
            } else {
                float sp = sqrtf(fmaf(v[0], v[0], fmaf(v[1], v[1], v[2] * v[2])));
                float c = cdrag * sp;
                for (int q = 0; q < 3; ++q) F[q] = F[q] - c * v[q];
            }
            float dt2 = dt * dt;
            for (int q = 0; q < 3; ++q) {
                float xn = (x[q] + v[q] * dt) + (F[q] * inv_m) * dt2;
                v[q] = damp * ((xn - x[q]) * inv_dt);
                x[q] = xn;
            }
        }
        t = t + dt;
    }
    free(deg); free(inc); free(fill); free(f);
    free(fdeg); free(finc); free(ff);
}

/* One face's share per corner (face_force_f32), for tests. */
void or_face_force(const float* x0, const float* x1, const float* x2, const float* v0, const float* v1,
                   const float* v2, float coef, float* out) {
    face_force_f32(x0, x1, x2, v0, v1, v2, coef, out);
}

/* Face forces of one robot: per mass the sum of the shares of its faces
 * (three distinct corners), faces in ascending order -- the term the water
 * step adds after the springs.  out: 3 per mass. */
void or_face_forces(int n_mass, const float* pos4, const float* vel4, int n_face, const uint16_t* faces3,
                    float coef, float* out) {
    memset(out, 0, sizeof(float) * 3 * (size_t)n_mass);
    for (int f = 0; f < n_face; ++f) {
        const uint16_t* c = faces3 + 3 * f;
        if (c[0] == c[1] || c[0] == c[2] || c[1] == c[2]) continue;
        float F[3];
        face_force_f32(pos4 + 4 * c[0], pos4 + 4 * c[1], pos4 + 4 * c[2], vel4 + 4 * c[0], vel4 + 4 * c[1],
                       vel4 + 4 * c[2], coef, F);
        for (int k = 0; k < 3; ++k)
            for (int q = 0; q < 3; ++q) out[3 * c[k] + q] = out[3 * c[k] + q] + F[q];
    }
}

/* face_off / faces may be NULL (no faces); with faces, env has 7 entries. */
int or_force_run(int mode, int n_robots, const int64_t* mass_off, float* pos, float* vel,
                 const int64_t* spring_off, const uint16_t* pairs, const uint8_t* mat,
                 const float* lbar, float* stress, const float* table, const float* env,
                 float dt, float t0, uint32_t steps, int track, int threads,
                 const int64_t* face_off, const uint16_t* faces) {
    if (mode != 1 && mode != 2) return -1;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int r = 0; r < n_robots; ++r) {
        int64_t m0 = mass_off[r], s0 = spring_off[r];
        const int64_t f0 = face_off ? face_off[r] : 0;
        const int nf = face_off ? (int)(face_off[r + 1] - f0) : 0;
        force_robot_f32(mode, (int)(mass_off[r + 1] - m0), pos + 4 * m0, vel + 4 * m0,
                        (int)(spring_off[r + 1] - s0), pairs + 2 * s0, mat + s0, lbar + s0,
                        stress ? stress + s0 : NULL, table, env, dt, t0, steps, track && stress,
                        nf, faces ? faces + 3 * f0 : NULL);
    }
    return 0;
}

/* FP64 transcription of the force modes (libm sin/sqrt), for drift. */
static void force_robot_f64(int mode, int nm, double* pos, double* vel, int ns,
                            const uint16_t* pairs, const uint8_t* mat, const double* lbar,
                            const float* table, const double* env, double dt, double t0,
                            uint32_t steps) {
    double* F = (double*)malloc(sizeof(double) * 3 * (size_t)(nm + 1));
    const double g = env[0], kfl = env[1], mus = env[2], muk = env[3], cdrag = env[4], damp = env[5];
    for (uint32_t step = 0; step < steps; ++step) {
        double tn = t0 + dt * (double)step;
        memset(F, 0, sizeof(double) * 3 * (size_t)nm);
        for (int s = 0; s < ns; ++s) {
            int m = mat[s];
            if (!m) continue;
            int a = pairs[2 * s], b = pairs[2 * s + 1];
            double L = lbar[s] * (1.0 + (double)table[4 * m + 1] * sin((double)table[4 * m + 2] * tn + (double)table[4 * m + 3]));
            double dx = pos[4 * a] - pos[4 * b], dy = pos[4 * a + 1] - pos[4 * b + 1], dz = pos[4 * a + 2] - pos[4 * b + 2];
            double d = sqrt(dx * dx + dy * dy + dz * dz);
            double c = -(double)table[4 * m] * (d - L) / (d + 1e-12);
            F[3 * a] += c * dx; F[3 * a + 1] += c * dy; F[3 * a + 2] += c * dz;
            F[3 * b] -= c * dx; F[3 * b + 1] -= c * dy; F[3 * b + 2] -= c * dz;
        }
        for (int i = 0; i < nm; ++i) {
            double* x = pos + 4 * i;
            double* v = vel + 4 * i;
            double* Fi = F + 3 * i;
            double mass = x[3];
            if (mode == 1) {
                Fi[2] -= mass * g;
                if (x[2] < 0.0) {
                    double fn = kfl * (-x[2]);
                    Fi[2] += fn;
                    double hx = v[0] + Fi[0] / mass * dt, hy = v[1] + Fi[1] / mass * dt;
                    double hs = sqrt(hx * hx + hy * hy);
                    if (hs <= mus * fn / mass * dt) {
                        Fi[0] = -mass * v[0] / dt;
                        Fi[1] = -mass * v[1] / dt;
                    } else {
                        Fi[0] -= muk * fn * hx / hs;
                        Fi[1] -= muk * fn * hy / hs;
                    }
                }
            } else {
                double sp = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                for (int q = 0; q < 3; ++q) Fi[q] -= cdrag * sp * v[q];
            }
            for (int q = 0; q < 3; ++q) {
                double xn = x[q] + v[q] * dt + Fi[q] / mass * dt * dt;
                v[q] = damp * (xn - x[q]) / dt;
                x[q] = xn;
            }
        }
    }
    free(F);
}

int or_force_run_f64(int mode, int n_robots, const int64_t* mass_off, double* pos, double* vel,
                     const int64_t* spring_off, const uint16_t* pairs, const uint8_t* mat,
                     const double* lbar, const float* table, const double* env, double dt,
                     double t0, uint32_t steps) {
    if (mode != 1 && mode != 2) return -1;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int r = 0; r < n_robots; ++r) {
        int64_t m0 = mass_off[r], s0 = spring_off[r];
        force_robot_f64(mode, (int)(mass_off[r + 1] - m0), pos + 4 * m0, vel + 4 * m0,
                        (int)(spring_off[r + 1] - s0), pairs + 2 * s0, mat + s0, lbar + s0,
                        table, env, dt, t0, steps);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Centre of mass of the non-air masses of each robot.
 *
 * or_com_device: the fixed reduction order of the CUDA kernels -- 32 lanes,
 * lane l sums masses l, l+32, ... in double, then an xor butterfly over
 * offsets 16, 8, 4, 2, 1; mean = sum / count, rounded to float.
 *
 * or_com_reference: SoftBody::updateCOM (SoftBody.cpp:112-121), a float
 * running mean mean += (p - mean) / (i + 1). */
void or_com_device(int n_robots, const int64_t* mass_off, const float* pos,
                   const uint8_t* mass_mat, float* com) {
    for (int r = 0; r < n_robots; ++r) {
        for (int c = 0; c < 3; ++c) {
            double lane[32];
            long cnt[32];
            for (int l = 0; l < 32; ++l) { lane[l] = 0.0; cnt[l] = 0; }
            int64_t n = mass_off[r + 1] - mass_off[r];
            for (int64_t i = 0; i < n; ++i) {
                int64_t g = mass_off[r] + i;
                if (!mass_mat[g]) continue;
                lane[i & 31] += (double)pos[4 * g + c];
                cnt[i & 31] += 1;
            }
            for (int off = 16; off >= 1; off >>= 1) {
                double nl[32];
                long nc[32];
                for (int l = 0; l < 32; ++l) { nl[l] = lane[l] + lane[l ^ off]; nc[l] = cnt[l] + cnt[l ^ off]; }
                for (int l = 0; l < 32; ++l) { lane[l] = nl[l]; cnt[l] = nc[l]; }
            }
            com[3 * r + c] = cnt[0] ? (float)(lane[0] / (double)cnt[0]) : 0.0f;
        }
    }
}

void or_com_reference(int n_robots, const int64_t* mass_off, const float* pos,
                      const uint8_t* mass_mat, float* com) {
    for (int r = 0; r < n_robots; ++r) {
        float mean[3] = {0.0f, 0.0f, 0.0f};
        volatile float i = 0.0f;
        for (int64_t g = mass_off[r]; g < mass_off[r + 1]; ++g) {
            if (!mass_mat[g]) continue;
            float den = i + 1.0f;
            for (int c = 0; c < 3; ++c) {
                float d = (pos[4 * g + c] - mean[c]) * 1.0f;
                mean[c] = mean[c] + d / den;
            }
            i = i + 1.0f;
        }
        for (int c = 0; c < 3; ++c) com[3 * r + c] = mean[c];
    }
}

/* ------------------------------------------------------------------ */
/* Development: replace each robot's highest-stress springs with springs
 * between random mass pairs (Simulator::Devo, Simulator.cu:640-668;
 * replaceSprings, devo_kernel.cu:81-168).
 *
 * Per robot r with n springs and m masses:
 *   1. rank the springs by accumulated stress, descending (the reference's
 *      CUB segmented radix sort, Simulator.cu:597-631), ties by ascending
 *      spring index (the radix sort is stable).  Order of the floats: -0 and
 *      +0 are equal; a NaN with the sign bit clear ranks above +inf, one with
 *      it set below -inf.
 *   2. replace the springs of ranks [lo, hi): lo = 0 and hi = min(k, n); or,
 *      with the "reference ranks" flag, lo = min(r k, n), hi = min(r k + k, n)
 *      -- the window the reference's indexing actually selects
 *      (devo_kernel.cu:112-116 offsets the global replacement index into
 *      robot r's sorted segment); ranks past the robot's own springs are
 *      dropped instead of spilling into the next robot's.  Robots with fewer
 *      than two masses are left alone.
 *   3. the spring of rank lo + j gets the pair (a, b) drawn by or_devo_pair
 *      for (seed, r, j), the composite material of the two masses
 *      (devo_kernel.cu:131-148), and the mean length
 *      |x_a - x_b| / (1 + dL0 sin(omega t + phi)) of that material at clock t
 *      (devo_kernel.cu:150-157), with the arithmetic of the step (fmaf phase,
 *      or_sin, sqrtf of the fmaf dot product, correctly rounded division).
 *      Stresses are left as they are (the reference does not reset them).
 *
 * Random pairs: the reference draws them with cuRAND (XORWOW) in a kernel
 * whose loop stride makes blocks overwrite one another (devo_kernel.cu:56-73),
 * so its pairs are not reproducible.  This build uses a counter-based
 * generator instead: SplitMix64's output function (Steele, Lea and Flood,
 * "Fast splittable pseudorandom number generators", OOPSLA 2014) over
 * (seed, robot, j, draw), mapped to [0, m) by Lemire's multiply-shift.  a is
 * draw 0; b is draw 1, redrawn (draws 2..63) while it equals a, then a+1 mod
 * m.
 *
 * out (optional, 4 words per replaced spring, robot-major, rank order):
 * global spring index, a | b << 16, material, mean-length bits.  Returns the
 * number of springs replaced. */
#define OR_DEVO_REFERENCE_RANKS 1u

static uint64_t or_mix64(uint64_t z) {
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static uint32_t or_devo_draw(uint64_t key, uint32_t j, uint32_t n, uint32_t m) {
    uint64_t u = or_mix64(key + 0xD1B54A32D192ED03ULL * ((((uint64_t)j << 8) | n) + 1));
    return (uint32_t)(((u >> 32) * (uint64_t)m) >> 32);
}

void or_devo_pair(uint64_t seed, uint32_t robot, uint32_t j, uint32_t m, uint32_t* a, uint32_t* b) {
    uint64_t key = or_mix64(seed + 0x9E3779B97F4A7C15ULL * ((uint64_t)robot + 1));
    uint32_t x = or_devo_draw(key, j, 0, m), y = or_devo_draw(key, j, 1, m);
    for (uint32_t n = 2; y == x && n < 64; ++n) y = or_devo_draw(key, j, n, m);
    if (y == x) y = (x + 1) % m;
    *a = x;
    *b = y;
}

/* Key whose ascending order is descending stress. */
uint32_t or_stress_key(float s) {
    uint32_t u;
    memcpy(&u, &s, 4);
    if (u == 0x80000000u) u = 0;
    uint32_t ord = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ~ord;
}

static int or_cmp_u64(const void* x, const void* y) {
    uint64_t a = *(const uint64_t*)x, b = *(const uint64_t*)y;
    return a < b ? -1 : (a > b);
}

long or_devo(int n_robots, const int64_t* mass_off, const float* pos, const uint8_t* mass_mat,
             const int64_t* spring_off, uint16_t* pairs, uint8_t* mat, float* lbar,
             const float* stress, const float* table, float t, uint32_t k, uint64_t seed,
             uint32_t flags, uint32_t* out) {
    long total = 0;
    for (int r = 0; r < n_robots; ++r) {
        const int64_t m0 = mass_off[r], s0 = spring_off[r];
        const uint32_t m = (uint32_t)(mass_off[r + 1] - m0), n = (uint32_t)(spring_off[r + 1] - s0);
        if (m < 2 || n == 0 || k == 0) continue;
        uint64_t lo = 0, hi = k < n ? k : n;
        if (flags & OR_DEVO_REFERENCE_RANKS) {
            lo = (uint64_t)r * k;
            hi = lo + k;
            if (lo > n) lo = n;
            if (hi > n) hi = n;
        }
        if (hi <= lo) continue;
        uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * n);
        for (uint32_t i = 0; i < n; ++i) keys[i] = ((uint64_t)or_stress_key(stress[s0 + i]) << 32) | i;
        qsort(keys, n, sizeof(uint64_t), or_cmp_u64);
        for (uint64_t q = lo; q < hi; ++q) {
            const uint32_t j = (uint32_t)(q - lo);
            const int64_t s = s0 + (int64_t)(uint32_t)keys[q];
            uint32_t a, b;
            or_devo_pair(seed, (uint32_t)r, j, m, &a, &b);
            const int id = or_composite_id(mass_mat[m0 + a], mass_mat[m0 + b]);
            const float* pa = pos + 4 * (m0 + a);
            const float* pb = pos + 4 * (m0 + b);
            float dx = pa[0] - pb[0], dy = pa[1] - pb[1], dz = pa[2] - pb[2];
            float d = sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
            float arg = fmaf(table[4 * id + 2], t, table[4 * id + 3]);
            float sn = (float)or_sin((double)arg);
            float rc = table[4 * id + 1] * sn;
            float den = 1.0f + rc;
            float L = d / den;
            pairs[2 * s] = (uint16_t)a;
            pairs[2 * s + 1] = (uint16_t)b;
            mat[s] = (uint8_t)id;
            lbar[s] = L;
            if (out) {
                uint32_t* o = out + 4 * total;
                o[0] = (uint32_t)s;
                o[1] = a | (b << 16);
                o[2] = (uint32_t)id;
                memcpy(&o[3], &L, 4);
            }
            ++total;
        }
        free(keys);
    }
    return total;
}
