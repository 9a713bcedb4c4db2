// fluid_oracle.cpp — CPU oracle for the DFSPH substep (TEST INFRASTRUCTURE).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline load this
// library; the product never links it. Every function cites the reference
// file:line it restates (paths inside Screendead/fluid-simulation-app).
//
// Arithmetic rules, so the CUDA path can be held to it bit for bit:
//   - IEEE binary32, round to nearest, no FMA contraction (-ffp-contract=off);
//   - WGSL expressions keep their left-to-right association;
//   - dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z; mix(a, b, t) = a*(1-t) + b*t;
//   - exp inside a kernel is or_exp below (a fixed Cody-Waite + Taylor
//     evaluation); exp of a per-substep constant is libm expf on the host;
//   - every global sum is exact: per-particle FP64 terms in 2^-28 fixed point,
//     summed as 64-bit integers, so the total does not depend on order.
//
// The substep's arithmetic type is Real: float, the oracle above. Compiled
// with -DOR_REAL=double the same source is the FP64 oracle (same algorithm,
// same float constants, every operation in double) that the FP32 path's
// errors are stated against; its C API still takes and returns float, plus
// or_sim_get_state64 for the double state. (The tracer and field helpers
// stay float in both.)
#include "fluid_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef OR_REAL
#define OR_REAL float
#endif

namespace {

typedef OR_REAL Real;

constexpr float kPi = 3.14159265358979323846f;
constexpr float kRestDensity = 998.2f;                // sim.rs:6
constexpr float kWorldScale = 4.0f;                   // lib.rs:13
constexpr float kSlabDepth = kWorldScale * 0.00765f;  // sim.rs:10

// sim_solve.wgsl:84-172
constexpr float XSPH_RATE = 6.0f;
constexpr float TOUCH_RATE = 40.0f;
constexpr float LENS_RATE = 20.0f;
constexpr float K_NEAR = 3000.0f;
constexpr float DYNAMIC_VISCOSITY = 1.002e-3f;
constexpr float HEAT_CAPACITY = 4184.0f;
constexpr float CONDUCTIVITY = 0.598f;
constexpr float EXPANSION = 2.07e-4f;
constexpr float SIGMA_WATER = 0.0728f;
constexpr float LATTICE_SIGMA = 0.8665f;
constexpr float COS_CONTACT = -0.342f;
// sim_tracers.wgsl:39-52
constexpr float FIXED = 65536.0f;
constexpr float TAU = 3.0f;
constexpr float TAU_STRAY = 0.25f;
constexpr float T_CHARGE = 4.0f;
constexpr float HUGE_F = 1e30f;  // sim_solve.wgsl:792

struct V3 {
    Real x, y, z;
};
inline V3 v3(Real x, Real y, Real z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline V3 operator*(Real s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline V3 operator*(V3 a, Real s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 operator/(V3 a, Real s) { return v3(a.x / s, a.y / s, a.z / s); }
inline Real dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Real length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// WGSL max / min / clamp / mix (finite inputs), in the wider of the argument
// types (float with float is the float expression itself).
template <class A, class B>
inline auto fmaxw(A a, B b) -> decltype(a + b) {
    typedef decltype(a + b) T;
    return (T)a > (T)b ? (T)a : (T)b;
}
template <class A, class B>
inline auto fminw(A a, B b) -> decltype(a + b) {
    typedef decltype(a + b) T;
    return (T)a < (T)b ? (T)a : (T)b;
}
template <class A, class B, class C>
inline auto clampw(A e, B lo, C hi) -> decltype(e + lo + hi) {
    return fminw(fmaxw(e, lo), hi);
}
template <class A, class B, class C>
inline auto mixw(A a, B b, C t) -> decltype(a + b + t) {
    typedef decltype(a + b + t) T;
    return (T)a * ((T)1 - (T)t) + (T)b * (T)t;
}
inline V3 load3(const float *p) { return v3(p[0], p[1], p[2]); }
inline V3 load3(const double *p) { return v3((Real)p[0], (Real)p[1], (Real)p[2]); }

// exp for per-particle arguments, shared definition with the CUDA path:
// x = k ln2 + r by Cody-Waite (ln2 split in a 16-bit head and a tail),
// e^r by the degree-7 Taylor polynomial in Horner form, then 2^k by
// exponent bits. Relative error under 2e-7 on [-87, 88].
float or_exp(float x) {
    if (!(x > -87.0f)) return 0.0f;
    if (x > 88.0f) x = 88.0f;
    const float kf = std::rint(x * 1.44269504f);
    float r = x - kf * 0.693145752f;
    r = r - kf * 1.42860677e-6f;
    float p = 1.98412698e-4f;  // 1/5040
    p = p * r + 1.38888889e-3f;
    p = p * r + 8.33333333e-3f;
    p = p * r + 4.16666667e-2f;
    p = p * r + 1.66666667e-1f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    const int k = (int)kf;
    uint32_t bits;
    float scale;
    bits = (uint32_t)(k + 127) << 23;
    std::memcpy(&scale, &bits, 4);
    return p * scale;
}

inline float exp_r(float x) { return or_exp(x); }

inline uint32_t pcg(uint32_t x) {  // sim_tracers.wgsl:54-58
    uint32_t h = x * 747796405u + 2891336453u;
    h = ((h >> ((h >> 28u) + 4u)) ^ h) * 277803737u;
    return (h >> 22u) ^ h;
}

// 64-bit fixed-point accumulation of non-negative FP64 terms: 2^-28 units,
// each term capped at 16, so no sum over 2^32 particles can wrap.
constexpr double kFixedScale = 268435456.0;
inline int64_t fx(double term) {
    if (!(term > 0.0)) return 0;
    if (term > 16.0) term = 16.0;
    return (int64_t)std::llrint(term * kFixedScale);
}

// exp of a per-particle argument: or_exp in the float oracle, libm in the
// FP64 one.
inline float exp_r(float x);
inline double exp_r(double x) { return std::exp(x); }

// Slabs per cell along x in a simulation's grid keys; the library's
// fluid_sim_grid_slabs() must equal it.
#ifndef OR_SIM_SLABS
#define OR_SIM_SLABS 4
#endif
constexpr uint32_t kSimSlabs = OR_SIM_SLABS;

// WGSL's f32 -> u32 saturating conversion, and the grid's cell and stable
// counting sort over positions of either width (sim.rs:38-44;
// sim_grid.wgsl:36-58; sim_scan.wgsl:97-120).
template <class T>
inline uint32_t sat_u32_t(T v) {
    if (!(v > (T)0.0f)) return 0u;
    if (v >= (T)4294967296.0f) return 0xffffffffu;
    return (uint32_t)v;
}
template <class T>
uint32_t cell_of_t(const OrGrid *g, const T *pos) {
    uint32_t c[3];
    for (int i = 0; i < 3; ++i) {
        const uint32_t u = sat_u32_t((pos[i] - g->min[i]) / g->cell);
        c[i] = u < g->dims[i] - 1u ? u : g->dims[i] - 1u;
    }
    return (c[2] * g->dims[1] + c[1]) * g->dims[0] + c[0];
}
// Slab of a cell along x (the cell cut into `slabs` equal slabs across the
// axis): the number of slab boundaries at or below the position's offset in
// its cell. A NaN or negative offset gives 0.
template <class T>
uint32_t x_slab_t(const OrGrid *g, const T *pos, uint32_t cx, uint32_t slabs) {
    const T off = pos[0] - (g->min[0] + (T)(float)cx * g->cell);
    uint32_t s = 0;
    for (uint32_t k = 1; k < slabs; ++k) s += off >= (T)(g->cell * ((float)k / (float)slabs)) ? 1u : 0u;
    return s;
}
// The stable counting sort by key; with slabs > 1 the key is cell * slabs +
// the x slab, so each cell's slots are in slab order (one of the orders the
// reference's atomic scatter can produce) and starts has cells * slabs + 1
// entries.
template <class T>
void grid_build_t(const OrGrid *g, const T *pos4, uint32_t n, uint32_t *keys, uint32_t *starts,
                  uint32_t *perm, uint32_t slabs = 1) {
    const uint32_t cells = g->dims[0] * g->dims[1] * g->dims[2] * slabs;
    std::vector<uint32_t> counts(cells, 0u);
    std::vector<uint32_t> k(n);
    for (uint32_t i = 0; i < n; ++i) {
        const T *p = pos4 + 4 * (size_t)i;
        k[i] = cell_of_t(g, p);
        if (slabs > 1) k[i] = k[i] * slabs + x_slab_t(g, p, k[i] % g->dims[0], slabs);
        counts[k[i]]++;
    }
    uint32_t run = 0;
    for (uint32_t c = 0; c < cells; ++c) {
        starts[c] = run;
        run += counts[c];
    }
    starts[cells] = run;
    for (uint32_t c = 0; c < cells; ++c) counts[c] = starts[c];
    for (uint32_t i = 0; i < n; ++i) perm[counts[k[i]]++] = i;
    if (keys) std::memcpy(keys, k.data(), sizeof(uint32_t) * n);
}

// A field of the substep as float.
template <class V>
void copy_out(void *out, const V &v) {
    float *o = (float *)out;
    for (size_t k = 0; k < v.size(); ++k) o[k] = (float)v[k];
}

// The wall and wedge polynomials (sim_solve.wgsl:213-235, :249-293, :334-340)
// over the substep's Real; the exported float functions below are the
// float instances.
template <class T>
T wall_density_t(T t) {
    if (t >= 2.0f) return 0.0f;
    const T t3 = t * t * t;
    if (t < 1.0f) return 0.5f - 0.7f * t + t3 * (1.0f / 3.0f + t * t * (-0.15f + 0.05f * t));
    return 8.0f / 15.0f - 0.8f * t + t3 * (2.0f / 3.0f + t * (-0.5f + t * (0.15f - t / 60.0f)));
}
template <class T>
T wall_gradient_t(T t) {
    if (t >= 2.0f) return 0.0f;
    const T t2 = t * t;
    if (t < 1.0f) return 0.7f + t2 * (-1.0f + t2 * (0.75f - t * 0.3f));
    return 0.8f + t2 * (-2.0f + t * (2.0f + t * (-0.75f + t * 0.1f)));
}
template <class T>
T wedge_t(T t1, T t2) {
    if (t1 * t1 + t2 * t2 >= 4.0f) return 0.0f;
    return (2.5005807e-01f +
            t2 * (-3.4681153e-01f +
                  t2 * (-4.0986882e-02f +
                        t2 * (3.0301620e-01f +
                              t2 * (-1.9202736e-01f + t2 * (4.6947582e-02f + t2 * (-3.8543515e-03f))))))) +
           t1 * ((-3.4681153e-01f +
                  t2 * (4.8587248e-01f +
                        t2 * (1.0092180e-02f +
                              t2 * (-2.9978363e-01f + t2 * (1.5320335e-01f + t2 * (-2.2544282e-02f)))))) +
                 t1 * ((-4.0986882e-02f +
                        t2 * (1.0092180e-02f +
                              t2 * (-5.4145610e-02f + t2 * (7.9597369e-02f + t2 * (-2.3350373e-02f))))) +
                       t1 * ((3.0301620e-01f +
                              t2 * (-2.9978363e-01f + t2 * (7.9597369e-02f + t2 * (-8.2431946e-03f)))) +
                             t1 * ((-1.9202736e-01f + t2 * (1.5320335e-01f + t2 * (-2.3350373e-02f))) +
                                   t1 * ((4.6947582e-02f + t2 * (-2.2544282e-02f)) +
                                         t1 * (-3.8543515e-03f))))));
}
template <class T>
T wedge_d_t(T t1, T t2) {
    if (t1 * t1 + t2 * t2 >= 4.0f) return 0.0f;
    return (-3.4611994e-01f +
            t2 * (4.4757673e-01f +
                  t2 * (1.1932939e-01f +
                        t2 * (-4.6460101e-01f +
                              t2 * (2.7637253e-01f + t2 * (-6.2846025e-02f + t2 * (4.3871652e-03f))))))) +
           t1 * ((-6.3622823e-02f +
                  t2 * (2.0521006e-01f +
                        t2 * (-3.7311339e-01f +
                              t2 * (3.7508155e-01f + t2 * (-1.6629713e-01f + t2 * (2.5030129e-02f)))))) +
                 t1 * ((7.8352497e-01f +
                        t2 * (-1.2658344e+00f +
                              t2 * (5.8898945e-01f + t2 * (-1.0772903e-01f + t2 * (1.3535777e-02f))))) +
                       t1 * ((-4.9470084e-01f +
                              t2 * (9.1302071e-01f + t2 * (-3.4330355e-01f + t2 * (2.4034609e-02f)))) +
                             t1 * ((-2.5605481e-02f + t2 * (-2.0067981e-01f + t2 * (5.9854468e-02f))) +
                                   t1 * ((8.8898623e-02f + t2 * (3.9914838e-03f)) +
                                         t1 * (-1.7788321e-02f))))));
}
template <class T>
T wall_adhesion_t(T t) {
    const T u = clampw((T)2.0f - t, (T)0.0f, (T)2.0f);
    return u * u *
           (1.7847015e-3f +
            u * (3.3392196e-3f + u * (-4.3394677e-3f + u * (1.6711868e-3f + u * (-2.1788750e-4f)))));
}

}  // namespace

extern "C" {

float or_slab_depth(void) { return kSlabDepth; }
float or_rest_density(void) { return kRestDensity; }

// sim.rs:318-323
uint32_t or_hash(uint32_t x) {
    uint32_t h = x * 0x9E3779B9u;
    h ^= h >> 16;
    h = h * 0x85EBCA6Bu;
    return h ^ (h >> 13);
}

// sim.rs:49-60
float or_kernel(float r, float h) {
    const float q = r / h;
    const float sigma = 1.0f / (kPi * h * h * h);
    if (q < 1.0f) return sigma * (1.0f - 1.5f * q * q * (1.0f - 0.5f * q));
    if (q < 2.0f) {
        const float t = 2.0f - q;
        return sigma * 0.25f * t * t * t;
    }
    return 0.0f;
}

// sim_solve.wgsl:213-222 (the runtime copy; sim.rs:261-272 is the same
// polynomial in a different association and is checked by the tests)
float or_wall_density(float t) { return wall_density_t<float>(t); }

// sim_solve.wgsl:226-235
float or_wall_gradient(float t) { return wall_gradient_t<float>(t); }

// sim.rs:296-316 (FP64, the tests' copy)
double or_wedge64(double t1, double t2) {
    if (t1 * t1 + t2 * t2 >= 4.0) return 0.0;
    return (2.5005807e-01 +
            t2 * (-3.4681153e-01 +
                   t2 * (-4.0986882e-02 +
                         t2 * (3.0301620e-01 +
                               t2 * (-1.9202736e-01 + t2 * (4.6947582e-02 + t2 * (-3.8543515e-03))))))) +
           t1 * ((-3.4681153e-01 +
                  t2 * (4.8587248e-01 +
                        t2 * (1.0092180e-02 +
                              t2 * (-2.9978363e-01 + t2 * (1.5320335e-01 + t2 * (-2.2544282e-02)))))) +
                 t1 * ((-4.0986882e-02 +
                        t2 * (1.0092180e-02 +
                              t2 * (-5.4145610e-02 + t2 * (7.9597369e-02 + t2 * (-2.3350373e-02))))) +
                       t1 * ((3.0301620e-01 +
                              t2 * (-2.9978363e-01 + t2 * (7.9597369e-02 + t2 * (-8.2431946e-03)))) +
                             t1 * ((-1.9202736e-01 + t2 * (1.5320335e-01 + t2 * (-2.3350373e-02))) +
                                   t1 * ((4.6947582e-02 + t2 * (-2.2544282e-02)) +
                                         t1 * (-3.8543515e-03))))));
}

// sim.rs:571-592 (the test copy of the shader's wedge_d)
double or_wedge_d64(double t1, double t2) {
    if (t1 * t1 + t2 * t2 >= 4.0) return 0.0;
    return (-3.4611994e-01 +
            t2 * (4.4757673e-01 +
                  t2 * (1.1932939e-01 +
                        t2 * (-4.6460101e-01 +
                              t2 * (2.7637253e-01 + t2 * (-6.2846025e-02 + t2 * (4.3871652e-03))))))) +
           t1 * ((-6.3622823e-02 +
                  t2 * (2.0521006e-01 +
                        t2 * (-3.7311339e-01 +
                              t2 * (3.7508155e-01 + t2 * (-1.6629713e-01 + t2 * (2.5030129e-02)))))) +
                 t1 * ((7.8352497e-01 +
                        t2 * (-1.2658344e+00 +
                              t2 * (5.8898945e-01 + t2 * (-1.0772903e-01 + t2 * (1.3535777e-02))))) +
                       t1 * ((-4.9470084e-01 +
                              t2 * (9.1302071e-01 + t2 * (-3.4330355e-01 + t2 * (2.4034609e-02)))) +
                             t1 * ((-2.5605481e-02 + t2 * (-2.0067981e-01 + t2 * (5.9854468e-02))) +
                                   t1 * ((8.8898623e-02 + t2 * (3.9914838e-03)) +
                                         t1 * (-1.7788321e-02))))));
}

// sim.rs:700-706 (the test copy of the shader's wall_adhesion)
double or_wall_adhesion64(double t) {
    double u = 2.0 - t;
    u = u < 0.0 ? 0.0 : (u > 2.0 ? 2.0 : u);
    return u * u *
           (1.7847015e-3 +
            u * (3.3392196e-3 + u * (-4.3394677e-3 + u * (1.6711868e-3 + u * (-2.1788750e-4)))));
}

// sim_solve.wgsl:249-270
float or_wedge(float t1, float t2) { return wedge_t<float>(t1, t2); }

// sim_solve.wgsl:272-293
float or_wedge_d(float t1, float t2) { return wedge_d_t<float>(t1, t2); }

// sim_solve.wgsl:334-340
float or_wall_adhesion(float t) { return wall_adhesion_t<float>(t); }

// sim.rs:65-72
void or_lattice_dims(float spacing, const float extent[2], float fill, uint32_t out[3]) {
    const float size[3] = {2.0f * extent[0] - spacing, (2.0f * extent[1] - spacing) * fill,
                           kSlabDepth - spacing};
    for (int i = 0; i < 3; ++i) {
        const float v = size[i] / spacing;
        uint32_t n = v <= 0.0f ? 0u : (uint32_t)v;
        out[i] = n < 1u ? 1u : n;
    }
}

// sim.rs:77-100
uint32_t or_seed_slab(float spacing, const float extent[2], float fill, float *out4) {
    uint32_t n[3];
    or_lattice_dims(spacing, extent, fill, n);
    const uint32_t count = n[0] * n[1] * n[2];
    if (!out4) return count;
    const float origin[3] = {-0.5f * (float)n[0] * spacing, -extent[1] + 0.5f * spacing,
                             -0.5f * (float)n[2] * spacing};
    auto jitter = [](uint32_t h) { return ((float)h / 4294967295.0f - 0.5f) * 0.2f; };
    for (uint32_t iz = 0; iz < n[2]; ++iz)
        for (uint32_t iy = 0; iy < n[1]; ++iy)
            for (uint32_t ix = 0; ix < n[0]; ++ix) {
                const uint32_t i = (iz * n[1] + iy) * n[0] + ix;
                float *o = out4 + 4 * (size_t)i;
                o[0] = origin[0] + ((float)ix + 0.5f + jitter(or_hash(i * 3))) * spacing;
                o[1] = origin[1] + ((float)iy + jitter(or_hash(i * 3 + 1))) * spacing;
                o[2] = origin[2] + ((float)iz + 0.5f + jitter(or_hash(i * 3 + 2))) * spacing;
                o[3] = 0.0f;
            }
    return count;
}

// sim.rs:139-151
uint16_t or_half_bits(float x) {
    uint32_t xb;
    std::memcpy(&xb, &x, 4);
    const uint16_t sign = (uint16_t)((xb >> 16) & 0x8000u);
    const float a = std::fabs(x);
    uint32_t ab;
    std::memcpy(&ab, &a, 4);
    if (ab < (113u << 23)) {
        const uint32_t mb = 126u << 23;
        float magic;
        std::memcpy(&magic, &mb, 4);
        const float s = a + magic;
        uint32_t sb;
        std::memcpy(&sb, &s, 4);
        return (uint16_t)(sign | (uint16_t)(sb - mb));
    }
    return (uint16_t)(sign | (uint16_t)(((ab + 0x0fffu + ((ab >> 13) & 1u)) - (112u << 23)) >> 13));
}

// sim.rs:168-175
float or_half_value(uint16_t bits) {
    const uint32_t raw = bits;
    uint32_t ob = ((raw & 0x7fffu) << 13) + (112u << 23);
    float o;
    std::memcpy(&o, &ob, 4);
    if ((raw & 0x7c00u) == 0) {
        uint32_t b = ob + (1u << 23);
        float f, m;
        std::memcpy(&f, &b, 4);
        const uint32_t mbits = 113u << 23;
        std::memcpy(&m, &mbits, 4);
        o = f - m;
        std::memcpy(&ob, &o, 4);
    }
    ob |= (raw & 0x8000u) << 16;
    std::memcpy(&o, &ob, 4);
    return o;
}

// sim.rs:127-133
void or_pack_tracer(const float pos[3], float speed, const float extent[2], uint32_t out[2]) {
    auto unorm = [](float v, float e) {
        return (uint32_t)(clampw(v / e * 0.5f + 0.5f, 0.0f, 1.0f) * 65535.0f + 0.5f);
    };
    out[0] = unorm(pos[0], extent[0]) | (unorm(pos[1], extent[1]) << 16);
    out[1] = (uint32_t)or_half_bits(pos[2]) | ((uint32_t)or_half_bits(speed) << 16);
}

// sim.rs:156-164
void or_unpack_tracer(const uint32_t raw[2], const float extent[2], float out[4]) {
    auto unorm = [](uint32_t q, float e) { return ((float)q / 65535.0f * 2.0f - 1.0f) * e; };
    out[0] = unorm(raw[0] & 0xffffu, extent[0]);
    out[1] = unorm(raw[0] >> 16, extent[1]);
    out[2] = or_half_value((uint16_t)(raw[1] & 0xffffu));
    out[3] = or_half_value((uint16_t)(raw[1] >> 16));
}

// sim.rs:105-122
void or_seed_tracers(uint32_t count, const float extent[2], float fill, uint32_t *out2) {
    const float half[3] = {extent[0] - 0.001f, extent[1] - 0.001f, 0.5f * kSlabDepth - 0.001f};
    auto unit = [](uint32_t h) { return (float)h / 4294967295.0f; };
    for (uint32_t i = 0; i < count; ++i) {
        const float pos[3] = {(unit(or_hash(i * 3)) * 2.0f - 1.0f) * half[0],
                              -half[1] + unit(or_hash(i * 3 + 1)) * 2.0f * half[1] * fill,
                              (unit(or_hash(i * 3 + 2)) * 2.0f - 1.0f) * half[2]};
        or_pack_tracer(pos, 0.0f, extent, out2 + 2 * (size_t)i);
    }
}

// The box geometry's tracers (sim.rs:105-122 moved to a box): uniform over
// the region [lo, lo + size) from the same hash stream, stored relative to
// the tracer box centre and packed over its half extent e.
void or_seed_tracers_box(uint32_t count, const float lo[3], const float size[3], const float centre[3],
                         const float e[2], uint32_t *out2) {
    auto unit = [](uint32_t h) { return (float)h / 4294967295.0f; };
    for (uint32_t i = 0; i < count; ++i) {
        float rel[3];
        for (int a = 0; a < 3; ++a) rel[a] = lo[a] + unit(or_hash(i * 3 + a)) * size[a] - centre[a];
        or_pack_tracer(rel, 0.0f, e, out2 + 2 * (size_t)i);
    }
}

// sim.rs:215-252
void or_pack_step(const float force[3], const float omega[3], const float domega[3], float dt,
                  float v_clamp, uint32_t seed, uint32_t touch_n, float touch_r,
                  const float *touches4, uint8_t out[144]) {
    std::memset(out, 0, 144);
    const float head[11] = {force[0], force[1],  force[2],  dt,        omega[0], omega[1],
                            omega[2], v_clamp,   domega[0], domega[1], domega[2]};
    std::memcpy(out, head, sizeof head);
    std::memcpy(out + 44, &seed, 4);
    std::memcpy(out + 48, &touch_r, 4);
    std::memcpy(out + 52, &touch_n, 4);
    if (touches4) std::memcpy(out + 64, touches4, 5 * 16);
}

// sim.rs:330-350
void or_pack_sim_params(const OrGrid *g, uint32_t count, float h, float mass, float rho0,
                        uint8_t out[64]) {
    std::memset(out, 0, 64);
    auto put_f = [&](int off, float v) { std::memcpy(out + off, &v, 4); };
    for (int i = 0; i < 3; ++i) put_f(i * 4, g->min[i]);
    put_f(12, g->cell);
    put_f(32, h);
    put_f(36, mass);
    put_f(40, rho0);
    const float sigma = 1.0f / (kPi * h * h * h);
    put_f(44, 1.0f / h);
    put_f(48, sigma);
    put_f(52, sigma / h);
    put_f(56, 4.0f * h * h);
    for (int i = 0; i < 3; ++i) std::memcpy(out + 16 + 4 * i, &g->dims[i], 4);
    std::memcpy(out + 28, &count, 4);
}

// sim.rs:24-32
void or_grid_slab(const float extent[2], float support, OrGrid *g) {
    const float half[3] = {extent[0], extent[1], kSlabDepth * 0.5f};
    for (int i = 0; i < 3; ++i) {
        g->dims[i] = (uint32_t)std::ceil(2.0f * half[i] / support) + 2u;
        g->min[i] = -half[i] - support;
    }
    g->cell = support;
}

// The same construction over [lo, hi]: one guard cell each side.
void or_grid_box(const float lo[3], const float hi[3], float support, OrGrid *g) {
    for (int i = 0; i < 3; ++i) {
        g->dims[i] = (uint32_t)std::ceil((hi[i] - lo[i]) / support) + 2u;
        g->min[i] = lo[i] - support;
    }
    g->cell = support;
}

uint32_t or_cell_of(const OrGrid *g, const float pos[3]) { return cell_of_t(g, pos); }

// sim_grid.wgsl:44-58 + sim_scan.wgsl:97-120, with the stable order.
void or_grid_build(const OrGrid *g, const float *pos4, uint32_t n, uint32_t *keys,
                   uint32_t *starts, uint32_t *perm) {
    grid_build_t(g, pos4, n, keys, starts, perm);
}

static void derive_kernel_consts(OrParams *p, float h) {
    p->h = h;
    p->inv_h = 1.0f / h;
    p->sigma = 1.0f / (kPi * h * h * h);
    p->sigma_h = p->sigma / h;
    p->support_sq = 4.0f * h * h;
}

// render.rs:1477-1478, :1610; sim_solve.wgsl:237-239 (walls), :311-312
void or_params_slab(const float extent[2], float spacing, float h_ratio, uint32_t count,
                    OrParams *p) {
    std::memset(p, 0, sizeof *p);
    const float h = h_ratio * spacing;
    OrGrid g;
    or_grid_slab(extent, 2.0f * h, &g);
    for (int i = 0; i < 3; ++i) {
        p->box_min[i] = g.min[i];
        p->dims[i] = g.dims[i];
    }
    p->cell = g.cell;
    p->count = count;
    derive_kernel_consts(p, h);
    p->rho0 = kRestDensity;
    p->mass = kRestDensity * spacing * spacing * spacing;
    for (int i = 0; i < 3; ++i) {
        p->wall_lo[i] = p->box_min[i] + p->cell;
        p->wall_hi[i] = -p->wall_lo[i];
        p->tracer_c[i] = 0.0f;
        p->tracer_e[i] = -(p->box_min[i] + p->cell);  // sim_tracers.wgsl:60-62
    }
    p->xsph_blend = -1.0f;
    p->nbr_cap = 96;
}

void or_params_box(const float lo[3], const float hi[3], float spacing, float h_ratio,
                   float rho0, uint32_t count, OrParams *p) {
    std::memset(p, 0, sizeof *p);
    const float h = h_ratio * spacing;
    OrGrid g;
    or_grid_box(lo, hi, 2.0f * h, &g);
    for (int i = 0; i < 3; ++i) {
        p->box_min[i] = g.min[i];
        p->dims[i] = g.dims[i];
    }
    p->cell = g.cell;
    p->count = count;
    derive_kernel_consts(p, h);
    p->rho0 = rho0;
    p->mass = rho0 * spacing * spacing * spacing;
    for (int i = 0; i < 3; ++i) {
        p->wall_lo[i] = lo[i];
        p->wall_hi[i] = hi[i];
        p->tracer_c[i] = (lo[i] + hi[i]) * 0.5f;
        p->tracer_e[i] = (hi[i] - lo[i]) * 0.5f;
    }
    p->xsph_blend = -1.0f;
    p->nbr_cap = 96;
}

static inline uint64_t splitmix64(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint32_t or_seed_block(const float lo[3], float spacing, const uint32_t n[3], float jitter,
                       uint64_t seed, float *out4) {
    const uint32_t count = n[0] * n[1] * n[2];
    if (!out4) return count;
    uint64_t s = seed;
    const float amp = jitter * spacing;
    size_t i = 0;
    for (uint32_t iz = 0; iz < n[2]; ++iz)
        for (uint32_t iy = 0; iy < n[1]; ++iy)
            for (uint32_t ix = 0; ix < n[0]; ++ix, ++i) {
                const uint32_t idx[3] = {ix, iy, iz};
                for (int a = 0; a < 3; ++a) {
                    const float u = (float)(splitmix64(&s) >> 40) * (1.0f / 16777216.0f);
                    out4[4 * i + a] =
                        lo[a] + ((float)idx[a] + 0.5f) * spacing + (2.0f * u - 1.0f) * amp;
                }
                out4[4 * i + 3] = 0.0f;
            }
    return count;
}

// ---------------------------------------------------------------------------
// The substep
// ---------------------------------------------------------------------------
struct OrSim {
    OrParams p;
    uint32_t n, cells, ntr;
    // resting set (slot order of the last integrate) and working set
    std::vector<Real> pos, vel, pvel, pp, temp;  // pos/vel/pvel are float4
    std::vector<uint32_t> id;
    std::vector<Real> wpos, wvel, wpvel, wpp, wtemp;
    std::vector<uint32_t> wid;
    std::vector<uint32_t> keys, starts, perm;
    std::vector<Real> density, alpha, kd, pressure, pinc;
    std::vector<Real> accel, xsph, wgrad;  // float4
    std::vector<uint32_t> nbr, nbr_n;       // nbr[k * n + i]
    uint32_t clamp_count, nbr_over;
    std::vector<uint32_t> tracers;
    std::vector<int32_t> vel_grid, vel_flat;
};

static int g_threads = 0;
void or_sim_set_threads(int threads) { g_threads = threads; }
uint32_t or_sim_slabs(void) { return kSimSlabs; }
static int nthreads() {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

OrSim *or_sim_new(const OrParams *p, uint32_t tracer_count) {
    OrSim *s = new OrSim();
    s->p = *p;
    s->n = p->count;
    s->cells = p->dims[0] * p->dims[1] * p->dims[2];
    s->ntr = tracer_count;
    const size_t n = s->n;
    s->pos.assign(4 * n, 0.f);
    s->vel.assign(4 * n, 0.f);
    s->pvel.assign(4 * n, 0.f);
    s->pp.assign(n, 0.f);
    s->temp.assign(n, 293.15f);
    s->id.resize(n);
    for (size_t i = 0; i < n; ++i) s->id[i] = (uint32_t)i;
    s->wpos.assign(4 * n, 0.f);
    s->wvel.assign(4 * n, 0.f);
    s->wpvel.assign(4 * n, 0.f);
    s->wpp.assign(n, 0.f);
    s->wtemp.assign(n, 0.f);
    s->wid.assign(n, 0u);
    s->keys.assign(n, 0u);
    s->starts.assign((size_t)s->cells * kSimSlabs + 1, 0u);
    s->perm.assign(n, 0u);
    s->density.assign(n, 0.f);
    s->alpha.assign(n, 0.f);
    s->kd.assign(n, 0.f);
    s->pressure.assign(n, 0.f);
    s->pinc.assign(n, 0.f);
    s->accel.assign(4 * n, 0.f);
    s->xsph.assign(4 * n, 0.f);
    s->wgrad.assign(4 * n, 0.f);
    s->nbr.assign((size_t)p->nbr_cap * n, 0u);
    s->nbr_n.assign(n, 0u);
    s->clamp_count = 0;
    s->nbr_over = 0;
    s->tracers.assign(2 * (size_t)tracer_count, 0u);
    s->vel_grid.assign(4 * (size_t)s->cells, 0);
    s->vel_flat.assign(4 * (size_t)s->cells, 0);
    return s;
}

void or_sim_free(OrSim *s) { delete s; }

void or_sim_set_state(OrSim *s, const float *pos4, const float *vel4, const float *prev_vel4,
                      const float *prev_p, const float *temp, const uint32_t *id) {
    const size_t n = s->n;
    auto in = [](std::vector<Real> &dst, const float *src, size_t m) {
        if (src)
            for (size_t k = 0; k < m; ++k) dst[k] = (Real)src[k];
    };
    in(s->pos, pos4, 4 * n);
    in(s->vel, vel4, 4 * n);
    in(s->pvel, prev_vel4, 4 * n);
    in(s->pp, prev_p, n);
    in(s->temp, temp, n);
    if (id) std::memcpy(s->id.data(), id, 4 * n);
}

void or_sim_get_state(const OrSim *s, float *pos4, float *vel4, float *prev_vel4, float *prev_p,
                      float *temp, uint32_t *id) {
    const size_t n = s->n;
    auto out = [](float *dst, const std::vector<Real> &src, size_t m) {
        if (dst)
            for (size_t k = 0; k < m; ++k) dst[k] = (float)src[k];
    };
    out(pos4, s->pos, 4 * n);
    out(vel4, s->vel, 4 * n);
    out(prev_vel4, s->pvel, 4 * n);
    out(prev_p, s->pp, n);
    out(temp, s->temp, n);
    if (id) std::memcpy(id, s->id.data(), 4 * n);
}

void or_sim_get_state64(const OrSim *s, double *pos4, double *vel4) {
    const size_t n = s->n;
    for (size_t k = 0; pos4 && k < 4 * n; ++k) pos4[k] = (double)s->pos[k];
    for (size_t k = 0; vel4 && k < 4 * n; ++k) vel4[k] = (double)s->vel[k];
}

int or_sim_real_bytes(void) { return (int)sizeof(Real); }

void or_sim_set_tracers(OrSim *s, const uint32_t *packed2) {
    std::memcpy(s->tracers.data(), packed2, 8 * (size_t)s->ntr);
}
void or_sim_get_tracers(const OrSim *s, uint32_t *packed2) {
    std::memcpy(packed2, s->tracers.data(), 8 * (size_t)s->ntr);
}

namespace {

OrGrid grid_of(const OrParams &p) {
    OrGrid g;
    for (int i = 0; i < 3; ++i) {
        g.min[i] = p.box_min[i];
        g.dims[i] = p.dims[i];
    }
    g.cell = p.cell;
    return g;
}

// count, scan, stable scatter of the five records plus the id
// (sim_grid.wgsl:44-72, sim_scan.wgsl:97-120).
void rebuild(OrSim *s) {
    const OrGrid g = grid_of(s->p);
    grid_build_t(&g, s->pos.data(), s->n, s->keys.data(), s->starts.data(), s->perm.data(), kSimSlabs);
    const int64_t n = s->n;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        const size_t i = s->perm[k];
        std::memcpy(&s->wpos[4 * k], &s->pos[4 * i], 4 * sizeof(Real));
        std::memcpy(&s->wvel[4 * k], &s->vel[4 * i], 4 * sizeof(Real));
        std::memcpy(&s->wpvel[4 * k], &s->pvel[4 * i], 4 * sizeof(Real));
        s->wpp[k] = s->pp[i];
        s->wtemp[k] = s->temp[i];
        s->wid[k] = s->id[i];
    }
}

inline Real kernel_q(const OrParams &p, Real q) {  // sim_solve.wgsl:176-182
    if (q < 1.0f) return p.sigma * (1.0f - 1.5f * q * q * (1.0f - 0.5f * q));
    const Real t = 2.0f - q;
    return p.sigma * 0.25f * t * t * t;
}

inline V3 grad_q(const OrParams &p, V3 x, Real r, Real q) {  // sim_solve.wgsl:184-196
    if (r < 1e-9f) return v3(0.f, 0.f, 0.f);
    Real dw;
    if (q < 1.0f) {
        dw = p.sigma_h * (-3.0f * q + 2.25f * q * q);
    } else {
        const Real t = 2.0f - q;
        dw = p.sigma_h * (-0.75f * t * t);
    }
    return (dw / r) * x;
}

inline Real cohesion(Real r, Real c, Real k, Real near) {  // sim_solve.wgsl:201-210
    if (r >= c || r < 1e-9f) return 0.0f;
    const Real a = (c - r) * (c - r) * (c - r) * r * r * r;
    if (2.0f * r > c) return k * a;
    return k * (2.0f * a - near);
}

inline Real wedge_dsum(Real t, Real a, Real b, Real c, Real d) {  // :295-297
    return wedge_d_t(t, a) + wedge_d_t(t, b) + wedge_d_t(t, c) + wedge_d_t(t, d);
}

inline Real wedge_sum(V3 tl, V3 th) {  // sim_solve.wgsl:299-304
    Real w = wedge_t(tl.x, tl.y) + wedge_t(tl.x, th.y) + wedge_t(th.x, tl.y) +
              wedge_t(th.x, th.y);
    w += wedge_t(tl.x, tl.z) + wedge_t(tl.x, th.z) + wedge_t(th.x, tl.z) + wedge_t(th.x, th.z);
    w += wedge_t(tl.y, tl.z) + wedge_t(tl.y, th.z) + wedge_t(th.y, tl.z) + wedge_t(th.y, th.z);
    return w;
}

V3 wall_grad_sum(const OrParams &p, V3 pos) {  // sim_solve.wgsl:310-328
    const V3 lo = load3(p.wall_lo), hi = load3(p.wall_hi);
    const Real inv_h = 1.0f / p.h;
    const V3 tl = (pos - lo) * inv_h;
    const V3 th = (hi - pos) * inv_h;
    const Real scale = p.rho0 * inv_h;
    V3 g = v3(0.f, 0.f, 0.f);
    g.x -= scale * (wall_gradient_t(tl.x) + wedge_dsum(tl.x, tl.y, th.y, tl.z, th.z));
    g.x += scale * (wall_gradient_t(th.x) + wedge_dsum(th.x, tl.y, th.y, tl.z, th.z));
    g.y -= scale * (wall_gradient_t(tl.y) + wedge_dsum(tl.y, tl.x, th.x, tl.z, th.z));
    g.y += scale * (wall_gradient_t(th.y) + wedge_dsum(th.y, tl.x, th.x, tl.z, th.z));
    g.z -= scale * (wall_gradient_t(tl.z) + wedge_dsum(tl.z, tl.x, th.x, tl.y, th.y));
    g.z += scale * (wall_gradient_t(th.z) + wedge_dsum(th.z, tl.x, th.x, tl.y, th.y));
    return g;
}

V3 wall_adh_sum(const OrParams &p, V3 pos) {  // sim_solve.wgsl:349-361
    const V3 lo = load3(p.wall_lo), hi = load3(p.wall_hi);
    const Real inv_h = 1.0f / p.h;
    V3 a = v3(0.f, 0.f, 0.f);
    a.x -= wall_adhesion_t((pos.x - lo.x) * inv_h);
    a.x += wall_adhesion_t((hi.x - pos.x) * inv_h);
    a.y -= wall_adhesion_t((pos.y - lo.y) * inv_h);
    a.y += wall_adhesion_t((hi.y - pos.y) * inv_h);
    a.z -= wall_adhesion_t((pos.z - lo.z) * inv_h);
    a.z += wall_adhesion_t((hi.z - pos.z) * inv_h);
    return a;
}

inline uint32_t base_coord(const OrParams &p, Real v, int axis) {  // :363-368
    const uint32_t u = sat_u32_t((v - p.box_min[axis]) / p.cell);
    return u < p.dims[axis] - 1u ? u : p.dims[axis] - 1u;
}

// density_div, sim_solve.wgsl:411-518. Returns the divergence residual
// term sum (fixed point) of max(drho, 0) dt / rho0.
int64_t density_div(OrSim *s, Real dt) {
    const OrParams &p = s->p;
    const int64_t n = s->n;
    const uint32_t cap = p.nbr_cap;
    int64_t res = 0;
    uint32_t over = 0;
#pragma omp parallel for num_threads(nthreads()) schedule(static) reduction(+ : res, over)
    for (int64_t pi = 0; pi < n; ++pi) {
        const V3 pos = load3(&s->wpos[4 * pi]);
        const V3 vel = load3(&s->wvel[4 * pi]);
        const uint32_t bx = base_coord(p, pos.x, 0), by = base_coord(p, pos.y, 1),
                       bz = base_coord(p, pos.z, 2);
        Real w_sum = p.sigma;
        Real rho_near = 0.0f;
        V3 grad_sum = v3(0.f, 0.f, 0.f);
        Real grad_sq = 0.0f;
        Real drho = 0.0f;
        uint32_t found = 0;
        for (int cell = 0; cell < 27; ++cell) {
            const int cx = (int)bx + (cell % 3) - 1;
            const int cy = (int)by + ((cell / 3) % 3) - 1;
            const int cz = (int)bz + (cell / 9) - 1;
            if (cx < 0 || cy < 0 || cz < 0 || cx >= (int)p.dims[0] || cy >= (int)p.dims[1] ||
                cz >= (int)p.dims[2])
                continue;
            const uint32_t c = ((uint32_t)cz * p.dims[1] + (uint32_t)cy) * p.dims[0] + (uint32_t)cx;
            const uint32_t end = s->starts[(c + 1) * kSimSlabs];
            for (uint32_t k = s->starts[c * kSimSlabs]; k < end; ++k) {
                if ((int64_t)k == pi) continue;
                const V3 x = pos - load3(&s->wpos[4 * (size_t)k]);
                const Real r2 = dot(x, x);
                if (r2 >= p.support_sq) continue;
                const Real r = std::sqrt(r2);
                const Real q = r * p.inv_h;
                w_sum += kernel_q(p, q);
                const Real wn = fmaxw(1.0f - q, 0.0f);
                rho_near += wn * wn * wn;
                const V3 gw = grad_q(p, x, r, q);
                grad_sum = grad_sum + gw;
                grad_sq += dot(gw, gw);
                drho += dot(vel - load3(&s->wvel[4 * (size_t)k]), gw);
                if (found < cap) s->nbr[(size_t)found * n + pi] = k;
                found++;
            }
        }
        s->nbr_n[pi] = found < cap ? found : cap;
        if (found > cap) over += found - cap;
        Real rho = p.mass * w_sum;
        grad_sq = p.mass * p.mass * grad_sq;
        drho = p.mass * drho;
        grad_sum = p.mass * grad_sum;
        const V3 lo = load3(p.wall_lo), hi = load3(p.wall_hi);
        const V3 tl = (pos - lo) * p.inv_h;
        const V3 th = (hi - pos) * p.inv_h;
        Real fill = 0.0f;
        fill += wall_density_t(tl.x) + wall_density_t(th.x);
        fill += wall_density_t(tl.y) + wall_density_t(th.y);
        fill += wall_density_t(tl.z) + wall_density_t(th.z);
        fill -= wedge_sum(tl, th);
        rho += p.rho0 * fill;
        const V3 wg = wall_grad_sum(p, pos);
        s->wgrad[4 * pi + 0] = wg.x;
        s->wgrad[4 * pi + 1] = wg.y;
        s->wgrad[4 * pi + 2] = wg.z;
        s->wgrad[4 * pi + 3] = 0.0f;
        grad_sum = grad_sum + wg;
        s->density[pi] = rho;
        s->wpos[4 * pi + 3] = rho_near;
        const Real a = rho / fmaxw(dot(grad_sum, grad_sum) + grad_sq, 1e-4f);
        s->alpha[pi] = a;
        drho += dot(vel, wg);
        s->kd[pi] = fmaxw(drho, 0.0f) * a / fmaxw(dt, 1e-9f) / rho;
        res += fx((double)fmaxw(drho, 0.0f) * (double)dt / (double)p.rho0);
    }
    s->nbr_over += over;
    return res;
}

// Neighbour gradient, recomputed bit-for-bit as density_div wrote it.
inline V3 nbr_grad(const OrSim *s, V3 pos, uint32_t j) {
    const V3 x = pos - load3(&s->wpos[4 * (size_t)j]);
    const Real r2 = dot(x, x);
    const Real r = std::sqrt(r2);
    const Real q = r * s->p.inv_h;
    return grad_q(s->p, x, r, q);
}

// kappa_partial, sim_solve.wgsl:596-606, sequential over the list.
inline V3 kappa_sum(const OrSim *s, int64_t pi, V3 pos) {
    const int64_t n = s->n;
    const uint32_t cnt = s->nbr_n[pi];
    const Real kd_i = s->kd[pi];
    V3 dv = v3(0.f, 0.f, 0.f);
    for (uint32_t k = 0; k < cnt; ++k) {
        const uint32_t j = s->nbr[(size_t)k * n + pi];
        const V3 e = nbr_grad(s, pos, j);
        dv = dv + (kd_i + s->kd[j]) * e;
    }
    return dv;
}

// apply_kappa_wide (div_apply / den_apply), sim_solve.wgsl:608-621, and the
// applied pressure kappa*rho for the density iterations.
void apply_kappa(OrSim *s, Real dt, bool add_pressure) {
    const OrParams &p = s->p;
    const int64_t n = s->n;
    std::vector<Real> out(4 * (size_t)n);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int64_t pi = 0; pi < n; ++pi) {
        const V3 pos = load3(&s->wpos[4 * pi]);
        const V3 total = kappa_sum(s, pi, pos);
        const V3 dv_full = p.mass * total + s->kd[pi] * load3(&s->wgrad[4 * pi]);
        const V3 was = load3(&s->wvel[4 * pi]);
        const V3 v = was - dt * dv_full;
        out[4 * pi + 0] = v.x;
        out[4 * pi + 1] = v.y;
        out[4 * pi + 2] = v.z;
        out[4 * pi + 3] = s->wvel[4 * pi + 3];
    }
    s->wvel.swap(out);
    if (add_pressure)
        for (int64_t pi = 0; pi < n; ++pi) s->pressure[pi] += s->pinc[pi];
}

// The divergence predictor for a second or later divergence iteration: the
// density_div sums again over the list, with this iteration's velocities.
int64_t div_kappa(OrSim *s, Real dt) {
    const OrParams &p = s->p;
    const int64_t n = s->n;
    int64_t res = 0;
#pragma omp parallel for num_threads(nthreads()) schedule(static) reduction(+ : res)
    for (int64_t pi = 0; pi < n; ++pi) {
        const V3 pos = load3(&s->wpos[4 * pi]);
        const V3 vel = load3(&s->wvel[4 * pi]);
        const uint32_t cnt = s->nbr_n[pi];
        Real drho = 0.0f;
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t j = s->nbr[(size_t)k * n + pi];
            const V3 e = nbr_grad(s, pos, j);
            drho += dot(vel - load3(&s->wvel[4 * (size_t)j]), e);
        }
        drho = p.mass * drho;
        drho += dot(vel, load3(&s->wgrad[4 * pi]));
        const Real rho = s->density[pi];
        s->kd[pi] = fmaxw(drho, 0.0f) * s->alpha[pi] / fmaxw(dt, 1e-9f) / rho;
        res += fx((double)fmaxw(drho, 0.0f) * (double)dt / (double)p.rho0);
    }
    return res;
}

// forces_eval, sim_solve.wgsl:524-592.
void forces_eval(OrSim *s) {
    const OrParams &p = s->p;
    const int64_t n = s->n;
    const Real coh_c = 2.0f * p.h;
    const Real c3 = coh_c * coh_c * coh_c;
    const Real coh_k = 32.0f / (3.14159265f * c3 * c3 * c3);
    const Real coh_near = c3 * c3 / 64.0f;
    const Real c = 2.0f * p.h;
    const Real gamma = SIGMA_WATER * 7040.0f / (21.0f * LATTICE_SIGMA * p.rho0 * p.rho0 * c * c);
    const Real beta =
        SIGMA_WATER * (1.0f + COS_CONTACT) * 1558.4f / (LATTICE_SIGMA * p.rho0 * p.rho0 * c * c);
    const Real visc_k = 2.0f * DYNAMIC_VISCOSITY;
    const Real heat_k = 2.0f * CONDUCTIVITY / HEAT_CAPACITY;
    const Real diss_k = 0.5f * DYNAMIC_VISCOSITY / HEAT_CAPACITY;
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int64_t pi = 0; pi < n; ++pi) {
        const Real *pos4 = &s->wpos[4 * pi];
        const V3 pos = load3(pos4);
        const V3 vel = load3(&s->wvel[4 * pi]);
        const Real temp = s->wtemp[pi];
        const Real rho_i = s->density[pi];
        const uint32_t cnt = s->nbr_n[pi];
        V3 visc = v3(0.f, 0.f, 0.f), blend = v3(0.f, 0.f, 0.f), near = v3(0.f, 0.f, 0.f),
           tension = v3(0.f, 0.f, 0.f);
        Real heat = 0.0f;
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t j = s->nbr[(size_t)k * n + pi];
            const V3 e = nbr_grad(s, pos, j);
            const Real *pj = &s->wpos[4 * (size_t)j];
            const V3 x = pos - load3(pj);
            const Real r2 = dot(x, x);
            const Real r = std::sqrt(r2);
            const Real rho_j = s->density[j];
            const Real f = dot(x, e) / (r2 + 0.01f * p.h * p.h);
            const Real pair = p.mass / (rho_i * rho_j) * f;
            const V3 dv = vel - load3(&s->wvel[4 * (size_t)j]);
            const Real wn = fmaxw(1.0f - r * p.inv_h, 0.0f);
            near = near + ((pos4[3] + pj[3]) * wn * wn) * (x / fmaxw(r, 1e-5f));
            visc = visc + (visc_k * pair) * dv;
            blend = blend - (p.mass / rho_j * kernel_q(p, r * p.inv_h)) * dv;
            heat += heat_k * pair * (temp - s->wtemp[j]);
            heat -= diss_k * pair * dot(dv, dv);
            const Real corr = 2.0f * p.rho0 / (rho_i + rho_j);
            tension = tension - ((corr * p.mass * cohesion(r, coh_c, coh_k, coh_near)) * x) /
                                    fmaxw(r, 1e-9f);
        }
        const V3 adh = (beta * p.rho0) * wall_adh_sum(p, pos);
        const V3 acc = visc + K_NEAR * near + gamma * tension + adh;
        s->accel[4 * pi + 0] = acc.x;
        s->accel[4 * pi + 1] = acc.y;
        s->accel[4 * pi + 2] = acc.z;
        s->accel[4 * pi + 3] = heat;
        s->xsph[4 * pi + 0] = blend.x;
        s->xsph[4 * pi + 1] = blend.y;
        s->xsph[4 * pi + 2] = blend.z;
        s->xsph[4 * pi + 3] = 0.0f;
        const Real rho = s->density[pi];
        const Real half = 0.5f * s->wpp[pi];
        s->kd[pi] = half / (rho * rho);
        s->pressure[pi] = half;
    }
}

// fingers, sim_solve.wgsl:103-127.
V3 fingers(const OrStep &st, V3 pos, V3 v) {
    Real px = 0.0f, py = 0.0f, weight = 0.0f;
    for (uint32_t i = 0; i < st.touch_n && i < 5; ++i) {
        const float *t = st.touches[i];
        const Real dx = pos.x - t[0], dy = pos.y - t[1];
        const Real q2 = (dx * dx + dy * dy) / (st.touch_r * st.touch_r);
        if (q2 < 1.0f) {
            const Real w = (1.0f - q2) * (1.0f - q2);
            px += w * t[2];
            py += w * t[3];
            weight += w;
        }
    }
    if (weight <= 0.0f) return v;
    const Real a = 1.0f - exp_r(-TOUCH_RATE * weight * st.dt);
    return v3(mixw(v.x, px / weight, a), mixw(v.y, py / weight, a), v.z);
}

// forces_den_apply, sim_solve.wgsl:630-663.
void forces_den_apply(OrSim *s, const OrStep &st, Real xsph_blend) {
    const OrParams &p = s->p;
    const int64_t n = s->n;
    const V3 force = load3(st.force), omega = load3(st.omega), domega = load3(st.domega);
    std::vector<Real> out(4 * (size_t)n);
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int64_t pi = 0; pi < n; ++pi) {
        const V3 pos = load3(&s->wpos[4 * pi]);
        const V3 total = kappa_sum(s, pi, pos);
        const Real *a = &s->accel[4 * pi];
        const V3 r = pos;
        const V3 v = load3(&s->wvel[4 * pi]);
        const V3 fict =
            -cross(domega, r) - cross(omega, cross(omega, r)) - 2.0f * cross(omega, v);
        const V3 forced = fingers(
            st, r, v + st.dt * (force + fict + load3(a)) + xsph_blend * load3(&s->xsph[4 * pi]));
        s->wtemp[pi] += st.dt * a[3];
        const V3 dv_full = p.mass * total + s->kd[pi] * load3(&s->wgrad[4 * pi]);
        const V3 o = forced - st.dt * dv_full;
        out[4 * pi + 0] = o.x;
        out[4 * pi + 1] = o.y;
        out[4 * pi + 2] = o.z;
        out[4 * pi + 3] = s->wvel[4 * pi + 3];
    }
    s->wvel.swap(out);
}

// den_kappa, sim_solve.wgsl:674-698; the applied pressure k*rho is held in
// pinc until den_apply applies the kappa it belongs to. Returns the density
// residual sum (fixed point) of max(rho*/rho0 - 1, 0).
int64_t den_kappa(OrSim *s, Real dt) {
    const OrParams &p = s->p;
    const int64_t n = s->n;
    int64_t res = 0;
#pragma omp parallel for num_threads(nthreads()) schedule(static) reduction(+ : res)
    for (int64_t pi = 0; pi < n; ++pi) {
        const V3 pos = load3(&s->wpos[4 * pi]);
        const V3 vel = load3(&s->wvel[4 * pi]);
        const uint32_t cnt = s->nbr_n[pi];
        Real drho = 0.0f;
        for (uint32_t k = 0; k < cnt; ++k) {
            const uint32_t j = s->nbr[(size_t)k * n + pi];
            const V3 e = nbr_grad(s, pos, j);
            drho += dot(vel - load3(&s->wvel[4 * (size_t)j]), e);
        }
        const Real rho = s->density[pi];
        drho = p.mass * drho + dot(vel, load3(&s->wgrad[4 * pi]));
        const Real rho_star = rho + dt * drho;
        const Real k = fmaxw(rho_star - p.rho0, 0.0f) * s->alpha[pi] / (dt * dt);
        s->kd[pi] = k / rho;
        s->pinc[pi] = k * rho;
        res += fx((double)rho_star / (double)p.rho0 - 1.0);
    }
    return res;
}

// integrate, sim_solve.wgsl:709-756, with the lens chase precomputed.
void integrate(OrSim *s, const OrStep &st, Real chase) {
    const OrParams &p = s->p;
    const int64_t n = s->n;
    const V3 lo = load3(p.wall_lo), hi = load3(p.wall_hi);
    uint32_t clamps = 0;
#pragma omp parallel for num_threads(nthreads()) schedule(static) reduction(+ : clamps)
    for (int64_t i = 0; i < n; ++i) {
        const Real *was = &s->wvel[4 * i];
        V3 v = load3(was);
        const Real speed = length(v);
        const Real ceiling = s->density[i] < 0.5f * p.rho0 ? 3.0f * st.v_clamp : st.v_clamp;
        if (speed > ceiling) {
            v = v * (ceiling / speed);
            clamps++;
        }
        const Real *pv = &s->wpvel[4 * i];
        const Real accel = length(v - load3(pv)) / st.dt;
        const V3 pp = load3(&s->wpos[4 * i]) + v * st.dt;
        const V3 cl = v3(clampw(pp.x, lo.x, hi.x), clampw(pp.y, lo.y, hi.y), clampw(pp.z, lo.z, hi.z));
        if (cl.x != pp.x) v.x = 0.0f;
        if (cl.y != pp.y) v.y = 0.0f;
        if (cl.z != pp.z) v.z = 0.0f;
        s->pos[4 * i + 0] = cl.x;
        s->pos[4 * i + 1] = cl.y;
        s->pos[4 * i + 2] = cl.z;
        s->pos[4 * i + 3] = 0.0f;
        s->vel[4 * i + 0] = v.x;
        s->vel[4 * i + 1] = v.y;
        s->vel[4 * i + 2] = v.z;
        s->vel[4 * i + 3] = mixw(was[3], accel, chase);
        s->pvel[4 * i + 0] = v.x;
        s->pvel[4 * i + 1] = v.y;
        s->pvel[4 * i + 2] = v.z;
        s->pvel[4 * i + 3] = mixw(pv[3], s->pressure[i], chase);
        const Real dp = s->pressure[i] - s->wpp[i];
        s->pp[i] = s->pressure[i];
        const Real t = s->wtemp[i];
        s->temp[i] = t + t * EXPANSION / (s->density[i] * HEAT_CAPACITY) * dp;
        s->id[i] = s->wid[i];
    }
    s->clamp_count += clamps;
}

Real step_xsph_blend(const OrParams &p, Real dt) {
    return p.xsph_blend >= 0.0f ? p.xsph_blend : 1.0f - std::exp(-XSPH_RATE * dt);
}

}  // namespace

void or_sim_substep(OrSim *s, const OrStep *st, uint32_t div_iters, uint32_t den_iters) {
    rebuild(s);
    density_div(s, st->dt);
    if (st->dt == 0.0f) return;
    for (uint32_t i = 0; i < div_iters; ++i) {
        if (i > 0) div_kappa(s, st->dt);
        apply_kappa(s, st->dt, false);
    }
    forces_eval(s);
    forces_den_apply(s, *st, step_xsph_blend(s->p, st->dt));
    for (uint32_t i = 0; i < den_iters; ++i) {
        den_kappa(s, st->dt);
        apply_kappa(s, st->dt, true);
    }
    integrate(s, *st, 1.0f - std::exp(-LENS_RATE * st->dt));
}

// The tolerance schedule. Divergence: density_div predicts, then apply and
// re-predict while the mean positive divergence exceeds div_tol (at least
// one apply, as the reference). Density: after the warm-start apply, predict
// and apply while the mean positive predicted compression exceeds den_tol.
// Both stop at max_iters applies. The residual that stops each loop is the
// one measured after its last apply.
void or_sim_substep_tol(OrSim *s, const OrStep *st, float div_tol, float den_tol,
                        uint32_t max_iters, uint32_t out_iters[2], double out_res[2]) {
    const double n = (double)s->n;
    auto mean = [n](int64_t acc) { return (double)acc / kFixedScale / n; };
    rebuild(s);
    int64_t acc = density_div(s, st->dt);
    out_iters[0] = out_iters[1] = 0;
    out_res[0] = mean(acc);
    out_res[1] = 0.0;
    if (st->dt == 0.0f) return;
    uint32_t it = 0;
    double res = mean(acc);
    while (it < max_iters && (it < 1 || res > (double)div_tol)) {
        apply_kappa(s, st->dt, false);
        it++;
        res = mean(div_kappa(s, st->dt));
    }
    out_iters[0] = it;
    out_res[0] = res;
    forces_eval(s);
    forces_den_apply(s, *st, step_xsph_blend(s->p, st->dt));
    res = mean(den_kappa(s, st->dt));
    it = 0;
    while (it < max_iters && res > (double)den_tol) {
        apply_kappa(s, st->dt, true);
        it++;
        res = mean(den_kappa(s, st->dt));
    }
    out_iters[1] = it;
    out_res[1] = res;
    integrate(s, *st, 1.0f - std::exp(-LENS_RATE * st->dt));
}

// One kernel of the substep on the current working set, for the per-kernel
// checks of the tests (the substep functions above run them in order).
double or_sim_kernel(OrSim *s, int kernel, const OrStep *st) {
    const double n = (double)s->n;
    switch (kernel) {
    case OR_KERNEL_DENSITY:
        rebuild(s);
        return (double)density_div(s, st->dt) / kFixedScale / n;
    case OR_KERNEL_DIV_APPLY: apply_kappa(s, st->dt, false); return 0.0;
    case OR_KERNEL_DIV_KAPPA: return (double)div_kappa(s, st->dt) / kFixedScale / n;
    case OR_KERNEL_FORCES_EVAL: forces_eval(s); return 0.0;
    case OR_KERNEL_FORCES_APPLY: forces_den_apply(s, *st, step_xsph_blend(s->p, st->dt)); return 0.0;
    case OR_KERNEL_DEN_KAPPA: return (double)den_kappa(s, st->dt) / kFixedScale / n;
    case OR_KERNEL_DEN_APPLY: apply_kappa(s, st->dt, true); return 0.0;
    case OR_KERNEL_INTEGRATE: integrate(s, *st, 1.0f - std::exp(-LENS_RATE * st->dt)); return 0.0;
    default: return -1.0;
    }
}

float or_det_exp(float x) { return or_exp(x); }

// reduce_stats, sim_solve.wgsl:800-874; the compression sum is exact.
void or_sim_stats(OrSim *s, float out[14]) {
    const OrParams &p = s->p;
    const size_t n = s->n;
    int64_t sum = 0;
    Real m = 0.0f, lo = HUGE_F, hi = -HUGE_F;
    for (size_t i = 0; i < n; ++i) {
        const Real c = s->density[i] / p.rho0 - 1.0f;
        sum += fx((double)fmaxw(c, 0.0f));
        m = fmaxw(m, c);
        lo = fminw(lo, s->density[i]);
        hi = fmaxw(hi, s->density[i]);
    }
    out[0] = (Real)((double)sum / kFixedScale / (double)n);
    out[1] = fmaxw(m, 0.0f);
    out[2] = lo;
    out[3] = hi;
    Real v_lo = HUGE_F, v_hi = -HUGE_F, a_lo = HUGE_F, a_hi = -HUGE_F;
    Real p_lo = HUGE_F, p_hi = -HUGE_F, t_lo = HUGE_F, t_hi = -HUGE_F;
    for (size_t i = 0; i < n; ++i) {
        const Real *q = &s->vel[4 * i];
        const Real speed = length(load3(q));
        v_lo = fminw(v_lo, speed);
        v_hi = fmaxw(v_hi, speed);
        a_lo = fminw(a_lo, q[3]);
        a_hi = fmaxw(a_hi, q[3]);
        const Real pr = s->pvel[4 * i + 3];
        p_lo = fminw(p_lo, pr);
        p_hi = fmaxw(p_hi, pr);
        t_lo = fminw(t_lo, s->temp[i]);
        t_hi = fmaxw(t_hi, s->temp[i]);
    }
    out[11] = v_lo;
    out[6] = v_hi;
    out[12] = a_lo;
    out[13] = a_hi;
    out[4] = p_lo;
    out[5] = p_hi;
    out[7] = t_lo;
    out[8] = t_hi;
    out[9] = (Real)s->clamp_count;
    out[10] = (Real)s->nbr_over;
}

namespace {

inline void store_tracer(OrSim *s, uint32_t i, V3 pos, float speed) {  // :75-80
    const OrParams &p = s->p;
    const float ux = clampw((pos.x - p.tracer_c[0]) / p.tracer_e[0] * 0.5f + 0.5f, 0.0f, 1.0f);
    const float uy = clampw((pos.y - p.tracer_c[1]) / p.tracer_e[1] * 0.5f + 0.5f, 0.0f, 1.0f);
    const uint32_t qx = (uint32_t)(ux * 65535.0f + 0.5f);
    const uint32_t qy = (uint32_t)(uy * 65535.0f + 0.5f);
    s->tracers[2 * (size_t)i] = qx | (qy << 16);
    s->tracers[2 * (size_t)i + 1] =
        (uint32_t)or_half_bits(pos.z - p.tracer_c[2]) | ((uint32_t)or_half_bits(speed) << 16);
}

inline void load_tracer(const OrSim *s, uint32_t i, float out[4]) {  // :64-69
    const OrParams &p = s->p;
    const uint32_t a = s->tracers[2 * (size_t)i], b = s->tracers[2 * (size_t)i + 1];
    out[0] = ((float)(a & 0xffffu) / 65535.0f * 2.0f - 1.0f) * p.tracer_e[0] + p.tracer_c[0];
    out[1] = ((float)(a >> 16) / 65535.0f * 2.0f - 1.0f) * p.tracer_e[1] + p.tracer_c[1];
    out[2] = or_half_value((uint16_t)(b & 0xffffu)) + p.tracer_c[2];
    out[3] = or_half_value((uint16_t)(b >> 16));
}

inline V3 tracer_clamp(const OrParams &p, V3 v) {
    return v3(clampw(v.x, p.tracer_c[0] - p.tracer_e[0], p.tracer_c[0] + p.tracer_e[0]),
              clampw(v.y, p.tracer_c[1] - p.tracer_e[1], p.tracer_c[1] + p.tracer_e[1]),
              clampw(v.z, p.tracer_c[2] - p.tracer_e[2], p.tracer_c[2] + p.tracer_e[2]));
}

void respawn(OrSim *s, uint32_t slot, uint32_t r) {  // sim_tracers.wgsl:82-92
    const OrParams &p = s->p;
    const uint32_t r1 = pcg(r), r2 = pcg(r1), r3 = pcg(r2), r4 = pcg(r3);
    const float half_cell = p.cell * 0.5f;
    const V3 jit = v3(((float)(r2 >> 20) / 4096.0f - 0.5f) * half_cell,
                      ((float)(r3 >> 20) / 4096.0f - 0.5f) * half_cell,
                      ((float)(r4 >> 20) / 4096.0f - 0.5f) * half_cell);
    const uint32_t j = r1 % p.count;
    store_tracer(s, slot, tracer_clamp(p, load3(&s->pos[4 * (size_t)j]) + jit),
                 length(load3(&s->vel[4 * (size_t)j])));
}

inline int32_t to_fixed(float v) {  // WGSL i32(f32): clamp, then toward zero
    const float f = v * FIXED;
    if (!(f == f)) return 0;
    if (f >= 2147483648.0f) return 2147483647;
    if (f <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)f;
}

}  // namespace

void or_sim_advect(OrSim *s, const OrStep *st) {  // sim_tracers.wgsl:140-183
    const OrParams &p = s->p;
    const float decay = std::exp(-st->dt / T_CHARGE);
    const float p_respawn = st->dt / TAU;
    const float p_stray = st->dt / TAU_STRAY;
    const uint32_t seed_h = pcg(st->seed);
    const uint32_t cells_x = p.dims[0], cells_y = p.dims[1];
#pragma omp parallel for num_threads(nthreads()) schedule(static)
    for (int64_t ii = 0; ii < (int64_t)s->ntr; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const uint32_t r0 = pcg(i ^ seed_h);
        if ((float)r0 / 4294967296.0f < p_respawn) {
            respawn(s, i, r0);
            continue;
        }
        float old[4];
        load_tracer(s, i, old);
        V3 pos = v3(old[0], old[1], old[2]);
        const float gp[3] = {(float)((pos.x - p.box_min[0]) / p.cell - 0.5f),
                             (float)((pos.y - p.box_min[1]) / p.cell - 0.5f),
                             (float)((pos.z - p.box_min[2]) / p.cell - 0.5f)};
        uint32_t base[3];
        float f[3];
        for (int a = 0; a < 3; ++a) {
            const float fl = std::floor(gp[a]);
            int32_t bi;
            if (!(fl == fl)) bi = 0;
            else if (fl >= 2147483648.0f) bi = 2147483647;
            else if (fl <= -2147483648.0f) bi = (int32_t)0x80000000u;
            else bi = (int32_t)fl;
            const int32_t top = (int32_t)p.dims[a] - 2;
            bi = bi < 0 ? 0 : (bi > top ? top : bi);
            base[a] = (uint32_t)bi;
            f[a] = clampw(gp[a] - (float)base[a], 0.0f, 1.0f);
        }
        float mx = 0.0f, my = 0.0f, mz = 0.0f, wc = 0.0f;
        for (uint32_t k = 0; k < 8; ++k) {
            const uint32_t ox = k & 1u, oy = (k >> 1) & 1u, oz = (k >> 2) & 1u;
            const float wx = ox ? f[0] : 1.0f - f[0];
            const float wy = oy ? f[1] : 1.0f - f[1];
            const float wz = oz ? f[2] : 1.0f - f[2];
            const float weight = wx * wy * wz;
            const uint32_t c = ((base[2] + oz) * cells_y + (base[1] + oy)) * cells_x + (base[0] + ox);
            const int32_t *cell = &s->vel_flat[4 * (size_t)c];
            mx += weight * (float)cell[0];
            my += weight * (float)cell[1];
            mz += weight * (float)cell[2];
            wc += weight * (float)cell[3];
        }
        V3 v = v3(0.f, 0.f, 0.f);
        if (wc > 0.0f) {
            const float den = wc * FIXED;
            v = v3(mx / den, my / den, mz / den);
        } else if ((float)pcg(r0 ^ 0x85ebca6bu) / 4294967296.0f < p_stray) {
            respawn(s, i, pcg(r0 ^ 0x632be59bu));
            continue;
        }
        pos = pos + v * st->dt;
        store_tracer(s, i, tracer_clamp(p, pos), fmaxw(length(v), old[3] * decay));
    }
}

void or_sim_tracers(OrSim *s, const OrStep *st) {
    const OrParams &p = s->p;
    const OrGrid g = grid_of(p);
    // splat (sim_tracers.wgsl:98-114): integer sums, order-free
    for (size_t i = 0; i < s->n; ++i) {
        const uint32_t c = cell_of_t(&g, &s->pos[4 * i]);
        const Real *v = &s->vel[4 * i];
        int32_t *cell = &s->vel_grid[4 * (size_t)c];
        cell[0] = (int32_t)((uint32_t)cell[0] + (uint32_t)to_fixed(v[0]));
        cell[1] = (int32_t)((uint32_t)cell[1] + (uint32_t)to_fixed(v[1]));
        cell[2] = (int32_t)((uint32_t)cell[2] + (uint32_t)to_fixed(v[2]));
        cell[3] = (int32_t)((uint32_t)cell[3] + 1u);
    }
    // resolve (:122-138)
    std::memcpy(s->vel_flat.data(), s->vel_grid.data(), 4 * s->vel_grid.size());
    std::fill(s->vel_grid.begin(), s->vel_grid.end(), 0);
    or_sim_advect(s, st);
}

void or_sim_field(const OrSim *s, int field, void *out) {
    const size_t n = s->n;
    switch (field) {
    case OR_FIELD_DENSITY: copy_out(out, s->density); break;
    case OR_FIELD_ALPHA: copy_out(out, s->alpha); break;
    case OR_FIELD_KD: copy_out(out, s->kd); break;
    case OR_FIELD_PRESSURE: copy_out(out, s->pressure); break;
    case OR_FIELD_NBR_N: std::memcpy(out, s->nbr_n.data(), 4 * n); break;
    case OR_FIELD_STARTS: std::memcpy(out, s->starts.data(), 4 * s->starts.size()); break;
    case OR_FIELD_PERM: std::memcpy(out, s->perm.data(), 4 * n); break;
    case OR_FIELD_WORK_POS: copy_out(out, s->wpos); break;
    case OR_FIELD_WORK_VEL: copy_out(out, s->wvel); break;
    case OR_FIELD_ACCEL: copy_out(out, s->accel); break;
    case OR_FIELD_XSPH: copy_out(out, s->xsph); break;
    case OR_FIELD_WALL_GRAD: copy_out(out, s->wgrad); break;
    case OR_FIELD_WORK_PREV_VEL: copy_out(out, s->wpvel); break;
    case OR_FIELD_WORK_PREV_P: copy_out(out, s->wpp); break;
    case OR_FIELD_WORK_TEMP: copy_out(out, s->wtemp); break;
    case OR_FIELD_PINC: copy_out(out, s->pinc); break;
    case OR_FIELD_NBR: {
        uint32_t *o = (uint32_t *)out;
        const uint32_t cap = s->p.nbr_cap;
        for (size_t i = 0; i < n; ++i)
            for (uint32_t k = 0; k < cap; ++k) o[i * cap + k] = k < s->nbr_n[i] ? s->nbr[(size_t)k * n + i] : 0xffffffffu;
        break;
    }
    case OR_FIELD_COUNTERS: {
        uint32_t *o = (uint32_t *)out;
        o[0] = s->clamp_count;
        o[1] = s->nbr_over;
        break;
    }
    default: break;
    }
}



// ---- the render-side thickness field ------------------------------------------

static float or_clampf(float e, float lo, float hi) { return std::fmin(std::fmax(e, lo), hi); }

// sim_sprites.wgsl lens_at
static float or_lens_value(uint32_t lens, const float *v, const float *pv, float rho, float lo, float hi) {
    float m;
    switch (lens) {
    case 1u: m = v[3]; break;
    case 2u: m = pv[3]; break;
    case 3u: m = rho; break;
    default: m = std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]); break;
    }
    return or_clampf((m - lo) / (hi - lo), 0.0f, 1.0f);
}

// Weights summed as 2^-20 fixed-point integers (order-free), then the decay
// and the blend constant per texel in FP32.
void or_field_splat(const float *pos4, const float *vel4, const float *pvel4, const float *density,
                    uint32_t n, const float geom[7], uint32_t w, uint32_t h, uint32_t lens, float keep,
                    float *field2) {
    const float gcx = geom[0], gcy = geom[1], ex = geom[2], ey = geom[3], radius = geom[4];
    const float lo = geom[5], hi = geom[6];
    const double scale = 1048576.0;
    std::vector<unsigned long long> acc(2 * (size_t)w * h, 0ull);
    const float W = (float)w, H = (float)h;
    for (uint32_t i = 0; i < n; ++i) {
        const float *p = &pos4[4 * (size_t)i];
        const float px = (p[0] - gcx) / ex, py = (p[1] - gcy) / ey;
        const float rx = radius / ex, ry = radius / ey;
        int tx0 = (int)std::floor((px - rx + 1.0f) * 0.5f * W - 0.5f) - 1;
        int tx1 = (int)std::ceil((px + rx + 1.0f) * 0.5f * W - 0.5f) + 1;
        int ty0 = (int)std::floor((1.0f - (py + ry)) * 0.5f * H - 0.5f) - 1;
        int ty1 = (int)std::ceil((1.0f - (py - ry)) * 0.5f * H - 0.5f) + 1;
        tx0 = tx0 < 0 ? 0 : tx0;
        ty0 = ty0 < 0 ? 0 : ty0;
        tx1 = tx1 > (int)w - 1 ? (int)w - 1 : tx1;
        ty1 = ty1 > (int)h - 1 ? (int)h - 1 : ty1;
        const float lv = lens ? or_lens_value(lens, &vel4[4 * (size_t)i], &pvel4[4 * (size_t)i], density[i], lo, hi)
                              : 0.0f;
        for (int ty = ty0; ty <= ty1; ++ty) {
            const float yt = 1.0f - ((float)ty + 0.5f) / H * 2.0f;
            const float cy = (yt - py) / ry;
            for (int tx = tx0; tx <= tx1; ++tx) {
                const float xt = ((float)tx + 0.5f) / W * 2.0f - 1.0f;
                const float cx = (xt - px) / rx;
                const float falloff = std::fmax(1.0f - (cx * cx + cy * cy), 0.0f);
                const float wt = falloff * falloff * 0.5f;
                if (wt > 0.0f) {
                    unsigned long long *a = &acc[2 * ((size_t)ty * w + tx)];
                    a[0] += (unsigned long long)std::llrint((double)wt * scale);
                    if (lens) a[1] += (unsigned long long)std::llrint((double)(wt * lv) * scale);
                }
            }
        }
    }
    const float splat = 1.0f - keep;
    for (size_t t = 0; t < (size_t)w * h; ++t) {
        const float r = (float)((double)acc[2 * t] / scale);
        const float g = (float)((double)acc[2 * t + 1] / scale);
        field2[2 * t] = field2[2 * t] * keep + splat * r;
        field2[2 * t + 1] = field2[2 * t + 1] * keep + splat * g;
    }
}

// The tile computation of field_filter written per texel: H blurs along x
// over edge-clamped taps, V blurs H along y, and the differences take V at
// the four neighbours (which may lie one texel past the edge, as the tile's
// apron does).
void or_field_filter(const float *field2, uint32_t w, uint32_t h, float ex, float ey, float *out4) {
    const float B[4] = {0.3125f, 0.234375f, 0.09375f, 0.015625f};
    auto cl = [](int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); };
    auto raw = [&](int x, int y) { return field2[2 * ((size_t)cl(y, (int)h - 1) * w + cl(x, (int)w - 1))]; };
    auto hblur = [&](int x, int y) {
        float a = raw(x, y) * B[0];
        for (int k = 1; k <= 3; ++k) a += (raw(x + k, y) + raw(x - k, y)) * B[k];
        return a;
    };
    auto vblur = [&](int x, int y) {
        float a = hblur(x, y) * B[0];
        for (int k = 1; k <= 3; ++k) a += (hblur(x, y + k) + hblur(x, y - k)) * B[k];
        return a;
    };
    const float sx = 2.0f * ex / (float)w, sy = 2.0f * ey / (float)h;
    const float aspect = (sx * sx) / (sy * sy);
    for (int y = 0; y < (int)h; ++y)
        for (int x = 0; x < (int)w; ++x) {
            const float d = vblur(x, y), xp = vblur(x + 1, y), xm = vblur(x - 1, y);
            const float yp = vblur(x, y + 1), ym = vblur(x, y - 1);
            const float lap = (xp + xm - 2.0f * d) + (yp + ym - 2.0f * d) * aspect;
            float *o = &out4[4 * ((size_t)y * w + x)];
            o[0] = d;
            o[1] = xp - xm;
            o[2] = ym - yp;
            o[3] = lap;
        }
}

}  // extern "C"
