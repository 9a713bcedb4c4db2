// common.cuh — shared device definitions for libfluidcu.
//
// Arithmetic contract: every physics kernel is compiled with -fmad=false,
// IEEE division and square root, no flush-to-zero. WGSL expressions keep
// their left-to-right association (dot = (x*x' + y*y') + z*z'), so each
// particle's result is a fixed function of its inputs and the neighbour
// order (stencil cells 0..26 with x fastest, slot order inside a cell).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/fluid_cu.h"

namespace fcu {

// Physical constants of the solver (sim_solve.wgsl:84-172, :792).
constexpr float TOUCH_RATE = 40.0f;
constexpr float K_NEAR = 3000.0f;
constexpr float DYNAMIC_VISCOSITY = 1.002e-3f;
constexpr float HEAT_CAPACITY = 4184.0f;
constexpr float CONDUCTIVITY = 0.598f;
constexpr float EXPANSION = 2.07e-4f;
constexpr float SIGMA_WATER = 0.0728f;
constexpr float LATTICE_SIGMA = 0.8665f;
constexpr float COS_CONTACT = -0.342f;
constexpr float HUGE_F = 1e30f;

// Device error flags (sticky, OR-ed into a device word).
enum : uint32_t {
    ERRF_SCAN_TIMEOUT = 1u,  // a decoupled look-back wait gave up
    ERRF_SORT_TIMEOUT = 2u,
};

// How long a look-back spin may poll one predecessor before it gives up:
// each poll is one L2 round trip (~0.5-1 us), so this is far above any
// legitimate wait and well below a second.
constexpr uint32_t kSpinLimit = 1u << 20;

struct DevParams {
    float box_min[3];
    float cell;
    uint32_t dims[3];
    uint32_t count;
    float h, mass, rho0, inv_h, sigma, sigma_h, support_sq;
    float wall_lo[3];
    float wall_hi[3];
    float tracer_c[3];
    float tracer_e[3];
    float xsph_blend;
    uint32_t nbr_cap;
};
static_assert(sizeof(DevParams) == sizeof(FluidSimParams), "params layout");

// The Step block as kernels read it, plus constants the host derives once
// per substep from dt (libm expf on the host, identical for every thread).
struct DevStep {
    FluidStep s;
    float xsph_blend;  // 1 - exp(-6 dt), or the configured blend
    float chase;       // 1 - exp(-20 dt)
    float decay;       // exp(-dt / 4), tracer charge
    float pad;
};

// Residual accumulators: one slot per iteration of a fixed schedule (the
// slots are cleared at the start of every substep), slot 0 reused by the
// tolerance loop (cleared by the kernel that reads it).
constexpr int kAccSlots = 128;
constexpr uint32_t kMaxIters = kAccSlots - 2;

// Per-substep solver counters the host reads back (the head, up to
// acc_div, is what a statistics read copies), then the accumulators.
struct DevSolve {
    double div_res, den_res;
    uint32_t div_iters, den_iters;
    uint32_t clamp_count, nbr_over;  // cumulative
    uint32_t error;
    uint32_t cursor;  // step ring read position
    unsigned long long substeps;
    unsigned long long total_div_iters;  // cumulative applies since create
    unsigned long long total_den_iters;
    uint32_t div_active, den_active;     // the box's tolerance loops go on
    unsigned long long acc_div[kAccSlots];  // fixed-point residual sums (2^-28)
    unsigned long long acc_den[kAccSlots];
};
constexpr size_t kSolveHeadBytes = 72;
static_assert(offsetof(DevSolve, acc_div) == kSolveHeadBytes, "DevSolve head");

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 operator-(F3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ F3 operator/(F3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len(F3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ F3 xyz(float4 v) { return f3(v.x, v.y, v.z); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float clampf(float e, float lo, float hi) { return fminf(fmaxf(e, lo), hi); }

// Cell coordinate of one axis: WGSL's saturating u32 conversion (negative
// and NaN to 0), then min with dims - 1 (sim_grid.wgsl:36-42).
__device__ __forceinline__ uint32_t axis_cell(float v, float mn, float cell, uint32_t dim) {
    const uint32_t u = __float2uint_rz((v - mn) / cell);
    return u < dim - 1u ? u : dim - 1u;
}

// Slabs per cell along x in a simulation's grid keys (GridGeom::slabs).
// Four measured on the 1M tilt workload: density_div 0.643 -> 0.610 ms
// (about 30 % fewer candidates), the list sweeps 2-3 % faster, the grid
// build 0.11 -> 0.12 ms (four times the starts), the plain step 4 % faster.
#ifndef FCU_SLABS
#define FCU_SLABS 4
#endif
constexpr uint32_t kSimSlabs = FCU_SLABS;

// Slab of coordinate v inside its cell c of one axis: the cell cut into
// `slabs` equal slabs across the axis, 0 .. slabs - 1, counted by threshold
// tests (a NaN offset, or one below the cell, gives 0; one past it, the last
// slab). Monotonic in v for a fixed c, and with the cell, so the key
// cell * slabs + slab orders an axis like its coordinate.
__device__ __forceinline__ uint32_t axis_slab(float v, float mn, float cell, uint32_t c, uint32_t slabs) {
    const float off = v - (mn + (float)c * cell);
    uint32_t s = 0;
    for (uint32_t k = 1; k < slabs; ++k) s += off >= cell * ((float)k / (float)slabs) ? 1u : 0u;
    return s;
}

// Fixed-point scale of the residual sums: 2^-28 per unit, each term capped
// at 16, so a 64-bit sum over 2^32 particles cannot wrap.
constexpr double kFixedScale = 268435456.0;
__device__ __forceinline__ unsigned long long fixed_term(double t) {
    if (!(t > 0.0)) return 0ull;
    if (t > 16.0) t = 16.0;
    return (unsigned long long)__double2ll_rn(t * kFixedScale);
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Adds one thread's fixed-point term into *acc: warp sum, then one atomic
// per warp. Integer sums, so the total does not depend on the order.
__device__ __forceinline__ void accumulate_fixed(unsigned long long *acc, unsigned long long v) {
    v = warp_sum_u64(v);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(acc, v);
}

// The same when lanes may add to different accumulators (a warp that
// straddles two boxes): one atomic per warp when they all share one, one
// per lane otherwise. Every lane of the warp must call it.
__device__ __forceinline__ void accumulate_at(unsigned long long *acc, unsigned long long v) {
    const uint32_t peers = __match_any_sync(0xffffffffu, (unsigned long long)acc);
    if (peers == 0xffffffffu) {
        v = warp_sum_u64(v);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(acc, v);
    } else if (v) {
        atomicAdd(acc, v);
    }
}

// Adds `v` to a per-box 32-bit counter the same way.
__device__ __forceinline__ void count_at(uint32_t *ctr, uint32_t v) {
    const uint32_t peers = __match_any_sync(0xffffffffu, (unsigned long long)ctr);
    if (peers == 0xffffffffu) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(ctr, v);
    } else if (v) {
        atomicAdd(ctr, v);
    }
}

}  // namespace fcu
