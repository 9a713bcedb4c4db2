// solve.cu — DFSPH sweeps for sm_100a, one thread per particle.
//
// Reference: crates/fluid-core/src/sim_solve.wgsl (whole file). The reference
// splits each particle over 8 subgroup lanes; here a particle is one thread
// (a million particles fill 148 SMs many times over) and its neighbours are
// summed in one fixed order: the 27 stencil cells with x fastest, walked as
// nine rows of three x-adjacent cells, which are one contiguous slot range of
// the cell-ordered working set; slots ascending. A neighbour list entry is 8
// bytes, the slot j and the kernel-gradient scale dw / r density_div found
// (slot-major, so a warp's k-th entries are adjacent); later sweeps form the
// gradient (dw / r) * (x_i - x_j) from the positions, which do not move
// inside a substep, bit for bit the value density_div had.
//
// Compiled with -fmad=false: no product-sum is fused unless written so.
#include <cuda_fp16.h>

#include "solve.cuh"

// Neighbour batches of the list sweeps (see walk below): entries whose
// records are loaded before any is used. Position + kappa records, position
// + velocity records, and forces_eval's five records; FCU_MINB is the
// minimum resident blocks per SM the sweeps are compiled for (0: none).
#ifndef FCU_B_KD
#define FCU_B_KD 4
#endif
#ifndef FCU_B_PV
#define FCU_B_PV 4
#endif
#ifndef FCU_B_N5
#define FCU_B_N5 1
#endif
// Minimum resident blocks per SM that density_div (at 128 threads a block;
// scaled for other block sizes; a batch too: its instance measured 3 %
// faster held to it) and the one box's kappa sweeps are compiled for (0:
// none), and density_div's hits staged per round.
// density_div at 8 blocks (64 registers, 24 bytes spilled) measured 0.590
// against 0.608 ms at 7 (72 registers) and 0.624 at 6 on the 1M workload
// with four x slabs per cell.
#ifndef FCU_MINB_DD
#define FCU_MINB_DD 8
#endif
// The batch's instance (box lookups) spills 58 bytes at 8 blocks.
#ifndef FCU_MINB_DD_BATCH
#define FCU_MINB_DD_BATCH 7
#endif
#ifndef FCU_MINB_KAPPA
#define FCU_MINB_KAPPA 0
#endif
// The batch's kappa sweeps (box lookups and per-box accumulators) would take
// 87-88 registers; held to the one box's 80 so that as many threads stay
// resident (768 a SM).
constexpr int kBatchKappaThreads = 768;
#ifndef FCU_STAGE
#define FCU_STAGE 32
#endif
// Candidates density_div loads before testing any (a round may then stage
// up to FCU_STAGE + FCU_DD_CHUNK - 1 hits).
#ifndef FCU_DD_P2
#define FCU_DD_P2 2
#endif
#ifndef FCU_DD_CHUNK
#define FCU_DD_CHUNK 4
#endif
#ifndef FCU_MINB
#define FCU_MINB 0
#endif
// One box's forces_eval (plain and with the divergence prediction) at 8
// blocks of 128 threads per SM (64 registers; the fused one spills 24
// bytes): frames 1.1 % shorter on the 1M workload than at its 72 / 76
// registers (7 / 6 blocks). Scaled for other block sizes like density_div.
#ifndef FCU_MINB_FORCES
#define FCU_MINB_FORCES 8
#endif
// The batch's forces_eval at 7 blocks of 128 per SM (scaled likewise):
// batched_256 8.88 against 9.05 ms a substep with no floor, 9.12 at 8.
#ifndef FCU_MINB_FORCES_BATCH
#define FCU_MINB_FORCES_BATCH 7
#endif

namespace fcu {

namespace {

// The kernel's constants a neighbour pair needs, apart from the rest of a
// box's parameters: a batch's sweeps keep these four in registers and read
// the others from the box's entry where they are used.
struct KernelConsts {
    float sigma, sigma_h, inv_h, support_sq;
};
__device__ __forceinline__ KernelConsts kernel_consts(const DevParams &P) {
    return KernelConsts{P.sigma, P.sigma_h, P.inv_h, P.support_sq};
}

template <class KP>
__device__ __forceinline__ float kernel_q(const KP &P, float q) {  // :176-182
    if (q < 1.0f) return P.sigma * (1.0f - 1.5f * q * q * (1.0f - 0.5f * q));
    const float t = 2.0f - q;
    return P.sigma * 0.25f * t * t * t;
}

// grad_q (sim_solve.wgsl:184-196) returns (dw / r) * x; this is its scalar
// dw / r, and 0 under the r < 1e-9 guard (0 * x sums exactly like the
// guard's zero vector: a signed zero added to any sum leaves it unchanged).
template <class KP>
__device__ __forceinline__ float grad_scale(const KP &P, float r, float q) {
    if (r < 1e-9f) return 0.0f;
    float dw;
    if (q < 1.0f) {
        dw = P.sigma_h * (-3.0f * q + 2.25f * q * q);
    } else {
        const float t = 2.0f - q;
        dw = P.sigma_h * (-0.75f * t * t);
    }
    return dw / r;
}

__device__ __forceinline__ float cohesion(float r, float c, float k, float near) {  // :201-210
    if (r >= c || r < 1e-9f) return 0.0f;
    const float a = (c - r) * (c - r) * (c - r) * r * r * r;
    if (2.0f * r > c) return k * a;
    return k * (2.0f * a - near);
}

__device__ __forceinline__ float wall_density(float t) {  // :213-222
    if (t >= 2.0f) return 0.0f;
    const float t3 = t * t * t;
    if (t < 1.0f) return 0.5f - 0.7f * t + t3 * (1.0f / 3.0f + t * t * (-0.15f + 0.05f * t));
    return 8.0f / 15.0f - 0.8f * t + t3 * (2.0f / 3.0f + t * (-0.5f + t * (0.15f - t / 60.0f)));
}

__device__ __forceinline__ float wall_gradient(float t) {  // :226-235
    if (t >= 2.0f) return 0.0f;
    const float t2 = t * t;
    if (t < 1.0f) return 0.7f + t2 * (-1.0f + t2 * (0.75f - t * 0.3f));
    return 0.8f + t2 * (-2.0f + t * (2.0f + t * (-0.75f + t * 0.1f)));
}

__device__ __forceinline__ float wedge(float t1, float t2) {  // :249-270
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

__device__ __forceinline__ float wedge_d(float t1, float t2) {  // :272-293
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

__device__ __forceinline__ float wall_adhesion(float t) {  // :334-340
    const float u = clampf(2.0f - t, 0.0f, 2.0f);
    return u * u *
           (1.7847015e-3f +
            u * (3.3392196e-3f + u * (-4.3394677e-3f + u * (1.6711868e-3f + u * (-2.1788750e-4f)))));
}

__device__ __forceinline__ float wedge_dsum(float t, float a, float b, float c, float d) {  // :295
    return wedge_d(t, a) + wedge_d(t, b) + wedge_d(t, c) + wedge_d(t, d);
}

__device__ __forceinline__ float wedge_sum(F3 tl, F3 th) {  // :299-304
    float w = wedge(tl.x, tl.y) + wedge(tl.x, th.y) + wedge(th.x, tl.y) + wedge(th.x, th.y);
    w += wedge(tl.x, tl.z) + wedge(tl.x, th.z) + wedge(th.x, tl.z) + wedge(th.x, th.z);
    w += wedge(tl.y, tl.z) + wedge(tl.y, th.z) + wedge(th.y, tl.z) + wedge(th.y, th.z);
    return w;
}

__device__ __forceinline__ F3 wall_lo(const DevParams &P) { return f3(P.wall_lo[0], P.wall_lo[1], P.wall_lo[2]); }
__device__ __forceinline__ F3 wall_hi(const DevParams &P) { return f3(P.wall_hi[0], P.wall_hi[1], P.wall_hi[2]); }

__device__ F3 wall_grad_sum(const DevParams &P, F3 pos) {  // :310-328
    const F3 lo = wall_lo(P), hi = wall_hi(P);
    const float inv_h = 1.0f / P.h;
    const F3 tl = (pos - lo) * inv_h;
    const F3 th = (hi - pos) * inv_h;
    const float scale = P.rho0 * inv_h;
    F3 g = f3(0.f, 0.f, 0.f);
    g.x -= scale * (wall_gradient(tl.x) + wedge_dsum(tl.x, tl.y, th.y, tl.z, th.z));
    g.x += scale * (wall_gradient(th.x) + wedge_dsum(th.x, tl.y, th.y, tl.z, th.z));
    g.y -= scale * (wall_gradient(tl.y) + wedge_dsum(tl.y, tl.x, th.x, tl.z, th.z));
    g.y += scale * (wall_gradient(th.y) + wedge_dsum(th.y, tl.x, th.x, tl.z, th.z));
    g.z -= scale * (wall_gradient(tl.z) + wedge_dsum(tl.z, tl.x, th.x, tl.y, th.y));
    g.z += scale * (wall_gradient(th.z) + wedge_dsum(th.z, tl.x, th.x, tl.y, th.y));
    return g;
}

__device__ F3 wall_adh_sum(const DevParams &P, F3 pos) {  // :349-361
    const F3 lo = wall_lo(P), hi = wall_hi(P);
    const float inv_h = 1.0f / P.h;
    F3 a = f3(0.f, 0.f, 0.f);
    a.x -= wall_adhesion((pos.x - lo.x) * inv_h);
    a.x += wall_adhesion((hi.x - pos.x) * inv_h);
    a.y -= wall_adhesion((pos.y - lo.y) * inv_h);
    a.y += wall_adhesion((hi.y - pos.y) * inv_h);
    a.z -= wall_adhesion((pos.z - lo.z) * inv_h);
    a.z += wall_adhesion((hi.z - pos.z) * inv_h);
    return a;
}

// exp for per-particle arguments: Cody-Waite reduction by ln2 (16-bit head,
// tail), degree-7 Taylor polynomial of e^r in Horner form, scale by 2^k
// through the exponent bits. The CPU oracle evaluates the same sequence.
__device__ __forceinline__ float det_exp(float x) {
    if (!(x > -87.0f)) return 0.0f;
    if (x > 88.0f) x = 88.0f;
    const float kf = rintf(x * 1.44269504f);
    float r = x - kf * 0.693145752f;
    r = r - kf * 1.42860677e-6f;
    float p = 1.98412698e-4f;
    p = p * r + 1.38888889e-3f;
    p = p * r + 8.33333333e-3f;
    p = p * r + 4.16666667e-2f;
    p = p * r + 1.66666667e-1f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    const int k = (int)kf;
    return p * __uint_as_float((uint32_t)(k + 127) << 23);
}

// The neighbour's kernel gradient, bit for bit what grad_q returned for the
// pair in density_div: its stored scale dw / r times x_i - x_j.
__device__ __forceinline__ F3 pair_grad(float scale, F3 pos, float4 pj) {
    return scale * (pos - xyz(pj));
}

// Walks particle i's neighbour list in list order, B entries at a time: the
// B list entries are loaded, then the B neighbours' records, and only then
// is any of them used, so one batch's loads overlap instead of each
// neighbour waiting on the round trip of the one before. The partial last
// batch loads the particle's own record in its empty places and skips them.
// `use(scale, record)` sees the neighbours in the same order as a plain
// loop, so every sum is the same sum.
// A list entry is read once per sweep: with FCU_LIST_CS it is loaded with
// the streaming (evict-first) hint, leaving the caches to the neighbours'
// records. With FCU_PREFETCH the entries of the next batch are requested
// before the current batch's records are used.
#ifndef FCU_LIST_CS
#define FCU_LIST_CS 1
#endif
#ifndef FCU_PREFETCH
#define FCU_PREFETCH 1
#endif
// FCU_L2PF > 0: each batch also asks L2 for the list rows FCU_L2PF batches
// past the next one (no registers held), so the entries' DRAM round trip
// starts earlier.
#ifndef FCU_L2PF
#define FCU_L2PF 1
#endif
__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
__device__ __forceinline__ uint2 list_ld(const uint2 *p) {
#if FCU_LIST_CS
    return __ldcs(p);
#else
    return __ldg(p);
#endif
}

template <int B, class T, class Load, class Use>
__device__ __forceinline__ void walk(const uint2 *__restrict__ nbr, uint32_t n, uint32_t i,
                                     uint32_t cnt, Load load, Use use) {
#if FCU_PREFETCH
    uint2 e[B];
#pragma unroll
    for (int u = 0; u < B; ++u) e[u] = ((uint32_t)u < cnt) ? list_ld(&nbr[(size_t)u * n + i]) : make_uint2(i, 0u);
    for (uint32_t k = 0; k < cnt; k += B) {
        T v[B];
#pragma unroll
        for (int u = 0; u < B; ++u) v[u] = load(e[u].x);
        uint2 en[B];
#pragma unroll
        for (int u = 0; u < B; ++u)
            en[u] = (k + B + u < cnt) ? list_ld(&nbr[(size_t)(k + B + u) * n + i]) : make_uint2(i, 0u);
#if FCU_L2PF
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const uint32_t kf = k + B * (1 + FCU_L2PF) + u;
            if (kf < cnt) prefetch_l2(&nbr[(size_t)kf * n + i]);
        }
#endif
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (k + u < cnt) use(__uint_as_float(e[u].y), v[u]);
#pragma unroll
        for (int u = 0; u < B; ++u) e[u] = en[u];
    }
#else
    for (uint32_t k = 0; k < cnt; k += B) {
        uint2 e[B];
#pragma unroll
        for (int u = 0; u < B; ++u)
            e[u] = (k + u < cnt) ? list_ld(&nbr[(size_t)(k + u) * n + i]) : make_uint2(i, 0u);
        T v[B];
#pragma unroll
        for (int u = 0; u < B; ++u) v[u] = load(e[u].x);
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (k + u < cnt) use(__uint_as_float(e[u].y), v[u]);
    }
#endif
}

struct PosKd {
    float4 p;
    float kd;
};
struct PosVel {
    float4 p, v;
};
struct Nbr5 {
    float4 p, v;
    float rho, temp, near;
};

// Particle counts stay below 2^28 (the host rejects more), so masking a list
// entry's slot changes no slot. forces_eval's loader applies the mask before
// forming its five record addresses: measured 13 % faster on the 1M-particle
// workload (0.58 against 0.67 ms); in the kappa sweeps it measured slower and
// is left out.
constexpr uint32_t kSlotMask = (1u << 28) - 1u;
__device__ __forceinline__ uint32_t list_slot(uint32_t code) { return code & kSlotMask; }

// ---- gather into the working set (sim_grid.wgsl:52-63) -------------------
__global__ void __launch_bounds__(256) k_gather(SimBufs b, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t i = __ldg(&b.perm[k]);
    if (i >= n) i = k;  // only after a grid build that gave up; keeps reads in bounds
    b.wpos[k] = __ldg(&b.pos[i]);
    b.wvel[k] = __ldg(&b.vel[i]);
    b.wpvel[k] = __ldg(&b.pvel[i]);
    b.wpp[k] = __ldg(&b.pp[i]);
    b.wtemp[k] = __ldg(&b.temp[i]);
    b.wid[k] = __ldg(&b.id[i]);
}

// Per-box views of a Geo. kB (batch) is a template flag so the one-box
// kernels keep their constants in parameter space and their sums on the
// plain warp-aggregated atomics.
template <bool kB>
__device__ __forceinline__ uint32_t box_index(const Geo &g, uint32_t i) {
    return kB ? (uint32_t)__ldg(&g.box_of[i]) : 0u;
}
template <bool kB>
__device__ __forceinline__ DevParams params_of(const Geo &g, uint32_t bi) {
    if (kB) return g.box[bi];
    return g.one;
}
// The same by reference: the box's entry in global memory (batch), or the
// kernel's own parameter space (one box: the kernel takes Geo as
// __grid_constant__, so no copy is made).
template <bool kB>
__device__ __forceinline__ const DevParams &params_ref(const Geo &g, uint32_t bi) {
    return kB ? g.box[bi] : g.one;
}
template <bool kB>
__device__ __forceinline__ uint32_t cell_base_of(const Geo &g, uint32_t bi) {
    return kB ? __ldg(&g.cell_base[bi]) : 0u;
}
template <bool kB>
__device__ __forceinline__ uint32_t first_of(const Geo &g, uint32_t bi) {
    return kB ? __ldg(&g.first[bi]) : 0u;
}
// Adds a thread's fixed-point term to its box's accumulator; every lane of
// the warp calls it.
template <bool kB>
__device__ __forceinline__ void add_term(unsigned long long *acc, unsigned long long v) {
    if (kB) accumulate_at(acc, v);
    else accumulate_fixed(acc, v);
}

// One row (oz, oy) of a particle's 27-cell stencil: three x-adjacent cells,
// one contiguous slot range of the cell-ordered working set. Cell culling: a
// stencil cell whose nearest point lies beyond the support holds no
// neighbour, so skipping it changes neither the neighbour set nor its order.
// The distances to the own cell's faces are shrunk by a margin far above
// their rounding error (1e-3 cell plus 1e-6 |pos|, ~8 ulp of the
// coordinates), so a cell is culled only when every candidate in it would
// fail r2 < support^2. Returns false for a row outside the grid or culled.
struct Stencil {
    int bx, by, bz;
    float xl, xh, yl, yh, zl, zh;
    float px, margin;
};

__device__ __forceinline__ Stencil stencil_of(const DevParams &P, F3 pos) {
    Stencil t;
    t.bx = (int)axis_cell(pos.x, P.box_min[0], P.cell, P.dims[0]);
    t.by = (int)axis_cell(pos.y, P.box_min[1], P.cell, P.dims[1]);
    t.bz = (int)axis_cell(pos.z, P.box_min[2], P.cell, P.dims[2]);
    const float margin = 1e-3f * P.cell + 1e-6f * (fabsf(pos.x) + fabsf(pos.y) + fabsf(pos.z));
    const float fx = pos.x - (P.box_min[0] + (float)t.bx * P.cell);
    const float fy = pos.y - (P.box_min[1] + (float)t.by * P.cell);
    const float fz = pos.z - (P.box_min[2] + (float)t.bz * P.cell);
    t.xl = fmaxf(fx - margin, 0.0f);
    t.xh = fmaxf(P.cell - fx - margin, 0.0f);
    t.yl = fmaxf(fy - margin, 0.0f);
    t.yh = fmaxf(P.cell - fy - margin, 0.0f);
    t.zl = fmaxf(fz - margin, 0.0f);
    t.zh = fmaxf(P.cell - fz - margin, 0.0f);
    t.px = pos.x;
    t.margin = margin;
    return t;
}

// Key of coordinate x along the first axis with K slabs per cell.
template <int K>
__device__ __forceinline__ uint32_t x_key(const DevParams &P, float x) {
    const uint32_t c = axis_cell(x, P.box_min[0], P.cell, P.dims[0]);
    return K > 1 ? c * K + axis_slab(x, P.box_min[0], P.cell, c, K) : c;
}

//
// With K slabs per cell (the cells' slots in slab order along x), the row's
// range is cut further to the slabs that can hold a point within the
// support in x: every candidate whose x differs from the particle's by the
// support's half-chord at the row's nearest perpendicular distance, widened
// by 0.1 % and the margin, or more fails r2 < support^2, and keys are
// monotonic in x, so the slabs of x -/+ that width bound every neighbour's.
template <int K>
__device__ __forceinline__ bool stencil_row(const DevParams &P, uint32_t cell_base,
                                            const uint32_t *__restrict__ starts, uint32_t n,
                                            const Stencil &t, int oz, int oy, uint32_t &s,
                                            uint32_t &e) {
    const int cz = t.bz + oz, cy = t.by + oy;
    if (cz < 0 || cz >= (int)P.dims[2] || cy < 0 || cy >= (int)P.dims[1]) return false;
    const float dzp = oz < 0 ? t.zl * t.zl : (oz > 0 ? t.zh * t.zh : 0.0f);
    const float dperp = dzp + (oy < 0 ? t.yl * t.yl : (oy > 0 ? t.yh * t.yh : 0.0f));
    if (dperp >= P.support_sq) return false;
    const int cx0 = (t.bx > 0 && dperp + t.xl * t.xl < P.support_sq) ? t.bx - 1 : t.bx;
    const int cx1 = (t.bx + 1 < (int)P.dims[0] && dperp + t.xh * t.xh < P.support_sq) ? t.bx + 1 : t.bx;
    const uint32_t row = ((uint32_t)cz * P.dims[1] + (uint32_t)cy) * P.dims[0];
    if (K > 1) {
        const float w = sqrtf(P.support_sq - dperp) * 1.001f + t.margin;
        const uint32_t klo = max(x_key<K>(P, t.px - w), (uint32_t)cx0 * K);
        const uint32_t khi = min(x_key<K>(P, t.px + w), (uint32_t)cx1 * K + (K - 1));
        s = __ldg(&starts[cell_base + row * K + klo]);
        e = __ldg(&starts[cell_base + row * K + khi + 1]);
    } else {
        s = __ldg(&starts[cell_base + row + cx0]);
        e = __ldg(&starts[cell_base + row + cx1 + 1]);
    }
    if (e > n) e = n;  // starts never exceed n unless a scan gave up
    return s < e;
}

// The pair terms density_div sums over one neighbour (sim_solve.wgsl:449-466).
struct DensitySums {
    float w_sum, rho_near, grad_sq, drho;
    F3 grad_sum;
};

template <class KP>
__device__ __forceinline__ float density_pair(const KP &P, DensitySums &d, F3 pos, F3 vel,
                                              F3 x, float r2, float4 vj) {
    const float r = sqrtf(r2);
    const float q = r * P.inv_h;
    d.w_sum += kernel_q(P, q);
    const float wn = fmaxf(1.0f - q, 0.0f);
    d.rho_near += wn * wn * wn;
    const float gs = grad_scale(P, r, q);
    const F3 gw = gs * x;
    d.grad_sum = d.grad_sum + gw;
    d.grad_sq += dot(gw, gw);
    d.drho += dot(vel - xyz(vj), gw);
    return gs;
}

// ---- threads ordered by neighbour count -------------------------------------
// A list sweep's warp runs as many iterations as its longest list, so lanes
// whose particles have fewer neighbours idle. A block can hand its slots to
// its threads in order of list length instead (a counting sort of the
// block's slots by nbr_n in shared memory), so each warp holds particles of
// similar counts. Which thread computes a particle changes nothing in its
// sums, so the results are the same bits. Returns this thread's slot, or
// g.n when the block has fewer slots than threads. forces_eval, issue-bound
// on its per-pair divisions, gains (0.474 -> 0.439 ms on the 1M workload);
// the L1-bound sweeps (apply 0.108 -> 0.125, forces_apply 0.10 -> 0.127 ms)
// lose more on their scattered own-record and list loads, and keep slot
// order, and density_div ordered by each particle's neighbour count of the
// last substep measured slower too (0.643 -> 0.672 ms).
#ifndef FCU_SORTED_FORCES
#define FCU_SORTED_FORCES 1
#endif
#if FCU_SORTED_FORCES
constexpr int kCountBins = 64;  // nbr_n / 2, the last bin open-ended

template <int TPB>
__device__ __forceinline__ uint32_t slot_by_count(const uint32_t *__restrict__ counts, uint32_t n) {
    __shared__ uint32_t s_bin[kCountBins];
    __shared__ uint32_t s_slot[TPB];
    const uint32_t base = blockIdx.x * TPB, tid = threadIdx.x;
    const uint32_t i0 = base + tid;
    const bool live = i0 < n;
    if (tid < (uint32_t)kCountBins) s_bin[tid] = 0u;
    __syncthreads();
    uint32_t bin = 0, rank = 0;
    if (live) {
        const uint32_t c = __ldg(&counts[i0]) >> 1;
        bin = c < (uint32_t)kCountBins ? c : (uint32_t)kCountBins - 1u;
        rank = atomicAdd(&s_bin[bin], 1u);
    }
    __syncthreads();
    if (tid < 32u) {  // exclusive scan of the 64 bins, two a lane
        const uint32_t a0 = s_bin[2 * tid], a1 = s_bin[2 * tid + 1];
        uint32_t x = a0 + a1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (tid >= (uint32_t)o) x += y;
        }
        const uint32_t excl = x - a0 - a1;
        s_bin[2 * tid] = excl;
        s_bin[2 * tid + 1] = excl + a0;
    }
    __syncthreads();
    if (live) s_slot[s_bin[bin] + rank] = i0;
    __syncthreads();
    const uint32_t count = n > base ? (n - base < (uint32_t)TPB ? n - base : (uint32_t)TPB) : 0u;
    return tid < count ? s_slot[tid] : n;
}
#endif

// ---- density_div (sim_solve.wgsl:411-518) --------------------------------
// One thread per particle, in rounds of two phases. Phase 1: the thread walks
// its own stencil candidates in order and stages each hit as a (row, offset)
// code in its column of shared memory, until kStage hits are staged or the
// stencil is done. Phase 2: it forms the sums over the staged hits, in order,
// and writes their list entries. A plain loop that sums each hit where it is
// found runs the long hit path at every candidate where any lane of the warp
// hits (ncu: 12 of 32 lanes active per instruction, 73 % issue-bound on the
// 1M-particle workload) and scatters its list stores; here the warp's lanes
// take their k-th staged hit together, so the hit path is not divergent and
// the stores of a round coalesce. The neighbours are summed in the same
// order as the plain loop, so every sum is the same sum. A stencil row wider
// than a code's 4,096-slot offset falls back to the plain loop.
constexpr int kStage = FCU_STAGE;
constexpr int kP2 = FCU_DD_P2;
constexpr uint32_t kRowSpan = 4096;

// The plain loop over every candidate, each hit summed and the first `cap`
// listed. Returns the hits found.
template <int K>
__device__ __forceinline__ uint32_t density_scan_all(const DevParams &P, uint32_t base, const SimBufs &b,
                                                  uint32_t n, uint32_t i, F3 pos, F3 vel,
                                                  const Stencil &t, DensitySums &d) {
    uint32_t found = 0;
    for (int oz = -1; oz <= 1; ++oz)
        for (int oy = -1; oy <= 1; ++oy) {
            uint32_t s, e;
            if (!stencil_row<K>(P, base, b.starts, n, t, oz, oy, s, e)) continue;
            for (uint32_t k = s; k < e; ++k) {
                if (k == i) continue;
                const F3 x = pos - xyz(__ldg(&b.wpos[k]));
                const float r2 = dot(x, x);
                if (r2 >= P.support_sq) continue;
                const float gs = density_pair(P, d, pos, vel, x, r2, __ldg(&b.wvel[k]));
                if (found < P.nbr_cap) b.nbr[(size_t)found * n + i] = make_uint2(k, __float_as_uint(gs));
                found++;
            }
        }
    return found;
}

template <bool kB, int TPB>
__global__ void __launch_bounds__(TPB, (kB ? FCU_MINB_DD_BATCH : FCU_MINB_DD) * 128 / TPB)
    k_density_div(const __grid_constant__ Geo g, SimBufs b, int slot) {
    __shared__ uint16_t s_hit[kStage + FCU_DD_CHUNK - 1][TPB];
    __shared__ uint32_t s_beg[9][TPB];
    __shared__ uint32_t s_end[9][TPB];
    const uint32_t n = g.n;
    const uint32_t tid = threadIdx.x;
    const uint32_t i = blockIdx.x * blockDim.x + tid;
    const bool live = i < n;
    const uint32_t bi = box_index<kB>(g, live ? i : n - 1);
    unsigned long long term = 0;
    if (live) {
        const DevParams &P = params_ref<kB>(g, bi);
        const KernelConsts K = kernel_consts(P);
        const uint32_t base = cell_base_of<kB>(g, bi);
        const float dt = g.st[bi].s.dt;
        const F3 pos = xyz(__ldg(&b.wpos[i]));
        const F3 vel = xyz(__ldg(&b.wvel[i]));
        const Stencil t = stencil_of(P, pos);
        const uint32_t cap = P.nbr_cap;
        DensitySums d;
        d.w_sum = P.sigma;  // lane 0's self term W(0), sim_solve.wgsl:426
        d.rho_near = 0.0f;
        d.grad_sq = 0.0f;
        d.drho = 0.0f;
        d.grad_sum = f3(0.f, 0.f, 0.f);
        bool wide = false;
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            uint32_t s = 0, e = 0;
            if (!stencil_row<(int)kSimSlabs>(P, base, b.starts, n, t, r / 3 - 1, r % 3 - 1, s, e)) s = e = 0;
            s_beg[r][tid] = s;
            s_end[r][tid] = e;
            wide = wide || (e - s > kRowSpan);
        }
        uint32_t found = 0;
        if (!wide) {
            uint32_t r = 0, k = s_beg[0][tid], e = s_end[0][tid], rs = k;
            bool more = true;
            while (more) {
                // phase 1: stage up to kStage hits
                uint32_t staged = 0;
                while (staged < (uint32_t)kStage) {
                    if (k >= e) {
                        if (++r >= 9u) {
                            more = false;
                            break;
                        }
                        k = rs = s_beg[r][tid];
                        e = s_end[r][tid];
                        continue;
                    }
#if FCU_DD_CHUNK > 1
                    {
                        float4 pc[FCU_DD_CHUNK];
#pragma unroll
                        for (int u = 0; u < FCU_DD_CHUNK; ++u) {
                            const uint32_t ku = k + u;
                            pc[u] = __ldg(&b.wpos[ku < e ? ku : i]);
                        }
                        // every squared distance first, then the tests: the
                        // candidates' arithmetic overlaps (0.88 -> 0.82 ms
                        // against testing each as it is formed)
                        float r2[FCU_DD_CHUNK];
#pragma unroll
                        for (int u = 0; u < FCU_DD_CHUNK; ++u) {
                            const F3 x = pos - xyz(pc[u]);
                            r2[u] = dot(x, x);
                        }
#pragma unroll
                        for (int u = 0; u < FCU_DD_CHUNK; ++u) {
                            const uint32_t ku = k + u;
                            if (ku < e && ku != i && r2[u] < K.support_sq) {
                                s_hit[staged][tid] = (uint16_t)((r << 12) | (ku - rs));
                                ++staged;
                            }
                        }
                        k = (e - k > (uint32_t)FCU_DD_CHUNK) ? k + FCU_DD_CHUNK : e;
                    }
#else
                    if (k != i) {
                        const F3 x = pos - xyz(__ldg(&b.wpos[k]));
                        if (dot(x, x) < K.support_sq) {
                            s_hit[staged][tid] = (uint16_t)((r << 12) | (k - rs));
                            ++staged;
                        }
                    }
                    ++k;
#endif
                }
                // phase 2: the staged hits, in order, kP2 loads in flight
                for (uint32_t h = 0; h < staged; h += kP2) {
                    uint32_t j[kP2];
#pragma unroll
                    for (int u = 0; u < kP2; ++u) {
                        const bool ok = h + u < staged;
                        const uint32_t code = ok ? (uint32_t)s_hit[h + u][tid] : 0u;
                        j[u] = ok ? s_beg[code >> 12][tid] + (code & (kRowSpan - 1u)) : i;
                    }
                    float4 pj[kP2], vj[kP2];
#pragma unroll
                    for (int u = 0; u < kP2; ++u) {
                        pj[u] = __ldg(&b.wpos[j[u]]);
                        vj[u] = __ldg(&b.wvel[j[u]]);
                    }
#pragma unroll
                    for (int u = 0; u < kP2; ++u) {
                        if (h + u < staged) {
                            const F3 x = pos - xyz(pj[u]);
                            const float gs = density_pair(K, d, pos, vel, x, dot(x, x), vj[u]);
                            const uint32_t idx = found + h + u;
                            if (idx < cap) b.nbr[(size_t)idx * n + i] = make_uint2(j[u], __float_as_uint(gs));
                        }
                    }
                }
                found += staged;
            }
        } else {
            found = density_scan_all<(int)kSimSlabs>(P, base, b, n, i, pos, vel, t, d);
        }
        // sim_solve.wgsl:475-517
        b.nbr_n[i] = found < cap ? found : cap;
        if (found > cap) atomicAdd(&g.solve[bi].nbr_over, found - cap);
        float rho = P.mass * d.w_sum;
        const float rho_near = d.rho_near;
        const float grad_sq = P.mass * P.mass * d.grad_sq;
        float drho = P.mass * d.drho;
        F3 grad_sum = P.mass * d.grad_sum;
        const F3 lo = wall_lo(P), hi = wall_hi(P);
        const F3 tl = (pos - lo) * P.inv_h;
        const F3 th = (hi - pos) * P.inv_h;
        float fill = 0.0f;
        fill += wall_density(tl.x) + wall_density(th.x);
        fill += wall_density(tl.y) + wall_density(th.y);
        fill += wall_density(tl.z) + wall_density(th.z);
        fill -= wedge_sum(tl, th);
        rho += P.rho0 * fill;
        const F3 wg = wall_grad_sum(P, pos);
        b.wgrad[i] = make_float4(wg.x, wg.y, wg.z, 0.0f);
        grad_sum = grad_sum + wg;
        b.density[i] = rho;
        b.rho_near[i] = rho_near;
        const float a = rho / fmaxf(dot(grad_sum, grad_sum) + grad_sq, 1e-4f);
        b.alpha[i] = a;
        drho += dot(vel, wg);
        const float kdv = fmaxf(drho, 0.0f) * a / fmaxf(dt, 1e-9f) / rho;
        b.kd[i] = kdv;
        b.wpk[i] = make_float4(pos.x, pos.y, pos.z, kdv);
        term = fixed_term((double)fmaxf(drho, 0.0f) * (double)dt / (double)P.rho0);
    }
    add_term<kB>(&g.solve[bi].acc_div[slot], term);
}

// Whether box bi's tolerance loop `gate` has stopped (its kernels skip it).
template <bool kB>
__device__ __forceinline__ bool gated_out(const Geo &g, uint32_t bi, int gate) {
    if (!kB || gate == kGateNone) return false;
    const DevSolve &sv = g.solve[bi];
    return (gate == kGateDiv ? sv.div_active : sv.den_active) == 0u;
}


// ---- divergence predictor for a later divergence iteration ---------------
// density_div's divergence sums again over the list, with this
// iteration's velocities.
template <bool kB, int TPB>
__global__ void __launch_bounds__(TPB, kB ? kBatchKappaThreads / TPB : FCU_MINB_KAPPA) k_div_kappa(Geo g, SimBufs b, int slot,
                                                                       int gate) {
    const uint32_t n = g.n;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const uint32_t bi = box_index<kB>(g, live ? i : n - 1);
    unsigned long long term = 0;
    if (live && !gated_out<kB>(g, bi, gate)) {
        const DevParams P = params_of<kB>(g, bi);
        const float dt = g.st[bi].s.dt;
        const F3 pos = xyz(__ldg(&b.wpos[i]));
        const F3 vel = xyz(__ldg(&b.wvel[i]));
        const uint32_t cnt = __ldg(&b.nbr_n[i]);
        float drho = 0.0f;
        walk<FCU_B_PV, PosVel>(
            b.nbr, n, i, cnt,
            [&](uint32_t j) { return PosVel{__ldg(&b.wpos[j]), __ldg(&b.wvel[j])}; },
            [&](float gs, const PosVel &q) { drho += dot(vel - xyz(q.v), pair_grad(gs, pos, q.p)); });
        drho = P.mass * drho;
        drho += dot(vel, xyz(__ldg(&b.wgrad[i])));
        const float rho = __ldg(&b.density[i]);
        const float kdv = fmaxf(drho, 0.0f) * __ldg(&b.alpha[i]) / fmaxf(dt, 1e-9f) / rho;
        b.kd[i] = kdv;
        b.wpk[i] = make_float4(pos.x, pos.y, pos.z, kdv);
        term = fixed_term((double)fmaxf(drho, 0.0f) * (double)dt / (double)P.rho0);
    }
    add_term<kB>(&g.solve[bi].acc_div[slot], term);
}

// kappa_partial (sim_solve.wgsl:596-606), sequential over the list.
__device__ __forceinline__ F3 kappa_sum(const SimBufs &b, uint32_t i, uint32_t n, F3 pos, float kd_i) {
    const uint32_t cnt = __ldg(&b.nbr_n[i]);
    F3 dv = f3(0.f, 0.f, 0.f);
    walk<FCU_B_KD, PosKd>(
        b.nbr, n, i, cnt, [&](uint32_t j) {
            const float4 q = __ldg(&b.wpk[j]);
            return PosKd{q, q.w};
        },
        [&](float gs, const PosKd &q) { dv = dv + (kd_i + q.kd) * pair_grad(gs, pos, q.p); });
    return dv;
}

// ---- apply_kappa_wide: div_apply / den_apply (sim_solve.wgsl:608-621) -----
// For the density iterations the applied pressure k*rho that den_kappa held
// back joins the pressure here, with the kappa it belongs to.
template <bool kB>
__device__ __forceinline__ void apply_at(const Geo &g, const SimBufs &b, uint32_t i, int add_pressure,
                                         int gate) {
    const uint32_t n = g.n;
    const uint32_t bi = box_index<kB>(g, i);
    if (gated_out<kB>(g, bi, gate)) return;
    const float mass = params_of<kB>(g, bi).mass;
    const float dt = g.st[bi].s.dt;
    const F3 pos = xyz(__ldg(&b.wpos[i]));
    const float kd_i = b.kd[i];
    const F3 total = kappa_sum(b, i, n, pos, kd_i);
    const F3 dv_full = mass * total + kd_i * xyz(__ldg(&b.wgrad[i]));
    const float4 was = b.wvel[i];
    const F3 v = xyz(was) - dt * dv_full;
    b.wvel[i] = make_float4(v.x, v.y, v.z, was.w);
    if (add_pressure) b.pressure[i] += b.pinc[i];
}

template <bool kB, int TPB>
__global__ void __launch_bounds__(TPB, FCU_MINB) k_apply(Geo g, SimBufs b, int add_pressure, int gate) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < g.n) apply_at<kB>(g, b, i, add_pressure, gate);
}

// ---- forces_eval (sim_solve.wgsl:524-592) ---------------------------------
// With kDiv, the same walk also forms the divergence prediction of
// k_div_kappa (the same pair terms, in the same order, so the same sums):
// its kappa goes to kd2 / wpk2 and its residual term to acc_div[slot], and
// boxes whose divergence loop has stopped (gate) are skipped. The tolerance
// schedule runs this after each divergence apply, so the prediction that
// only decides whether the loop stops costs no sweep of its own.
template <bool kB, bool kDiv>
__device__ __forceinline__ void forces_eval_body(const Geo &g, const SimBufs &b, uint32_t i, bool live,
                                                 int slot, int gate) {
    const uint32_t n = g.n;
    if (!kDiv && !live) return;
    const uint32_t bi = box_index<kB>(g, live ? i : n - 1);
    unsigned long long term = 0;
    if (live && !(kDiv && gated_out<kB>(g, bi, gate))) {
    // a batch reads its box's constants from the box's entry where they are
    // used, keeping the pair loop's few in registers; one box copies them
    // from parameter space as before
    DevParams Pc;
    if (!kB) Pc = g.one;
    const DevParams &P = kB ? g.box[bi] : Pc;
    const KernelConsts K = kernel_consts(P);
    const float mass = P.mass, inv_h = P.inv_h, rho0 = P.rho0, soft = 0.01f * P.h * P.h;
    const float coh_c = 2.0f * P.h;
    const float c3 = coh_c * coh_c * coh_c;
    const float coh_k = 32.0f / (3.14159265f * c3 * c3 * c3);
    const float coh_near = c3 * c3 / 64.0f;
    const float c = 2.0f * P.h;
    const float gamma = SIGMA_WATER * 7040.0f / (21.0f * LATTICE_SIGMA * P.rho0 * P.rho0 * c * c);
    const float beta =
        SIGMA_WATER * (1.0f + COS_CONTACT) * 1558.4f / (LATTICE_SIGMA * P.rho0 * P.rho0 * c * c);
    const float visc_k = 2.0f * DYNAMIC_VISCOSITY;
    const float heat_k = 2.0f * CONDUCTIVITY / HEAT_CAPACITY;
    const float diss_k = 0.5f * DYNAMIC_VISCOSITY / HEAT_CAPACITY;

    const F3 pos = xyz(__ldg(&b.wpos[i]));
    const float near_i = __ldg(&b.rho_near[i]);
    const F3 vel = xyz(__ldg(&b.wvel[i]));
    const float temp = __ldg(&b.wtemp[i]);
    const float rho_i = __ldg(&b.density[i]);
    const uint32_t cnt = __ldg(&b.nbr_n[i]);
    F3 visc = f3(0.f, 0.f, 0.f), blend = f3(0.f, 0.f, 0.f), near = f3(0.f, 0.f, 0.f),
       tension = f3(0.f, 0.f, 0.f);
    float heat = 0.0f, drho = 0.0f;
    auto load = [&](uint32_t code) {
        const uint32_t j = list_slot(code);
        return Nbr5{__ldg(&b.wpos[j]), __ldg(&b.wvel[j]), __ldg(&b.density[j]), __ldg(&b.wtemp[j]),
                    __ldg(&b.rho_near[j])};
    };
    walk<FCU_B_N5, Nbr5>(b.nbr, n, i, cnt, load, [&](float gs, const Nbr5 &q) {
        const float4 pj = q.p;
        const F3 e = pair_grad(gs, pos, pj);
        const F3 x = pos - xyz(pj);
        const float r2 = dot(x, x);
        const float r = sqrtf(r2);
        const float rho_j = q.rho;
        const float f = dot(x, e) / (r2 + soft);
        const float pair = mass / (rho_i * rho_j) * f;
        const F3 dv = vel - xyz(q.v);
        if (kDiv) drho += dot(dv, e);
        const float wn = fmaxf(1.0f - r * inv_h, 0.0f);
        near = near + ((near_i + q.near) * wn * wn) * (x / fmaxf(r, 1e-5f));
        visc = visc + (visc_k * pair) * dv;
        blend = blend - (mass / rho_j * kernel_q(K, r * inv_h)) * dv;
        heat += heat_k * pair * (temp - q.temp);
        heat -= diss_k * pair * dot(dv, dv);
        const float corr = 2.0f * rho0 / (rho_i + rho_j);
        tension = tension - ((corr * mass * cohesion(r, coh_c, coh_k, coh_near)) * x) / fmaxf(r, 1e-9f);
    });
    const F3 adh = (beta * P.rho0) * wall_adh_sum(P, pos);
    const F3 acc = visc + K_NEAR * near + gamma * tension + adh;
    b.accel[i] = make_float4(acc.x, acc.y, acc.z, heat);
    b.xsph[i] = make_float4(blend.x, blend.y, blend.z, 0.0f);
    const float half = 0.5f * __ldg(&b.wpp[i]);
    const float kdv = half / (rho_i * rho_i);
    b.kd[i] = kdv;
    b.wpk[i] = make_float4(pos.x, pos.y, pos.z, kdv);
    b.pressure[i] = half;
    if (kDiv) {  // k_div_kappa's prediction
        const float dt = g.st[bi].s.dt;
        drho = P.mass * drho;
        drho += dot(vel, xyz(__ldg(&b.wgrad[i])));
        const float kdd = fmaxf(drho, 0.0f) * __ldg(&b.alpha[i]) / fmaxf(dt, 1e-9f) / rho_i;
        b.kd2[i] = kdd;
        b.wpk2[i] = make_float4(pos.x, pos.y, pos.z, kdd);
        term = fixed_term((double)fmaxf(drho, 0.0f) * (double)dt / (double)P.rho0);
    }
    }
    if (kDiv) add_term<kB>(&g.solve[bi].acc_div[slot], term);
}

template <bool kB, int TPB>
__global__ void __launch_bounds__(TPB, kB ? FCU_MINB_FORCES_BATCH * 128 / TPB : FCU_MINB_FORCES * 128 / TPB) k_forces_plain(Geo g, SimBufs b, int slot, int gate) {
#if FCU_SORTED_FORCES
    const uint32_t i = slot_by_count<TPB>(b.nbr_n, g.n);
#else
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
#endif
    forces_eval_body<kB, false>(g, b, i, i < g.n, slot, gate);
}
template <bool kB, int TPB>
__global__ void __launch_bounds__(TPB, kB ? FCU_MINB_FORCES_BATCH * 128 / TPB : FCU_MINB_FORCES * 128 / TPB) k_forces_fused(Geo g, SimBufs b, int slot, int gate) {
#if FCU_SORTED_FORCES
    const uint32_t i = slot_by_count<TPB>(b.nbr_n, g.n);
#else
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
#endif
    forces_eval_body<kB, true>(g, b, i, i < g.n, slot, gate);
}

// fingers (sim_solve.wgsl:103-127)
__device__ __forceinline__ F3 fingers(const FluidStep &st, F3 pos, F3 v) {
    float px = 0.0f, py = 0.0f, weight = 0.0f;
    const uint32_t tn = st.touch_n < 5u ? st.touch_n : 5u;
    for (uint32_t t = 0; t < tn; ++t) {
        const float *tc = st.touches[t];
        const float dx = pos.x - tc[0], dy = pos.y - tc[1];
        const float q2 = (dx * dx + dy * dy) / (st.touch_r * st.touch_r);
        if (q2 < 1.0f) {
            const float w = (1.0f - q2) * (1.0f - q2);
            px += w * tc[2];
            py += w * tc[3];
            weight += w;
        }
    }
    if (weight <= 0.0f) return v;
    const float a = 1.0f - det_exp(-TOUCH_RATE * weight * st.dt);
    return f3(mixf(v.x, px / weight, a), mixf(v.y, py / weight, a), v.z);
}

// ---- forces_den_apply (sim_solve.wgsl:630-663) -----------------------------
template <bool kB, int TPB>
__global__ void __launch_bounds__(TPB, FCU_MINB) k_forces_apply(Geo g, SimBufs b) {
    const uint32_t n = g.n;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t bi = box_index<kB>(g, i);
    const float mass = params_of<kB>(g, bi).mass;
    const DevStep *stp = &g.st[bi];
    const FluidStep &st = stp->s;
    const float dt = st.dt;
    const F3 pos = xyz(__ldg(&b.wpos[i]));
    const float kd_i = b.kd[i];
    const F3 total = kappa_sum(b, i, n, pos, kd_i);
    const float4 a = __ldg(&b.accel[i]);
    const F3 r = pos;
    const float4 was = b.wvel[i];
    const F3 v = xyz(was);
    const F3 force = f3(st.force[0], st.force[1], st.force[2]);
    const F3 omega = f3(st.omega[0], st.omega[1], st.omega[2]);
    const F3 domega = f3(st.domega[0], st.domega[1], st.domega[2]);
    const F3 fict = -cross(domega, r) - cross(omega, cross(omega, r)) - 2.0f * cross(omega, v);
    const F3 forced = fingers(st, r, v + dt * (force + fict + xyz(a)) + stp->xsph_blend * xyz(__ldg(&b.xsph[i])));
    b.wtemp[i] += dt * a.w;
    const F3 dv_full = mass * total + kd_i * xyz(__ldg(&b.wgrad[i]));
    const F3 o = forced - dt * dv_full;
    b.wvel[i] = make_float4(o.x, o.y, o.z, was.w);
}

// ---- den_kappa (sim_solve.wgsl:674-698) ------------------------------------
template <bool kB>
__device__ __forceinline__ void den_kappa_at(const Geo &g, const SimBufs &b, uint32_t i, bool live, int slot,
                                             int gate) {
    const uint32_t n = g.n;
    const uint32_t bi = box_index<kB>(g, live ? i : n - 1);
    unsigned long long term = 0;
    if (live && !gated_out<kB>(g, bi, gate)) {
        const DevParams P = params_of<kB>(g, bi);
        const float mass = P.mass, rho0 = P.rho0;
        const float dt = g.st[bi].s.dt;
        const F3 pos = xyz(__ldg(&b.wpos[i]));
        const F3 vel = xyz(__ldg(&b.wvel[i]));
        const uint32_t cnt = __ldg(&b.nbr_n[i]);
        float drho = 0.0f;
        walk<FCU_B_PV, PosVel>(
            b.nbr, n, i, cnt,
            [&](uint32_t j) { return PosVel{__ldg(&b.wpos[j]), __ldg(&b.wvel[j])}; },
            [&](float gs, const PosVel &q) { drho += dot(vel - xyz(q.v), pair_grad(gs, pos, q.p)); });
        const float rho = __ldg(&b.density[i]);
        drho = mass * drho + dot(vel, xyz(__ldg(&b.wgrad[i])));
        const float rho_star = rho + dt * drho;
        const float kk = fmaxf(rho_star - rho0, 0.0f) * __ldg(&b.alpha[i]) / (dt * dt);
        const float kdv = kk / rho;
        b.kd[i] = kdv;
        b.wpk[i] = make_float4(pos.x, pos.y, pos.z, kdv);
        b.pinc[i] = kk * rho;
        term = fixed_term((double)rho_star / (double)rho0 - 1.0);
    }
    add_term<kB>(&g.solve[bi].acc_den[slot], term);
}

template <bool kB, int TPB>
__global__ void __launch_bounds__(TPB, kB ? kBatchKappaThreads / TPB : FCU_MINB_KAPPA) k_den_kappa(Geo g, SimBufs b, int slot,
                                                                       int gate) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    den_kappa_at<kB>(g, b, i, i < g.n, slot, gate);
}

// ---- integrate (sim_solve.wgsl:709-756) ------------------------------------
// With div_slot >= 0 (the fixed schedule) each box's first slot also records
// the box's residuals from the accumulator slots of the last divergence and
// density predictions, and the iteration counts.
template <bool kB, int TPB>
__global__ void __launch_bounds__(TPB) k_integrate(Geo g, SimBufs b, int div_slot, int den_slot,
                                                   int div_iters, int den_iters) {
    const uint32_t n = g.n;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const uint32_t bi = box_index<kB>(g, live ? i : n - 1);
    uint32_t clamped_speed = 0;
    if (live) {
        const DevParams P = params_of<kB>(g, bi);
        const DevStep *stp = &g.st[bi];
        const FluidStep &st = stp->s;
        const float4 was = __ldg(&b.wvel[i]);
        F3 v = xyz(was);
        const float speed = len(v);
        const float rho = __ldg(&b.density[i]);
        const float ceiling = rho < 0.5f * P.rho0 ? 3.0f * st.v_clamp : st.v_clamp;
        if (speed > ceiling) {
            v = v * (ceiling / speed);
            clamped_speed = 1;
        }
        const float4 pv = __ldg(&b.wpvel[i]);
        const float accel = len(v - xyz(pv)) / st.dt;
        const F3 pp = xyz(__ldg(&b.wpos[i])) + v * st.dt;
        const F3 cl = f3(clampf(pp.x, P.wall_lo[0], P.wall_hi[0]), clampf(pp.y, P.wall_lo[1], P.wall_hi[1]),
                         clampf(pp.z, P.wall_lo[2], P.wall_hi[2]));
        if (cl.x != pp.x) v.x = 0.0f;
        if (cl.y != pp.y) v.y = 0.0f;
        if (cl.z != pp.z) v.z = 0.0f;
        const float chase = stp->chase;
        const float pressure = __ldg(&b.pressure[i]);
        b.pos[i] = make_float4(cl.x, cl.y, cl.z, 0.0f);
        b.vel[i] = make_float4(v.x, v.y, v.z, mixf(was.w, accel, chase));
        b.pvel[i] = make_float4(v.x, v.y, v.z, mixf(pv.w, pressure, chase));
        const float dp = pressure - __ldg(&b.wpp[i]);
        b.pp[i] = pressure;
        const float t = __ldg(&b.wtemp[i]);
        b.temp[i] = t + t * EXPANSION / (rho * HEAT_CAPACITY) * dp;
        b.id[i] = __ldg(&b.wid[i]);
        if (i == first_of<kB>(g, bi)) {
            DevSolve *sv = &g.solve[bi];
            const double nb = (double)P.count;
            sv->substeps += 1ull;
            if (div_slot >= 0) {
                sv->div_res = (double)sv->acc_div[div_slot] / kFixedScale / nb;
                sv->den_res = den_slot >= 0 ? (double)sv->acc_den[den_slot] / kFixedScale / nb : 0.0;
                sv->div_iters = (uint32_t)div_iters;
                sv->den_iters = (uint32_t)den_iters;
                sv->total_div_iters += (unsigned long long)div_iters;
                sv->total_den_iters += (unsigned long long)den_iters;
            }
        }
    }
    if (kB) {
        count_at(&g.solve[bi].clamp_count, clamped_speed);
    } else {
        const uint32_t m = __ballot_sync(0xffffffffu, clamped_speed != 0u);
        if ((threadIdx.x & 31) == 0 && m) atomicAdd(&g.solve[0].clamp_count, __popc(m));
    }
}

// The tolerance loops' bookkeeping, one block over the boxes: for each box
// whose loop runs (every box on the first call), read and clear its
// residual accumulator of `which` (0 divergence, 1 density), count the
// iteration unless `first`, record the residual, and go on while under
// max_iters and above tol (the divergence loop always makes its first
// apply, as the reference). The graph's loop continues while any box does.
__global__ void __launch_bounds__(256) k_tol_finish(Geo g, int which, int first, float tol,
                                                    uint32_t max_iters,
                                                    cudaGraphConditionalHandle handle) {
    int any = 0;
    for (uint32_t bi = threadIdx.x; bi < g.nboxes; bi += blockDim.x) {
        DevSolve *sv = &g.solve[bi];
        uint32_t *active = which == 0 ? &sv->div_active : &sv->den_active;
        if (!first && !*active) continue;
        unsigned long long *acc = which == 0 ? &sv->acc_div[0] : &sv->acc_den[0];
        const uint32_t cnt = g.box_of ? g.box[bi].count : g.one.count;
        const double res = (double)*acc / kFixedScale / (double)cnt;
        *acc = 0ull;
        uint32_t *iters = which == 0 ? &sv->div_iters : &sv->den_iters;
        const uint32_t it = first ? 0u : *iters + 1u;
        *iters = it;
        if (!first) {
            if (which == 0) sv->total_div_iters += 1ull;
            else sv->total_den_iters += 1ull;
        }
        if (which == 0) sv->div_res = res;
        else sv->den_res = res;
        const bool go = it < max_iters && (res > (double)tol || (which == 0 && it < 1u));
        *active = go ? 1u : 0u;
        any |= go ? 1 : 0;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) cudaGraphSetConditional(handle, any ? 1u : 0u);
}

// ---- reduce_stats (sim_solve.wgsl:800-874) ---------------------------------
// Per box, per-chunk partials (block (chunk, box) strides through the box's
// slots), then one block per box folds them; min and max are exact in any
// order and the compression sum is an integer sum.
template <bool kB>
__global__ void __launch_bounds__(kStatsThreads) k_stats_partial(Geo g, SimBufs b) {
    const uint32_t bi = blockIdx.y;
    const DevParams P = params_of<kB>(g, bi);
    const uint32_t first = first_of<kB>(g, bi);
    const uint32_t end = first + P.count;
    __shared__ float sh[12][kStatsThreads / 32];
    __shared__ unsigned long long ssum[kStatsThreads / 32];
    float m = 0.0f, lo = HUGE_F, hi = -HUGE_F;
    float v_lo = HUGE_F, v_hi = -HUGE_F, a_lo = HUGE_F, a_hi = -HUGE_F;
    float p_lo = HUGE_F, p_hi = -HUGE_F, t_lo = HUGE_F, t_hi = -HUGE_F;
    unsigned long long sum = 0;
    const float rho0 = P.rho0;
    for (uint32_t i = first + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
        const float d = __ldg(&b.density[i]);
        const float c = d / rho0 - 1.0f;
        sum += fixed_term((double)fmaxf(c, 0.0f));
        m = fmaxf(m, c);
        lo = fminf(lo, d);
        hi = fmaxf(hi, d);
        const float4 q = __ldg(&b.vel[i]);
        const float speed = len(xyz(q));
        v_lo = fminf(v_lo, speed);
        v_hi = fmaxf(v_hi, speed);
        a_lo = fminf(a_lo, q.w);
        a_hi = fmaxf(a_hi, q.w);
        const float pr = __ldg(&b.pvel[i]).w;
        p_lo = fminf(p_lo, pr);
        p_hi = fmaxf(p_hi, pr);
        const float t = __ldg(&b.temp[i]);
        t_lo = fminf(t_lo, t);
        t_hi = fmaxf(t_hi, t);
    }
    float vals[12] = {m, lo, hi, v_lo, v_hi, a_lo, a_hi, p_lo, p_hi, t_lo, t_hi, 0.0f};
    const bool is_max[12] = {true, false, true, false, true, false, true, false, true, false, true, true};
#pragma unroll
    for (int q = 0; q < 11; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float y = __shfl_xor_sync(0xffffffffu, vals[q], o);
            vals[q] = is_max[q] ? fmaxf(vals[q], y) : fminf(vals[q], y);
        }
    }
    sum = warp_sum_u64(sum);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 11; ++q) sh[q][warp] = vals[q];
        ssum[warp] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float out[11];
        unsigned long long s = 0;
        for (int q = 0; q < 11; ++q) out[q] = sh[q][0];
        for (int w = 0; w < kStatsThreads / 32; ++w) {
            for (int q = 0; q < 11; ++q) out[q] = is_max[q] ? fmaxf(out[q], sh[q][w]) : fminf(out[q], sh[q][w]);
            s += ssum[w];
        }
        float *part = b.stats_part + ((size_t)bi * gridDim.x + blockIdx.x) * 12;
        for (int q = 0; q < 11; ++q) part[q] = out[q];
        atomicAdd(&b.stats_acc[bi], s);
    }
}

template <bool kB>
__global__ void __launch_bounds__(kStatsThreads) k_stats_final(Geo g, SimBufs b, uint32_t chunks) {
    // one block per box: thread t folds chunks t, t + blockDim, ..., then the
    // warps and the block fold the threads (min and max are exact in any order)
    const uint32_t bi = blockIdx.x;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ float s_w[kStatsThreads / 32][11];
    const bool is_max[11] = {true, false, true, false, true, false, true, false, true, false, true};
    const float *part = b.stats_part + (size_t)bi * chunks * 12;
    float out[11];
    const uint32_t k0 = threadIdx.x < chunks ? threadIdx.x : 0u;
#pragma unroll
    for (int q = 0; q < 11; ++q) out[q] = part[k0 * 12 + q];
    for (uint32_t k = threadIdx.x + blockDim.x; k < chunks; k += blockDim.x)
#pragma unroll
        for (int q = 0; q < 11; ++q) {
            const float v = part[k * 12 + q];
            out[q] = is_max[q] ? fmaxf(out[q], v) : fminf(out[q], v);
        }
#pragma unroll
    for (int q = 0; q < 11; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float v = __shfl_xor_sync(0xffffffffu, out[q], o);
            out[q] = is_max[q] ? fmaxf(out[q], v) : fminf(out[q], v);
        }
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 11; ++q) s_w[warp][q] = out[q];
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (uint32_t w = 1; w < blockDim.x / 32; ++w)
#pragma unroll
        for (int q = 0; q < 11; ++q) out[q] = is_max[q] ? fmaxf(out[q], s_w[w][q]) : fminf(out[q], s_w[w][q]);
    float *s = b.stats + (size_t)bi * 16;
    s[0] = (float)((double)b.stats_acc[bi] / kFixedScale / (double)params_of<kB>(g, bi).count);
    b.stats_acc[bi] = 0ull;
    s[1] = fmaxf(out[0], 0.0f);
    s[2] = out[1];
    s[3] = out[2];
    s[11] = out[3];
    s[6] = out[4];
    s[12] = out[5];
    s[13] = out[6];
    s[4] = out[7];
    s[5] = out[8];
    s[7] = out[9];
    s[8] = out[10];
    s[9] = (float)g.solve[bi].clamp_count;
    s[10] = (float)g.solve[bi].nbr_over;
}

// ---- tracers (sim_tracers.wgsl) ----------------------------------------------
__device__ __forceinline__ uint32_t pcg(uint32_t x) {  // :54-58
    uint32_t h = x * 747796405u + 2891336453u;
    h = ((h >> ((h >> 28u) + 4u)) ^ h) * 277803737u;
    return (h >> 22u) ^ h;
}

__device__ __forceinline__ int32_t to_fixed(float v) {  // i32(v * 65536): saturating, toward zero
    return __float2int_rz(v * 65536.0f);
}

// The lanes of a warp whose particles share a cell add their fixed-point
// velocities first (__reduce_add_sync over the match_any group: wrapping
// 32-bit sums, like the atomics, so the cell totals are the same bits) and
// one lane adds the group's total: slots are in cell order, so a warp's
// particles sit in a few cells.
__global__ void __launch_bounds__(256) k_splat(DevParams P, SimBufs b) {  // :98-114
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < P.count;
    uint32_t c = 0xffffffffu;
    uint32_t fx = 0, fy = 0, fz = 0;
    if (live) {
        const float4 p = __ldg(&b.pos[i]);
        const uint32_t cx = axis_cell(p.x, P.box_min[0], P.cell, P.dims[0]);
        const uint32_t cy = axis_cell(p.y, P.box_min[1], P.cell, P.dims[1]);
        const uint32_t cz = axis_cell(p.z, P.box_min[2], P.cell, P.dims[2]);
        c = ((cz * P.dims[1] + cy) * P.dims[0] + cx) * 4u;
        const float4 v = __ldg(&b.vel[i]);
        fx = (uint32_t)to_fixed(v.x);
        fy = (uint32_t)to_fixed(v.y);
        fz = (uint32_t)to_fixed(v.z);
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, c);
    fx = __reduce_add_sync(peers, fx);
    fy = __reduce_add_sync(peers, fy);
    fz = __reduce_add_sync(peers, fz);
    if (live && (threadIdx.x & 31u) == (uint32_t)(__ffs(peers) - 1)) {
        atomicAdd(&b.vel_grid[c], (int32_t)fx);
        atomicAdd(&b.vel_grid[c + 1], (int32_t)fy);
        atomicAdd(&b.vel_grid[c + 2], (int32_t)fz);
        atomicAdd(&b.vel_grid[c + 3], __popc(peers));
    }
}

__global__ void __launch_bounds__(256) k_resolve(SimBufs b, uint32_t cells) {  // :122-138
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    int4 *g = reinterpret_cast<int4 *>(b.vel_grid);
    b.vel_flat[c] = g[c];
    g[c] = make_int4(0, 0, 0, 0);
}

__device__ __forceinline__ void store_tracer(const DevParams &P, uint32_t *tr, uint32_t i, F3 pos,
                                             float speed) {  // :75-80
    const float ux = clampf((pos.x - P.tracer_c[0]) / P.tracer_e[0] * 0.5f + 0.5f, 0.0f, 1.0f);
    const float uy = clampf((pos.y - P.tracer_c[1]) / P.tracer_e[1] * 0.5f + 0.5f, 0.0f, 1.0f);
    const uint32_t qx = (uint32_t)(ux * 65535.0f + 0.5f);
    const uint32_t qy = (uint32_t)(uy * 65535.0f + 0.5f);
    const uint32_t hz = __half_as_ushort(__float2half_rn(pos.z - P.tracer_c[2]));
    const uint32_t hs = __half_as_ushort(__float2half_rn(speed));
    reinterpret_cast<uint2 *>(tr)[i] = make_uint2(qx | (qy << 16), hz | (hs << 16));
}

__device__ __forceinline__ F3 tracer_clamp(const DevParams &P, F3 v) {
    return f3(clampf(v.x, P.tracer_c[0] - P.tracer_e[0], P.tracer_c[0] + P.tracer_e[0]),
              clampf(v.y, P.tracer_c[1] - P.tracer_e[1], P.tracer_c[1] + P.tracer_e[1]),
              clampf(v.z, P.tracer_c[2] - P.tracer_e[2], P.tracer_c[2] + P.tracer_e[2]));
}

__device__ void respawn(const DevParams &P, const SimBufs &b, uint32_t slot, uint32_t r) {  // :82-92
    const uint32_t r1 = pcg(r), r2 = pcg(r1), r3 = pcg(r2), r4 = pcg(r3);
    const float half_cell = P.cell * 0.5f;
    const F3 jit = f3(((float)(r2 >> 20) / 4096.0f - 0.5f) * half_cell,
                      ((float)(r3 >> 20) / 4096.0f - 0.5f) * half_cell,
                      ((float)(r4 >> 20) / 4096.0f - 0.5f) * half_cell);
    const uint32_t j = r1 % P.count;
    store_tracer(P, b.tracers, slot, tracer_clamp(P, xyz(b.pos[j]) + jit), len(xyz(b.vel[j])));
}

__global__ void __launch_bounds__(256) k_advect(DevParams P, SimBufs b, DevStep stv,
                                                uint32_t ntr) {  // :140-183
    const DevStep *stp = &stv;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntr) return;
    const float dt = stp->s.dt;
    const float p_respawn = dt / 3.0f;
    const float p_stray = dt / 0.25f;
    const uint32_t r0 = pcg(i ^ pcg(stp->s.seed));
    if ((float)r0 / 4294967296.0f < p_respawn) {
        respawn(P, b, i, r0);
        return;
    }
    const uint2 t = reinterpret_cast<const uint2 *>(b.tracers)[i];
    float old[4];
    old[0] = ((float)(t.x & 0xffffu) / 65535.0f * 2.0f - 1.0f) * P.tracer_e[0] + P.tracer_c[0];
    old[1] = ((float)(t.x >> 16) / 65535.0f * 2.0f - 1.0f) * P.tracer_e[1] + P.tracer_c[1];
    old[2] = __half2float(__ushort_as_half((unsigned short)(t.y & 0xffffu))) + P.tracer_c[2];
    old[3] = __half2float(__ushort_as_half((unsigned short)(t.y >> 16)));
    F3 pos = f3(old[0], old[1], old[2]);
    const float gp[3] = {(pos.x - P.box_min[0]) / P.cell - 0.5f, (pos.y - P.box_min[1]) / P.cell - 0.5f,
                         (pos.z - P.box_min[2]) / P.cell - 0.5f};
    uint32_t base[3];
    float f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int32_t bi = __float2int_rz(floorf(gp[a]));
        const int32_t top = (int32_t)P.dims[a] - 2;
        bi = bi < 0 ? 0 : (bi > top ? top : bi);
        base[a] = (uint32_t)bi;
        f[a] = clampf(gp[a] - (float)base[a], 0.0f, 1.0f);
    }
    float mx = 0.0f, my = 0.0f, mz = 0.0f, wc = 0.0f;
#pragma unroll
    for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t ox = k & 1u, oy = (k >> 1) & 1u, oz = (k >> 2) & 1u;
        const float wx = ox ? f[0] : 1.0f - f[0];
        const float wy = oy ? f[1] : 1.0f - f[1];
        const float wz = oz ? f[2] : 1.0f - f[2];
        const float weight = wx * wy * wz;
        const uint32_t c = ((base[2] + oz) * P.dims[1] + (base[1] + oy)) * P.dims[0] + (base[0] + ox);
        const int4 cell = b.vel_flat[c];
        mx += weight * (float)cell.x;
        my += weight * (float)cell.y;
        mz += weight * (float)cell.z;
        wc += weight * (float)cell.w;
    }
    F3 v = f3(0.f, 0.f, 0.f);
    if (wc > 0.0f) {
        const float den = wc * 65536.0f;
        v = f3(mx / den, my / den, mz / den);
    } else if ((float)pcg(r0 ^ 0x85ebca6bu) / 4294967296.0f < p_stray) {
        respawn(P, b, i, pcg(r0 ^ 0x632be59bu));
        return;
    }
    pos = pos + v * dt;
    store_tracer(P, b.tracers, i, tracer_clamp(P, pos), fmaxf(len(v), old[3] * stp->decay));
}

inline uint32_t blocks_for(uint32_t n, uint32_t t) { return (n + t - 1) / t; }

}  // namespace

void launch_gather(cudaStream_t s, const SimBufs &b, uint32_t n) {
    if (n) k_gather<<<blocks_for(n, 256), 256, 0, s>>>(b, n);
}

// One launch of `kern` over g.n particles: the batch instance when the
// geometry has a box map, the one-box instance otherwise, at the block size
// the geometry's tuning table holds for the kernel (or the default).
#define FCU_SWEEP_AT(kern, T, ...)                                                      \
    do {                                                                                \
        const uint32_t blocks_ = blocks_for(g.n, T);                                    \
        if (g.box_of) kern<true, T><<<blocks_, T, 0, s>>>(__VA_ARGS__);                 \
        else kern<false, T><<<blocks_, T, 0, s>>>(__VA_ARGS__);                         \
    } while (0)
#define FCU_SWEEP(kern, slot_id, deflt, ...)                                            \
    do {                                                                                \
        if (!g.n) return;                                                               \
        const int tpb_ = g.tpb[slot_id] ? (int)g.tpb[slot_id] : (deflt);                \
        if (tpb_ == 64) FCU_SWEEP_AT(kern, 64, __VA_ARGS__);                            \
        else if (tpb_ == 256) FCU_SWEEP_AT(kern, 256, __VA_ARGS__);                     \
        else FCU_SWEEP_AT(kern, 128, __VA_ARGS__);                                      \
    } while (0)

void launch_density_div(cudaStream_t s, const Geo &g, const SimBufs &b, int slot) {
    FCU_SWEEP(k_density_div, kTuneDensity, kSolveThreads, g, b, slot);
}
void launch_div_kappa(cudaStream_t s, const Geo &g, const SimBufs &b, int slot, int gate) {
    FCU_SWEEP(k_div_kappa, kTuneDivKappa, kSolveThreads, g, b, slot, gate);
}
void launch_apply(cudaStream_t s, const Geo &g, const SimBufs &b, bool add_pressure, int gate) {
    FCU_SWEEP(k_apply, kTuneApply, kSolveThreads, g, b, add_pressure ? 1 : 0, gate);
}
void launch_forces_eval(cudaStream_t s, const Geo &g, const SimBufs &b) {
    FCU_SWEEP(k_forces_plain, kTuneForcesEval, kSolveThreads, g, b, 0, kGateNone);
}
void launch_forces_div(cudaStream_t s, const Geo &g, const SimBufs &b, int slot, int gate) {
    FCU_SWEEP(k_forces_fused, kTuneForcesEval, kSolveThreads, g, b, slot, gate);
}
void launch_forces_apply(cudaStream_t s, const Geo &g, const SimBufs &b) {
    FCU_SWEEP(k_forces_apply, kTuneForcesApply, kSolveThreads, g, b);
}
void launch_den_kappa(cudaStream_t s, const Geo &g, const SimBufs &b, int slot, int gate) {
    FCU_SWEEP(k_den_kappa, kTuneDenKappa, kSolveThreads, g, b, slot, gate);
}
void launch_integrate(cudaStream_t s, const Geo &g, const SimBufs &b, int div_slot, int den_slot,
                      int div_iters, int den_iters) {
    FCU_SWEEP(k_integrate, kTuneIntegrate, 256, g, b, div_slot, den_slot, div_iters, den_iters);
}
#undef FCU_SWEEP_AT
#undef FCU_SWEEP

void launch_tol_finish(cudaStream_t s, const Geo &g, int which, int first, float tol,
                       uint32_t max_iters, cudaGraphConditionalHandle handle) {
    uint32_t threads = (g.nboxes + 31u) & ~31u;
    if (threads > 256u) threads = 256u;
    if (threads < 32u) threads = 32u;
    k_tol_finish<<<1, threads, 0, s>>>(g, which, first, tol, max_iters, handle);
}
void launch_stats(cudaStream_t s, const Geo &g, const SimBufs &b, uint32_t chunks) {
    if (!g.nboxes || !chunks) return;
    const dim3 grid(chunks, g.nboxes);
    if (g.box_of) {
        k_stats_partial<true><<<grid, kStatsThreads, 0, s>>>(g, b);
        k_stats_final<true><<<g.nboxes, kStatsThreads, 0, s>>>(g, b, chunks);
    } else {
        k_stats_partial<false><<<grid, kStatsThreads, 0, s>>>(g, b);
        k_stats_final<false><<<g.nboxes, kStatsThreads, 0, s>>>(g, b, chunks);
    }
}
void launch_splat(cudaStream_t s, const DevParams &P, const SimBufs &b) {
    if (P.count) k_splat<<<blocks_for(P.count, 256), 256, 0, s>>>(P, b);
}
void launch_resolve(cudaStream_t s, const DevParams &P, const SimBufs &b) {
    const uint32_t cells = P.dims[0] * P.dims[1] * P.dims[2];
    k_resolve<<<blocks_for(cells, 256), 256, 0, s>>>(b, cells);
}
void launch_advect(cudaStream_t s, const DevParams &P, const SimBufs &b, const DevStep &st,
                   uint32_t ntr) {
    if (ntr) k_advect<<<blocks_for(ntr, 256), 256, 0, s>>>(P, b, st, ntr);
}

}  // namespace fcu
