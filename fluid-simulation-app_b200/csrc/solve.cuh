// solve.cuh — the DFSPH substep's sweeps, integrate, statistics, tracers.
#pragma once

#include "common.cuh"

namespace fcu {


// Device pointers of the particle state and scratch: one box, or a batch of
// boxes laid end to end (box b owns slots first[b] .. first[b] + count - 1 in
// both sets, for good: its cell keys sit above every earlier box's, and the
// stable sort keeps each box's slots in place).
struct SimBufs {
    // resting set (slot order of the last integrate)
    float4 *pos, *vel, *pvel;
    float *pp, *temp;
    uint32_t *id;
    // working set (this substep's cell order)
    float4 *wpos, *wvel, *wpvel;
    float *wpp, *wtemp;
    uint32_t *wid;
    // scratch
    uint32_t *keys, *starts, *perm;
    float *density, *alpha, *kd, *pressure, *pinc, *rho_near;
    float4 *accel, *xsph, *wgrad;
    float4 *wpk;  // position and kd of the last prediction: apply's one record per neighbour
    // the divergence loop's own kd and (position, kd) in the tolerance
    // schedule, where forces_eval also forms the divergence prediction
    float *kd2;
    float4 *wpk2;
    // Neighbour list, slot-major (entry k of particle i at k * n + i): the
    // neighbour's slot and the bits of its kernel-gradient scale dw / r,
    // so a sweep forms the gradient (dw / r) * (x_i - x_j) without the
    // square root and the division density_div already did.
    uint2 *nbr;
    uint32_t *nbr_n;
    // tracers (one box)
    uint32_t *tracers;  // 2 words each
    int32_t *vel_grid;  // 4 per cell, atomic sums
    int4 *vel_flat;
    // stats, per box
    float *stats_part;  // [box][chunk][12]
    unsigned long long *stats_acc;  // [box]
    float *stats;       // [box][16]
};

// The sweeps whose block size can be tuned (entries of Geo::tpb).
enum TuneSlot : int {
    kTuneDensity = 0,
    kTuneDivKappa,
    kTuneApply,
    kTuneForcesEval,
    kTuneForcesApply,
    kTuneDenKappa,
    kTuneIntegrate,
    kTuneCount
};

// Which box a slot belongs to, and the per-box constants, Step blocks and
// solver counters. One box: box_of is null, the constants travel by value
// in `one` (the kernel's parameter space), solve and st point at one entry.
// A batch: box_of, box, cell_base and first are device arrays. tpb: the
// launch's block size per tuned sweep (64, 128 or 256; 0 = the default),
// read by the host-side launchers only.
struct Geo {
    uint16_t tpb[8];
    DevParams one;                           // the box, when there is one
    const DevParams *__restrict__ box;       // [nboxes] (batch)
    const uint16_t *__restrict__ box_of;     // [n] (batch) or null
    const uint32_t *__restrict__ cell_base;  // [nboxes] first cell key of each box (batch)
    const uint32_t *__restrict__ first;      // [nboxes] first slot of each box (batch)
    DevSolve *solve;                         // [nboxes]
    const DevStep *st;                       // [nboxes] this substep's Step blocks
    uint32_t n;                              // particles in all boxes
    uint32_t nboxes;
};

constexpr int kSolveThreads = 128;
constexpr int kStatsChunks = 592;  // 4 blocks of kStatsThreads per SM at 1M particles
constexpr int kStatsThreads = 256;

// A tolerance loop's gate: the kernel skips boxes whose loop has stopped.
enum Gate : int { kGateNone = 0, kGateDiv = 1, kGateDen = 2 };

// Enqueue helpers: each launches one kernel on `s`.
void launch_gather(cudaStream_t s, const SimBufs &b, uint32_t n);
void launch_density_div(cudaStream_t s, const Geo &g, const SimBufs &b, int slot);
void launch_div_kappa(cudaStream_t s, const Geo &g, const SimBufs &b, int slot, int gate);
void launch_apply(cudaStream_t s, const Geo &g, const SimBufs &b, bool add_pressure, int gate);
void launch_forces_eval(cudaStream_t s, const Geo &g, const SimBufs &b);
// forces_eval that also forms the divergence prediction (kappa into kd2 /
// wpk2, residual term into acc_div[slot]), skipping boxes whose divergence
// loop has stopped.
void launch_forces_div(cudaStream_t s, const Geo &g, const SimBufs &b, int slot, int gate);
void launch_forces_apply(cudaStream_t s, const Geo &g, const SimBufs &b);

void launch_den_kappa(cudaStream_t s, const Geo &g, const SimBufs &b, int slot, int gate);
// div_slot >= 0: record each box's residuals from those accumulator slots
// and the fixed iteration counts (the fixed schedule).
void launch_integrate(cudaStream_t s, const Geo &g, const SimBufs &b, int div_slot, int den_slot,
                      int div_iters, int den_iters);
// The tolerance loop's step after a prediction sweep: records each box's
// residual of `which` (0 divergence, 1 density), counts the iteration,
// keeps each box's loop going or stops it, and sets `handle` while any goes.
void launch_tol_finish(cudaStream_t s, const Geo &g, int which, int first, float tol,
                       uint32_t max_iters, cudaGraphConditionalHandle handle);
// reduce_stats of every box (chunks: blocks per box).
void launch_stats(cudaStream_t s, const Geo &g, const SimBufs &b, uint32_t chunks);
void launch_splat(cudaStream_t s, const DevParams &P, const SimBufs &b);
void launch_resolve(cudaStream_t s, const DevParams &P, const SimBufs &b);
void launch_advect(cudaStream_t s, const DevParams &P, const SimBufs &b, const DevStep &st,
                   uint32_t ntr);

}  // namespace fcu
