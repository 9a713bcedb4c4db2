// solve.cuh — the DFSPH substep's sweeps, integrate, statistics, tracers.
#pragma once

#include "common.cuh"

namespace fcu {

// Device pointers of one box's particle state and scratch.
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
    // Neighbour list, slot-major (entry k of particle i at k * n + i): the
    // neighbour's slot and the bits of its kernel-gradient scale dw / r,
    // so a sweep forms the gradient (dw / r) * (x_i - x_j) without the
    // square root and the division density_div already did.
    uint2 *nbr;
    uint32_t *nbr_n;
    // tracers
    uint32_t *tracers;  // 2 words each
    int32_t *vel_grid;  // 4 per cell, atomic sums
    int4 *vel_flat;
    // stats
    float *stats_part;  // [blocks][12]
    unsigned long long *stats_acc;
    float *stats;       // 14
};

constexpr int kSolveThreads = 128;
constexpr int kStatsBlocks = 148;
constexpr int kStatsThreads = 256;

// Enqueue helpers: each launches one kernel on `s`.
void launch_gather(cudaStream_t s, const SimBufs &b, uint32_t n);
void launch_density_div(cudaStream_t s, const DevParams &P, const SimBufs &b, const DevStep *st,
                        DevSolve *solve, unsigned long long *acc);
void launch_div_kappa(cudaStream_t s, const DevParams &P, const SimBufs &b, const DevStep *st,
                      unsigned long long *acc);
void launch_apply(cudaStream_t s, const DevParams &P, const SimBufs &b, const DevStep *st,
                  bool add_pressure);
void launch_forces_eval(cudaStream_t s, const DevParams &P, const SimBufs &b);
void launch_forces_apply(cudaStream_t s, const DevParams &P, const SimBufs &b, const DevStep *st);
void launch_den_kappa(cudaStream_t s, const DevParams &P, const SimBufs &b, const DevStep *st,
                      unsigned long long *acc);
void launch_integrate(cudaStream_t s, const DevParams &P, const SimBufs &b, const DevStep *st,
                      DevSolve *solve, int div_slot, int den_slot, int div_iters, int den_iters);
// The tolerance loop's step after a prediction sweep: records the residual
// of `which` (0 divergence, 1 density), counts the iteration, sets `handle`.
void launch_tol_finish(cudaStream_t s, DevSolve *solve, uint32_t n, int which, int first, float tol,
                       uint32_t max_iters, cudaGraphConditionalHandle handle);
void launch_stats(cudaStream_t s, const DevParams &P, const SimBufs &b, DevSolve *solve);
void launch_splat(cudaStream_t s, const DevParams &P, const SimBufs &b);
void launch_resolve(cudaStream_t s, const DevParams &P, const SimBufs &b);
void launch_advect(cudaStream_t s, const DevParams &P, const SimBufs &b, const DevStep &st,
                   uint32_t ntr);

}  // namespace fcu
