/*
 * fluid_oracle.h — CPU oracle for the DFSPH substep.
 *
 * TEST INFRASTRUCTURE. This is the correctness oracle and the timed CPU
 * baseline, nothing else: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py may load it. The product path
 * (include/fluid_cu.h) never links or calls it.
 *
 * It restates, in plain C++ with IEEE single precision and no FMA
 * contraction, the reference's own CPU substrate and compute shaders:
 *   crates/fluid-core/src/sim.rs           grid, kernel, walls, seeding, packers
 *   crates/fluid-core/src/sim_grid.wgsl    count / scatter
 *   crates/fluid-core/src/sim_scan.wgsl    exclusive scan, starts[C] = N
 *   crates/fluid-core/src/sim_solve.wgsl   density_div .. integrate, reduce_stats
 *   crates/fluid-core/src/sim_tracers.wgsl splat / resolve / advect
 *   crates/fluid-core/src/render.rs        dispatch order (:3175-3229, :3924-3981)
 *
 * Ordering conventions (the reference leaves them free):
 *   - the cell sort is the stable counting sort (ascending previous slot
 *     inside a cell), the order validate_bench assumes (render.rs:2703-2715);
 *   - each particle sums its neighbours sequentially: stencil cells
 *     0..26 with x fastest (sim_solve.wgsl:436-438), particles in slot order
 *     inside a cell, one accumulator per quantity, self term first.
 */
#ifndef FLUID_ORACLE_H
#define FLUID_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Grid geometry, sim.rs:14-44 (Grid) generalised to any [lo, hi] box. */
typedef struct OrGrid {
    float min[3];
    float cell;
    uint32_t dims[3];
} OrGrid;

/* Everything a substep reads besides the particle state (the reference's
 * SimParams, sim_solve.wgsl:11-23, plus the box walls made explicit). */
typedef struct OrParams {
    float box_min[3];
    float cell;
    uint32_t dims[3];
    uint32_t count;
    float h, mass, rho0, inv_h, sigma, sigma_h, support_sq;
    float wall_lo[3];
    float wall_hi[3];
    float tracer_c[3]; /* tracer box centre: 0 for the reference slab */
    float tracer_e[3]; /* tracer box half extent */
    float xsph_blend;  /* < 0: the reference's 1 - exp(-6 dt) per substep */
    uint32_t nbr_cap;  /* 96 in the reference (sim_solve.wgsl:388) */
} OrParams;

/* The 144-byte Step block, sim.rs:215-252 / sim_solve.wgsl:29-41. */
typedef struct OrStep {
    float force[3];
    float dt;
    float omega[3];
    float v_clamp;
    float domega[3];
    uint32_t seed;
    float touch_r;
    uint32_t touch_n;
    uint32_t pad[2];
    float touches[5][4];
} OrStep;

/* ---- sim.rs CPU substrate ------------------------------------------------ */
uint32_t or_hash(uint32_t x);
float or_kernel(float r, float h);
float or_wall_density(float t);
float or_wall_gradient(float t);
double or_wedge64(double t1, double t2);
double or_wedge_d64(double t1, double t2);
double or_wall_adhesion64(double t);
float or_wedge(float t1, float t2);
float or_wedge_d(float t1, float t2);
float or_wall_adhesion(float t);
void or_lattice_dims(float spacing, const float extent[2], float fill, uint32_t out[3]);
uint32_t or_seed_slab(float spacing, const float extent[2], float fill, float *out4);
void or_seed_tracers(uint32_t count, const float extent[2], float fill, uint32_t *out2);
/* Tracers of a box: uniform over [lo, lo + size), relative to centre,
 * packed over the half extent e (the same hash stream as the slab's). */
void or_seed_tracers_box(uint32_t count, const float lo[3], const float size[3], const float centre[3],
                         const float e[2], uint32_t *out2);
uint16_t or_half_bits(float x);
float or_half_value(uint16_t bits);
void or_pack_tracer(const float pos[3], float speed, const float extent[2], uint32_t out[2]);
void or_unpack_tracer(const uint32_t raw[2], const float extent[2], float out[4]);
void or_pack_step(const float force[3], const float omega[3], const float domega[3], float dt,
                  float v_clamp, uint32_t seed, uint32_t touch_n, float touch_r,
                  const float *touches4, uint8_t out[144]);
void or_pack_sim_params(const OrGrid *g, uint32_t count, float h, float mass, float rho0,
                        uint8_t out[64]);
float or_slab_depth(void);
float or_rest_density(void);

/* ---- grid -------------------------------------------------------------- */
void or_grid_slab(const float extent[2], float support, OrGrid *g);
void or_grid_box(const float lo[3], const float hi[3], float support, OrGrid *g);
uint32_t or_cell_of(const OrGrid *g, const float pos[3]);
/* count -> exclusive scan (starts[C] = n) -> stable scatter of the index. */
void or_grid_build(const OrGrid *g, const float *pos4, uint32_t n, uint32_t *keys,
                   uint32_t *starts, uint32_t *perm);

/* Parameters of the reference slab (render.rs:1477-1612): h = h_ratio * spacing,
 * cell = 2h, rest density 998.2, walls at box_min + cell and its negation. */
void or_params_slab(const float extent[2], float spacing, float h_ratio, uint32_t count,
                    OrParams *p);
/* Parameters of an arbitrary box [lo, hi], walls on the box faces. */
void or_params_box(const float lo[3], const float hi[3], float spacing, float h_ratio,
                   float rho0, uint32_t count, OrParams *p);

/* Lattice block at the box's low corner, seeded splitmix64 jitter of
 * +-jitter*spacing per axis; the same stream the product seeds with. */
uint32_t or_seed_block(const float lo[3], float spacing, const uint32_t n[3], float jitter,
                       uint64_t seed, float *out4);

/* ---- the substep --------------------------------------------------------- */
typedef struct OrSim OrSim;
OrSim *or_sim_new(const OrParams *p, uint32_t tracer_count);
void or_sim_free(OrSim *s);
void or_sim_set_threads(int threads);
/* Slabs per cell along x in a simulation's grid keys (cell * slabs + slab):
 * each cell's slots are in slab order, and the starts field holds
 * cells * slabs + 1 entries. */
uint32_t or_sim_slabs(void);
/* Resting set, in its slot order. Any pointer may be null (zero fill,
 * temperature 293.15, id = slot). */
void or_sim_set_state(OrSim *s, const float *pos4, const float *vel4, const float *prev_vel4,
                      const float *prev_p, const float *temp, const uint32_t *id);
void or_sim_get_state(const OrSim *s, float *pos4, float *vel4, float *prev_vel4, float *prev_p,
                      float *temp, uint32_t *id);
void or_sim_set_tracers(OrSim *s, const uint32_t *packed2);
void or_sim_get_tracers(const OrSim *s, uint32_t *packed2);
/* One substep at the fixed schedule: div_iters divergence applies (the
 * reference: 1) and den_iters constant-density pairs (the reference: 5 or
 * 2). dt == 0 runs the rebuild and density_div alone, as render.rs:3904-3955
 * does at zero substeps. */
void or_sim_substep(OrSim *s, const OrStep *st, uint32_t div_iters, uint32_t den_iters);
/* One substep with tolerance-driven iteration counts (FP64 residuals). */
void or_sim_substep_tol(OrSim *s, const OrStep *st, float div_tol, float den_tol,
                        uint32_t max_iters, uint32_t out_iters[2], double out_res[2]);
/* The state in double: the FP64 oracle's own values (the float oracle's,
 * widened). Either pointer may be null. */
void or_sim_get_state64(const OrSim *s, double *pos4, double *vel4);
/* sizeof the substep's arithmetic type: 4 (the oracle), 8 (the FP64 oracle). */
int or_sim_real_bytes(void);
/* One kernel of the substep on the current working set, in isolation (the
 * per-kernel checks of the tests): DENSITY is the rebuild and density_div;
 * the kappa kernels return their mean residual, the others 0. */
enum {
    OR_KERNEL_DENSITY = 0,
    OR_KERNEL_DIV_APPLY = 1,
    OR_KERNEL_DIV_KAPPA = 2,
    OR_KERNEL_FORCES_EVAL = 3,
    OR_KERNEL_FORCES_APPLY = 4,
    OR_KERNEL_DEN_KAPPA = 5,
    OR_KERNEL_DEN_APPLY = 6,
    OR_KERNEL_INTEGRATE = 7
};
double or_sim_kernel(OrSim *s, int kernel, const OrStep *st);
/* The per-particle exp of the finger blend (sim_solve.wgsl:122), the
 * deterministic evaluation the CUDA path shares. */
float or_det_exp(float x);

/* reduce_stats into out[14] (sim_solve.wgsl:800-874). */
void or_sim_stats(OrSim *s, float out[14]);
/* One tracer pass (splat, resolve, advect), sim_tracers.wgsl. */
void or_sim_tracers(OrSim *s, const OrStep *st);
/* Advect alone, on the velocity field the last resolve left. */
void or_sim_advect(OrSim *s, const OrStep *st);

enum {
    OR_FIELD_DENSITY = 0, /* float[n], working order */
    OR_FIELD_ALPHA = 1,
    OR_FIELD_KD = 2,
    OR_FIELD_PRESSURE = 3,
    OR_FIELD_NBR_N = 4,    /* uint32[n] */
    OR_FIELD_STARTS = 5,   /* uint32[C+1] */
    OR_FIELD_PERM = 6,     /* uint32[n] */
    OR_FIELD_WORK_POS = 7, /* float4[n] */
    OR_FIELD_WORK_VEL = 8, /* float4[n] */
    OR_FIELD_ACCEL = 9,    /* float4[n] */
    OR_FIELD_XSPH = 10,    /* float4[n] */
    OR_FIELD_WALL_GRAD = 11,
    OR_FIELD_COUNTERS = 12, /* uint32[2]: clamp count, neighbour overflow */
    OR_FIELD_WORK_PREV_VEL = 13, /* float4[n], working order */
    OR_FIELD_WORK_PREV_P = 14,   /* float[n], working order */
    OR_FIELD_WORK_TEMP = 15,     /* float[n], working order */
    OR_FIELD_PINC = 16,          /* float[n]: k*rho of the last den_kappa */
    OR_FIELD_NBR = 17            /* uint32[n][cap]: each particle's list, 0xffffffff past nbr_n */
};
void or_sim_field(const OrSim *s, int field, void *out);

/* The render-side thickness field. geom = {cx, cy, ex, ey, radius, lo, hi}:
 * the field spans world x in cx +- ex, y in cy +- ey. The body splat of
 * sim_sprites.wgsl (`body`, `weight`, `lens_at`; lens 0 none, 1 accel lens,
 * 2 pressure lens, 3 density, 4 speed) with the decay draw of render.rs:
 * 3233-3282: field2[h][w][2] = field2 * keep + (1 - keep) * splat. */
void or_field_splat(const float *pos4, const float *vel4, const float *pvel4, const float *density,
                    uint32_t n, const float geom[7], uint32_t w, uint32_t h, uint32_t lens, float keep,
                    float *field2);
/* sim_surface.wgsl field_filter: out4[h][w] = (blurred, x difference,
 * y difference, Laplacian) of field2's thickness channel. */
void or_field_filter(const float *field2, uint32_t w, uint32_t h, float ex, float ey, float *out4);

#ifdef __cplusplus
}
#endif
#endif
