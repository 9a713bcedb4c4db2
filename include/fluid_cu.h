/*
 * fluid_cu.h — C ABI of the B200 DFSPH step (libfluidcu.so).
 *
 * The drop-in boundary for fluid-core's per-frame simulation step. It keeps
 * the conventions of the reference's C ABI (crates/fluid-ffi/include/
 * fluid_ffi.h:11-182, crates/fluid-ffi/src/lib.rs:72-285): an opaque handle,
 * plain-old-data structs passed by value or pointer, create returning null
 * with the reason available as text. Rendering and surfaces are not part of
 * it. Unlike the reference, every call that can fail returns a status code.
 *
 * Threading: one handle per host thread. Calls are ordered on the handle's
 * CUDA stream and return before the GPU finishes, except those documented
 * as synchronising (stats, reads, sync).
 */
#ifndef FLUID_CU_H
#define FLUID_CU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define FLUID_OK 0
#define FLUID_ERR_ARG -1     /* bad argument or size */
#define FLUID_ERR_CUDA -2    /* a CUDA call failed; see fluid_last_error() */
#define FLUID_ERR_TIMEOUT -3 /* a bounded device-side wait gave up */
#define FLUID_ERR_NAN -4     /* a non-finite value reached the statistics */
#define FLUID_ERR_STATE -5   /* call not valid in the handle's state */
#define FLUID_ERR_OOM -6     /* device allocation failed */

/* Replaces fluid_ffi.h:58 FLUID_TOUCH_SLOTS; sim.rs:180 MAX_TOUCHES. */
#define FLUID_TOUCH_SLOTS 5
/* sim_solve.wgsl:388 NBR_CAP. */
#define FLUID_NBR_CAP_DEFAULT 96

typedef struct FluidSim FluidSim;

/* fluid_ffi.h:17-21 */
typedef struct FluidVec3 {
    float x;
    float y;
    float z;
} FluidVec3;

/* The 144-byte Step block, byte for byte: sim.rs:200-252 (pack_step),
 * sim_solve.wgsl:29-41. force is the body force (tilt gravity), m/s^2 in the
 * box frame; dt the substep; omega / domega the box's angular velocity and
 * acceleration; v_clamp the CFL speed; seed the tracer seed; the fingers'
 * shared radius, count and (x, y, vx, vy) each. */
typedef struct FluidStep {
    float force[3];
    float dt;
    float omega[3];
    float v_clamp;
    float domega[3];
    uint32_t seed;
    float touch_r;
    uint32_t touch_n;
    uint32_t pad[2];
    float touches[FLUID_TOUCH_SLOTS][4];
} FluidStep;

#define FLUID_GEOMETRY_SLAB 0 /* the reference slab: +-extent in x, y; +-slab depth/2 in z */
#define FLUID_GEOMETRY_BOX 1  /* any axis-aligned box [box_lo, box_hi] */

#define FLUID_SEED_SLAB 0  /* sim.rs:77-100 seed_slab at `fill` */
#define FLUID_SEED_BLOCK 1 /* lattice block of `block` dims at box_lo, splitmix64 jitter */
#define FLUID_SEED_NONE 2  /* `count` particles at the origin until set_state */

#define FLUID_SOLVE_FIXED 0     /* div_iters / den_iters applies (reference: 1 / 5) */
#define FLUID_SOLVE_TOLERANCE 1 /* iterate to div_tol / den_tol, FP64 residuals, capped */

/* What fluid_renderer_create's sim arguments (fluid_ffi.h:74-83) and
 * Sim::new (render.rs:1468-1612) decide, made explicit. */
typedef struct FluidSimConfig {
    uint32_t geometry;
    float extent[2]; /* slab half width and height, m */
    float box_lo[3]; /* box corners, m */
    float box_hi[3];
    float spacing;      /* lattice spacing d, m */
    float h_ratio;      /* kernel h / d; the reference uses 1.2 (render.rs:1477) */
    float rest_density; /* kg/m^3; 0 selects the reference's 998.2 (sim.rs:6) */
    uint32_t seeding;
    float fill;         /* seed_slab's height fraction (0.5 in the reference) */
    uint32_t block[3];  /* FLUID_SEED_BLOCK lattice dims */
    float jitter;       /* FLUID_SEED_BLOCK jitter amplitude, fraction of d */
    uint64_t seed;      /* FLUID_SEED_BLOCK stream seed */
    uint32_t count;     /* FLUID_SEED_NONE particle count */
    uint32_t tracers;   /* passive tracers, seeded as sim.rs:105-122 */
    float xsph_blend;   /* < 0: the reference's 1 - exp(-6 dt) per substep */
    float temperature;  /* initial K (293.15 in the reference) */
    uint32_t solve;
    uint32_t div_iters;
    uint32_t den_iters;
    float div_tol;      /* mean positive divergence * dt / rho0 */
    float den_tol;      /* mean positive predicted compression */
    uint32_t max_iters;
    uint32_t nbr_cap;   /* neighbours kept per particle (overflow counted) */
    int32_t device;     /* CUDA device ordinal */
} FluidSimConfig;

/* The derived constants every kernel reads (SimParams, sim_solve.wgsl:11-23,
 * plus the walls and tracer box made explicit). */
typedef struct FluidSimParams {
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
} FluidSimParams;

/* The reduce_stats block (sim_solve.wgsl:800-874; the sim half of
 * FluidRenderStats, fluid_ffi.h:23-47) plus the solver's own counters. */
typedef struct FluidSimStats {
    float compression_avg; /* mean max(rho/rho0 - 1, 0): the density error */
    float compression_max;
    float density_min;
    float density_max;
    float pressure_min;
    float pressure_max;
    float v_max;
    float temperature_min;
    float temperature_max;
    uint32_t clamp_count;        /* cumulative CFL clamps */
    uint32_t neighbour_overflow; /* cumulative neighbours past nbr_cap */
    float v_min;
    float accel_min;
    float accel_max;
    uint32_t div_iters;    /* last substep */
    uint32_t den_iters;    /* last substep, warm start excluded */
    double div_residual;   /* last substep, after its last divergence apply */
    double den_residual;   /* last substep, after its last density apply */
    uint64_t substeps;     /* substeps run since create */
    uint64_t total_div_iters; /* divergence applies since create */
    uint64_t total_den_iters; /* density applies since create, warm starts excluded */
    uint32_t substeps_last_frame;
    int32_t error;         /* sticky device error (FLUID_ERR_*) */
} FluidSimStats;

/* Internal buffers a test may read back (render.rs tests read starts,
 * density and the working set the same way). */
#define FLUID_FIELD_DENSITY 0   /* float[n], working order */
#define FLUID_FIELD_ALPHA 1
#define FLUID_FIELD_KD 2
#define FLUID_FIELD_PRESSURE 3
#define FLUID_FIELD_NBR_N 4     /* uint32[n] */
#define FLUID_FIELD_STARTS 5    /* uint32[C * fluid_sim_grid_slabs() + 1] */
#define FLUID_FIELD_PERM 6      /* uint32[n] */
#define FLUID_FIELD_WORK_POS 7  /* float4[n] */
#define FLUID_FIELD_WORK_VEL 8  /* float4[n] */
#define FLUID_FIELD_ACCEL 9     /* float4[n] */
#define FLUID_FIELD_XSPH 10     /* float4[n] */
#define FLUID_FIELD_WALL_GRAD 11
#define FLUID_FIELD_COUNTERS 12 /* uint32[2]: clamp count, neighbour overflow */

/* Text of the last error on this thread ("" if none). */
const char *fluid_last_error(void);

/* The reference's defaults: slab geometry, seed_slab at fill 0.5, h = 1.2 d,
 * rest density 998.2, 293.15 K, fixed schedule 1 / 5, 96 neighbours. */
void fluid_sim_default_config(FluidSimConfig *cfg);

/* Replaces fluid_renderer_create (fluid_ffi.h:74-83; lib.rs:72-109) for the
 * sim alone: builds the particles, the grid and every device buffer, and
 * captures the substep as a CUDA graph. At most 2^28 - 1 particles (a
 * batch too, over all its boxes). Null on failure, reason in
 * fluid_last_error() and on stderr. */
FluidSim *fluid_sim_create(const FluidSimConfig *cfg);

/* Replaces fluid_renderer_destroy (fluid_ffi.h:182; lib.rs:283-285). */
void fluid_sim_destroy(FluidSim *sim);

int32_t fluid_sim_params(const FluidSim *sim, FluidSimParams *out);
uint32_t fluid_sim_count(const FluidSim *sim);
uint32_t fluid_sim_tracer_count(const FluidSim *sim);
/* The handle's cudaStream_t. */
void *fluid_sim_stream(FluidSim *sim);

/* One substep (render.rs:3175-3202 per substep): rebuild, density and
 * factor, the divergence solve, forces, the constant-density solve,
 * integrate. dt == 0 runs the rebuild and the density sweep alone, as the
 * reference's zero-substep test path (render.rs:3904-3955). Asynchronous. */
int32_t fluid_sim_step(FluidSim *sim, const FluidStep *step);

/* `n` substeps from an array of Step blocks, one upload. Asynchronous. */
int32_t fluid_sim_run(FluidSim *sim, const FluidStep *steps, uint32_t n);

/* reduce_stats on the current state (render.rs:3203). Asynchronous. */
int32_t fluid_sim_reduce_stats(FluidSim *sim);

/* One tracer pass (splat, resolve, advect; render.rs:3204-3228) with the
 * frame's dt and seed from `step`. Asynchronous. */
int32_t fluid_sim_tracers(FluidSim *sim, const FluidStep *step);
/* advect alone on the last resolved field (render.rs:5770-5787). */
int32_t fluid_sim_advect(FluidSim *sim, const FluidStep *step);

/* One frame the way Renderer::frame encodes it (render.rs:3090-3228), minus
 * drawing: `substeps` substeps of dt/substeps (0 selects substeps_for on the
 * last frame's v_max, capped at `cap`), v_clamp = 0.4 d / dt_sub, refine
 * passes by refine_passes(dt_sub) in the fixed schedule, then reduce_stats
 * and, with tracers, one tracer pass at the frame dt and `seed`. A dt of 0
 * encodes nothing (render.rs:3165-3168). Asynchronous; the stats it uses
 * for v_max are the previous frame's, read without blocking. */
int32_t fluid_sim_frame(FluidSim *sim, FluidVec3 force, FluidVec3 omega, FluidVec3 domega,
                        float dt, uint32_t substeps, uint32_t cap, uint32_t seed);

/* ---- the frame controller (host only) ------------------------------------ */

/* One reading of the motion sensors, MotionSample (lib.rs:21-37): gravity
 * and user acceleration in g, device frame; rotation rate in rad/s. */
typedef struct FluidMotion {
    FluidVec3 gravity;
    FluidVec3 user_acceleration;
    FluidVec3 rotation_rate;
} FluidMotion;

/* What one frame of Renderer::frame decides before encoding
 * (render.rs:3021-3098). */
typedef struct FluidFramePlan {
    FluidStep step;     /* the Step block each substep runs (dt_sub, v_clamp, fingers) */
    FluidVec3 force;    /* smoothed body force, m/s^2 */
    FluidVec3 omega;    /* smoothed angular velocity */
    FluidVec3 domega;   /* its derivative, clamped to +-200 */
    float dt;           /* frame dt, clamped to 1/30 s; 0 encodes nothing */
    float deviation;    /* the force filter's raw-to-smooth deviation */
    uint32_t substeps;  /* substeps_for on the given v_max; 0 with dt 0 */
    uint32_t refine;    /* refine_passes(dt / substeps) */
    uint32_t seed;      /* the frame's tracer seed */
    uint32_t asleep;    /* 1: the idle gate skipped the frame */
    uint64_t frames;    /* frames planned (not asleep) */
    uint64_t idle_frames;
} FluidFramePlan;

typedef struct FluidController FluidController;

/* render.rs:63-65, :76-78, :97-106: the substep floor, the refine passes of
 * a substep, and the substep count of a frame. */
uint32_t fluid_substep_floor(float dt, float dt_sub_max);
uint32_t fluid_refine_passes(float dt_sub);
uint32_t fluid_substeps_for(float dt, float v_max, float spacing, uint32_t cap);

/* The controller state Renderer keeps across frames: ForceFilter,
 * RotationTracker, Fingers, IdleGate (render.rs:862-1105). `extent` is the
 * box half width and height the fingers map onto; `cap` the substep cap.
 * Null on bad arguments. */
FluidController *fluid_controller_create(float spacing, const float extent[2], uint32_t cap);
void fluid_controller_destroy(FluidController *ctl);
/* Replaces fluid_renderer_touch (fluid_ffi.h:132-136): slot's finger at
 * normalised drawable (x, y), or lifted when down is 0. */
int32_t fluid_controller_touch(FluidController *ctl, uint32_t slot, float x, float y, uint32_t down);
/* One frame's plan from a motion sample at now_ms (CADisplayLink time) and
 * the one-frame-stale v_max (FluidSimStats.v_max). */
int32_t fluid_controller_plan(FluidController *ctl, const FluidMotion *motion, double now_ms,
                              float v_max, FluidFramePlan *out);
/* The idle gate alone (IdleGate, render.rs:1024-1105): asleep() is true
 * while a settled, untouched, unmoved pool's frame may be skipped. */
typedef struct FluidIdleGate FluidIdleGate;
FluidIdleGate *fluid_idle_gate_create(void);
void fluid_idle_gate_destroy(FluidIdleGate *gate);
uint32_t fluid_idle_gate_still_frames(void);
uint32_t fluid_idle_gate_asleep(FluidIdleGate *gate, uint32_t touched, const float smooth[3],
                                float dev, const float omega[3], float v_max);

/* Runs a plan on the GPU (render.rs:3168-3229 minus drawing): its substeps
 * with its Step block, reduce_stats, and a tracer pass at the frame dt. A
 * plan that is asleep or has dt 0 encodes nothing. Asynchronous. */
int32_t fluid_sim_frame_plan(FluidSim *sim, const FluidFramePlan *plan);

/* Waits for the handle's stream. Returns a sticky device error if one was
 * raised (a bounded wait that gave up). */
int32_t fluid_sim_sync(FluidSim *sim);

/* Replaces fluid_renderer_stats (fluid_ffi.h:175): the last reduce_stats
 * plus the solver counters. Synchronises. */
int32_t fluid_sim_stats(FluidSim *sim, FluidSimStats *out);

/* The resting set in slot order, any pointer may be null. Synchronises. */
int32_t fluid_sim_get_state(FluidSim *sim, float *pos4, float *vel4, float *prev_vel4,
                            float *prev_p, float *temp, uint32_t *id);
/* Replaces the resting set; null pointers leave that record unchanged.
 * Resets the warm start and the counters' baselines nowhere: the state is
 * taken as is. */
int32_t fluid_sim_set_state(FluidSim *sim, const float *pos4, const float *vel4,
                            const float *prev_vel4, const float *prev_p, const float *temp,
                            const uint32_t *id);
/* Positions and velocities ordered by particle id (the seed's order): the
 * particle-readback interface. Synchronises. */
int32_t fluid_sim_read_particles(FluidSim *sim, float *pos4, float *vel4);

/* Tracers as packed 8-byte records (sim_tracers.wgsl:64-80). */
int32_t fluid_sim_get_tracers(FluidSim *sim, uint32_t *packed2);
int32_t fluid_sim_set_tracers(FluidSim *sim, const uint32_t *packed2);

/* Copies an internal buffer (FLUID_FIELD_*) to host memory. Synchronises. */
int32_t fluid_sim_read_field(FluidSim *sim, int32_t field, void *out, uint64_t bytes);

/* Times one substep kernel by kernel with CUDA events on the handle's
 * stream: writes up to `cap` durations (ms) and names, returns the count. */
int32_t fluid_sim_profile_step(FluidSim *sim, const FluidStep *step, float *ms,
                               const char **names, uint32_t cap);
/* Kernel launches one substep issues at the current schedule (fixed mode). */
uint32_t fluid_sim_kernels_per_substep(const FluidSim *sim);
/* Slabs per cell along x in a simulation's neighbour grid: the grid keys
 * are cell * slabs + slab, so each cell's slots are in slab order (the
 * reference's scatter, sim_grid.wgsl:60-72, ranks a cell's particles by
 * atomic arrival, so any order inside a cell is one it can produce), and
 * FLUID_FIELD_STARTS holds cells * slabs + 1 entries. fluid_grid_build and
 * fluid_grid_build_static sort by cell alone. */
uint32_t fluid_sim_grid_slabs(void);

/* ---- the render-side thickness field ---------------------------------------
 * The body splat of sim_sprites.wgsl (`body`, `weight`, radius 1.5 h, an
 * orthographic view of the box's x-y extent) with the decay draw of the
 * field pass (render.rs:3233-3282), and sim_surface.wgsl `field_filter`,
 * as CUDA into device buffers the handle owns: no graphics stack. */
typedef struct FluidFieldParams {
    uint32_t width, height; /* texels (the reference uses a quarter of the drawable per axis) */
    float keep;             /* fraction of the previous field kept (0: a fresh splat) */
    uint32_t lens;          /* g channel: 0 none, 1 accel lens, 2 pressure lens, 3 density, 4 speed */
    float lo, hi;           /* the lens ramp's ends (sim_sprites.wgsl lens_at) */
} FluidFieldParams;

/* field = field * keep + (1 - keep) * splat of every particle: r the
 * thickness, g the thickness weighted by the lens. (Re)allocates and zeroes
 * the field when its size changes. Asynchronous. */
int32_t fluid_sim_field_splat(FluidSim *sim, const FluidFieldParams *p);
/* field_filter of the current field: (blurred thickness, x difference,
 * y difference, Laplacian) per texel. Asynchronous. */
int32_t fluid_sim_field_filter(FluidSim *sim);
/* Reads the field [height][width][2] and the filtered field
 * [height][width][4] (either may be null). Synchronises. */
int32_t fluid_sim_field_read(FluidSim *sim, float *field2, float *filtered4);
/* The field's keep fraction for a v_max (render.rs:1107-1111): 0.8 at rest,
 * down to 0 across 0.05-0.25 m/s. */
float fluid_field_keep_target(float v_max);

/* ---- batched boxes --------------------------------------------------------
 * Many independent boxes stepped by the same launches: each kernel of a
 * substep covers every box, a substep is one graph launch, and in the
 * tolerance mode each box stops its own loops (the graph loops while any box
 * is above tolerance). Each box's trajectory, iteration counts and residuals
 * are bit-identical to fluid_sim_create of its configuration. The reference
 * has no batch (one Sim per renderer, render.rs:1468-1612); this replaces
 * stepping many Sims one after another. */
typedef struct FluidBatch FluidBatch;

/* boxes[nboxes] (1..65535): per-box geometry, seeding, xsph_blend and
 * temperature; solve, div/den_iters, div/den_tol, max_iters, nbr_cap and
 * device must match boxes[0]; tracers must be 0. Null on failure. */
FluidBatch *fluid_batch_create(const FluidSimConfig *boxes, uint32_t nboxes);
void fluid_batch_destroy(FluidBatch *batch);
uint32_t fluid_batch_boxes(const FluidBatch *batch);
uint32_t fluid_batch_count(const FluidBatch *batch, uint32_t box);
uint32_t fluid_batch_total(const FluidBatch *batch);
void *fluid_batch_stream(FluidBatch *batch);
int32_t fluid_batch_params(const FluidBatch *batch, uint32_t box, FluidSimParams *out);
/* One substep of every box; steps[nboxes], box k takes steps[k] (dt > 0). */
int32_t fluid_batch_step(FluidBatch *batch, const FluidStep *steps);
/* `count` substeps; steps[count][nboxes]. Asynchronous. */
int32_t fluid_batch_run(FluidBatch *batch, const FluidStep *steps, uint32_t count);
/* reduce_stats of every box (sim_solve.wgsl:800-874). */
int32_t fluid_batch_reduce_stats(FluidBatch *batch);
/* Per-box statistics, out[nboxes]. Synchronises. */
int32_t fluid_batch_stats(FluidBatch *batch, FluidSimStats *out);
int32_t fluid_batch_sync(FluidBatch *batch);
/* One box's resting set (slot order), as fluid_sim_get_state. */
int32_t fluid_batch_get_state(FluidBatch *batch, uint32_t box, float *pos4, float *vel4,
                              float *prev_vel4, float *prev_p, float *temp, uint32_t *id);

/* The tuned sweeps, in this order, for the block-size calls below: density,
 * divergence prediction, apply, forces, forces apply, density prediction,
 * integrate. */
#define FLUID_TUNED_SWEEPS 7
/* Chooses each tuned sweep's block size (64, 128 or 256 threads) by timing
 * one substep of every candidate, Step blocks steps[nboxes], on the batch's
 * current state, which is restored afterwards (the batch does not advance).
 * Later substeps launch with the choices; results do not depend on them.
 * chosen[7] receives the sizes and ms[3][7] the times (candidate-major),
 * either may be null. Synchronises; allocates a snapshot of the state. */
int32_t fluid_batch_autotune(FluidBatch *batch, const FluidStep *steps, uint32_t *chosen,
                             float *ms);
/* Sets (0: the default) or reads the block size of each tuned sweep. */
int32_t fluid_batch_set_blocks(FluidBatch *batch, const uint32_t *tpb);
int32_t fluid_batch_get_blocks(const FluidBatch *batch, uint32_t *tpb);

/* ---- the adjoint -----------------------------------------------------------
 * A differentiable model of the substep (density, divergence solve, forces,
 * density solve, advection; particles in a fixed order, neighbour lists
 * rebuilt every substep) with hand-written adjoint kernels. Controls: one
 * body force per frame (the tilt-control sequence) and the XSPH
 * coefficient. Loss: |COM(final) - target|^2 + mean((rho/rho0 - 1)^2).
 * Each substep's neighbour lists, iteration counts and clamp branches are
 * held fixed under differentiation; the counts are decided by the
 * tolerance rule on the first forward (or set) and then frozen. The state
 * is checkpointed every `checkpoint_every` frames; the backward pass
 * recomputes each segment from its checkpoint. Precision 32 or 64 (the
 * FP64 instance is what finite differences check). The reference has no
 * adjoint (no counterpart). */
typedef struct FluidAdjoint FluidAdjoint;

FluidAdjoint *fluid_adjoint_create(const FluidSimConfig *cfg, uint32_t frames,
                                   uint32_t substeps_per_frame, float frame_dt, float v_clamp,
                                   uint32_t checkpoint_every, uint32_t precision);
void fluid_adjoint_destroy(FluidAdjoint *adj);
uint32_t fluid_adjoint_count(const FluidAdjoint *adj);
/* forces[frames][3], the XSPH coefficient, target[3]; writes the loss.
 * Synchronises. */
int32_t fluid_adjoint_forward(FluidAdjoint *adj, const double *forces, double xsph,
                              const double target[3], double *loss);
/* Gradients of the last forward's loss: grad_forces[frames][3], grad_xsph
 * (either may be null). Needs a forward since the last backward. */
int32_t fluid_adjoint_backward(FluidAdjoint *adj, double *grad_forces, double *grad_xsph);
/* The frozen per-substep iteration counts, [frames * substeps_per_frame]. */
int32_t fluid_adjoint_get_schedule(const FluidAdjoint *adj, uint32_t *div_iters,
                                   uint32_t *den_iters);
int32_t fluid_adjoint_set_schedule(FluidAdjoint *adj, const uint32_t *div_iters,
                                   const uint32_t *den_iters);
/* Final positions and velocities of the last forward, [count][3]. */
int32_t fluid_adjoint_final_state(FluidAdjoint *adj, double *pos3, double *vel3);
/* Device time of the last forward and backward, ms. */
int32_t fluid_adjoint_timing(const FluidAdjoint *adj, float *forward_ms, float *backward_ms);

/* ---- the neighbour grid alone ------------------------------------------ */

/* Grid geometry: sim.rs:14-44 (Grid). Key of a position:
 * (z * dims.y + y) * dims.x + x of min(u32((p - min) / cell), dims - 1). */
typedef struct FluidGrid {
    float min[3];
    float cell;
    uint32_t dims[3];
} FluidGrid;

/* Device workspace bytes fluid_grid_build needs for n positions. */
uint64_t fluid_grid_workspace_bytes(uint32_t n, const FluidGrid *grid);

/* The counting sort of sim_grid.wgsl:44-72 and sim_density.wgsl:36-55 with
 * the scan of sim_scan.wgsl:97-120, stable: starts[C+1] (starts[C] = n) and
 * the permutation perm[n] (slot -> input index, ascending index inside a
 * cell). All pointers are device memory; keys may be null. `stream` is a
 * cudaStream_t (null: the legacy default stream). Asynchronous. */
int32_t fluid_grid_build(const float *pos4, uint32_t n, const FluidGrid *grid, uint32_t *keys,
                         uint32_t *starts, uint32_t *perm, void *workspace, uint64_t ws_bytes,
                         void *stream);

/* Whether the fluid_grid_build last run on `workspace` (with the same n and
 * grid) completed: FLUID_OK, or FLUID_ERR_TIMEOUT (reason in
 * fluid_last_error()) when one of its bounded look-back waits gave up, in
 * which case its starts and permutation are invalid (a missing prefix was
 * counted as zero, so slots may repeat). Reads the build's error word on
 * `stream` after the work queued there and waits for it; allocates nothing.
 * Follows the reference's convention that a failure carries its reason
 * (crates/fluid-ffi/src/lib.rs:86-108). */
int32_t fluid_grid_build_status(const void *workspace, uint32_t n, const FluidGrid *grid,
                                void *stream);

/* The same from and to host memory (allocates, copies, synchronises). */
int32_t fluid_grid_build_host(const float *pos4, uint32_t n, const FluidGrid *grid,
                              uint32_t *starts, uint32_t *perm);

/* Scratch bytes compiled into the library for fluid_grid_build_static,
 * one area per device. */
#define FLUID_GRID_STATIC_SCRATCH_BYTES (16u << 20)

/* fluid_grid_build for callers that cannot allocate: the same keys, starts
 * and permutation, with no workspace argument and no allocation of any kind;
 * the scratch is a fixed area of FLUID_GRID_STATIC_SCRATCH_BYTES inside the
 * library. No counterpart in the reference (its grid build runs on buffers
 * the simulation owns). A build needing more scratch than that
 * (fluid_grid_workspace_bytes above the limit) returns FLUID_ERR_ARG. The
 * first call on each device sets up the scratch address; make it before any
 * stream capture begins. One scratch area per device: calls whose work
 * overlaps on the device race and must be ordered by the caller (one stream,
 * or events). Asynchronous on `stream`. */
int32_t fluid_grid_build_static(const float *pos4, uint32_t n, const FluidGrid *grid,
                                uint32_t *keys, uint32_t *starts, uint32_t *perm, void *stream);

/* Whether the last fluid_grid_build_static on the current device completed:
 * FLUID_OK, or FLUID_ERR_TIMEOUT when a bounded look-back wait gave up and
 * its starts and permutation are invalid. The error word lives in the fixed
 * scratch, so read it after that build and before the next call on the
 * device, which clears it. Reads on `stream` and waits; allocates nothing. */
int32_t fluid_grid_build_static_status(void *stream);

/* Failure detection, exercised (no counterpart in the reference): runs one
 * block of the grid's look-back scan whose predecessor never publishes, so
 * the scan's bounded wait (2^20 polls) gives up. Returns FLUID_ERR_TIMEOUT
 * when the wait gave up and recorded it, as it should; *ms (if not null)
 * the kernel's time. Nothing faults or hangs, and the device stays usable. */
int32_t fluid_selftest_scan_wait(int32_t device, float *ms);

/* The same for a radix digit pass of the grid build: one block claims the
 * second tile while the first never publishes its digit counts, so every
 * digit's bounded look-back (2^20 polls) gives up. FLUID_ERR_TIMEOUT when it
 * gave up and recorded it, as it should; *ms (if not null) the kernel's
 * time. The give-up is read back through fluid_grid_build_status on the
 * workspace the pass ran on. Nothing faults or hangs, and the device stays
 * usable. */
int32_t fluid_selftest_radix_wait(int32_t device, float *ms);

/* The same stalled digit pass on fluid_grid_build_static's fixed scratch,
 * laid out as its builds lay it out, reported through
 * fluid_grid_build_static_status: FLUID_ERR_TIMEOUT, as it should.
 * Allocates nothing. */
int32_t fluid_selftest_static_radix_wait(int32_t device, float *ms);

#ifdef __cplusplus
}
#endif
#endif
