// sim.cu — the FluidSim handle behind include/fluid_cu.h.
//
// Replaces Sim::new / the per-frame encode of crates/fluid-core/src/render.rs
// (:1468-1612 buffers and initial state, :3168-3229 the dispatch sequence)
// and the C ABI of crates/fluid-ffi/src/lib.rs. The substep is captured once
// as a CUDA graph per schedule and replayed; the Step block of every substep
// travels through a device ring that the first kernel of the substep reads,
// so a run of substeps needs one upload and no host synchronisation.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "field.cuh"
#include "grid.cuh"
#include "solve.cuh"

using namespace fcu;

namespace {

thread_local std::string g_last_error;

int32_t fail(int32_t code, const std::string &msg) {
    g_last_error = msg;
    fprintf(stderr, "fluid: %s\n", msg.c_str());
    return code;
}

#define CK(expr)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(e_ == cudaErrorMemoryAllocation ? FLUID_ERR_OOM : FLUID_ERR_CUDA,    \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

constexpr float kPi = 3.14159265358979323846f;
constexpr float kRestDensity = 998.2f;                 // sim.rs:6
constexpr float kSlabDepth = 4.0f * 0.00765f;          // sim.rs:10, lib.rs:13
constexpr uint32_t kRing = 1024;                       // Step blocks in flight

uint32_t hash32(uint32_t x) {  // sim.rs:318-323
    uint32_t h = x * 0x9E3779B9u;
    h ^= h >> 16;
    h = h * 0x85EBCA6Bu;
    return h ^ (h >> 13);
}

uint64_t splitmix64(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// IEEE half bits, round to nearest even (pack2x16float; sim.rs:139-151).
uint16_t half_bits(float x) {
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

void pack_tracer(const float pos[3], float speed, const float e[2], uint32_t out[2]) {  // sim.rs:127-133
    auto unorm = [](float v, float ex) {
        float u = v / ex * 0.5f + 0.5f;
        u = u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
        return (uint32_t)(u * 65535.0f + 0.5f);
    };
    out[0] = unorm(pos[0], e[0]) | (unorm(pos[1], e[1]) << 16);
    out[1] = (uint32_t)half_bits(pos[2]) | ((uint32_t)half_bits(speed) << 16);
}

}  // namespace

namespace fcu {
// Records an error for fluid_last_error from another translation unit.
int32_t report_error(int32_t code, const std::string &msg) { return fail(code, msg); }
void host_step_constants(float xsph_cfg, const FluidStep &st, DevStep &d);
}  // namespace fcu

struct FluidSim {
    FluidSimConfig cfg{};
    DevParams P{};
    uint32_t n = 0, cells = 0, ntr = 0;
    uint32_t keyspace = 0;  // grid keys: cells * kSimSlabs
    int device = 0;
    cudaStream_t stream = nullptr;
    SimBufs b{};
    GridWork gw{};
    void *grid_ws = nullptr;
    DevStep *ring = nullptr, *cur = nullptr;
    DevSolve *solve = nullptr;
    DevStep *h_ring = nullptr;  // pinned mirror of the ring
    uint64_t h_cursor = 0, synced_cursor = 0;
    std::map<std::pair<uint32_t, uint32_t>, cudaGraphExec_t> graphs;
    cudaGraphExec_t density_graph = nullptr;
    cudaGraphExec_t tol_graph = nullptr;
    cudaStream_t side = nullptr;  // captures the loop bodies
    std::vector<void *> allocs;
    float stats_host[14]{};
    uint32_t last_frame_substeps = 0;
    // one-frame-stale stats for the frame controller (render.rs:3418-3514)
    float *h_stats_stale = nullptr;
    cudaEvent_t stats_ready = nullptr;
    bool stats_pending = false;
    float v_max_stale = 0.0f;
    // the render-side thickness field (fluid_sim_field_*), allocated on use
    float2 *field = nullptr;
    float4 *field_filtered = nullptr;
    unsigned long long *field_acc = nullptr;
    FieldGeom fgeom{};

    // The sweeps' view of this one-box simulation.
    Geo geo() const {
        Geo g{};
        g.one = P;
        g.solve = solve;
        g.st = cur;
        g.n = n;
        g.nboxes = 1;
        return g;
    }
    uint32_t stats_chunks() const {
        const uint32_t c = (n + kStatsThreads - 1) / kStatsThreads;
        return c < 1u ? 1u : (c > (uint32_t)kStatsChunks ? (uint32_t)kStatsChunks : c);
    }

    template <class T>
    cudaError_t alloc(T **p, size_t count) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 16);
        if (e == cudaSuccess) {
            allocs.push_back(q);
            *p = (T *)q;
        }
        return e;
    }
};

namespace {

void derive_params(const FluidSimConfig &c, uint32_t count, DevParams &P) {
    std::memset(&P, 0, sizeof P);
    const float h = c.h_ratio * c.spacing;
    const float support = 2.0f * h;
    if (c.geometry == FLUID_GEOMETRY_SLAB) {
        // sim.rs:24-32 and render.rs:1477-1478
        const float half[3] = {c.extent[0], c.extent[1], kSlabDepth * 0.5f};
        for (int i = 0; i < 3; ++i) {
            P.dims[i] = (uint32_t)std::ceil(2.0f * half[i] / support) + 2u;
            P.box_min[i] = -half[i] - support;
        }
    } else {
        for (int i = 0; i < 3; ++i) {
            P.dims[i] = (uint32_t)std::ceil((c.box_hi[i] - c.box_lo[i]) / support) + 2u;
            P.box_min[i] = c.box_lo[i] - support;
        }
    }
    P.cell = support;
    P.count = count;
    // sim.rs:330-350 (pack_sim_params)
    P.h = h;
    P.inv_h = 1.0f / h;
    P.sigma = 1.0f / (kPi * h * h * h);
    P.sigma_h = P.sigma / h;
    P.support_sq = 4.0f * h * h;
    P.rho0 = c.rest_density > 0.0f ? c.rest_density : kRestDensity;
    P.mass = P.rho0 * c.spacing * c.spacing * c.spacing;  // render.rs:1610
    for (int i = 0; i < 3; ++i) {
        if (c.geometry == FLUID_GEOMETRY_SLAB) {
            // sim_solve.wgsl:237-239, :311-312; sim_tracers.wgsl:60-62
            P.wall_lo[i] = P.box_min[i] + P.cell;
            P.wall_hi[i] = -P.wall_lo[i];
            P.tracer_c[i] = 0.0f;
            P.tracer_e[i] = -(P.box_min[i] + P.cell);
        } else {
            P.wall_lo[i] = c.box_lo[i];
            P.wall_hi[i] = c.box_hi[i];
            P.tracer_c[i] = (c.box_lo[i] + c.box_hi[i]) * 0.5f;
            P.tracer_e[i] = (c.box_hi[i] - c.box_lo[i]) * 0.5f;
        }
    }
    P.xsph_blend = c.xsph_blend;
    P.nbr_cap = c.nbr_cap;
}

// sim.rs:65-72
void lattice_dims(float spacing, const float extent[2], float fill, uint32_t out[3]) {
    const float size[3] = {2.0f * extent[0] - spacing, (2.0f * extent[1] - spacing) * fill,
                           kSlabDepth - spacing};
    for (int i = 0; i < 3; ++i) {
        const float v = size[i] / spacing;
        const uint32_t k = v <= 0.0f ? 0u : (uint32_t)v;
        out[i] = k < 1u ? 1u : k;
    }
}

// sim.rs:77-100
void seed_slab(float spacing, const float extent[2], float fill, std::vector<float> &out) {
    uint32_t n[3];
    lattice_dims(spacing, extent, fill, n);
    out.assign(4ull * n[0] * n[1] * n[2], 0.0f);
    const float origin[3] = {-0.5f * (float)n[0] * spacing, -extent[1] + 0.5f * spacing,
                             -0.5f * (float)n[2] * spacing};
    auto jitter = [](uint32_t h) { return ((float)h / 4294967295.0f - 0.5f) * 0.2f; };
    for (uint32_t iz = 0; iz < n[2]; ++iz)
        for (uint32_t iy = 0; iy < n[1]; ++iy)
            for (uint32_t ix = 0; ix < n[0]; ++ix) {
                const uint32_t i = (iz * n[1] + iy) * n[0] + ix;
                float *o = &out[4ull * i];
                o[0] = origin[0] + ((float)ix + 0.5f + jitter(hash32(i * 3))) * spacing;
                o[1] = origin[1] + ((float)iy + jitter(hash32(i * 3 + 1))) * spacing;
                o[2] = origin[2] + ((float)iz + 0.5f + jitter(hash32(i * 3 + 2))) * spacing;
            }
}

// A lattice block at box_lo: cell centres (i + 1/2) d, each axis jittered by
// a uniform draw in [-jitter, jitter) d from one splitmix64 stream.
void seed_block(const FluidSimConfig &c, std::vector<float> &out) {
    const uint64_t n = (uint64_t)c.block[0] * c.block[1] * c.block[2];
    out.assign(4 * n, 0.0f);
    uint64_t s = c.seed;
    const float amp = c.jitter * c.spacing;
    size_t i = 0;
    for (uint32_t iz = 0; iz < c.block[2]; ++iz)
        for (uint32_t iy = 0; iy < c.block[1]; ++iy)
            for (uint32_t ix = 0; ix < c.block[0]; ++ix, ++i) {
                const uint32_t idx[3] = {ix, iy, iz};
                for (int a = 0; a < 3; ++a) {
                    const float u = (float)(splitmix64(&s) >> 40) * (1.0f / 16777216.0f);
                    out[4 * i + a] = c.box_lo[a] + ((float)idx[a] + 0.5f) * c.spacing + (2.0f * u - 1.0f) * amp;
                }
            }
}

// sim.rs:105-122 for the slab; over the block's region for a box.
void seed_tracers(const FluidSimConfig &c, const DevParams &P, uint32_t count,
                  std::vector<uint32_t> &out) {
    out.assign(2ull * count, 0u);
    auto unit = [](uint32_t h) { return (float)h / 4294967295.0f; };
    if (c.geometry == FLUID_GEOMETRY_SLAB) {
        const float half[3] = {c.extent[0] - 0.001f, c.extent[1] - 0.001f, 0.5f * kSlabDepth - 0.001f};
        for (uint32_t i = 0; i < count; ++i) {
            const float pos[3] = {(unit(hash32(i * 3)) * 2.0f - 1.0f) * half[0],
                                  -half[1] + unit(hash32(i * 3 + 1)) * 2.0f * half[1] * c.fill,
                                  (unit(hash32(i * 3 + 2)) * 2.0f - 1.0f) * half[2]};
            pack_tracer(pos, 0.0f, c.extent, &out[2ull * i]);
        }
        return;
    }
    float size[3];
    for (int a = 0; a < 3; ++a) {
        const uint32_t nb = c.seeding == FLUID_SEED_BLOCK ? c.block[a] : 0u;
        size[a] = nb ? (float)nb * c.spacing : (c.box_hi[a] - c.box_lo[a]);
    }
    for (uint32_t i = 0; i < count; ++i) {
        float rel[3];
        for (int a = 0; a < 3; ++a)
            rel[a] = c.box_lo[a] + unit(hash32(i * 3 + a)) * size[a] - P.tracer_c[a];
        const float e[2] = {P.tracer_e[0], P.tracer_e[1]};
        pack_tracer(rel, 0.0f, e, &out[2ull * i]);
    }
}

void fill_step(const FluidSim *s, const FluidStep &st, DevStep &d) {
    host_step_constants(s->cfg.xsph_blend, st, d);
}

GridGeom geom_of(const DevParams &P) {
    GridGeom g;
    for (int i = 0; i < 3; ++i) {
        g.min[i] = P.box_min[i];
        g.dims[i] = P.dims[i];
    }
    g.cell = P.cell;
    g.slabs = kSimSlabs;
    return g;
}

// One substep's launches at a fixed schedule (render.rs:3175-3202):
// div_iters divergence applies, den_iters constant-density pairs. With
// density_only the substep stops after density_div (the zero-dt path).
// `mark`, when set, is called after every launch with the kernel's name.
template <class Mark>
cudaError_t enqueue_substep(FluidSim *s, cudaStream_t st, uint32_t div_iters, uint32_t den_iters,
                            bool density_only, Mark mark) {
    cudaError_t e = cudaMemsetAsync(s->solve->acc_div, 0, 2 * kAccSlots * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    e = grid_build_enqueue(st, s->b.pos, s->n, geom_of(s->P), s->b.keys, s->b.starts, s->b.perm, s->gw,
                           s->ring, s->cur, s->solve, kRing);
    if (e != cudaSuccess) return e;
    mark("grid");
    const Geo g = s->geo();
    launch_gather(st, s->b, s->n);
    mark("gather");
    launch_density_div(st, g, s->b, 0);
    mark("density_div");
    if (density_only) return cudaGetLastError();
    for (uint32_t d = 0; d < div_iters; ++d) {
        if (d > 0) {
            launch_div_kappa(st, g, s->b, (int)d, kGateNone);
            mark("div_kappa");
        }
        launch_apply(st, g, s->b, false, kGateNone);
        mark("div_apply");
    }
    launch_forces_eval(st, g, s->b);
    mark("forces_eval");
    launch_forces_apply(st, g, s->b);
    mark("forces_den_apply");
    for (uint32_t k = 0; k < den_iters; ++k) {
        launch_den_kappa(st, g, s->b, (int)k, kGateNone);
        mark("den_kappa");
        launch_apply(st, g, s->b, true, kGateNone);
        mark("den_apply");
    }
    const int div_slot = div_iters > 0 ? (int)div_iters - 1 : 0;
    launch_integrate(st, g, s->b, div_slot, den_iters > 0 ? (int)den_iters - 1 : -1, (int)div_iters,
                     (int)den_iters);
    mark("integrate");
    return cudaGetLastError();
}

int32_t capture(FluidSim *s, uint32_t div_iters, uint32_t den_iters, bool density_only,
                cudaGraphExec_t *out) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_substep(s, s->stream, div_iters, den_iters, density_only, [](const char *) {});
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess) return fail(FLUID_ERR_CUDA, std::string("substep capture: ") + cudaGetErrorString(e));
    if (e2 != cudaSuccess) return fail(FLUID_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(e2));
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(FLUID_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    return FLUID_OK;
}

int32_t graph_for(FluidSim *s, uint32_t div_iters, uint32_t den_iters, cudaGraphExec_t *out) {
    auto key = std::make_pair(div_iters, den_iters);
    auto it = s->graphs.find(key);
    if (it != s->graphs.end()) {
        *out = it->second;
        return FLUID_OK;
    }
    int32_t rc = capture(s, div_iters, den_iters, false, out);
    if (rc == FLUID_OK) s->graphs[key] = *out;
    return rc;
}

// Adds a WHILE node after the capture's current frontier and makes it the
// frontier; returns its body graph.
int32_t add_while(cudaStream_t st, cudaGraph_t g, cudaGraphConditionalHandle h, cudaGraph_t *body) {
    cudaStreamCaptureStatus status;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(st, &status, nullptr, nullptr, &deps, &nd));
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &p));
    *body = p.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return FLUID_OK;
}

// The tolerance substep: the same sweeps as the fixed schedule, with the
// divergence and density iterations as device-side loops (graph WHILE
// nodes) that a one-thread kernel continues or stops from the exact FP64
// residual, so no iteration waits on the host.
int32_t capture_tolerance(FluidSim *s, cudaGraphExec_t *out) {
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle hdiv, hden;
    CK(cudaGraphConditionalHandleCreate(&hdiv, g, 0, 0));
    CK(cudaGraphConditionalHandleCreate(&hden, g, 0, 0));
    const FluidSimConfig &c = s->cfg;
    cudaStream_t st = s->stream;
    cudaGraph_t bdiv = nullptr, bden = nullptr;
    CK(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int32_t rc = FLUID_OK;
    cudaError_t e = cudaMemsetAsync(s->solve->acc_div, 0, 2 * kAccSlots * sizeof(unsigned long long), st);
    if (e == cudaSuccess)
        e = grid_build_enqueue(st, s->b.pos, s->n, geom_of(s->P), s->b.keys, s->b.starts, s->b.perm, s->gw,
                               s->ring, s->cur, s->solve, kRing);
    const Geo geo = s->geo();
    // With at least one divergence apply, forces_eval runs after every one
    // and also forms the divergence prediction that decides whether the
    // loop goes on (its kappa in kd2 / wpk2, which the loop's applies read).
    const bool fused = c.max_iters >= 1;
    SimBufs bd = s->b;
    if (fused) {
        bd.kd = s->b.kd2;
        bd.wpk = s->b.wpk2;
    }
    if (e == cudaSuccess) {
        launch_gather(st, s->b, s->n);
        launch_density_div(st, geo, bd, 0);
        launch_tol_finish(st, geo, 0, 1, c.div_tol, c.max_iters, hdiv);
        rc = add_while(st, g, hdiv, &bdiv);
    }
    if (e == cudaSuccess && rc == FLUID_OK) {
        if (!fused) launch_forces_eval(st, geo, s->b);
        launch_forces_apply(st, geo, s->b);
        launch_den_kappa(st, geo, s->b, 0, kGateNone);
        launch_tol_finish(st, geo, 1, 1, c.den_tol, c.max_iters, hden);
        rc = add_while(st, g, hden, &bden);
    }
    if (e == cudaSuccess && rc == FLUID_OK) launch_integrate(st, geo, s->b, -1, -1, 0, 0);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaGraph_t g2 = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(st, &g2);
    if (rc != FLUID_OK || e != cudaSuccess || e2 != cudaSuccess) {
        cudaGraphDestroy(g);
        if (rc != FLUID_OK) return rc;
        return fail(FLUID_ERR_CUDA, std::string("tolerance capture: ") +
                                        cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    // loop bodies
    CK(cudaStreamBeginCaptureToGraph(s->side, bdiv, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launch_apply(s->side, geo, bd, false, kGateDiv);
    if (fused) launch_forces_div(s->side, geo, s->b, 0, kGateDiv);
    else launch_div_kappa(s->side, geo, s->b, 0, kGateDiv);
    launch_tol_finish(s->side, geo, 0, 0, c.div_tol, c.max_iters, hdiv);
    CK(cudaStreamEndCapture(s->side, &bdiv));
    CK(cudaStreamBeginCaptureToGraph(s->side, bden, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launch_apply(s->side, geo, s->b, true, kGateDen);
    launch_den_kappa(s->side, geo, s->b, 0, kGateDen);
    launch_tol_finish(s->side, geo, 1, 0, c.den_tol, c.max_iters, hden);
    CK(cudaStreamEndCapture(s->side, &bden));
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(FLUID_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    return FLUID_OK;
}

// The graph of one substep in the handle's schedule.
int32_t substep_graph(FluidSim *s, uint32_t den_fixed, cudaGraphExec_t *out) {
    if (s->cfg.solve == FLUID_SOLVE_TOLERANCE) {
        if (!s->tol_graph) {
            int32_t rc = capture_tolerance(s, &s->tol_graph);
            if (rc != FLUID_OK) return rc;
        }
        *out = s->tol_graph;
        return FLUID_OK;
    }
    return graph_for(s, s->cfg.div_iters, den_fixed, out);
}


// Places `count` Step blocks in the ring (pinned mirror, then one or two
// copies) for the next `count` substeps.
int32_t upload_steps(FluidSim *s, const FluidStep *steps, uint32_t count) {
    if (s->h_cursor + count - s->synced_cursor > kRing) {
        // The mirror slots about to be rewritten may still wait for their copy.
        CK(cudaStreamSynchronize(s->stream));
        s->synced_cursor = s->h_cursor;
    }
    uint32_t done = 0;
    while (done < count) {
        const uint32_t slot = (uint32_t)((s->h_cursor + done) % kRing);
        uint32_t m = count - done;
        if (m > kRing - slot) m = kRing - slot;
        for (uint32_t k = 0; k < m; ++k) fill_step(s, steps[done + k], s->h_ring[slot + k]);
        CK(cudaMemcpyAsync(s->ring + slot, s->h_ring + slot, m * sizeof(DevStep), cudaMemcpyHostToDevice,
                           s->stream));
        done += m;
    }
    s->h_cursor += count;
    return FLUID_OK;
}

// One frame on the GPU (render.rs:3168-3229 minus drawing): n substeps of
// the Step block `st` (the fixed schedule runs `refine` density pairs), then
// reduce_stats, a tracer pass at the frame dt and seed, and the stale-stats
// copy the next frame's substep policy reads without blocking.
int32_t run_frame(FluidSim *s, const FluidStep &st, uint32_t n, uint32_t refine, float frame_dt,
                  uint32_t seed) {
    std::vector<FluidStep> steps(n, st);
    int32_t rc = upload_steps(s, steps.data(), n);
    if (rc != FLUID_OK) return rc;
    cudaGraphExec_t g;
    rc = substep_graph(s, refine, &g);
    if (rc != FLUID_OK) return rc;
    for (uint32_t k = 0; k < n; ++k) CK(cudaGraphLaunch(g, s->stream));
    launch_stats(s->stream, s->geo(), s->b, s->stats_chunks());
    if (s->ntr) {
        FluidStep tr;
        std::memset(&tr, 0, sizeof tr);
        tr.force[0] = st.force[0];
        tr.force[1] = st.force[1];
        tr.force[2] = st.force[2];
        tr.dt = frame_dt;
        tr.seed = seed;
        DevStep d;
        fill_step(s, tr, d);
        launch_splat(s->stream, s->P, s->b);
        launch_resolve(s->stream, s->P, s->b);
        launch_advect(s->stream, s->P, s->b, d, s->ntr);
    }
    CK(cudaGetLastError());
    if (!s->stats_pending) {
        CK(cudaMemcpyAsync(s->h_stats_stale, s->b.stats, 16 * sizeof(float), cudaMemcpyDeviceToHost,
                           s->stream));
        CK(cudaEventRecord(s->stats_ready, s->stream));
        s->stats_pending = true;
    }
    s->last_frame_substeps = n;
    return FLUID_OK;
}

bool valid_config(const FluidSimConfig *c, std::string &why) {
    if (!c) return why = "null config", false;
    if (!(c->spacing > 0.0f) || !(c->h_ratio > 0.0f)) return why = "spacing and h_ratio must be positive", false;
    if (c->geometry > FLUID_GEOMETRY_BOX) return why = "unknown geometry", false;
    if (c->geometry == FLUID_GEOMETRY_SLAB && !(c->extent[0] > 0.0f && c->extent[1] > 0.0f))
        return why = "slab extent must be positive", false;
    if (c->geometry == FLUID_GEOMETRY_BOX)
        for (int i = 0; i < 3; ++i)
            if (!(c->box_hi[i] > c->box_lo[i])) return why = "box_hi must exceed box_lo", false;
    if (c->seeding > FLUID_SEED_NONE) return why = "unknown seeding", false;
    if (c->seeding == FLUID_SEED_BLOCK && c->geometry != FLUID_GEOMETRY_BOX)
        return why = "block seeding needs the box geometry", false;
    if (c->seeding == FLUID_SEED_SLAB && c->geometry != FLUID_GEOMETRY_SLAB)
        return why = "slab seeding needs the slab geometry", false;
    if (c->nbr_cap == 0 || c->nbr_cap > 1024) return why = "nbr_cap must be in 1..1024", false;
    if (c->solve > FLUID_SOLVE_TOLERANCE) return why = "unknown solve mode", false;
    if (c->div_iters > kMaxIters || c->den_iters > kMaxIters || c->max_iters > kMaxIters)
        return why = "iteration counts are capped at 126", false;
    return true;
}

}  // namespace

// Host steps the batch handle (batch.cu) shares with the one-box handle.
namespace fcu {
bool host_valid_config(const FluidSimConfig *c, std::string &why) { return valid_config(c, why); }
void host_params(const FluidSimConfig &c, uint32_t count, DevParams &P) { derive_params(c, count, P); }
void host_seed(const FluidSimConfig &c, std::vector<float> &pos) {
    if (c.seeding == FLUID_SEED_SLAB) seed_slab(c.spacing, c.extent, c.fill, pos);
    else if (c.seeding == FLUID_SEED_BLOCK) seed_block(c, pos);
    else pos.assign(4ull * c.count, 0.0f);
}
// The reference evaluates these per thread (sim_solve.wgsl:657, :741;
// sim_tracers.wgsl:182); they depend on dt alone, so once per substep.
void host_step_constants(float xsph_cfg, const FluidStep &st, DevStep &d) {
    d.s = st;
    const float dt = st.dt;
    d.xsph_blend = xsph_cfg >= 0.0f ? xsph_cfg : 1.0f - std::exp(-6.0f * dt);
    d.chase = 1.0f - std::exp(-20.0f * dt);
    d.decay = std::exp(-dt / 4.0f);
    d.pad = 0.0f;
}
int32_t host_add_while(cudaStream_t st, cudaGraph_t g, cudaGraphConditionalHandle h, cudaGraph_t *body) {
    return add_while(st, g, h, body);
}
}  // namespace fcu

extern "C" {

const char *fluid_last_error(void) { return g_last_error.c_str(); }

void fluid_sim_default_config(FluidSimConfig *c) {
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->geometry = FLUID_GEOMETRY_SLAB;
    c->extent[0] = 4.0f * 0.0357f;  // render.rs:3868 TEST_EXTENT
    c->extent[1] = 4.0f * 0.0774f;
    c->spacing = 4.0f * 0.0025f;    // render.rs:1353 SIM_SPACING
    c->h_ratio = 1.2f;
    c->rest_density = 0.0f;
    c->seeding = FLUID_SEED_SLAB;
    c->fill = 0.5f;
    c->jitter = 0.005f;
    c->seed = 1;
    c->tracers = 0;
    c->xsph_blend = -1.0f;
    c->temperature = 293.15f;
    c->solve = FLUID_SOLVE_FIXED;
    c->div_iters = 1;
    c->den_iters = 5;
    c->div_tol = 0.01f;
    c->den_tol = 0.001f;
    c->max_iters = 100;
    c->nbr_cap = FLUID_NBR_CAP_DEFAULT;
    c->device = 0;
}

void fluid_sim_destroy(FluidSim *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
    if (s->density_graph) cudaGraphExecDestroy(s->density_graph);
    if (s->tol_graph) cudaGraphExecDestroy(s->tol_graph);
    for (void *p : s->allocs) cudaFree(p);
    if (s->grid_ws) cudaFree(s->grid_ws);
    if (s->h_ring) cudaFreeHost(s->h_ring);
    if (s->h_stats_stale) cudaFreeHost(s->h_stats_stale);
    if (s->stats_ready) cudaEventDestroy(s->stats_ready);
    if (s->field) cudaFree(s->field);
    if (s->field_filtered) cudaFree(s->field_filtered);
    if (s->field_acc) cudaFree(s->field_acc);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

static int32_t create_into(FluidSim *s, const FluidSimConfig *cfg) {
    s->cfg = *cfg;
    s->device = cfg->device;
    CK(cudaSetDevice(s->device));
    std::vector<float> pos;
    if (cfg->seeding == FLUID_SEED_SLAB) seed_slab(cfg->spacing, cfg->extent, cfg->fill, pos);
    else if (cfg->seeding == FLUID_SEED_BLOCK) seed_block(*cfg, pos);
    else pos.assign(4ull * cfg->count, 0.0f);
    const uint64_t n64 = pos.size() / 4;
    // a neighbour list entry holds the slot in 28 bits
    if (n64 == 0 || n64 > 0x0fffffffull) return fail(FLUID_ERR_ARG, "particle count must be in 1..2^28-1");
    s->n = (uint32_t)n64;
    derive_params(*cfg, s->n, s->P);
    const uint64_t cells64 = (uint64_t)s->P.dims[0] * s->P.dims[1] * s->P.dims[2];
    if (cells64 >= 0xffffffffull) return fail(FLUID_ERR_ARG, "grid has too many cells");
    s->cells = (uint32_t)cells64;
    if (cells64 * kSimSlabs >= 0xffffffffull) return fail(FLUID_ERR_ARG, "grid has too many cells");
    s->keyspace = (uint32_t)(cells64 * kSimSlabs);
    s->ntr = cfg->tracers;
    if ((uint64_t)s->n * cfg->nbr_cap > (1ull << 40)) return fail(FLUID_ERR_ARG, "neighbour lists too large");

    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    const size_t n = s->n, C = s->cells;
    SimBufs &b = s->b;
    CK(s->alloc(&b.pos, n));
    CK(s->alloc(&b.vel, n));
    CK(s->alloc(&b.pvel, n));
    CK(s->alloc(&b.pp, n));
    CK(s->alloc(&b.temp, n));
    CK(s->alloc(&b.id, n));
    CK(s->alloc(&b.wpos, n));
    CK(s->alloc(&b.wvel, n));
    CK(s->alloc(&b.wpvel, n));
    CK(s->alloc(&b.wpp, n));
    CK(s->alloc(&b.wtemp, n));
    CK(s->alloc(&b.wid, n));
    CK(s->alloc(&b.keys, n));
    CK(s->alloc(&b.starts, (size_t)s->keyspace + 1));
    CK(s->alloc(&b.perm, n));
    CK(s->alloc(&b.density, n));
    CK(s->alloc(&b.alpha, n));
    CK(s->alloc(&b.kd, n));
    CK(s->alloc(&b.wpk, n));
    CK(s->alloc(&b.kd2, n));
    CK(s->alloc(&b.wpk2, n));
    CK(s->alloc(&b.pressure, n));
    CK(s->alloc(&b.pinc, n));
    CK(s->alloc(&b.rho_near, n));
    CK(s->alloc(&b.accel, n));
    CK(s->alloc(&b.xsph, n));
    CK(s->alloc(&b.wgrad, n));
    CK(s->alloc(&b.nbr, n * cfg->nbr_cap));
    CK(s->alloc(&b.nbr_n, n));
    CK(s->alloc(&b.tracers, 2 * (size_t)(s->ntr > 0 ? s->ntr : 1)));
    CK(s->alloc(&b.vel_grid, 4 * C));
    CK(s->alloc(&b.vel_flat, C));
    CK(s->alloc(&b.stats_part, (size_t)kStatsChunks * 12));
    CK(s->alloc(&b.stats_acc, 1));
    CK(s->alloc(&b.stats, 16));
    CK(s->alloc(&s->ring, kRing));
    CK(s->alloc(&s->cur, 1));
    CK(s->alloc(&s->solve, 1));
    const size_t wsb = grid_work_bytes(s->n, s->keyspace);
    CK(cudaMalloc(&s->grid_ws, wsb));
    s->gw = grid_work_carve(s->grid_ws, s->n, s->keyspace, &s->solve->error);
    CK(cudaMallocHost(&s->h_ring, kRing * sizeof(DevStep)));
    CK(cudaMallocHost(&s->h_stats_stale, 16 * sizeof(float)));
    CK(cudaEventCreateWithFlags(&s->stats_ready, cudaEventDisableTiming));

    // Initial state (render.rs:1484-1555): the seed, at rest, at temperature.
    std::vector<float> zeros4(4 * n, 0.0f), zeros(n, 0.0f), temp(n, cfg->temperature);
    std::vector<uint32_t> ids(n);
    for (size_t i = 0; i < n; ++i) ids[i] = (uint32_t)i;
    CK(cudaMemcpy(b.pos, pos.data(), 16 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.vel, zeros4.data(), 16 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.pvel, zeros4.data(), 16 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.pp, zeros.data(), 4 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.temp, temp.data(), 4 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.id, ids.data(), 4 * n, cudaMemcpyHostToDevice));
    for (float *z : {b.density, b.alpha, b.kd, b.pressure, b.pinc, b.rho_near}) CK(cudaMemset(z, 0, 4 * n));
    CK(cudaMemset(b.nbr_n, 0, 4 * n));
    CK(cudaMemset(b.vel_grid, 0, 16 * C));
    CK(cudaMemset(b.vel_flat, 0, 16 * C));
    CK(cudaMemset(b.stats_acc, 0, 8));
    CK(cudaMemset(b.stats, 0, 64));
    CK(cudaMemset(s->solve, 0, sizeof(DevSolve)));
    if (s->ntr) {
        std::vector<uint32_t> tr;
        seed_tracers(*cfg, s->P, s->ntr, tr);
        CK(cudaMemcpy(b.tracers, tr.data(), 8ull * s->ntr, cudaMemcpyHostToDevice));
    }
    CK(cudaDeviceSynchronize());
    CK(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    cudaGraphExec_t g;
    int32_t rc = substep_graph(s, cfg->den_iters, &g);
    if (rc != FLUID_OK) return rc;
    return FLUID_OK;
}

FluidSim *fluid_sim_create(const FluidSimConfig *cfg) {
    std::string why;
    if (!valid_config(cfg, why)) {
        fail(FLUID_ERR_ARG, why);
        return nullptr;
    }
    FluidSim *s = new FluidSim();
    if (create_into(s, cfg) != FLUID_OK) {
        std::string keep = g_last_error;
        fluid_sim_destroy(s);
        g_last_error = keep;
        return nullptr;
    }
    g_last_error.clear();
    return s;
}

int32_t fluid_sim_params(const FluidSim *s, FluidSimParams *out) {
    if (!s || !out) return fail(FLUID_ERR_ARG, "null argument");
    std::memcpy(out, &s->P, sizeof *out);
    return FLUID_OK;
}

uint32_t fluid_sim_count(const FluidSim *s) { return s ? s->n : 0u; }
uint32_t fluid_sim_tracer_count(const FluidSim *s) { return s ? s->ntr : 0u; }
void *fluid_sim_stream(FluidSim *s) { return s ? (void *)s->stream : nullptr; }

int32_t fluid_sim_run(FluidSim *s, const FluidStep *steps, uint32_t count) {
    if (!s || (!steps && count)) return fail(FLUID_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    for (uint32_t k = 0; k < count; ++k)
        if (!(steps[k].dt >= 0.0f) || !std::isfinite(steps[k].dt)) return fail(FLUID_ERR_ARG, "dt must be finite and >= 0");
    uint32_t done = 0;
    while (done < count) {
        uint32_t m = count - done;
        if (m > kRing / 2) m = kRing / 2;
        int32_t rc = upload_steps(s, steps + done, m);
        if (rc != FLUID_OK) return rc;
        for (uint32_t k = 0; k < m; ++k) {
            cudaGraphExec_t g;
            if (steps[done + k].dt == 0.0f) {
                if (!s->density_graph) {
                    rc = capture(s, 0, 0, true, &s->density_graph);
                    if (rc != FLUID_OK) return rc;
                }
                g = s->density_graph;
            } else {
                rc = substep_graph(s, s->cfg.den_iters, &g);
                if (rc != FLUID_OK) return rc;
            }
            CK(cudaGraphLaunch(g, s->stream));
        }
        done += m;
    }
    return FLUID_OK;
}

int32_t fluid_sim_step(FluidSim *s, const FluidStep *step) { return fluid_sim_run(s, step, 1); }

int32_t fluid_sim_reduce_stats(FluidSim *s) {
    if (!s) return fail(FLUID_ERR_ARG, "null handle");
    CK(cudaSetDevice(s->device));
    launch_stats(s->stream, s->geo(), s->b, s->stats_chunks());
    CK(cudaGetLastError());
    return FLUID_OK;
}

int32_t fluid_sim_tracers(FluidSim *s, const FluidStep *step) {
    if (!s || !step) return fail(FLUID_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    if (!s->ntr) return FLUID_OK;
    DevStep d;
    fill_step(s, *step, d);
    launch_splat(s->stream, s->P, s->b);
    launch_resolve(s->stream, s->P, s->b);
    launch_advect(s->stream, s->P, s->b, d, s->ntr);
    CK(cudaGetLastError());
    return FLUID_OK;
}

int32_t fluid_sim_advect(FluidSim *s, const FluidStep *step) {
    if (!s || !step) return fail(FLUID_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    DevStep d;
    fill_step(s, *step, d);
    launch_advect(s->stream, s->P, s->b, d, s->ntr);
    CK(cudaGetLastError());
    return FLUID_OK;
}

int32_t fluid_sim_sync(FluidSim *s) {
    if (!s) return fail(FLUID_ERR_ARG, "null handle");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    uint32_t err = 0;
    CK(cudaMemcpy(&err, &s->solve->error, 4, cudaMemcpyDeviceToHost));
    if (err) return fail(FLUID_ERR_TIMEOUT, "a bounded device wait gave up (error flags " + std::to_string(err) + ")");
    return FLUID_OK;
}

int32_t fluid_sim_stats(FluidSim *s, FluidSimStats *out) {
    if (!s || !out) return fail(FLUID_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    float st[16];
    DevSolve sv;
    CK(cudaMemcpy(st, s->b.stats, sizeof st, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&sv, s->solve, kSolveHeadBytes, cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof *out);
    out->compression_avg = st[0];
    out->compression_max = st[1];
    out->density_min = st[2];
    out->density_max = st[3];
    out->pressure_min = st[4];
    out->pressure_max = st[5];
    out->v_max = st[6];
    out->temperature_min = st[7];
    out->temperature_max = st[8];
    out->clamp_count = sv.clamp_count;
    out->neighbour_overflow = sv.nbr_over;
    out->v_min = st[11];
    out->accel_min = st[12];
    out->accel_max = st[13];
    out->div_iters = sv.div_iters;
    out->den_iters = sv.den_iters;
    out->div_residual = sv.div_res;
    out->den_residual = sv.den_res;
    out->substeps = sv.substeps;
    out->total_div_iters = sv.total_div_iters;
    out->total_den_iters = sv.total_den_iters;
    out->substeps_last_frame = s->last_frame_substeps;
    out->error = sv.error ? FLUID_ERR_TIMEOUT : FLUID_OK;
    bool finite = true;
    for (int k = 0; k < 14; ++k) finite = finite && std::isfinite(st[k]);
    if (!finite) out->error = FLUID_ERR_NAN;
    return out->error;
}

int32_t fluid_sim_get_state(FluidSim *s, float *pos4, float *vel4, float *prev_vel4, float *prev_p,
                            float *temp, uint32_t *id) {
    if (!s) return fail(FLUID_ERR_ARG, "null handle");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    const size_t n = s->n;
    if (pos4) CK(cudaMemcpy(pos4, s->b.pos, 16 * n, cudaMemcpyDeviceToHost));
    if (vel4) CK(cudaMemcpy(vel4, s->b.vel, 16 * n, cudaMemcpyDeviceToHost));
    if (prev_vel4) CK(cudaMemcpy(prev_vel4, s->b.pvel, 16 * n, cudaMemcpyDeviceToHost));
    if (prev_p) CK(cudaMemcpy(prev_p, s->b.pp, 4 * n, cudaMemcpyDeviceToHost));
    if (temp) CK(cudaMemcpy(temp, s->b.temp, 4 * n, cudaMemcpyDeviceToHost));
    if (id) CK(cudaMemcpy(id, s->b.id, 4 * n, cudaMemcpyDeviceToHost));
    return FLUID_OK;
}

int32_t fluid_sim_set_state(FluidSim *s, const float *pos4, const float *vel4, const float *prev_vel4,
                            const float *prev_p, const float *temp, const uint32_t *id) {
    if (!s) return fail(FLUID_ERR_ARG, "null handle");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    const size_t n = s->n;
    if (pos4) CK(cudaMemcpy(s->b.pos, pos4, 16 * n, cudaMemcpyHostToDevice));
    if (vel4) CK(cudaMemcpy(s->b.vel, vel4, 16 * n, cudaMemcpyHostToDevice));
    if (prev_vel4) CK(cudaMemcpy(s->b.pvel, prev_vel4, 16 * n, cudaMemcpyHostToDevice));
    if (prev_p) CK(cudaMemcpy(s->b.pp, prev_p, 4 * n, cudaMemcpyHostToDevice));
    if (temp) CK(cudaMemcpy(s->b.temp, temp, 4 * n, cudaMemcpyHostToDevice));
    if (id) {
        std::vector<uint8_t> seen(n, 0);
        for (size_t i = 0; i < n; ++i) {
            if (id[i] >= n || seen[id[i]]) return fail(FLUID_ERR_ARG, "ids must be a permutation of 0..n-1");
            seen[id[i]] = 1;
        }
        CK(cudaMemcpy(s->b.id, id, 4 * n, cudaMemcpyHostToDevice));
    }
    return FLUID_OK;
}

int32_t fluid_sim_read_particles(FluidSim *s, float *pos4, float *vel4) {
    if (!s) return fail(FLUID_ERR_ARG, "null handle");
    const size_t n = s->n;
    std::vector<float> p(4 * n), v(4 * n);
    std::vector<uint32_t> id(n);
    int32_t rc = fluid_sim_get_state(s, p.data(), v.data(), nullptr, nullptr, nullptr, id.data());
    if (rc != FLUID_OK) return rc;
    for (size_t k = 0; k < n; ++k) {
        const uint32_t i = id[k];
        if (pos4) std::memcpy(pos4 + 4 * (size_t)i, &p[4 * k], 16);
        if (vel4) std::memcpy(vel4 + 4 * (size_t)i, &v[4 * k], 16);
    }
    return FLUID_OK;
}

int32_t fluid_sim_get_tracers(FluidSim *s, uint32_t *packed2) {
    if (!s || !packed2) return fail(FLUID_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    if (s->ntr) CK(cudaMemcpy(packed2, s->b.tracers, 8ull * s->ntr, cudaMemcpyDeviceToHost));
    return FLUID_OK;
}

int32_t fluid_sim_set_tracers(FluidSim *s, const uint32_t *packed2) {
    if (!s || !packed2) return fail(FLUID_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    if (s->ntr) CK(cudaMemcpy(s->b.tracers, packed2, 8ull * s->ntr, cudaMemcpyHostToDevice));
    return FLUID_OK;
}

// sim_sprites.wgsl body + weight and the field pass of render.rs:3233-3282:
// the decay draw (field *= keep) and one splat of every particle at blend
// constant 1 - keep, into the handle's float2 field.
int32_t fluid_sim_field_splat(FluidSim *s, const FluidFieldParams *p) {
    if (!s || !p) return fail(FLUID_ERR_ARG, "null argument");
    if (p->width == 0 || p->height == 0 || (uint64_t)p->width * p->height > (1ull << 26))
        return fail(FLUID_ERR_ARG, "field size must be 1..2^26 texels");
    if (!(p->keep >= 0.0f && p->keep <= 1.0f)) return fail(FLUID_ERR_ARG, "keep must be in [0, 1]");
    if (p->lens > 4u) return fail(FLUID_ERR_ARG, "lens codes are 0..4");
    if (p->lens && !(p->hi != p->lo)) return fail(FLUID_ERR_ARG, "the lens ramp needs hi != lo");
    CK(cudaSetDevice(s->device));
    const size_t texels = (size_t)p->width * p->height;
    if (!s->field || s->fgeom.w != p->width || s->fgeom.h != p->height) {
        CK(cudaStreamSynchronize(s->stream));
        if (s->field) cudaFree(s->field);
        if (s->field_filtered) cudaFree(s->field_filtered);
        if (s->field_acc) cudaFree(s->field_acc);
        s->field = nullptr;
        s->field_filtered = nullptr;
        s->field_acc = nullptr;
        CK(cudaMalloc(&s->field, texels * sizeof(float2)));
        CK(cudaMalloc(&s->field_filtered, texels * sizeof(float4)));
        CK(cudaMalloc(&s->field_acc, texels * 2 * sizeof(unsigned long long)));
        CK(cudaMemsetAsync(s->field, 0, texels * sizeof(float2), s->stream));
        CK(cudaMemsetAsync(s->field_filtered, 0, texels * sizeof(float4), s->stream));
        CK(cudaMemsetAsync(s->field_acc, 0, texels * 2 * sizeof(unsigned long long), s->stream));
    }
    FieldGeom &g = s->fgeom;
    g.cx = s->P.tracer_c[0];  // the slab's extent -(box_min + cell), or the box's centre and half size
    g.cy = s->P.tracer_c[1];
    g.ex = s->P.tracer_e[0];
    g.ey = s->P.tracer_e[1];
    g.radius = s->P.h * 1.5f;  // SPLAT_RADIUS, sim_sprites.wgsl
    g.w = p->width;
    g.h = p->height;
    g.lens = p->lens;
    g.lo = p->lo;
    g.hi = p->hi;
    launch_field_splat(s->stream, g, s->b.pos, s->b.vel, s->b.pvel, s->b.density, s->n, p->keep, 1.0f - p->keep,
                       s->field, s->field_acc);
    CK(cudaGetLastError());
    return FLUID_OK;
}

// sim_surface.wgsl field_filter over the current field.
int32_t fluid_sim_field_filter(FluidSim *s) {
    if (!s) return fail(FLUID_ERR_ARG, "null handle");
    if (!s->field) return fail(FLUID_ERR_STATE, "no field yet: splat first");
    CK(cudaSetDevice(s->device));
    launch_field_filter(s->stream, s->fgeom, s->field, s->field_filtered);
    CK(cudaGetLastError());
    return FLUID_OK;
}

int32_t fluid_sim_field_read(FluidSim *s, float *field2, float *filtered4) {
    if (!s) return fail(FLUID_ERR_ARG, "null handle");
    if (!s->field) return fail(FLUID_ERR_STATE, "no field yet: splat first");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    const size_t texels = (size_t)s->fgeom.w * s->fgeom.h;
    if (field2) CK(cudaMemcpy(field2, s->field, texels * sizeof(float2), cudaMemcpyDeviceToHost));
    if (filtered4) CK(cudaMemcpy(filtered4, s->field_filtered, texels * sizeof(float4), cudaMemcpyDeviceToHost));
    return FLUID_OK;
}

int32_t fluid_sim_read_field(FluidSim *s, int32_t field, void *out, uint64_t bytes) {
    if (!s || !out) return fail(FLUID_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    const uint64_t n = s->n;
    const void *src = nullptr;
    uint64_t need = 0;
    switch (field) {
    case FLUID_FIELD_DENSITY: src = s->b.density; need = 4 * n; break;
    case FLUID_FIELD_ALPHA: src = s->b.alpha; need = 4 * n; break;
    case FLUID_FIELD_KD: src = s->b.kd; need = 4 * n; break;
    case FLUID_FIELD_PRESSURE: src = s->b.pressure; need = 4 * n; break;
    case FLUID_FIELD_NBR_N: src = s->b.nbr_n; need = 4 * n; break;
    case FLUID_FIELD_STARTS: src = s->b.starts; need = 4ull * (s->keyspace + 1); break;
    case FLUID_FIELD_PERM: src = s->b.perm; need = 4 * n; break;
    case FLUID_FIELD_WORK_POS: src = s->b.wpos; need = 16 * n; break;
    case FLUID_FIELD_WORK_VEL: src = s->b.wvel; need = 16 * n; break;
    case FLUID_FIELD_ACCEL: src = s->b.accel; need = 16 * n; break;
    case FLUID_FIELD_XSPH: src = s->b.xsph; need = 16 * n; break;
    case FLUID_FIELD_WALL_GRAD: src = s->b.wgrad; need = 16 * n; break;
    case FLUID_FIELD_COUNTERS: {
        if (bytes < 8) return fail(FLUID_ERR_ARG, "buffer too small");
        DevSolve sv;
        CK(cudaMemcpy(&sv, s->solve, kSolveHeadBytes, cudaMemcpyDeviceToHost));
        ((uint32_t *)out)[0] = sv.clamp_count;
        ((uint32_t *)out)[1] = sv.nbr_over;
        return FLUID_OK;
    }
    default: return fail(FLUID_ERR_ARG, "unknown field");
    }
    if (bytes < need) return fail(FLUID_ERR_ARG, "buffer too small");
    CK(cudaMemcpy(out, src, need, cudaMemcpyDeviceToHost));
    if (field == FLUID_FIELD_WORK_POS) {
        // The reference keeps rho_near in the working position's w
        // (sim_solve.wgsl:502-507); this build keeps it in its own array.
        std::vector<float> rn(n);
        CK(cudaMemcpy(rn.data(), s->b.rho_near, 4 * n, cudaMemcpyDeviceToHost));
        float *o = (float *)out;
        for (uint64_t i = 0; i < n; ++i) o[4 * i + 3] = rn[i];
    }
    return FLUID_OK;
}

uint32_t fluid_sim_grid_slabs(void) { return kSimSlabs; }

uint32_t fluid_sim_kernels_per_substep(const FluidSim *s) {
    if (!s) return 0;
    const uint32_t passes = (uint32_t)radix_passes(s->keyspace);
    // keys + one per radix pass + starts scan + gather + density_div
    //   + div applies (+ div_kappa after the first) + forces pair
    //   + den pairs + integrate
    const uint32_t d = s->cfg.div_iters, k = s->cfg.den_iters;
    return 2 + passes + 1 + 1 + (d ? 2 * d - 1 : 0) + 2 + 2 * k + 1;
}

int32_t fluid_sim_profile_step(FluidSim *s, const FluidStep *step, float *ms, const char **names,
                               uint32_t cap) {
    if (!s || !step || !ms) return fail(FLUID_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    int32_t rc = upload_steps(s, step, 1);
    if (rc != FLUID_OK) return rc;
    std::vector<cudaEvent_t> ev;
    std::vector<const char *> nm;
    cudaEvent_t e0;
    CK(cudaEventCreate(&e0));
    CK(cudaEventRecord(e0, s->stream));
    ev.push_back(e0);
    cudaError_t err = cudaSuccess;
    auto mark = [&](const char *name) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        cudaEventRecord(e, s->stream);
        ev.push_back(e);
        nm.push_back(name);
    };
    if (step->dt == 0.0f) err = enqueue_substep(s, s->stream, 0, 0, true, mark);
    else err = enqueue_substep(s, s->stream, s->cfg.div_iters, s->cfg.den_iters, false, mark);
    CK(err);
    CK(cudaStreamSynchronize(s->stream));
    uint32_t k = 0;
    for (; k + 1 < ev.size() && k < cap; ++k) {
        cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]);
        if (names) names[k] = nm[k];
    }
    for (auto e : ev) cudaEventDestroy(e);
    return (int32_t)k;
}

int32_t fluid_sim_frame(FluidSim *s, FluidVec3 force, FluidVec3 omega, FluidVec3 domega, float dt,
                        uint32_t substeps, uint32_t cap, uint32_t seed) {
    if (!s) return fail(FLUID_ERR_ARG, "null handle");
    if (!std::isfinite(dt) || dt < 0.0f) return fail(FLUID_ERR_ARG, "dt must be finite and >= 0");
    CK(cudaSetDevice(s->device));
    // The one-frame-stale v_max (render.rs:3090-3094): take last frame's
    // stats if their copy has landed, never wait for them.
    if (s->stats_pending && cudaEventQuery(s->stats_ready) == cudaSuccess) {
        s->v_max_stale = s->h_stats_stale[6];
        s->stats_pending = false;
    }
    // A dt of zero encodes nothing (render.rs:3165-3168).
    if (dt == 0.0f) {
        s->last_frame_substeps = 0;
        return FLUID_OK;
    }
    uint32_t n = substeps ? substeps
                          : fluid_substeps_for(dt, s->v_max_stale, s->cfg.spacing, cap ? cap : 16u);
    if (n == 0) n = 1;
    const float dt_sub = dt / (float)n;
    FluidStep st;
    std::memset(&st, 0, sizeof st);
    st.force[0] = force.x;
    st.force[1] = force.y;
    st.force[2] = force.z;
    st.dt = dt_sub;
    st.omega[0] = omega.x;
    st.omega[1] = omega.y;
    st.omega[2] = omega.z;
    st.v_clamp = 0.4f * s->cfg.spacing / dt_sub;  // render.rs:3171
    st.domega[0] = domega.x;
    st.domega[1] = domega.y;
    st.domega[2] = domega.z;
    return run_frame(s, st, n, fluid_refine_passes(dt_sub), dt, seed);
}

int32_t fluid_sim_frame_plan(FluidSim *s, const FluidFramePlan *plan) {
    if (!s || !plan) return fail(FLUID_ERR_ARG, "null argument");
    CK(cudaSetDevice(s->device));
    if (s->stats_pending && cudaEventQuery(s->stats_ready) == cudaSuccess) {
        s->v_max_stale = s->h_stats_stale[6];
        s->stats_pending = false;
    }
    if (plan->asleep || plan->dt == 0.0f || plan->substeps == 0) {
        s->last_frame_substeps = 0;
        return FLUID_OK;
    }
    if (!std::isfinite(plan->dt) || plan->dt < 0.0f || !(plan->step.dt > 0.0f))
        return fail(FLUID_ERR_ARG, "plan dt must be finite and positive");
    return run_frame(s, plan->step, plan->substeps, plan->refine ? plan->refine : 5u, plan->dt,
                     plan->seed);
}

uint64_t fluid_grid_workspace_bytes(uint32_t n, const FluidGrid *grid) {
    if (!grid) return 0;
    const uint64_t cells = (uint64_t)grid->dims[0] * grid->dims[1] * grid->dims[2];
    if (cells == 0 || cells >= 0xffffffffull) return 0;
    return grid_work_bytes(n, (uint32_t)cells);
}

int32_t fluid_grid_build(const float *pos4, uint32_t n, const FluidGrid *grid, uint32_t *keys,
                         uint32_t *starts, uint32_t *perm, void *workspace, uint64_t ws_bytes,
                         void *stream) {
    if (!grid || !starts || (n && (!pos4 || !perm)) || !workspace) return fail(FLUID_ERR_ARG, "null argument");
    if (!(grid->cell > 0.0f)) return fail(FLUID_ERR_ARG, "cell must be positive");
    for (int i = 0; i < 3; ++i)
        if (grid->dims[i] == 0) return fail(FLUID_ERR_ARG, "dims must be positive");
    const uint64_t cells = (uint64_t)grid->dims[0] * grid->dims[1] * grid->dims[2];
    if (cells >= 0xffffffffull) return fail(FLUID_ERR_ARG, "grid has too many cells");
    if (ws_bytes < grid_work_bytes(n, (uint32_t)cells)) return fail(FLUID_ERR_ARG, "workspace too small");
    if ((uintptr_t)workspace & 255u) return fail(FLUID_ERR_ARG, "workspace must be 256-byte aligned");
    if (((uintptr_t)pos4 & 15u)) return fail(FLUID_ERR_ARG, "positions must be 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    GridWork w = grid_work_carve(workspace, n, (uint32_t)cells, nullptr);
    CK(cudaMemsetAsync(w.err, 0, 4, st));
    // Without a caller buffer the keys live in k2: pass 0 reads them and
    // writes k1, and k2 is next written by pass 1, after they are consumed.
    uint32_t *k = keys ? keys : w.k2;
    GridGeom g;
    for (int i = 0; i < 3; ++i) {
        g.min[i] = grid->min[i];
        g.dims[i] = grid->dims[i];
    }
    g.cell = grid->cell;
    CK(grid_build_enqueue(st, (const float4 *)pos4, n, g, k, starts, perm, w, nullptr, nullptr, nullptr,
                          kRing));
    return FLUID_OK;
}

int32_t fluid_grid_build_host(const float *pos4, uint32_t n, const FluidGrid *grid, uint32_t *starts,
                              uint32_t *perm) {
    if (!grid || !starts || (n && (!pos4 || !perm))) return fail(FLUID_ERR_ARG, "null argument");
    const uint64_t cells = (uint64_t)grid->dims[0] * grid->dims[1] * grid->dims[2];
    const uint64_t wsb = fluid_grid_workspace_bytes(n, grid);
    if (!wsb) return fail(FLUID_ERR_ARG, "bad grid");
    float *d_pos = nullptr;
    uint32_t *d_starts = nullptr, *d_perm = nullptr, *d_keys = nullptr;
    void *d_ws = nullptr;
    int32_t rc = FLUID_OK;
    cudaError_t e = cudaSuccess;
    do {
        if ((e = cudaMalloc(&d_pos, 16ull * (n ? n : 1))) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_keys, 4ull * (n ? n : 1))) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_perm, 4ull * (n ? n : 1))) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_starts, 4ull * (cells + 1))) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_ws, wsb)) != cudaSuccess) break;
        if (n && (e = cudaMemcpy(d_pos, pos4, 16ull * n, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        rc = fluid_grid_build(d_pos, n, grid, d_keys, d_starts, d_perm, d_ws, wsb, nullptr);
        if (rc != FLUID_OK) break;
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) break;
        uint32_t err = 0;
        GridWork w = grid_work_carve(d_ws, n, (uint32_t)cells, nullptr);
        if ((e = cudaMemcpy(&err, w.err, 4, cudaMemcpyDeviceToHost)) != cudaSuccess) break;
        if (err) {
            rc = fail(FLUID_ERR_TIMEOUT, "a bounded look-back wait gave up");
            break;
        }
        if ((e = cudaMemcpy(starts, d_starts, 4ull * (cells + 1), cudaMemcpyDeviceToHost)) != cudaSuccess) break;
        if (n && (e = cudaMemcpy(perm, d_perm, 4ull * n, cudaMemcpyDeviceToHost)) != cudaSuccess) break;
    } while (0);
    cudaFree(d_pos);
    cudaFree(d_keys);
    cudaFree(d_perm);
    cudaFree(d_starts);
    cudaFree(d_ws);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? FLUID_ERR_OOM : FLUID_ERR_CUDA,
                    std::string("grid_build_host: ") + cudaGetErrorString(e));
    return rc;
}

}  // extern "C"
