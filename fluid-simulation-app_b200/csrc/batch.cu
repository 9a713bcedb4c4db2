// batch.cu — FluidBatch: many independent boxes stepped by the same launches.
//
// The boxes' particles are laid end to end (box b owns slots first[b] ..
// first[b] + count[b] - 1) and their grids likewise (box b's cell keys start
// at cell_base[b]), so one grid build sorts every box at once and keeps each
// box inside its own slot range, and each sweep of a substep is ONE launch
// over all boxes' particles. A particle finds its box's constants, Step
// block, residual accumulators and loop gates through the static slot ->
// box map. A substep is one CUDA graph launch, the tolerance loops device-
// side WHILE nodes that run while any box is above its tolerance; a box
// whose loop has stopped is skipped by the loop's kernels, so every box
// takes exactly the iterations it would take alone.
//
// Every box's trajectory is bit-identical to a one-box simulation of its
// configuration: the neighbour order, every per-particle sum and every
// residual (an integer sum) are the same.
//
// The reference has no batch: it runs one Sim per renderer
// (crates/fluid-core/src/render.rs:1468-1612); this replaces running many
// of them one after another.
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "grid.cuh"
#include "solve.cuh"

namespace fcu {
int32_t report_error(int32_t code, const std::string &msg);
bool host_valid_config(const FluidSimConfig *c, std::string &why);
void host_params(const FluidSimConfig &c, uint32_t count, DevParams &P);
void host_seed(const FluidSimConfig &c, std::vector<float> &pos);
void host_step_constants(float xsph_cfg, const FluidStep &st, DevStep &d);
int32_t host_add_while(cudaStream_t st, cudaGraph_t g, cudaGraphConditionalHandle h, cudaGraph_t *body);
}  // namespace fcu

using namespace fcu;

#define BK(expr)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return report_error(e_ == cudaErrorMemoryAllocation ? FLUID_ERR_OOM : FLUID_ERR_CUDA, \
                                std::string(#expr) + ": " + cudaGetErrorString(e_));              \
    } while (0)

namespace {

constexpr uint32_t kBatchRing = 128;  // substeps of Step blocks in flight
constexpr uint32_t kMaxBoxes = 65535;

// Clears every box's residual accumulators (the substep's first launch).
__global__ void __launch_bounds__(128) k_clear_acc(DevSolve *solve) {
    DevSolve *sv = &solve[blockIdx.x];
    for (int k = threadIdx.x; k < kAccSlots; k += blockDim.x) {
        sv->acc_div[k] = 0ull;
        sv->acc_den[k] = 0ull;
    }
}

}  // namespace

struct FluidBatch {
    FluidSimConfig common{};  // the solve settings every box shares
    std::vector<FluidSimConfig> cfg;
    std::vector<DevParams> P;
    std::vector<uint32_t> first, count, cell_base;
    uint32_t nboxes = 0, n = 0, cells = 0, chunks = 1;
    uint16_t tpb[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // block size per tuned sweep (0: default)
    int device = 0;
    cudaStream_t stream = nullptr, side = nullptr;
    SimBufs b{};
    GridWork gw{};
    void *grid_ws = nullptr;
    DevParams *d_box = nullptr;
    uint16_t *d_box_of = nullptr;
    uint32_t *d_cell_base = nullptr, *d_first = nullptr;
    DevStep *ring = nullptr, *cur = nullptr, *h_ring = nullptr;
    DevSolve *solve = nullptr;
    uint64_t h_cursor = 0, synced_cursor = 0;
    std::map<std::pair<uint32_t, uint32_t>, cudaGraphExec_t> graphs;
    cudaGraphExec_t tol_graph = nullptr;
    std::vector<void *> allocs;

    Geo geo() const {
        Geo g{};
        g.one = P[0];
        g.box = d_box;
        g.box_of = d_box_of;
        g.cell_base = d_cell_base;
        g.first = d_first;
        g.solve = solve;
        g.st = cur;
        g.n = n;
        g.nboxes = nboxes;
        for (int k = 0; k < 8; ++k) g.tpb[k] = tpb[k];
        return g;
    }
    BoxKeys keys() const { return BoxKeys{d_box_of, d_box, d_cell_base, nboxes, kSimSlabs}; }

    template <class T>
    cudaError_t alloc(T **p, size_t cnt) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, cnt * sizeof(T) > 0 ? cnt * sizeof(T) : 16);
        if (e == cudaSuccess) {
            allocs.push_back(q);
            *p = (T *)q;
        }
        return e;
    }
};

namespace {

// One substep of every box at a fixed schedule (the one-box sequence).
cudaError_t batch_enqueue(FluidBatch *s, cudaStream_t st, uint32_t div_iters, uint32_t den_iters) {
    k_clear_acc<<<s->nboxes, 128, 0, st>>>(s->solve);
    const BoxKeys bk = s->keys();
    cudaError_t e = grid_build_enqueue(st, s->b.pos, s->n, GridGeom{}, s->b.keys, s->b.starts, s->b.perm,
                                       s->gw, s->ring, s->cur, s->solve, kBatchRing, &bk);
    if (e != cudaSuccess) return e;
    const Geo g = s->geo();
    launch_gather(st, s->b, s->n);
    launch_density_div(st, g, s->b, 0);
    for (uint32_t d = 0; d < div_iters; ++d) {
        if (d > 0) launch_div_kappa(st, g, s->b, (int)d, kGateNone);
        launch_apply(st, g, s->b, false, kGateNone);
    }
    launch_forces_eval(st, g, s->b);
    launch_forces_apply(st, g, s->b);
    for (uint32_t k = 0; k < den_iters; ++k) {
        launch_den_kappa(st, g, s->b, (int)k, kGateNone);
        launch_apply(st, g, s->b, true, kGateNone);
    }
    const int div_slot = div_iters > 0 ? (int)div_iters - 1 : 0;
    launch_integrate(st, g, s->b, div_slot, den_iters > 0 ? (int)den_iters - 1 : -1, (int)div_iters,
                     (int)den_iters);
    return cudaGetLastError();
}

int32_t batch_graph_fixed(FluidBatch *s, uint32_t div_iters, uint32_t den_iters, cudaGraphExec_t *out) {
    auto key = std::make_pair(div_iters, den_iters);
    auto it = s->graphs.find(key);
    if (it != s->graphs.end()) {
        *out = it->second;
        return FLUID_OK;
    }
    cudaGraph_t g = nullptr;
    BK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = batch_enqueue(s, s->stream, div_iters, den_iters);
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return report_error(FLUID_ERR_CUDA, std::string("batch capture: ") +
                                                cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return report_error(FLUID_ERR_CUDA, std::string("batch instantiate: ") + cudaGetErrorString(e));
    s->graphs[key] = *out;
    return FLUID_OK;
}

// The tolerance substep over all boxes: the divergence and density loops
// are WHILE nodes; the loop kernels skip boxes whose loop has stopped.
int32_t batch_graph_tolerance(FluidBatch *s, cudaGraphExec_t *out) {
    if (s->tol_graph) {
        *out = s->tol_graph;
        return FLUID_OK;
    }
    cudaGraph_t g = nullptr;
    BK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle hdiv, hden;
    BK(cudaGraphConditionalHandleCreate(&hdiv, g, 0, 0));
    BK(cudaGraphConditionalHandleCreate(&hden, g, 0, 0));
    const FluidSimConfig &c = s->common;
    cudaStream_t st = s->stream;
    cudaGraph_t bdiv = nullptr, bden = nullptr;
    BK(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int32_t rc = FLUID_OK;
    k_clear_acc<<<s->nboxes, 128, 0, st>>>(s->solve);
    const BoxKeys bk = s->keys();
    cudaError_t e = grid_build_enqueue(st, s->b.pos, s->n, GridGeom{}, s->b.keys, s->b.starts, s->b.perm,
                                       s->gw, s->ring, s->cur, s->solve, kBatchRing, &bk);
    const Geo geo = s->geo();
    // forces_eval after every divergence apply, forming the prediction that
    // decides the loop (as the one-box tolerance substep)
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
        rc = host_add_while(st, g, hdiv, &bdiv);
    }
    if (e == cudaSuccess && rc == FLUID_OK) {
        if (!fused) launch_forces_eval(st, geo, s->b);
        launch_forces_apply(st, geo, s->b);
        launch_den_kappa(st, geo, s->b, 0, kGateNone);
        launch_tol_finish(st, geo, 1, 1, c.den_tol, c.max_iters, hden);
        rc = host_add_while(st, g, hden, &bden);
    }
    if (e == cudaSuccess && rc == FLUID_OK) launch_integrate(st, geo, s->b, -1, -1, 0, 0);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaGraph_t g2 = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(st, &g2);
    if (rc != FLUID_OK || e != cudaSuccess || e2 != cudaSuccess) {
        cudaGraphDestroy(g);
        if (rc != FLUID_OK) return rc;
        return report_error(FLUID_ERR_CUDA, std::string("batch tolerance capture: ") +
                                                cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    // Inside the loops every slot is launched and the boxes whose loop has
    // stopped return at once (a work list of the active boxes' tiles, walked
    // by persistent blocks, measured 7 % slower a substep).
    BK(cudaStreamBeginCaptureToGraph(s->side, bdiv, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launch_apply(s->side, geo, bd, false, kGateDiv);
    if (fused) launch_forces_div(s->side, geo, s->b, 0, kGateDiv);
    else launch_div_kappa(s->side, geo, s->b, 0, kGateDiv);
    launch_tol_finish(s->side, geo, 0, 0, c.div_tol, c.max_iters, hdiv);
    BK(cudaStreamEndCapture(s->side, &bdiv));
    BK(cudaStreamBeginCaptureToGraph(s->side, bden, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    launch_apply(s->side, geo, s->b, true, kGateDen);
    launch_den_kappa(s->side, geo, s->b, 0, kGateDen);
    launch_tol_finish(s->side, geo, 1, 0, c.den_tol, c.max_iters, hden);
    BK(cudaStreamEndCapture(s->side, &bden));
    e = cudaGraphInstantiate(&s->tol_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return report_error(FLUID_ERR_CUDA, std::string("batch instantiate: ") + cudaGetErrorString(e));
    *out = s->tol_graph;
    return FLUID_OK;
}

int32_t batch_graph(FluidBatch *s, cudaGraphExec_t *out) {
    if (s->common.solve == FLUID_SOLVE_TOLERANCE) return batch_graph_tolerance(s, out);
    return batch_graph_fixed(s, s->common.div_iters, s->common.den_iters, out);
}

// Places `count` substeps of Step blocks ([count][nboxes]) in the ring.
int32_t batch_upload(FluidBatch *s, const FluidStep *steps, uint32_t count) {
    if (s->h_cursor + count - s->synced_cursor > kBatchRing) {
        BK(cudaStreamSynchronize(s->stream));
        s->synced_cursor = s->h_cursor;
    }
    const size_t nb = s->nboxes;
    uint32_t done = 0;
    while (done < count) {
        const uint32_t slot = (uint32_t)((s->h_cursor + done) % kBatchRing);
        uint32_t m = count - done;
        if (m > kBatchRing - slot) m = kBatchRing - slot;
        for (uint32_t k = 0; k < m; ++k)
            for (size_t bx = 0; bx < nb; ++bx)
                host_step_constants(s->cfg[bx].xsph_blend, steps[(done + k) * nb + bx],
                                    s->h_ring[(slot + k) * nb + bx]);
        BK(cudaMemcpyAsync(s->ring + slot * nb, s->h_ring + slot * nb, m * nb * sizeof(DevStep),
                           cudaMemcpyHostToDevice, s->stream));
        done += m;
    }
    s->h_cursor += count;
    return FLUID_OK;
}

// The solve settings every box of a batch must share.
bool same_solve(const FluidSimConfig &a, const FluidSimConfig &b) {
    return a.solve == b.solve && a.div_iters == b.div_iters && a.den_iters == b.den_iters &&
           a.div_tol == b.div_tol && a.den_tol == b.den_tol && a.max_iters == b.max_iters &&
           a.nbr_cap == b.nbr_cap && a.device == b.device;
}

int32_t batch_create_into(FluidBatch *s, const FluidSimConfig *boxes, uint32_t nboxes) {
    s->common = boxes[0];
    s->device = boxes[0].device;
    s->nboxes = nboxes;
    s->cfg.assign(boxes, boxes + nboxes);
    BK(cudaSetDevice(s->device));
    std::vector<float> pos;
    std::vector<float> temp;
    std::vector<uint32_t> ids;
    std::vector<uint16_t> box_of;
    uint64_t n64 = 0, cells64 = 0;
    s->P.resize(nboxes);
    for (uint32_t bx = 0; bx < nboxes; ++bx) {
        std::vector<float> p;
        host_seed(boxes[bx], p);
        const uint64_t cnt = p.size() / 4;
        if (cnt == 0) return report_error(FLUID_ERR_ARG, "box " + std::to_string(bx) + " has no particles");
        host_params(boxes[bx], (uint32_t)cnt, s->P[bx]);
        const uint64_t c = (uint64_t)s->P[bx].dims[0] * s->P[bx].dims[1] * s->P[bx].dims[2];
        s->first.push_back((uint32_t)n64);
        s->count.push_back((uint32_t)cnt);
        // grid keys: each box's cells * kSimSlabs keys above the earlier boxes'
        s->cell_base.push_back((uint32_t)cells64);
        n64 += cnt;
        cells64 += c * kSimSlabs;
        if (n64 > 0x0fffffffull) return report_error(FLUID_ERR_ARG, "a batch holds at most 2^28-1 particles");
        if (cells64 >= 0xffffffffull) return report_error(FLUID_ERR_ARG, "the batch's grids have too many cells");
        pos.insert(pos.end(), p.begin(), p.end());
        temp.insert(temp.end(), cnt, boxes[bx].temperature);
        for (uint64_t k = 0; k < cnt; ++k) {
            ids.push_back((uint32_t)k);
            box_of.push_back((uint16_t)bx);
        }
    }
    s->n = (uint32_t)n64;
    s->cells = (uint32_t)cells64;
    if ((uint64_t)s->n * s->common.nbr_cap > (1ull << 40)) return report_error(FLUID_ERR_ARG, "neighbour lists too large");
    // stats: about 2048 particles per block, at least one block per box
    uint32_t maxc = 0;
    for (uint32_t c : s->count) maxc = c > maxc ? c : maxc;
    s->chunks = (maxc + 2047u) / 2048u;
    if (s->chunks < 1u) s->chunks = 1u;
    if (s->chunks > (uint32_t)kStatsChunks) s->chunks = kStatsChunks;

    BK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    BK(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
    const size_t n = s->n, C = s->cells, nb = nboxes;
    SimBufs &b = s->b;
    BK(s->alloc(&b.pos, n));
    BK(s->alloc(&b.vel, n));
    BK(s->alloc(&b.pvel, n));
    BK(s->alloc(&b.pp, n));
    BK(s->alloc(&b.temp, n));
    BK(s->alloc(&b.id, n));
    BK(s->alloc(&b.wpos, n));
    BK(s->alloc(&b.wvel, n));
    BK(s->alloc(&b.wpvel, n));
    BK(s->alloc(&b.wpp, n));
    BK(s->alloc(&b.wtemp, n));
    BK(s->alloc(&b.wid, n));
    BK(s->alloc(&b.keys, n));
    BK(s->alloc(&b.starts, C + 1));
    BK(s->alloc(&b.perm, n));
    BK(s->alloc(&b.density, n));
    BK(s->alloc(&b.alpha, n));
    BK(s->alloc(&b.kd, n));
    BK(s->alloc(&b.wpk, n));
    BK(s->alloc(&b.kd2, n));
    BK(s->alloc(&b.wpk2, n));
    BK(s->alloc(&b.pressure, n));
    BK(s->alloc(&b.pinc, n));
    BK(s->alloc(&b.rho_near, n));
    BK(s->alloc(&b.accel, n));
    BK(s->alloc(&b.xsph, n));
    BK(s->alloc(&b.wgrad, n));
    BK(s->alloc(&b.nbr, n * s->common.nbr_cap));
    BK(s->alloc(&b.nbr_n, n));
    BK(s->alloc(&b.stats_part, nb * s->chunks * 12));
    BK(s->alloc(&b.stats_acc, nb));
    BK(s->alloc(&b.stats, nb * 16));
    BK(s->alloc(&s->d_box, nb));
    BK(s->alloc(&s->d_box_of, n));
    BK(s->alloc(&s->d_cell_base, nb));
    BK(s->alloc(&s->d_first, nb));
    BK(s->alloc(&s->ring, (size_t)kBatchRing * nb));
    BK(s->alloc(&s->cur, nb));
    BK(s->alloc(&s->solve, nb));

    const size_t wsb = grid_work_bytes(s->n, s->cells);
    BK(cudaMalloc(&s->grid_ws, wsb));
    s->gw = grid_work_carve(s->grid_ws, s->n, s->cells, &s->solve[0].error);
    BK(cudaMallocHost(&s->h_ring, (size_t)kBatchRing * nb * sizeof(DevStep)));

    std::vector<float> zeros4(4 * n, 0.0f), zeros(n, 0.0f);
    BK(cudaMemcpy(b.pos, pos.data(), 16 * n, cudaMemcpyHostToDevice));
    BK(cudaMemcpy(b.vel, zeros4.data(), 16 * n, cudaMemcpyHostToDevice));
    BK(cudaMemcpy(b.pvel, zeros4.data(), 16 * n, cudaMemcpyHostToDevice));
    BK(cudaMemcpy(b.pp, zeros.data(), 4 * n, cudaMemcpyHostToDevice));
    BK(cudaMemcpy(b.temp, temp.data(), 4 * n, cudaMemcpyHostToDevice));
    BK(cudaMemcpy(b.id, ids.data(), 4 * n, cudaMemcpyHostToDevice));
    for (float *z : {b.density, b.alpha, b.kd, b.pressure, b.pinc, b.rho_near}) BK(cudaMemset(z, 0, 4 * n));
    BK(cudaMemset(b.nbr_n, 0, 4 * n));
    BK(cudaMemset(b.stats_acc, 0, 8 * nb));
    BK(cudaMemset(b.stats, 0, 64 * nb));
    BK(cudaMemcpy(s->d_box, s->P.data(), nb * sizeof(DevParams), cudaMemcpyHostToDevice));
    BK(cudaMemcpy(s->d_box_of, box_of.data(), 2 * n, cudaMemcpyHostToDevice));
    BK(cudaMemcpy(s->d_cell_base, s->cell_base.data(), 4 * nb, cudaMemcpyHostToDevice));
    BK(cudaMemcpy(s->d_first, s->first.data(), 4 * nb, cudaMemcpyHostToDevice));
    BK(cudaMemset(s->solve, 0, nb * sizeof(DevSolve)));
    BK(cudaDeviceSynchronize());
    cudaGraphExec_t g;
    return batch_graph(s, &g);
}

}  // namespace

extern "C" {

void fluid_batch_destroy(FluidBatch *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
    if (s->tol_graph) cudaGraphExecDestroy(s->tol_graph);
    for (void *p : s->allocs) cudaFree(p);
    if (s->grid_ws) cudaFree(s->grid_ws);
    if (s->h_ring) cudaFreeHost(s->h_ring);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

FluidBatch *fluid_batch_create(const FluidSimConfig *boxes, uint32_t nboxes) {
    if (!boxes || nboxes == 0 || nboxes > kMaxBoxes) {
        report_error(FLUID_ERR_ARG, "a batch needs 1..65535 box configurations");
        return nullptr;
    }
    for (uint32_t bx = 0; bx < nboxes; ++bx) {
        std::string why;
        if (!host_valid_config(&boxes[bx], why)) {
            report_error(FLUID_ERR_ARG, "box " + std::to_string(bx) + ": " + why);
            return nullptr;
        }
        if (boxes[bx].tracers) {
            report_error(FLUID_ERR_ARG, "box " + std::to_string(bx) + ": a batch carries no tracers");
            return nullptr;
        }
        if (!same_solve(boxes[bx], boxes[0])) {
            report_error(FLUID_ERR_ARG, "box " + std::to_string(bx) +
                                            ": solve settings, nbr_cap and device must match box 0");
            return nullptr;
        }
    }
    FluidBatch *s = new FluidBatch();
    if (batch_create_into(s, boxes, nboxes) != FLUID_OK) {
        std::string keep = fluid_last_error();
        fluid_batch_destroy(s);
        report_error(FLUID_ERR_ARG, keep);
        return nullptr;
    }
    return s;
}

uint32_t fluid_batch_boxes(const FluidBatch *s) { return s ? s->nboxes : 0u; }
uint32_t fluid_batch_count(const FluidBatch *s, uint32_t box) {
    return (s && box < s->nboxes) ? s->count[box] : 0u;
}
uint32_t fluid_batch_total(const FluidBatch *s) { return s ? s->n : 0u; }
void *fluid_batch_stream(FluidBatch *s) { return s ? (void *)s->stream : nullptr; }

int32_t fluid_batch_params(const FluidBatch *s, uint32_t box, FluidSimParams *out) {
    if (!s || !out || box >= s->nboxes) return report_error(FLUID_ERR_ARG, "bad batch, box or output");
    std::memcpy(out, &s->P[box], sizeof *out);
    return FLUID_OK;
}

int32_t fluid_batch_run(FluidBatch *s, const FluidStep *steps, uint32_t count) {
    if (!s || (!steps && count)) return report_error(FLUID_ERR_ARG, "null argument");
    BK(cudaSetDevice(s->device));
    const size_t nb = s->nboxes;
    for (size_t k = 0; k < (size_t)count * nb; ++k)
        if (!(steps[k].dt > 0.0f) || !std::isfinite(steps[k].dt))
            return report_error(FLUID_ERR_ARG, "batch steps need a finite dt > 0");
    cudaGraphExec_t g;
    int32_t rc = batch_graph(s, &g);
    if (rc != FLUID_OK) return rc;
    uint32_t done = 0;
    while (done < count) {
        uint32_t m = count - done;
        if (m > kBatchRing / 2) m = kBatchRing / 2;
        rc = batch_upload(s, steps + (size_t)done * nb, m);
        if (rc != FLUID_OK) return rc;
        for (uint32_t k = 0; k < m; ++k) BK(cudaGraphLaunch(g, s->stream));
        done += m;
    }
    return FLUID_OK;
}

int32_t fluid_batch_step(FluidBatch *s, const FluidStep *steps) { return fluid_batch_run(s, steps, 1); }

int32_t fluid_batch_reduce_stats(FluidBatch *s) {
    if (!s) return report_error(FLUID_ERR_ARG, "null handle");
    BK(cudaSetDevice(s->device));
    launch_stats(s->stream, s->geo(), s->b, s->chunks);
    BK(cudaGetLastError());
    return FLUID_OK;
}

int32_t fluid_batch_sync(FluidBatch *s) {
    if (!s) return report_error(FLUID_ERR_ARG, "null handle");
    BK(cudaSetDevice(s->device));
    BK(cudaStreamSynchronize(s->stream));
    uint32_t err = 0;
    BK(cudaMemcpy(&err, &s->solve[0].error, 4, cudaMemcpyDeviceToHost));
    if (err) return report_error(FLUID_ERR_TIMEOUT, "a bounded device wait gave up (error flags " + std::to_string(err) + ")");
    return FLUID_OK;
}

int32_t fluid_batch_stats(FluidBatch *s, FluidSimStats *out) {
    if (!s || !out) return report_error(FLUID_ERR_ARG, "null argument");
    BK(cudaSetDevice(s->device));
    BK(cudaStreamSynchronize(s->stream));
    const size_t nb = s->nboxes;
    std::vector<float> st(16 * nb);
    std::vector<DevSolve> sv(nb);
    BK(cudaMemcpy(st.data(), s->b.stats, 64 * nb, cudaMemcpyDeviceToHost));
    BK(cudaMemcpy2D(sv.data(), sizeof(DevSolve), s->solve, sizeof(DevSolve), kSolveHeadBytes, nb,
                    cudaMemcpyDeviceToHost));
    int32_t worst = FLUID_OK;
    const uint32_t err0 = sv[0].error;
    for (size_t bx = 0; bx < nb; ++bx) {
        const float *q = &st[16 * bx];
        FluidSimStats &o = out[bx];
        std::memset(&o, 0, sizeof o);
        o.compression_avg = q[0];
        o.compression_max = q[1];
        o.density_min = q[2];
        o.density_max = q[3];
        o.pressure_min = q[4];
        o.pressure_max = q[5];
        o.v_max = q[6];
        o.temperature_min = q[7];
        o.temperature_max = q[8];
        o.clamp_count = sv[bx].clamp_count;
        o.neighbour_overflow = sv[bx].nbr_over;
        o.v_min = q[11];
        o.accel_min = q[12];
        o.accel_max = q[13];
        o.div_iters = sv[bx].div_iters;
        o.den_iters = sv[bx].den_iters;
        o.div_residual = sv[bx].div_res;
        o.den_residual = sv[bx].den_res;
        o.substeps = sv[bx].substeps;
        o.total_div_iters = sv[bx].total_div_iters;
        o.total_den_iters = sv[bx].total_den_iters;
        o.error = err0 ? FLUID_ERR_TIMEOUT : FLUID_OK;
        bool finite = true;
        for (int k = 0; k < 14; ++k) finite = finite && std::isfinite(q[k]);
        if (!finite) o.error = FLUID_ERR_NAN;
        if (o.error != FLUID_OK) worst = o.error;
    }
    return worst;
}

int32_t fluid_batch_get_state(FluidBatch *s, uint32_t box, float *pos4, float *vel4, float *prev_vel4,
                              float *prev_p, float *temp, uint32_t *id) {
    if (!s || box >= s->nboxes) return report_error(FLUID_ERR_ARG, "bad batch or box");
    BK(cudaSetDevice(s->device));
    BK(cudaStreamSynchronize(s->stream));
    const size_t f = s->first[box], n = s->count[box];
    if (pos4) BK(cudaMemcpy(pos4, s->b.pos + f, 16 * n, cudaMemcpyDeviceToHost));
    if (vel4) BK(cudaMemcpy(vel4, s->b.vel + f, 16 * n, cudaMemcpyDeviceToHost));
    if (prev_vel4) BK(cudaMemcpy(prev_vel4, s->b.pvel + f, 16 * n, cudaMemcpyDeviceToHost));
    if (prev_p) BK(cudaMemcpy(prev_p, s->b.pp + f, 4 * n, cudaMemcpyDeviceToHost));
    if (temp) BK(cudaMemcpy(temp, s->b.temp + f, 4 * n, cudaMemcpyDeviceToHost));
    if (id) BK(cudaMemcpy(id, s->b.id + f, 4 * n, cudaMemcpyDeviceToHost));
    return FLUID_OK;
}

}  // extern "C"

namespace {

// The captured substeps launch with the block sizes of their capture: drop
// them so the next run captures with the current table.
void drop_graphs(FluidBatch *s) {
    cudaStreamSynchronize(s->stream);
    for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
    if (s->tol_graph) cudaGraphExecDestroy(s->tol_graph);
    s->tol_graph = nullptr;
}

// One substep of every box as direct launches at a fixed schedule (one
// divergence apply, two density pairs) with every tuned sweep at `tpb`,
// each sweep's launches timed with events: ms[slot] accumulates.
int32_t timed_substep(FluidBatch *s, int tpb, float *ms, cudaEvent_t *ev) {
    cudaStream_t st = s->stream;
    Geo g = s->geo();
    for (int k = 0; k < kTuneCount; ++k) g.tpb[k] = (uint16_t)tpb;
    k_clear_acc<<<s->nboxes, 128, 0, st>>>(s->solve);
    const BoxKeys bk = s->keys();
    BK(grid_build_enqueue(st, s->b.pos, s->n, GridGeom{}, s->b.keys, s->b.starts, s->b.perm, s->gw,
                          nullptr, nullptr, s->solve, kBatchRing, &bk));
    launch_gather(st, s->b, s->n);
    int e = 0;
    auto timed = [&](int slot, auto &&launch) {
        cudaEventRecord(ev[e], st);
        launch();
        cudaEventRecord(ev[e + 1], st);
        cudaEventSynchronize(ev[e + 1]);
        float t = 0.0f;
        cudaEventElapsedTime(&t, ev[e], ev[e + 1]);
        ms[slot] += t;
    };
    timed(kTuneDensity, [&] { launch_density_div(st, g, s->b, 0); });
    timed(kTuneApply, [&] { launch_apply(st, g, s->b, false, kGateNone); });
    timed(kTuneDivKappa, [&] { launch_div_kappa(st, g, s->b, 1, kGateNone); });
    timed(kTuneForcesEval, [&] { launch_forces_eval(st, g, s->b); });
    timed(kTuneForcesApply, [&] { launch_forces_apply(st, g, s->b); });
    for (int k = 0; k < 2; ++k) {
        timed(kTuneDenKappa, [&] { launch_den_kappa(st, g, s->b, k, kGateNone); });
        timed(kTuneApply, [&] { launch_apply(st, g, s->b, true, kGateNone); });
    }
    timed(kTuneIntegrate, [&] { launch_integrate(st, g, s->b, 0, 1, 1, 2); });
    BK(cudaGetLastError());
    return FLUID_OK;
}

}  // namespace

extern "C" {

int32_t fluid_batch_set_blocks(FluidBatch *s, const uint32_t *tpb) {
    if (!s || !tpb) return report_error(FLUID_ERR_ARG, "null argument");
    for (int k = 0; k < kTuneCount; ++k)
        if (tpb[k] != 0 && tpb[k] != 64 && tpb[k] != 128 && tpb[k] != 256)
            return report_error(FLUID_ERR_ARG, "block sizes are 64, 128 or 256 (0: default)");
    BK(cudaSetDevice(s->device));
    drop_graphs(s);
    for (int k = 0; k < kTuneCount; ++k) s->tpb[k] = (uint16_t)tpb[k];
    return FLUID_OK;
}

int32_t fluid_batch_get_blocks(const FluidBatch *s, uint32_t *tpb) {
    if (!s || !tpb) return report_error(FLUID_ERR_ARG, "null argument");
    for (int k = 0; k < kTuneCount; ++k) tpb[k] = s->tpb[k];
    return FLUID_OK;
}

int32_t fluid_batch_autotune(FluidBatch *s, const FluidStep *steps, uint32_t *chosen, float *ms_out) {
    if (!s || !steps) return report_error(FLUID_ERR_ARG, "null argument");
    const size_t nb = s->nboxes, n = s->n;
    for (size_t k = 0; k < nb; ++k)
        if (!(steps[k].dt > 0.0f) || !std::isfinite(steps[k].dt))
            return report_error(FLUID_ERR_ARG, "batch steps need a finite dt > 0");
    BK(cudaSetDevice(s->device));
    BK(cudaStreamSynchronize(s->stream));
    // the Step blocks of the timed substeps go straight to the current slots
    std::vector<DevStep> d(nb);
    for (size_t k = 0; k < nb; ++k) host_step_constants(s->cfg[k].xsph_blend, steps[k], d[k]);
    // snapshot of everything a substep changes that outlives it
    std::vector<void *> tmp;
    auto save = [&](const void *src, size_t bytes) -> void * {
        void *q = nullptr;
        if (cudaMalloc(&q, bytes) != cudaSuccess) return nullptr;
        tmp.push_back(q);
        cudaMemcpyAsync(q, src, bytes, cudaMemcpyDeviceToDevice, s->stream);
        return q;
    };
    struct Saved {
        void *dst;
        const void *src;
        size_t bytes;
    };
    std::vector<Saved> saved = {{s->b.pos, nullptr, 16 * n}, {s->b.vel, nullptr, 16 * n},
                                {s->b.pvel, nullptr, 16 * n}, {s->b.pp, nullptr, 4 * n},
                                {s->b.temp, nullptr, 4 * n},  {s->b.id, nullptr, 4 * n},
                                {s->solve, nullptr, nb * sizeof(DevSolve)}, {s->cur, nullptr, nb * sizeof(DevStep)}};
    int32_t rc = FLUID_OK;
    for (auto &v : saved) {
        v.src = save(v.dst, v.bytes);
        if (!v.src) rc = report_error(FLUID_ERR_OOM, "autotune: no room for the state snapshot");
    }
    auto restore = [&] {
        for (auto &v : saved)
            if (v.src) cudaMemcpyAsync(v.dst, v.src, v.bytes, cudaMemcpyDeviceToDevice, s->stream);
    };
    const int cand[3] = {64, 128, 256};
    float ms[3][kTuneCount] = {};
    cudaEvent_t ev[2];
    cudaEventCreate(&ev[0]);
    cudaEventCreate(&ev[1]);
    for (int c = 0; c < 3 && rc == FLUID_OK; ++c) {
        for (int rep = 0; rep < 2 && rc == FLUID_OK; ++rep) {  // the first run warms up
            restore();
            cudaMemcpyAsync(s->cur, d.data(), nb * sizeof(DevStep), cudaMemcpyHostToDevice, s->stream);
            float t[kTuneCount] = {};
            rc = timed_substep(s, cand[c], t, ev);
            if (rep == 1)
                for (int k = 0; k < kTuneCount; ++k) ms[c][k] = t[k];
        }
    }
    restore();
    cudaStreamSynchronize(s->stream);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    for (void *q : tmp) cudaFree(q);
    if (rc != FLUID_OK) return rc;
    BK(cudaGetLastError());
    drop_graphs(s);
    for (int k = 0; k < kTuneCount; ++k) {
        int best = 1;
        for (int c = 0; c < 3; ++c)
            if (ms[c][k] < ms[best][k]) best = c;
        s->tpb[k] = (uint16_t)cand[best];
        if (chosen) chosen[k] = (uint32_t)cand[best];
        if (ms_out)
            for (int c = 0; c < 3; ++c) ms_out[c * kTuneCount + k] = ms[c][k];
    }
    return FLUID_OK;
}

}  // extern "C"
