// grid.cu — neighbour grid build for sm_100a.
//
// Reference: count / scatter in crates/fluid-core/src/sim_grid.wgsl:36-72 and
// sim_density.wgsl:36-55; the scan in sim_scan.wgsl:97-120 (exclusive, with
// the total at starts[cells]). The reference's scatter ranks particles inside
// a cell by atomic arrival; this build is stable (ascending input index inside
// a cell), the order a sequential counting sort produces.
//
//   k_cell_keys      key = cell_of(pos), warp-aggregated histogram
//   k_scan_lookback  single-pass exclusive scan, decoupled look-back with
//                    warp shuffles and ballots; every spin is bounded
//   k_radix_hist     per-tile digit histograms (bin-major matrix)
//   k_radix_scatter  stable per-digit scatter: warp match_any ranking in
//                    input order, per-warp digit counts, tile offsets from
//                    the look-back scan of the histogram matrix
#include <string>

#include "grid.cuh"

namespace fcu {

namespace {

constexpr unsigned long long kFlagAgg = 1ull << 32;
constexpr unsigned long long kFlagPrefix = 2ull << 32;

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Cell key of every position, and the cell histogram. Block 0 also moves
// the substep's Step block from the ring into `cur` for the kernels after it.
__global__ void __launch_bounds__(256) k_cell_keys(const float4 *__restrict__ pos, uint32_t n,
                                                   GridGeom g, uint32_t *__restrict__ keys,
                                                   uint32_t *__restrict__ counts,
                                                   const DevStep *__restrict__ ring, DevStep *cur,
                                                   DevSolve *solve, uint32_t ring_size) {
    if (ring && blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t c = solve->cursor;
        *cur = ring[c % ring_size];
        solve->cursor = c + 1u;
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    uint32_t key = 0;
    if (live) {
        const float4 p = __ldg(&pos[i]);
        const uint32_t cx = axis_cell(p.x, g.min[0], g.cell, g.dims[0]);
        const uint32_t cy = axis_cell(p.y, g.min[1], g.cell, g.dims[1]);
        const uint32_t cz = axis_cell(p.z, g.min[2], g.cell, g.dims[2]);
        key = (cz * g.dims[1] + cy) * g.dims[0] + cx;
        keys[i] = key;
    }
    const uint32_t act = __ballot_sync(0xffffffffu, live);
    if (live) {
        const uint32_t peers = __match_any_sync(act, key);
        if ((threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&counts[key], __popc(peers));
    }
}

// The same over a batch of boxes: box b's key is cell_base[b] plus its
// cell in its own grid. Block 0 moves the substep's nboxes Step blocks
// (ring entry `cursor`, box-major) into cur[0 .. nboxes-1].
__global__ void __launch_bounds__(256) k_box_keys(const float4 *__restrict__ pos, uint32_t n,
                                                  BoxKeys bk, uint32_t *__restrict__ keys,
                                                  uint32_t *__restrict__ counts,
                                                  const DevStep *__restrict__ ring, DevStep *cur,
                                                  DevSolve *solve, uint32_t ring_size) {
    if (ring && blockIdx.x == 0) {
        const uint32_t c = solve->cursor;
        const DevStep *src = ring + (size_t)(c % ring_size) * bk.nboxes;
        for (uint32_t b = threadIdx.x; b < bk.nboxes; b += blockDim.x) cur[b] = src[b];
        __syncthreads();
        if (threadIdx.x == 0) solve->cursor = c + 1u;
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    uint32_t key = 0;
    if (live) {
        const uint32_t b = __ldg(&bk.box_of[i]);
        const DevParams *P = &bk.box[b];
        const float4 p = __ldg(&pos[i]);
        const float cell = __ldg(&P->cell);
        const uint32_t dx = __ldg(&P->dims[0]), dy = __ldg(&P->dims[1]), dz = __ldg(&P->dims[2]);
        const uint32_t cx = axis_cell(p.x, __ldg(&P->box_min[0]), cell, dx);
        const uint32_t cy = axis_cell(p.y, __ldg(&P->box_min[1]), cell, dy);
        const uint32_t cz = axis_cell(p.z, __ldg(&P->box_min[2]), cell, dz);
        key = __ldg(&bk.cell_base[b]) + (cz * dy + cy) * dx + cx;
        keys[i] = key;
    }
    const uint32_t act = __ballot_sync(0xffffffffu, live);
    if (live) {
        const uint32_t peers = __match_any_sync(act, key);
        if ((threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&counts[key], __popc(peers));
    }
}

// Exclusive scan of in[0..n) into out[0..n), single pass. Tiles are claimed
// in launch order through ctl[0]; ctl[1 + t] is tile t's status word: flag in
// the high half (1 aggregate, 2 inclusive prefix), value in the low half.
// With write_total, out[n] receives the grand total. With zero_in, the
// input is cleared after it is read (the counts die here, as the
// reference's scatter clears them for the next rebuild).
__global__ void __launch_bounds__(kScanThreads) k_scan_lookback(uint32_t *in, uint32_t *out,
                                                                uint32_t n,
                                                                unsigned long long *ctl,
                                                                uint32_t *err, int write_total,
                                                                int zero_in) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[kScanThreads / 32];
    __shared__ uint32_t s_excl;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd((unsigned int *)ctl, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    unsigned long long *status = ctl + 1;
    const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;

    uint32_t v[kScanItems];
    const bool vec = base + kScanItems <= n && ((uintptr_t)(in + base) & 15u) == 0 &&
                     ((uintptr_t)(out + base) & 15u) == 0;
    if (vec) {
        const uint4 *src = reinterpret_cast<const uint4 *>(in + base);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const uint4 x = src[q];
            v[4 * q + 0] = x.x;
            v[4 * q + 1] = x.y;
            v[4 * q + 2] = x.z;
            v[4 * q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v[k] = (base + k < n) ? in[base + k] : 0u;
    }
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) sum += v[k];

    // block-wide scan of the thread sums
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < kScanThreads / 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t block_total = s_warp[kScanThreads / 32 - 1];
    const uint32_t thread_excl = (warp > 0 ? s_warp[warp - 1] : 0u) + x - sum;

    // decoupled look-back, warp 0
    if (warp == 0) {
        uint32_t exclusive = 0;
        if (tile == 0) {
            if (lane == 0) st_relaxed(&status[0], kFlagPrefix | block_total);
        } else {
            if (lane == 0) st_relaxed(&status[tile], kFlagAgg | block_total);
            int64_t pred = (int64_t)tile - 1;
            while (true) {
                const int64_t idx = pred - (int64_t)lane;
                unsigned long long st = idx >= 0 ? ld_relaxed(&status[idx]) : kFlagPrefix;
                uint32_t spins = 0;
                while (true) {
                    const bool invalid = (st >> 32) == 0;
                    if (!__any_sync(0xffffffffu, invalid)) break;
                    if (++spins > kSpinLimit) {
                        if (lane == 0) atomicOr(err, ERRF_SCAN_TIMEOUT);
                        if (invalid) st = kFlagPrefix;  // give up: count it as zero
                        break;
                    }
                    if (invalid) st = ld_relaxed(&status[idx]);
                }
                const uint32_t pmask = __ballot_sync(0xffffffffu, (st >> 32) == 2ull);
                const uint32_t val = (uint32_t)st;
                if (pmask) {
                    const int j = __ffs(pmask) - 1;
                    exclusive += warp_sum_u32((int)lane <= j ? val : 0u);
                    break;
                }
                exclusive += warp_sum_u32(val);
                pred -= 32;
            }
            if (lane == 0) st_relaxed(&status[tile], kFlagPrefix | (unsigned long long)(exclusive + block_total));
        }
        if (lane == 0) s_excl = exclusive;
    }
    __syncthreads();
    uint32_t run = s_excl + thread_excl;
    if (vec) {
        uint32_t o[kScanItems];
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            o[k] = run;
            run += v[k];
        }
        uint4 *dst = reinterpret_cast<uint4 *>(out + base);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q)
            dst[q] = make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
        if (zero_in) {
            uint4 *z = reinterpret_cast<uint4 *>(in + base);
#pragma unroll
            for (int q = 0; q < kScanItems / 4; ++q) z[q] = make_uint4(0, 0, 0, 0);
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            if (base + k < n) {
                out[base + k] = run;
                if (zero_in) in[base + k] = 0u;
            }
            run += v[k];
        }
    }
    if (write_total && threadIdx.x == 0 && (uint64_t)(tile + 1) * kScanTile >= n)
        out[n] = s_excl + block_total;
}

// Digit histogram of one tile of keys, written bin-major: hist[d * tiles + t].
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint32_t *__restrict__ keys,
                                                             uint32_t n, int shift,
                                                             uint32_t *__restrict__ hist,
                                                             uint32_t tiles) {
    __shared__ uint32_t h[kRadix];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t tile = blockIdx.x;
    const uint64_t base = (uint64_t)tile * kSortTile;
#pragma unroll 4
    for (int r = 0; r < kSortItems; ++r) {
        const uint64_t i = base + (uint64_t)r * kSortThreads + threadIdx.x;
        const bool live = i < n;
        const uint32_t d = live ? (__ldg(&keys[i]) >> shift) & (kRadix - 1) : 0u;
        const uint32_t act = __ballot_sync(0xffffffffu, live);
        if (live) {
            const uint32_t peers = __match_any_sync(act, d);
            if ((threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&h[d], __popc(peers));
        }
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * tiles + tile] = h[threadIdx.x];
}

// Stable scatter of one digit pass. Warp w of tile t owns the contiguous
// run t*TILE + w*32*ITEMS .. +32*ITEMS; in round r lane l holds element
// run + r*32 + l, so (warp, round, lane) is input order and ranks taken in
// that order keep equal digits in input order. `vals_in` null means the
// identity (the first pass). `keys_out` may be null (the last pass).
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(
    const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t n,
    int shift, const uint32_t *__restrict__ offsets, uint32_t tiles,
    uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out) {
    __shared__ uint32_t s_hist[kSortWarps][kRadix];
    __shared__ uint32_t s_off[kRadix];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) s_hist[w][threadIdx.x] = 0;
    s_off[threadIdx.x] = offsets[(uint64_t)threadIdx.x * tiles + tile];
    __syncthreads();

    const uint64_t wbase = (uint64_t)tile * kSortTile + (uint64_t)warp * (32 * kSortItems);
    const uint32_t lt = lanemask_lt();
    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint64_t i = wbase + (uint64_t)r * 32 + lane;
        const bool live = i < n;
        key[r] = live ? __ldg(&keys_in[i]) : 0u;
        val[r] = live ? (vals_in ? __ldg(&vals_in[i]) : (uint32_t)i) : 0u;
        const uint32_t d = (key[r] >> shift) & (kRadix - 1);
        const uint32_t act = __ballot_sync(0xffffffffu, live);
        rank[r] = 0;
        if (live) {
            const uint32_t peers = __match_any_sync(act, d);
            const uint32_t before = s_hist[warp][d];
            rank[r] = before + __popc(peers & lt);
            __syncwarp(act);
            if (lane == (uint32_t)(__ffs(peers) - 1)) s_hist[warp][d] = before + __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t t = s_hist[w][threadIdx.x];
            s_hist[w][threadIdx.x] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint64_t i = wbase + (uint64_t)r * 32 + lane;
        if (i < n) {
            const uint32_t d = (key[r] >> shift) & (kRadix - 1);
            const uint32_t dst = s_off[d] + s_hist[warp][d] + rank[r];
            // Always below n when the offsets are right; the test keeps a
            // scan that gave up (garbage offsets) from writing out of bounds.
            if (dst < n) {
                vals_out[dst] = val[r];
                if (keys_out) keys_out[dst] = key[r];
            }
        }
    }
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t scan_region_bytes(uint32_t len) {
    return align256(8ull * (1ull + div_up(len, kScanTile)));
}

}  // namespace

size_t grid_work_bytes(uint32_t n, uint32_t cells) {
    const int passes = radix_passes(cells);
    const uint32_t tiles = div_up(n > 0 ? n : 1, kSortTile);
    size_t b = 0;
    b += align256(4ull * cells);
    b += scan_region_bytes(cells) + (size_t)passes * scan_region_bytes(kRadix * tiles);
    b += align256(4ull * kRadix * tiles);
    b += 4 * align256(4ull * (n > 0 ? n : 1));
    b += 256;  // err word when the caller gives none
    return b;
}

GridWork grid_work_carve(void *ws, uint32_t n, uint32_t cells, uint32_t *err) {
    GridWork w{};
    w.passes = radix_passes(cells);
    w.cells = cells;
    w.n = n;
    const uint32_t tiles = div_up(n > 0 ? n : 1, kSortTile);
    char *p = (char *)ws;
    w.counts = (uint32_t *)p;
    p += align256(4ull * cells);
    w.scan_ctl = (unsigned long long *)p;
    w.scan_ctl_bytes = scan_region_bytes(cells) + (size_t)w.passes * scan_region_bytes(kRadix * tiles);
    p += w.scan_ctl_bytes;
    w.hist = (uint32_t *)p;
    p += align256(4ull * kRadix * tiles);
    const size_t nb = align256(4ull * (n > 0 ? n : 1));
    w.k1 = (uint32_t *)p;
    p += nb;
    w.k2 = (uint32_t *)p;
    p += nb;
    w.v1 = (uint32_t *)p;
    p += nb;
    w.v2 = (uint32_t *)p;
    p += nb;
    w.err = err ? err : (uint32_t *)p;
    return w;
}

cudaError_t grid_build_enqueue(cudaStream_t stream, const float4 *pos, uint32_t n,
                               const GridGeom &g, uint32_t *keys, uint32_t *starts,
                               uint32_t *perm, GridWork &w, bool counts_zeroed,
                               const DevStep *ring, DevStep *cur, DevSolve *solve,
                               uint32_t ring_size, const BoxKeys *boxes) {
    cudaError_t e;
    const uint32_t cells = w.cells;
    if (!counts_zeroed) {
        e = cudaMemsetAsync(w.counts, 0, 4ull * cells, stream);
        if (e != cudaSuccess) return e;
    }
    e = cudaMemsetAsync(w.scan_ctl, 0, w.scan_ctl_bytes, stream);
    if (e != cudaSuccess) return e;
    if (n > 0 || ring) {
        const uint32_t blocks = div_up(n > 0 ? n : 1, 256);
        if (boxes)
            k_box_keys<<<blocks, 256, 0, stream>>>(pos, n, *boxes, keys, w.counts, ring, cur, solve, ring_size);
        else
            k_cell_keys<<<blocks, 256, 0, stream>>>(pos, n, g, keys, w.counts, ring, cur, solve, ring_size);
    }
    unsigned long long *ctl = w.scan_ctl;
    k_scan_lookback<<<div_up(cells > 0 ? cells : 1, kScanTile), kScanThreads, 0, stream>>>(
        w.counts, starts, cells, ctl, w.err, 1, 1);
    ctl += scan_region_bytes(cells) / 8;
    if (n == 0) return cudaGetLastError();
    const uint32_t tiles = div_up(n, kSortTile);
    const uint32_t *kin = keys;
    const uint32_t *vin = nullptr;
    for (int pass = 0; pass < w.passes; ++pass) {
        const int shift = pass * kRadixBits;
        const bool last = pass == w.passes - 1;
        uint32_t *kout = last ? nullptr : ((pass & 1) ? w.k2 : w.k1);
        uint32_t *vout = last ? perm : ((pass & 1) ? w.v2 : w.v1);
        k_radix_hist<<<tiles, kSortThreads, 0, stream>>>(kin, n, shift, w.hist, tiles);
        const uint32_t len = kRadix * tiles;
        k_scan_lookback<<<div_up(len, kScanTile), kScanThreads, 0, stream>>>(w.hist, w.hist, len, ctl,
                                                                             w.err, 0, 0);
        ctl += scan_region_bytes(len) / 8;
        k_radix_scatter<<<tiles, kSortThreads, 0, stream>>>(kin, vin, n, shift, w.hist, tiles, kout, vout);
        kin = kout;
        vin = vout;
    }
    return cudaGetLastError();
}

int32_t report_error(int32_t code, const std::string &msg);

}  // namespace fcu

// The look-back scan's bounded wait, run out on purpose: one block of the
// scan claims tile 1 (the tile counter starts at 1) over a status array in
// which tile 0 never publishes, so its look-back polls status[0] until the
// kSpinLimit bound, records ERRF_SCAN_TIMEOUT and treats the missing prefix
// as zero. Nothing faults or hangs; the context stays usable.
extern "C" int32_t fluid_selftest_scan_wait(int32_t device, float *ms) {
    using namespace fcu;
    auto fail = [](cudaError_t e) {
        return report_error(FLUID_ERR_CUDA, std::string("fluid_selftest_scan_wait: ") + cudaGetErrorString(e));
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e);
    const uint32_t n = 2 * kScanTile;
    uint32_t *in = nullptr, *out = nullptr, *err = nullptr;
    unsigned long long *ctl = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    uint32_t flags = 0;
    float t = 0.0f;
    const unsigned long long one = 1ull;
    do {
        if ((e = cudaMalloc(&in, 4ull * n)) != cudaSuccess) break;
        if ((e = cudaMalloc(&out, 4ull * (n + 1))) != cudaSuccess) break;
        if ((e = cudaMalloc(&ctl, 8ull * 4)) != cudaSuccess) break;
        if ((e = cudaMalloc(&err, 4)) != cudaSuccess) break;
        if ((e = cudaMemset(in, 0, 4ull * n)) != cudaSuccess) break;
        if ((e = cudaMemset(ctl, 0, 8ull * 4)) != cudaSuccess) break;
        if ((e = cudaMemset(err, 0, 4)) != cudaSuccess) break;
        if ((e = cudaMemcpy(ctl, &one, 8, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((e = cudaEventCreate(&ev[0])) != cudaSuccess) break;
        if ((e = cudaEventCreate(&ev[1])) != cudaSuccess) break;
        cudaEventRecord(ev[0]);
        k_scan_lookback<<<1, kScanThreads>>>(in, out, n, ctl, err, 0, 0);
        cudaEventRecord(ev[1]);
        if ((e = cudaEventSynchronize(ev[1])) != cudaSuccess) break;
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        cudaEventElapsedTime(&t, ev[0], ev[1]);
        if ((e = cudaMemcpy(&flags, err, 4, cudaMemcpyDeviceToHost)) != cudaSuccess) break;
    } while (false);
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    cudaFree(in);
    cudaFree(out);
    cudaFree(ctl);
    cudaFree(err);
    if (e != cudaSuccess) return fail(e);
    if (ms) *ms = t;
    if (flags & ERRF_SCAN_TIMEOUT)
        return report_error(FLUID_ERR_TIMEOUT, "fluid_selftest_scan_wait: the look-back wait gave up, as it should");
    return FLUID_OK;
}
