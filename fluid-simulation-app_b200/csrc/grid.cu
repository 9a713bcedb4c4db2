// grid.cu — neighbour grid build for sm_100a.
//
// Reference: count / scatter in crates/fluid-core/src/sim_grid.wgsl:36-72 and
// sim_density.wgsl:36-55; the scan in sim_scan.wgsl:97-120 (exclusive, with
// the total at starts[cells]). The reference's scatter ranks particles inside
// a cell by atomic arrival; this build is stable (ascending input index inside
// a cell), the order a sequential counting sort produces.
//
//   k_cell_keys      key = cell_of(pos), and every radix pass's digit
//                    counts over all keys
//   k_radix_pass     one stable 8-bit digit pass: warp ranking in input
//                    order (digit peers from eight ballots), each tile's
//                    digit offsets by decoupled look-back over the earlier
//                    tiles, the tile staged in shared memory in digit order
//                    and written out coalesced; the last pass also stores
//                    the end of every run of equal keys at starts[key + 1]
//   k_scan_lookback  single-pass scan (sum or max), decoupled look-back with
//                    warp shuffles and ballots; every spin is bounded. The
//                    inclusive max-scan of the run ends gives starts, the
//                    exclusive scan of the cell counts, without counting
#include <algorithm>
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
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// The lanes of `act` whose 8-bit digit equals this lane's: what
// __match_any_sync(act, d) returns, from one ballot per digit bit (cheaper
// than the general match on sm_100). Every lane of the warp calls it.
__device__ __forceinline__ uint32_t digit_peers(uint32_t act, uint32_t d) {
    uint32_t m = act;
#pragma unroll
    for (int b = 0; b < kRadixBits; ++b) {
        const uint32_t bit = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(0xffffffffu, bit);
        m &= bit ? bal : ~bal;
    }
    return m;
}

// Adds the run of equal digits this lane starts (in adjacent lanes) to the
// shared histogram h; positions in cell order give long runs. Every lane of
// the warp calls it.
__device__ __forceinline__ void count_digit_runs(uint32_t *h, bool live, uint32_t d) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t live_mask = __ballot_sync(0xffffffffu, live);
    const uint32_t prev = __shfl_up_sync(0xffffffffu, d, 1);
    const bool prev_live = lane > 0 && ((live_mask >> (lane - 1)) & 1u);
    const bool head = live && (!prev_live || prev != d);
    const uint32_t stops = __ballot_sync(0xffffffffu, head) | ~live_mask;
    if (head) {
        const uint32_t after = stops & ~((2u << lane) - 1u);  // stops above this lane
        const uint32_t end = after ? (uint32_t)(__ffs(after) - 1) : 32u;
        atomicAdd(&h[d], end - lane);
    }
}

// Every pass's digit counts over all keys: a block's shared histograms,
// then one global add per nonzero bin. Every lane of the block calls both.
__device__ __forceinline__ void count_digits(uint32_t (*h)[kRadix], int passes, bool live, uint32_t key) {
    for (int p = 0; p < passes; ++p) count_digit_runs(h[p], live, (key >> (p * kRadixBits)) & (kRadix - 1));
}
__device__ __forceinline__ void flush_digits(uint32_t (*h)[kRadix], int passes, uint32_t *digit_counts) {
    __syncthreads();
    for (int p = 0; p < passes; ++p) {
        const uint32_t c = h[p][threadIdx.x];
        if (c) atomicAdd(&digit_counts[p * kRadix + threadIdx.x], c);
    }
}

// Cell key of every position, and every radix pass's digit counts. A
// grid-stride loop over a capped grid, so the digit counts leave each block
// once. Block 0 also moves the substep's Step block from the ring into
// `cur` for the kernels after it.
__global__ void __launch_bounds__(kSortThreads) k_cell_keys(const float4 *__restrict__ pos, uint32_t n,
                                                            GridGeom g, uint32_t *__restrict__ keys,
                                                            int passes, uint32_t *digit_counts,
                                                            const DevStep *__restrict__ ring, DevStep *cur,
                                                            DevSolve *solve, uint32_t ring_size) {
    __shared__ uint32_t h[kMaxPasses][kRadix];
    if (ring && blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t c = solve->cursor;
        *cur = ring[c % ring_size];
        solve->cursor = c + 1u;
    }
    for (int p = 0; p < kMaxPasses; ++p) h[p][threadIdx.x] = 0;
    __syncthreads();
    // kKeyItems positions per thread and round, all loaded before any is used
    const uint64_t stride = (uint64_t)gridDim.x * kSortThreads * kKeyItems;
    for (uint64_t at = (uint64_t)blockIdx.x * kSortThreads * kKeyItems; at < n; at += stride) {
        float4 p[kKeyItems];
#pragma unroll
        for (int u = 0; u < kKeyItems; ++u) {
            const uint64_t i = at + (uint64_t)u * kSortThreads + threadIdx.x;
            p[u] = i < n ? __ldg(&pos[i]) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < kKeyItems; ++u) {
            const uint64_t i = at + (uint64_t)u * kSortThreads + threadIdx.x;
            const bool live = i < n;
            uint32_t key = 0;
            if (live) {
                const uint32_t cx = axis_cell(p[u].x, g.min[0], g.cell, g.dims[0]);
                const uint32_t cy = axis_cell(p[u].y, g.min[1], g.cell, g.dims[1]);
                const uint32_t cz = axis_cell(p[u].z, g.min[2], g.cell, g.dims[2]);
                key = (cz * g.dims[1] + cy) * g.dims[0] + cx;
                if (g.slabs > 1) key = key * g.slabs + axis_slab(p[u].x, g.min[0], g.cell, cx, g.slabs);
                keys[i] = key;
            }
            count_digits(h, passes, live, key);
        }
    }
    flush_digits(h, passes, digit_counts);
}

// The same over a batch of boxes: box b's key is cell_base[b] plus its
// cell in its own grid. Block 0 moves the substep's nboxes Step blocks
// (ring entry `cursor`, box-major) into cur[0 .. nboxes-1].
__global__ void __launch_bounds__(kSortThreads) k_box_keys(const float4 *__restrict__ pos, uint32_t n,
                                                           BoxKeys bk, uint32_t *__restrict__ keys,
                                                           int passes, uint32_t *digit_counts,
                                                           const DevStep *__restrict__ ring, DevStep *cur,
                                                           DevSolve *solve, uint32_t ring_size) {
    __shared__ uint32_t h[kMaxPasses][kRadix];
    if (ring && blockIdx.x == 0) {
        const uint32_t c = solve->cursor;
        const DevStep *src = ring + (size_t)(c % ring_size) * bk.nboxes;
        for (uint32_t b = threadIdx.x; b < bk.nboxes; b += blockDim.x) cur[b] = src[b];
        __syncthreads();  // every thread has read the cursor before it moves
        if (threadIdx.x == 0) solve->cursor = c + 1u;
    }
    for (int p = 0; p < kMaxPasses; ++p) h[p][threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t at = (uint64_t)blockIdx.x * kSortThreads; at < n; at += (uint64_t)gridDim.x * kSortThreads) {
        const uint64_t i = at + threadIdx.x;
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
            key = (cz * dy + cy) * dx + cx;
            if (bk.slabs > 1)
                key = key * bk.slabs + axis_slab(p.x, __ldg(&P->box_min[0]), cell, cx, bk.slabs);
            key += __ldg(&bk.cell_base[b]);
            keys[i] = key;
        }
        count_digits(h, passes, live, key);
    }
    flush_digits(h, passes, digit_counts);
}

// Combine of the single-pass scan: sum, or max (kMax); 0 is the identity of
// both on unsigned values.
template <bool kMax>
__device__ __forceinline__ uint32_t scan_op(uint32_t a, uint32_t b) {
    return kMax ? max(a, b) : a + b;
}
template <bool kMax>
__device__ __forceinline__ uint32_t warp_reduce(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = scan_op<kMax>(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Scan of in[0..n) into out[0..n), single pass: exclusive sums, or with
// kMax inclusive maxima. Tiles are claimed in launch order through ctl[0];
// ctl[1 + t] is tile t's status word: flag in the high half (1 aggregate,
// 2 inclusive prefix), value in the low half. With write_total, out[n]
// receives the grand total. With zero_in, the input is cleared after it is
// read.
template <bool kMax>
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
    for (int k = 0; k < kScanItems; ++k) sum = scan_op<kMax>(sum, v[k]);

    // block-wide scan of the thread sums
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x = scan_op<kMax>(x, y);
    }
    uint32_t x_before = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) x_before = 0u;
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < kScanThreads / 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w = scan_op<kMax>(w, y);
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t block_total = s_warp[kScanThreads / 32 - 1];
    const uint32_t thread_excl = scan_op<kMax>(warp > 0 ? s_warp[warp - 1] : 0u, x_before);

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
                    exclusive = scan_op<kMax>(exclusive, warp_reduce<kMax>((int)lane <= j ? val : 0u));
                    break;
                }
                exclusive = scan_op<kMax>(exclusive, warp_reduce<kMax>(val));
                pred -= 32;
            }
            if (lane == 0)
                st_relaxed(&status[tile], kFlagPrefix | (unsigned long long)scan_op<kMax>(exclusive, block_total));
        }
        if (lane == 0) s_excl = exclusive;
    }
    __syncthreads();
    uint32_t run = scan_op<kMax>(s_excl, thread_excl);
    if (vec) {
        uint32_t o[kScanItems];
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            if (kMax) {
                run = max(run, v[k]);
                o[k] = run;
            } else {
                o[k] = run;
                run += v[k];
            }
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
            if (kMax) run = max(run, v[k]);
            if (base + k < n) {
                out[base + k] = run;
                if (zero_in) in[base + k] = 0u;
            }
            if (!kMax) run += v[k];
        }
    }
    if (write_total && threadIdx.x == 0 && (uint64_t)(tile + 1) * kScanTile >= n)
        out[n] = scan_op<kMax>(s_excl, block_total);
}

// One stable digit pass. Tiles are claimed in launch order through
// *tile_ctr. Warp w of tile t owns the contiguous run t*TILE + w*32*ITEMS ..
// +32*ITEMS; in round r lane l holds element run + r*32 + l, so (warp,
// round, lane) is input order and ranks taken in that order keep equal
// digits in input order. The tile's count of each digit d is published in
// tile_status[t][d] (flag in the high half: 1 this tile's count, 2 the
// inclusive count over tiles 0..t), and the thread of digit d looks back
// over the tiles before it for their counts of d (decoupled look-back, one
// chain per digit, every spin bounded). A digit's output run starts at the
// number of smaller digits over all keys (digit_counts) plus its count in
// earlier tiles. The tile is laid out in shared memory in (digit, input)
// order and written out by consecutive threads to consecutive addresses.
// `vals_in` null means the identity (the first pass); `keys_out` may be
// null (the last pass). With `starts` (the last pass, keys now in final
// order) every run of equal keys also stores its end at starts[key + 1]:
// inside a tile's digit segment the next output element is the next staged
// one, and the last element of a segment, whose successor another tile
// writes, stores with atomicMax (the true end of its run is larger).
static_assert(kRadix == kSortThreads, "one thread per digit");
// Blocks per SM the pass kernel is compiled for: 4 (64 registers) measured
// 0.75 ms at 16.7M positions against 0.84 at 3 and 1.01 at 1.
#ifndef FCU_SORT_MINB
#define FCU_SORT_MINB 4
#endif
// FCU_SORT_MATCH: digit peers by __match_any_sync instead of eight ballots.
// Measured at 16.7M positions: 15 % slower on uniform keys, 4 % faster on
// clustered ones; the simulation's grid 6 % faster.
#ifndef FCU_SORT_MATCH
#define FCU_SORT_MATCH 0
#endif
// FCU_VAL_PREFETCH > 0: a digit pass asks L1 for the values of every
// FCU_VAL_PREFETCH-th round of its tile while it ranks the keys. Measured:
// grid_16m 0.683 -> 0.648 ms a build at 1 (0.676 at 4); the 1M workload's
// grid 0.1153 -> 0.1147 ms.
#ifndef FCU_VAL_PREFETCH
#define FCU_VAL_PREFETCH 1
#endif
// Earlier tiles' status words a digit's look-back loads at once. Measured:
// the 1M workload's grid 0.1215 ms at 1, 0.1158 at 4, 0.1157 at 8 (16 bytes
// spilled), 0.1203 at 16; grid_16m 0.70 / 0.68 / 0.69 / 0.74 ms a build.
#ifndef FCU_LOOK_WINDOW
#define FCU_LOOK_WINDOW 4
#endif
constexpr int kLookWindow = FCU_LOOK_WINDOW;

__global__ void __launch_bounds__(kSortThreads, FCU_SORT_MINB) k_radix_pass(
    const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t n, int shift,
    const uint32_t *__restrict__ digit_counts, unsigned long long *tile_status, uint32_t *tile_ctr,
    uint32_t *err, uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out,
    uint32_t *__restrict__ starts, uint32_t cells) {
    __shared__ uint32_t s_hist[kSortWarps][kRadix];
    __shared__ uint32_t s_off[kRadix];    // output index of this tile's first element of digit d
    __shared__ uint32_t s_start[kRadix];  // staged index of the tile's first element of digit d
    __shared__ uint32_t s_wsum[kSortWarps];
    __shared__ uint32_t s_gsum[kSortWarps];
    __shared__ uint32_t s_key[kSortTile];
    __shared__ uint32_t s_val[kSortTile];
    __shared__ uint32_t s_tile;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) s_hist[w][threadIdx.x] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;

    // Indices fit 32 bits: the last tile ends at ceil(n / kSortTile) *
    // kSortTile <= 2^32 for any 32-bit n. A full tile (every tile but the
    // last) takes the loads and ballots without per-element bounds.
    const uint32_t wbase = tile * kSortTile + warp * (32 * kSortItems);
    const bool full = (uint64_t)(tile + 1) * kSortTile <= n;
    const uint32_t lt = lanemask_lt();
    uint32_t key[kSortItems], rank[kSortItems];
    if (full) {
#pragma unroll
        for (int r = 0; r < kSortItems; ++r) key[r] = __ldg(&keys_in[wbase + r * 32 + lane]);
    } else {
#pragma unroll
        for (int r = 0; r < kSortItems; ++r) {
            const uint32_t i = wbase + r * 32 + lane;
            key[r] = i < n ? __ldg(&keys_in[i]) : 0u;
        }
    }
#if FCU_VAL_PREFETCH
    // the values are read only after the ranking and the look-back: ask L1
    // for them now (no registers held) so that read finds them there
    if (vals_in) {
#pragma unroll
        for (int r = 0; r < kSortItems; r += FCU_VAL_PREFETCH) {
            const uint32_t i = wbase + r * 32 + lane;
            if (full || i < n) asm volatile("prefetch.global.L1 [%0];" ::"l"(vals_in + i));
        }
    }
#endif
    // every round's digit peers first (ballots and registers only), then the
    // rounds in order: the leader of each group of peers adds the group to
    // the warp's count of its digit and hands the old count to the group
    if (full) {
#pragma unroll
        for (int r = 0; r < kSortItems; ++r) {
            const uint32_t d = (key[r] >> shift) & (kRadix - 1);
#if FCU_SORT_MATCH
            rank[r] = __match_any_sync(0xffffffffu, d);
#else
            rank[r] = digit_peers(0xffffffffu, d);
#endif
        }
    } else {
#pragma unroll
        for (int r = 0; r < kSortItems; ++r) {
            const bool live = wbase + r * 32 + lane < n;
            const uint32_t act = __ballot_sync(0xffffffffu, live);
            const uint32_t d = (key[r] >> shift) & (kRadix - 1);
#if FCU_SORT_MATCH
            const uint32_t pe = live ? __match_any_sync(act, d) : 0u;
#else
            const uint32_t pe = digit_peers(act, d);
#endif
            rank[r] = live ? pe : 0u;  // a live lane is its own peer, so nonzero
        }
    }
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t peers = rank[r];
        const uint32_t d = (key[r] >> shift) & (kRadix - 1);
        const uint32_t leader = peers ? (uint32_t)(__ffs(peers) - 1) : lane;
        uint32_t before = 0;
        if (peers && lane == leader) before = atomicAdd(&s_hist[warp][d], (uint32_t)__popc(peers));
        before = __shfl_sync(0xffffffffu, before, leader);
        rank[r] = before + __popc(peers & lt);
        __syncwarp();  // this round's adds land before the next round's
    }
    __syncthreads();
    // thread = digit d: the warps' exclusive counts of it, and its tile count
    const uint32_t dig = threadIdx.x;
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t t = s_hist[w][dig];
        s_hist[w][dig] = total;
        total += t;
    }
    unsigned long long *mine = tile_status + (uint64_t)tile * kRadix;
    st_relaxed(&mine[dig], (tile == 0 ? kFlagPrefix : kFlagAgg) | total);

    // exclusive scans over the digits: of the tile counts (staged starts)
    // and of the global counts (where each digit's output begins)
    const uint32_t gc = __ldg(&digit_counts[dig]);
    uint32_t x = total, y = gc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t xu = __shfl_up_sync(0xffffffffu, x, o);
        const uint32_t yu = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= (uint32_t)o) {
            x += xu;
            y += yu;
        }
    }
    if (lane == 31) {
        s_wsum[warp] = x;
        s_gsum[warp] = y;
    }

    // look-back over the earlier tiles' counts of this digit: the status
    // words of kLookWindow earlier tiles are loaded at once, then taken in
    // order (an entry read while unpublished is re-read until it is), adding
    // counts until the first inclusive one. A word read early as a tile's own
    // count is still that count, so the sum is the same as one tile at a
    // time; only the chain of L2 round trips is shorter (a single wave of
    // tiles, as at 1M keys, otherwise walks back one tile per round trip).
    uint32_t excl = 0;
    if (tile > 0) {
        int64_t pred = (int64_t)tile - 1;
        bool done = false;
        while (!done) {
            unsigned long long v[kLookWindow];
#pragma unroll
            for (int u = 0; u < kLookWindow; ++u)
                v[u] = pred - u >= 0 ? ld_relaxed(&tile_status[(uint64_t)(pred - u) * kRadix + dig]) : kFlagPrefix;
#pragma unroll
            for (int u = 0; u < kLookWindow; ++u) {
                if (done) continue;
                unsigned long long x = v[u];
                uint32_t spins = 0;
                while ((x >> 32) == 0) {
                    if (++spins > kSpinLimit) {
                        atomicOr(err, ERRF_SCAN_TIMEOUT);
                        x = kFlagPrefix;  // give up: count it as zero and stop
                        break;
                    }
                    x = ld_relaxed(&tile_status[(uint64_t)(pred - u) * kRadix + dig]);
                }
                excl += (uint32_t)x;
                if ((x >> 32) == 2ull) done = true;
            }
            pred -= kLookWindow;
        }
        st_relaxed(&mine[dig], kFlagPrefix | (unsigned long long)(excl + total));
    }
    __syncthreads();
    uint32_t wx = 0, wy = 0;
    for (uint32_t w = 0; w < warp; ++w) {
        wx += s_wsum[w];
        wy += s_gsum[w];
    }
    s_start[dig] = wx + x - total;
    s_off[dig] = wy + y - gc + excl;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t i = wbase + r * 32 + lane;
        if (full || i < n) {
            const uint32_t d = (key[r] >> shift) & (kRadix - 1);
            const uint32_t at = s_start[d] + s_hist[warp][d] + rank[r];
            s_key[at] = key[r];
            s_val[at] = vals_in ? __ldg(&vals_in[i]) : i;
        }
    }
    __syncthreads();
    const uint32_t tbase = tile * kSortTile;
    const uint32_t count = full ? kSortTile : n - tbase;
    for (uint32_t j = threadIdx.x; j < count; j += kSortThreads) {
        const uint32_t k = s_key[j];
        const uint32_t d = (k >> shift) & (kRadix - 1);
        const uint32_t dst = s_off[d] + (j - s_start[d]);
        // Always below n when the counts are right; the test keeps a
        // look-back that gave up (garbage offsets) from writing out of bounds.
        if (dst < n) {
            vals_out[dst] = s_val[j];
            if (keys_out) keys_out[dst] = k;
            if (starts && k < cells) {
                const uint32_t kn = j + 1 < count ? s_key[j + 1] : 0u;
                const bool seg_end = j + 1 == count || ((kn >> shift) & (kRadix - 1)) != d;
                if (seg_end) atomicMax(&starts[k + 1], dst + 1);
                else if (kn != k) starts[k + 1] = dst + 1;
            }
        }
    }
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t scan_region_bytes(uint32_t len) {
    return align256(8ull * (1ull + div_up(len, kScanTile)));
}

// The zeroed part of the workspace: the starts scan's look-back region,
// every pass's tile counter and tile status words, every pass's digit
// counts.
__global__ void k_fill_u32(uint32_t *p, uint32_t n, uint32_t v) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) p[i] = v;
}

struct SortRegion {
    unsigned long long *fill_ctl;
    uint32_t *tile_ctr[kMaxPasses];
    unsigned long long *tile_status[kMaxPasses];
    uint32_t *digit_counts;
    size_t bytes;
};

SortRegion sort_region(void *base, uint32_t n, uint32_t cells, int passes) {
    SortRegion r{};
    const uint32_t tiles = div_up(n > 0 ? n : 1, kSortTile);
    const uintptr_t b = reinterpret_cast<uintptr_t>(base);
    size_t off = 0;
    r.fill_ctl = reinterpret_cast<unsigned long long *>(b + off);
    off += scan_region_bytes(cells + 1);
    for (int q = 0; q < passes; ++q) {
        r.tile_ctr[q] = reinterpret_cast<uint32_t *>(b + off);
        off += 256;
        r.tile_status[q] = reinterpret_cast<unsigned long long *>(b + off);
        off += align256(8ull * kRadix * tiles);
    }
    r.digit_counts = reinterpret_cast<uint32_t *>(b + off);
    off += align256(4ull * kRadix * kMaxPasses);
    r.bytes = off;
    return r;
}

}  // namespace

size_t grid_work_bytes(uint32_t n, uint32_t cells) {
    size_t b = sort_region(nullptr, n, cells, radix_passes(cells)).bytes;
    b += 4 * align256(4ull * (n > 0 ? n : 1));
    b += 256;  // err word when the caller gives none
    return b;
}

GridWork grid_work_carve(void *ws, uint32_t n, uint32_t cells, uint32_t *err) {
    GridWork w{};
    w.passes = radix_passes(cells);
    w.cells = cells;
    w.n = n;
    char *p = (char *)ws;
    w.scan_ctl = (unsigned long long *)p;
    w.scan_ctl_bytes = sort_region(ws, n, cells, w.passes).bytes;
    p += w.scan_ctl_bytes;
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
                               uint32_t *perm, GridWork &w, const DevStep *ring, DevStep *cur,
                               DevSolve *solve, uint32_t ring_size, const BoxKeys *boxes) {
    cudaError_t e;
    const uint32_t cells = w.cells;
    const SortRegion r = sort_region(w.scan_ctl, n, cells, w.passes);
    e = cudaMemsetAsync(w.scan_ctl, 0, w.scan_ctl_bytes, stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(starts, 0, 4ull * cells + 4, stream);
    if (e != cudaSuccess) return e;
    if (n > 0 || ring) {
        const uint32_t per = boxes ? kSortThreads : kSortThreads * kKeyItems;
        const uint32_t blocks = std::min(div_up(n > 0 ? n : 1, per), kKeyBlocks);
        if (boxes)
            k_box_keys<<<blocks, kSortThreads, 0, stream>>>(pos, n, *boxes, keys, w.passes, r.digit_counts, ring,
                                                            cur, solve, ring_size);
        else
            k_cell_keys<<<blocks, kSortThreads, 0, stream>>>(pos, n, g, keys, w.passes, r.digit_counts, ring, cur,
                                                             solve, ring_size);
    }
    if (n > 0) {
        const uint32_t tiles = div_up(n, kSortTile);
        const uint32_t *kin = keys;
        const uint32_t *vin = nullptr;
        for (int pass = 0; pass < w.passes; ++pass) {
            const bool last = pass == w.passes - 1;
            uint32_t *kout = last ? nullptr : ((pass & 1) ? w.k2 : w.k1);
            uint32_t *vout = last ? perm : ((pass & 1) ? w.v2 : w.v1);
            k_radix_pass<<<tiles, kSortThreads, 0, stream>>>(
                kin, vin, n, pass * kRadixBits, r.digit_counts + pass * kRadix, r.tile_status[pass],
                r.tile_ctr[pass], w.err, kout, vout, last ? starts : nullptr, cells);
            kin = kout;
            vin = vout;
        }
    }
    k_scan_lookback<true><<<div_up(cells + 1ull, kScanTile), kScanThreads, 0, stream>>>(starts, starts, cells + 1,
                                                                                        r.fill_ctl, w.err, 0, 0);
    return cudaGetLastError();
}

int32_t report_error(int32_t code, const std::string &msg);

}  // namespace fcu

// The look-back scan's bounded wait, run out on purpose: one block of the
// scan claims tile 1 (the tile counter starts at 1) over a status array in
// which tile 0 never publishes, so its look-back polls status[0] until the
// kSpinLimit bound, records ERRF_SCAN_TIMEOUT and treats the missing prefix
// as zero. Nothing faults or hangs; the context stays usable.
namespace fcu {

int32_t read_build_status(const uint32_t *err, cudaStream_t st, const char *who) {
    uint32_t flags = 0;
    cudaError_t e = cudaMemcpyAsync(&flags, err, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return report_error(FLUID_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
    if (flags & (ERRF_SCAN_TIMEOUT | ERRF_SORT_TIMEOUT))
        return report_error(FLUID_ERR_TIMEOUT,
                            std::string(who) + ": a look-back wait of the build gave up; its starts and "
                                               "permutation are invalid");
    return FLUID_OK;
}

cudaError_t enqueue_stalled_radix_pass(const GridWork &w, cudaStream_t st) {
    if (w.n < 2 * kSortTile || w.passes < 1) return cudaErrorInvalidValue;
    const SortRegion r = sort_region(w.scan_ctl, w.n, w.cells, w.passes);
    cudaError_t e = cudaMemsetAsync(w.scan_ctl, 0, w.scan_ctl_bytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.k2, 0, 4ull * w.n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.err, 0, 4, st);
    if (e != cudaSuccess) return e;
    // the tile counter starts at 1, so the one block claims tile 1
    k_fill_u32<<<1, 32, 0, st>>>(r.tile_ctr[0], 1, 1u);
    k_radix_pass<<<1, kSortThreads, 0, st>>>(w.k2, nullptr, w.n, 0, r.digit_counts, r.tile_status[0],
                                             r.tile_ctr[0], w.err, w.k1, w.v1, nullptr, 1u);
    return cudaGetLastError();
}

}  // namespace fcu

extern "C" int32_t fluid_grid_build_status(const void *workspace, uint32_t n, const FluidGrid *grid,
                                           void *stream) {
    using namespace fcu;
    if (!grid || !workspace) return report_error(FLUID_ERR_ARG, "fluid_grid_build_status: null argument");
    const uint64_t cells = (uint64_t)grid->dims[0] * grid->dims[1] * grid->dims[2];
    if (cells == 0 || cells >= 0xffffffffull)
        return report_error(FLUID_ERR_ARG, "fluid_grid_build_status: bad grid dims");
    const GridWork w = grid_work_carve(const_cast<void *>(workspace), n, (uint32_t)cells, nullptr);
    return read_build_status(w.err, (cudaStream_t)stream, "fluid_grid_build_status");
}

// The bounded look-back wait of a radix digit pass, run out on purpose on a
// real build workspace and reported through fluid_grid_build_status, the
// query a device-pointer caller uses: one block claims tile 1 while tile 0
// never publishes its digit counts, so every digit's look-back gives up. The
// keys are all zero, so the give-up offsets still land inside the outputs.
extern "C" int32_t fluid_selftest_radix_wait(int32_t device, float *ms) {
    using namespace fcu;
    auto fail = [](cudaError_t e) {
        return report_error(FLUID_ERR_CUDA, std::string("fluid_selftest_radix_wait: ") + cudaGetErrorString(e));
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e);
    const uint32_t n = 2 * kSortTile;
    FluidGrid g{};
    g.cell = 1.0f;
    g.dims[0] = 16;
    g.dims[1] = 16;
    g.dims[2] = 1;
    const size_t bytes = grid_work_bytes(n, 256u);
    void *ws = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    float t = 0.0f;
    int32_t rc = FLUID_OK;
    do {
        if ((e = cudaMalloc(&ws, bytes)) != cudaSuccess) break;
        if ((e = cudaEventCreate(&ev[0])) != cudaSuccess) break;
        if ((e = cudaEventCreate(&ev[1])) != cudaSuccess) break;
        const GridWork w = grid_work_carve(ws, n, 256u, nullptr);
        cudaEventRecord(ev[0]);
        if ((e = enqueue_stalled_radix_pass(w, nullptr)) != cudaSuccess) break;
        cudaEventRecord(ev[1]);
        if ((e = cudaEventSynchronize(ev[1])) != cudaSuccess) break;
        cudaEventElapsedTime(&t, ev[0], ev[1]);
        rc = fluid_grid_build_status(ws, n, &g, nullptr);
    } while (false);
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    cudaFree(ws);
    if (e != cudaSuccess) return fail(e);
    if (ms) *ms = t;
    if (rc == FLUID_ERR_TIMEOUT)
        return report_error(FLUID_ERR_TIMEOUT,
                            "fluid_selftest_radix_wait: the digit look-back wait gave up, as it should, "
                            "and fluid_grid_build_status reported it");
    return rc;
}

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
        k_scan_lookback<false><<<1, kScanThreads>>>(in, out, n, ctl, err, 0, 0);
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
