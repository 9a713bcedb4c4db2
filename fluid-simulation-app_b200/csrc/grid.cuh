// grid.cuh — the neighbour grid: cell keys, look-back scan, stable sort.
#pragma once

#include "common.cuh"

namespace fcu {

struct GridGeom {
    float min[3];
    float cell;
    uint32_t dims[3];
    // slabs > 1: each cell is cut into that many slabs along x and the key
    // is cell * slabs + slab, so a cell's slots are in slab order
    uint32_t slabs = 1;
};

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;  // 4096 u32 per tile

constexpr int kRadixBits = 8;
constexpr uint32_t kRadix = 1u << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr uint32_t kSortTile = kSortThreads * kSortItems;  // 4096 keys per tile
constexpr int kMaxPasses = 4;                               // 32-bit keys
constexpr uint32_t kKeyBlocks = 148 * 8;                    // grid cap of the key kernels
#ifndef FCU_KEY_ITEMS
#define FCU_KEY_ITEMS 4
#endif
constexpr int kKeyItems = FCU_KEY_ITEMS;                    // positions per thread and round (cell keys)

inline uint32_t div_up(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Digit passes for keys below `cells`.
inline int radix_passes(uint32_t cells) {
    uint32_t maxkey = cells > 0 ? cells - 1 : 0;
    int bits = 0;
    while (maxkey) {
        bits++;
        maxkey >>= 1;
    }
    int p = (bits + kRadixBits - 1) / kRadixBits;
    return p < 1 ? 1 : p;
}

// Scratch of one grid build, carved from one device allocation.
struct GridWork {
    unsigned long long *scan_ctl;  // look-back words and digit counts, zeroed per build
    size_t scan_ctl_bytes;
    uint32_t *k1, *k2, *v1, *v2;   // ping-pong keys / values
    uint32_t *err;                 // device error word (may alias the sim's)
    int passes;
    uint32_t cells, n;
};

size_t grid_work_bytes(uint32_t n, uint32_t cells);
// Carves `ws` (at least grid_work_bytes) into a GridWork.
GridWork grid_work_carve(void *ws, uint32_t n, uint32_t cells, uint32_t *err);

// Reads a build's error word on `stream` (waiting for it): FLUID_OK, or
// FLUID_ERR_TIMEOUT with a reason when a bounded look-back wait gave up.
int32_t read_build_status(const uint32_t *err, cudaStream_t stream, const char *who);
// Enqueues one block of a radix digit pass on the scratch of `w` (carved for
// at least two tiles of keys) that claims tile 1 while tile 0 never
// publishes: its bounded look-back waits give up and set w.err.
cudaError_t enqueue_stalled_radix_pass(const GridWork &w, cudaStream_t stream);

// A batch of boxes sharing one grid: slot i belongs to box box_of[i], whose
// keys are cell_base[b] .. cell_base[b] + its cells * slabs - 1 (the boxes'
// key ranges laid end to end, in box order; key cell * slabs + x slab).
struct BoxKeys {
    const uint16_t *box_of;     // [n]
    const DevParams *box;       // [nboxes]
    const uint32_t *cell_base;  // [nboxes]
    uint32_t nboxes;
    uint32_t slabs = 1;
};

// Enqueues keys -> stable radix sort -> starts on `stream`. `keys` receives
// each input's cell key, `starts` the exclusive scan of the cell counts with
// starts[cells] = n, `perm` the stable permutation. `ring`/`cur`/`solve`
// (may be null) let the key kernel
// also fetch the substep's Step block from the ring. With `boxes`, the keys
// are the batch's (`g` unused) and every box's Step block of the substep
// (ring entry cursor holds nboxes of them) moves to cur[0 .. nboxes-1].
cudaError_t grid_build_enqueue(cudaStream_t stream, const float4 *pos, uint32_t n,
                               const GridGeom &g, uint32_t *keys, uint32_t *starts,
                               uint32_t *perm, GridWork &w, const DevStep *ring, DevStep *cur,
                               DevSolve *solve, uint32_t ring_size, const BoxKeys *boxes = nullptr);

}  // namespace fcu
