// grid_static.cu — fluid_grid_build_static: the neighbour-grid build on a
// scratch area compiled into the library, for callers that cannot allocate.
//
// fluid_grid_build needs a device workspace of fluid_grid_workspace_bytes
// from its caller. Some callers have none to give and may not let the
// library allocate one: an embedder that owns a fixed GPU memory budget and
// forbids its libraries to allocate outside it (an engine or visualiser
// whose pools are sized at start-up), a real-time frame callback in which a
// cudaMalloc / cudaFree pair would synchronise the device and stall the
// frame, or a foreign-function caller holding only host handles and no
// device buffer to pass. This entry point serves them: it allocates nothing
// (no cudaMalloc, no cudaFree, no allocating library routine) and takes its
// scratch from one file-scope device array of kStaticScratchBytes.
//
// The reference has no counterpart: its grid build always runs on buffers
// the simulation created with it (crates/fluid-core/src/render.rs:1468-1612).
//
// Set-up: the first call on each device, with that device current, looks up
// the array's device address with cudaGetSymbolAddress (which can load the
// library's device code); make that first call before any stream capture
// begins. Later calls on the device reuse the address.
//
// Zeroing: every call clears, on the caller's stream and before its kernels,
// what must start at zero: the cell counts, the look-back status words of
// the scans and the error word. Everything else in the scratch is written
// before it is read.
//
// Errors: the build's error word sits at a fixed place, the first 256 bytes
// of the scratch, and the rest is carved for the build behind it. A look-
// back wait that gives up sets it; fluid_grid_build_static_status reads it
// back (after the build, before the next call on the device clears it), so
// a caller learns that its starts and permutation are invalid.
//
// Races: there is ONE scratch area per device. Two calls whose work overlaps
// on the device (different streams, or different host threads, with no
// stream order or event between them) share it and corrupt each other's
// result. Order such calls on one stream or with events.
#include <cstdio>
#include <mutex>
#include <string>

#include "grid.cuh"

namespace fcu {

int32_t report_error(int32_t code, const std::string &msg);

namespace {

// 16 MiB: e.g. 2^19 positions over 2^20 cells need 12.1 MiB of scratch,
// 2^20 positions over 2^18 cells 17.3 MiB (refused).
constexpr size_t kStaticScratchBytes = (size_t)FLUID_GRID_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_scratch[kStaticScratchBytes];

// The error word's slot at the head of the scratch. grid_work_bytes counts
// 256 bytes for an error word of the workspace's own, which a build with
// its word elsewhere leaves unused, so the carve behind the slot still
// ends within grid_work_bytes.
constexpr size_t kErrBytes = 256;

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void *g_scratch_addr[kMaxDevices];  // the array's device address, per device

// The scratch address on the current device, looked up on first use.
cudaError_t scratch_address(int dev, void **out) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace fcu

using namespace fcu;

extern "C" int32_t fluid_grid_build_static(const float *pos4, uint32_t n, const FluidGrid *grid,
                                           uint32_t *keys, uint32_t *starts, uint32_t *perm,
                                           void *stream) {
    if (!grid || !starts || (n && (!pos4 || !perm)))
        return report_error(FLUID_ERR_ARG, "fluid_grid_build_static: null argument");
    if (!(grid->cell > 0.0f)) return report_error(FLUID_ERR_ARG, "fluid_grid_build_static: cell must be positive");
    for (int i = 0; i < 3; ++i)
        if (grid->dims[i] == 0) return report_error(FLUID_ERR_ARG, "fluid_grid_build_static: dims must be positive");
    const uint64_t cells = (uint64_t)grid->dims[0] * grid->dims[1] * grid->dims[2];
    if (cells >= 0xffffffffull)
        return report_error(FLUID_ERR_ARG, "fluid_grid_build_static: grid has too many cells");
    const size_t need = grid_work_bytes(n, (uint32_t)cells);
    if (need > kStaticScratchBytes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "fluid_grid_build_static: %u positions over %llu cells need %zu bytes of scratch, "
                 "above the fixed %zu; use fluid_grid_build with a workspace",
                 n, (unsigned long long)cells, need, kStaticScratchBytes);
        return report_error(FLUID_ERR_ARG, msg);
    }
    if ((uintptr_t)pos4 & 15u)
        return report_error(FLUID_ERR_ARG, "fluid_grid_build_static: positions must be 16-byte aligned");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return report_error(FLUID_ERR_CUDA, std::string("fluid_grid_build_static: cudaGetDevice: ") +
                                                cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return report_error(FLUID_ERR_ARG, "fluid_grid_build_static: device ordinal above 63");
    void *ws = nullptr;
    e = scratch_address(dev, &ws);
    if (e != cudaSuccess)
        return report_error(FLUID_ERR_CUDA, std::string("fluid_grid_build_static: cudaGetSymbolAddress: ") +
                                                cudaGetErrorString(e));
    cudaStream_t st = (cudaStream_t)stream;
    GridWork w = grid_work_carve(static_cast<char *>(ws) + kErrBytes, n, (uint32_t)cells,
                                 static_cast<uint32_t *>(ws));
    e = cudaMemsetAsync(w.err, 0, 4, st);
    // Without a caller buffer the keys live in k2: pass 0 reads them and
    // writes k1, and k2 is next written by pass 1, after they are consumed.
    GridGeom g;
    for (int i = 0; i < 3; ++i) {
        g.min[i] = grid->min[i];
        g.dims[i] = grid->dims[i];
    }
    g.cell = grid->cell;
    if (e == cudaSuccess)
        e = grid_build_enqueue(st, (const float4 *)pos4, n, g, keys ? keys : w.k2, starts, perm, w, nullptr,
                               nullptr, nullptr, 1);
    if (e != cudaSuccess)
        return report_error(FLUID_ERR_CUDA, std::string("fluid_grid_build_static: ") + cudaGetErrorString(e));
    return FLUID_OK;
}

// The error word of the last fluid_grid_build_static on the current device.
extern "C" int32_t fluid_grid_build_static_status(void *stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return report_error(FLUID_ERR_CUDA, std::string("fluid_grid_build_static_status: cudaGetDevice: ") +
                                                cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return report_error(FLUID_ERR_ARG, "fluid_grid_build_static_status: device ordinal above 63");
    void *ws = nullptr;
    e = scratch_address(dev, &ws);
    if (e != cudaSuccess)
        return report_error(FLUID_ERR_CUDA, std::string("fluid_grid_build_static_status: cudaGetSymbolAddress: ") +
                                                cudaGetErrorString(e));
    return read_build_status(static_cast<const uint32_t *>(ws), (cudaStream_t)stream,
                             "fluid_grid_build_static_status");
}

// A radix digit pass's bounded look-back run out on the fixed scratch, as a
// build of fluid_grid_build_static lays it out, and reported through
// fluid_grid_build_static_status. Allocates nothing.
extern "C" int32_t fluid_selftest_static_radix_wait(int32_t device, float *ms) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess)
        return report_error(FLUID_ERR_CUDA, std::string("fluid_selftest_static_radix_wait: ") + cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices)
        return report_error(FLUID_ERR_ARG, "fluid_selftest_static_radix_wait: device ordinal above 63");
    void *ws = nullptr;
    e = scratch_address(device, &ws);
    cudaEvent_t ev[2] = {nullptr, nullptr};
    float t = 0.0f;
    int32_t rc = FLUID_OK;
    do {
        if (e != cudaSuccess) break;
        if ((e = cudaEventCreate(&ev[0])) != cudaSuccess) break;
        if ((e = cudaEventCreate(&ev[1])) != cudaSuccess) break;
        const uint32_t n = 2 * kSortTile;
        const GridWork w = grid_work_carve(static_cast<char *>(ws) + kErrBytes, n, 256u,
                                           static_cast<uint32_t *>(ws));
        cudaEventRecord(ev[0]);
        if ((e = enqueue_stalled_radix_pass(w, nullptr)) != cudaSuccess) break;
        cudaEventRecord(ev[1]);
        if ((e = cudaEventSynchronize(ev[1])) != cudaSuccess) break;
        cudaEventElapsedTime(&t, ev[0], ev[1]);
        rc = fluid_grid_build_static_status(nullptr);
    } while (false);
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    if (e != cudaSuccess)
        return report_error(FLUID_ERR_CUDA, std::string("fluid_selftest_static_radix_wait: ") + cudaGetErrorString(e));
    if (ms) *ms = t;
    if (rc == FLUID_ERR_TIMEOUT)
        return report_error(FLUID_ERR_TIMEOUT,
                            "fluid_selftest_static_radix_wait: the digit look-back wait gave up, as it should, "
                            "and fluid_grid_build_static_status reported it");
    return rc;
}
