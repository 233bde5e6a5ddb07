// lyd_noalloc.cu -- FindActiveBins for callers that cannot allocate device memory.
//
// Some hosts of this library may not call cudaMalloc at all. Examples:
// - a simulation framework that owns every device allocation through its own pool;
// - a plugin that runs inside a caller's memory budget;
// - code that must not allocate once its time loop has started.
// Such callers hold their J, bin widths and cell volumes in device memory they allocated
// themselves, and need the active-bin window of FindActiveBins
// (src/UpdateLyaJandH.jl:47-97) without a lyd_ctx, whose creation allocates.
//
// The per-CTA partial sums that the reduction needs, the cloud record and the block work
// list therefore live in one file-scope __device__ array of fixed size (1 MiB of FP64 partials
// plus a tail of about 33 KiB). Every GPU that loads the library holds
// this array until the process exits. In host code the array's name is only a host-side
// stand-in, so its device address is fetched with cudaGetSymbolAddress, once per device,
// on the first call made with that device current.
//
// Every call shares the array and leaves its contents behind. Each call writes every
// partial it later reads, so nothing has to start at zero. Calls whose kernels overlap on
// the GPU (two streams, or two host threads) race on the array and must be serialised by
// the caller.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <mutex>

#include "lyd_internal.h"
#include "lyd_physics.cuh"
#include "lydion_m1.h"

namespace {

// 131072 doubles of partial sums (1 MiB), then the window, the cloud record and the work list.
constexpr size_t kScratchDoubles = 131072;
constexpr int kMaxItems = 2048;
struct Tail {
    int kwin[2];
    int pad[2];
    lyd::CloudDesc cloud;
    int4 items[kMaxItems];
};
constexpr size_t kTailDoubles = (sizeof(Tail) + sizeof(double) - 1) / sizeof(double);
static __device__ __align__(256) double g_active_scratch[kScratchDoubles + kTailDoubles];

constexpr int kMaxDevices = 64;
std::once_flag g_once[kMaxDevices];
void *g_addr[kMaxDevices];
cudaError_t g_status[kMaxDevices];

// Device address of the scratch array on the current device (set up on first use).
cudaError_t scratch_on_current_device(double **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::call_once(g_once[dev], [dev] {
        g_status[dev] = cudaGetSymbolAddress(&g_addr[dev], g_active_scratch);
    });
    *out = static_cast<double *>(g_addr[dev]);
    return g_status[dev];
}

}  // namespace

int lyd_find_active_bins_noalloc(const double *J, const double *dnu, const double *dV, int32_t n_nu, int32_t n_r,
                                 int32_t n_z, int32_t kcore_min, int32_t kcore_max, void *stream, int32_t *kmin,
                                 int32_t *kmax) {
    if (!J || !dnu || !dV || !kmin || !kmax) return LYD_ERR_ARG;
    if (n_nu < 4 || n_nu > 256 || n_r < 3 || n_z < 3) return LYD_ERR_ARG;
    if (kcore_min < 0 || kcore_max >= n_nu || kcore_min > kcore_max) return LYD_ERR_ARG;
    double *scratch = nullptr;
    if (scratch_on_current_device(&scratch) != cudaSuccess) return LYD_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return LYD_ERR_CUDA;
    const int ncell = n_r * n_z;
    int nblocks = lyd::freq_blocks(ncell, dev);
    const int cap = (int)(kScratchDoubles / (size_t)(n_nu + 1));
    if (nblocks > cap) nblocks = cap;
    if (nblocks > kMaxItems) nblocks = kMaxItems;
    // the cloud record and the work list are built on the host stack and copied into the
    // scratch tail (pageable copies: the call returns once the source has been staged)
    Tail h_tail;
    memset(&h_tail, 0, sizeof(h_tail));
    h_tail.cloud.nr = n_r;
    h_tail.cloud.nz = n_z;
    h_tail.cloud.pb0 = 0;
    const int cpb = (ncell + nblocks - 1) / nblocks;
    int nitems = 0;
    for (int b = 0; b < ncell; b += cpb) h_tail.items[nitems++] = make_int4(0, b, b + cpb < ncell ? b + cpb : ncell, 0);
    h_tail.cloud.npb = nitems;
    Tail *tail = reinterpret_cast<Tail *>(scratch + kScratchDoubles);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t head = offsetof(Tail, items);
    if (cudaMemcpyAsync(tail, &h_tail, head + (size_t)nitems * sizeof(int4), cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
        return LYD_ERR_CUDA;
    lyd::launch_find_active(0, J, n_nu, dnu, dV, &tail->cloud, tail->items, nitems, lyd::kJeps, scratch, st);
    lyd::RedArgs r{};
    r.partials = scratch;
    r.nblocks = nitems;
    r.nnu = n_nu;
    r.nclouds = 1;
    r.parts = lyd::PART_ACTIVE;
    r.kcore_min = kcore_min;
    r.kcore_max = kcore_max;
    r.j_scale = 1.0;
    r.cl = &tail->cloud;
    r.kwin = tail->kwin;
    lyd::launch_reduce(r, st);
    if (cudaGetLastError() != cudaSuccess) return LYD_ERR_CUDA;
    int h[2] = {0, 0};
    if (cudaMemcpyAsync(h, tail->kwin, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess) return LYD_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return LYD_ERR_CUDA;
    *kmin = h[0];
    *kmax = h[1];
    return LYD_OK;
}
