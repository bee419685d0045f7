// Direct-sum accelerations that allocate nothing.
//
// gtd_system_* keeps its bodies and its force kernel's per-row partial sums in buffers it allocates
// with cudaMalloc.  Some callers cannot let a library allocate: a process whose device memory is
// already handed to a pool (a PyTorch caching allocator holding the GPU, a simulation that reserves
// all its memory once at start-up) may not be able to get more, and in a running loop cudaMalloc /
// cudaFree synchronise the whole device, stalling every other stream.  This entry point takes the
// caller's device buffers for input and output and keeps the only scratch the force needs - the
// stream-K partial sums - in one fixed array compiled into the library.
#include <cuda_runtime.h>

#include <mutex>

#include "gtd_internal.cuh"

namespace gtd {

// The scratch: 8 MiB in device global memory, a file-scope __device__ array.  Every GPU that loads
// this library holds its own copy until the process exits.  From host code the name only stands in
// for the symbol; its device address comes from cudaGetSymbolAddress (below), once per device.
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

// The stream-K grid is capped so the partial sums of N = 65536 bodies fit the scratch.
constexpr int kNoAllocMaxGrid = 296;
constexpr int64_t kNoAllocMaxBodies = 65536;
constexpr int kMaxDevices = 64;

struct ScratchAddr {
    void *ptr = nullptr;
    bool ready = false;
};
static ScratchAddr g_scratch_addr[kMaxDevices];
static std::mutex g_scratch_mu;

// Sums the partials of body i (CTA order, as the integrate kernel does) into acc3[3 i .. 3 i + 2].
__global__ void noalloc_combine_kernel(int64_t n, int64_t tiles, int64_t total, int grid, int bi,
                                       const double *part, double *acc3) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t r = i / bi;
    const int l = (int)(i - r * bi);
    const int64_t g0 = ((r * tiles + 1) * (int64_t)grid - 1) / total;
    const int64_t g1 = (((r + 1) * tiles) * (int64_t)grid - 1) / total;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int64_t g = g0; g <= g1; ++g) {
        const double *slot = part + (size_t)(g + r) * 3 * bi;
        ax += slot[l];
        ay += slot[bi + l];
        az += slot[2 * bi + l];
    }
    acc3[3 * i] = ax;
    acc3[3 * i + 1] = ay;
    acc3[3 * i + 2] = az;
}

// Device address of the scratch on the current device; looked up on the first call per device.
static int scratch_on_current_device(void **out) {
    int dev = 0;
    GTD_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(GTD_ERR_CAPACITY, "device ordinal %d not supported", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    ScratchAddr &sa = g_scratch_addr[dev];
    if (!sa.ready) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        sa.ptr = p;
        sa.ready = true;
    }
    *out = sa.ptr;
    return GTD_OK;
}

}  // namespace gtd

using namespace gtd;

extern "C" int gtd_direct_accelerations_noalloc(int64_t n, const double *pm4, double G, int precision, double *acc3,
                                                void *stream) {
    if (n < 0) return fail(GTD_ERR_INVALID_ARGUMENT, "n must not be negative");
    if (n == 0) return GTD_OK;
    if (!pm4 || !acc3) return fail(GTD_ERR_INVALID_ARGUMENT, "pm4 and acc3 must be device pointers");
    if (precision != GTD_PREC_F64 && precision != GTD_PREC_MIXED)
        return fail(GTD_ERR_INVALID_ARGUMENT, "unknown precision %d", precision);
    if (reinterpret_cast<uintptr_t>(pm4) % 16 != 0)
        return fail(GTD_ERR_INVALID_ARGUMENT, "pm4 must be 16-byte aligned (it is read as double4 records)");
    if (n > kNoAllocMaxBodies)
        return fail(GTD_ERR_CAPACITY,
                    "gtd_direct_accelerations_noalloc holds its partial sums in a fixed %zu-byte device array and "
                    "accepts at most %lld bodies; got %lld (use gtd_system_accelerations for larger systems)",
                    kNoAllocScratchBytes, (long long)kNoAllocMaxBodies, (long long)n);
    void *scratch = nullptr;
    int rc = scratch_on_current_device(&scratch);
    if (rc) return rc;
    int dev = 0;
    GTD_CUDA(cudaGetDevice(&dev));
    ForcePlan p = make_plan(n, precision, dev, 0);
    if (p.grid > kNoAllocMaxGrid) {
        p.grid = kNoAllocMaxGrid;
        p.slots = p.grid + p.rows;
    }
    if (partial_bytes(p) > kNoAllocScratchBytes)
        return fail(GTD_ERR_CAPACITY, "%lld bodies need %zu bytes of partial sums; the fixed scratch holds %zu",
                    (long long)n, partial_bytes(p), kNoAllocScratchBytes);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    rc = launch_force(precision, p, reinterpret_cast<const double4 *>(pm4), G, static_cast<double *>(scratch), st);
    if (rc) return rc;
    noalloc_combine_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, p.tiles, p.total, p.grid, p.bi,
                                                                         static_cast<const double *>(scratch), acc3);
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}
