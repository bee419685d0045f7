// Direct-sum accelerations that allocate nothing.
//
// gtd_system_* keeps its bodies and its force kernel's per-row partial sums in buffers it allocates
// with cudaMalloc.  Some callers cannot let a library allocate: a process whose device memory is
// already handed to a pool (a PyTorch caching allocator holding the GPU, a simulation that reserves
// all its memory once at start-up) may not be able to get more, and in a running loop cudaMalloc /
// cudaFree synchronise the whole device, stalling every other stream.  This entry point takes the
// caller's device buffers for input and output and keeps the only scratch the force needs - the
// force kernel's partial sums (and, in mixed precision, its work-queue counter, zeroed on the
// stream before every launch) - in one fixed array compiled into the library.
#include <cuda_runtime.h>

#include <mutex>

#include "gtd_internal.cuh"

namespace gtd {

// The scratch: 8 MiB in device global memory, a file-scope __device__ array.  Every GPU that loads
// this library holds its own copy until the process exits.  From host code the name only stands in
// for the symbol; its device address comes from cudaGetSymbolAddress (below), once per device.
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

constexpr int64_t kNoAllocMaxBodies = 65536;
constexpr int kMaxDevices = 64;

struct ScratchAddr {
    void *ptr = nullptr;
    bool ready = false;
};
static ScratchAddr g_scratch_addr[kMaxDevices];
static std::mutex g_scratch_mu;

// Whether p is memory the current device can read and write: device or managed memory of that
// device.  A host pointer, or another device's buffer, is rejected before any launch.
static bool on_current_device(const void *p, int dev) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();  // the failed query leaves its error as the last error: clear it
        return false;
    }
    if (at.type == cudaMemoryTypeManaged) return true;
    return at.type == cudaMemoryTypeDevice && at.device == dev;
}

// Device address of the scratch on the current device; looked up on the first call per device and
// kept for the life of the process.  cudaDeviceReset discards the module and with it the array, so
// the kept address is not valid across a device reset: do not use this entry point after one.
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
    int dev = 0;
    GTD_CUDA(cudaGetDevice(&dev));
    if (!on_current_device(pm4, dev) || !on_current_device(acc3, dev))
        return fail(GTD_ERR_INVALID_ARGUMENT,
                    "pm4 and acc3 must be device (or managed) memory of the current device %d", dev);
    void *scratch = nullptr;
    int rc = scratch_on_current_device(&scratch);
    if (rc) return rc;
    // the split of the force into partial sums is narrowed until they fit the fixed scratch
    ForcePlan p = make_plan(n, precision, dev, 0);
    rc = fit_plan_partials(p, kNoAllocScratchBytes);
    if (rc) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    rc = launch_force(precision, p, reinterpret_cast<const double4 *>(pm4), G, static_cast<double *>(scratch), st);
    if (rc) return rc;
    return launch_sum_partials(p, static_cast<const double *>(scratch), acc3, st);
}
