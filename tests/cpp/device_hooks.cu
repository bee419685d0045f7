// Device callbacks written the way a user of gtd_system_evolve_callbacks writes them: plain C
// functions that enqueue their own kernels on the handle's stream (include/gtd_b200.h).  Built by
// tests/test_callbacks_gpu.py with nvcc into a scratch shared library.
#include <cuda_runtime.h>

#include "gtd_b200.h"

namespace {

// for_each_bod: every velocity scaled by a factor (the reference's `b.curr_vel *= f` per body).
__global__ void scale_velocities_kernel(int64_t n, double *vel, double f) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    vel[4 * i] *= f;
    vel[4 * i + 1] *= f;
    vel[4 * i + 2] *= f;
}

// continue_ev_if: true for the first `limit` evaluations (a counter in device memory).
__global__ void count_steps_kernel(unsigned long long *counter, unsigned long long limit, unsigned *cont) {
    *cont = (*counter)++ < limit ? 1u : 0u;
}

}  // namespace

extern "C" {

struct scale_args {
    double factor;
};

int hook_scale_velocities(void *user, const gtd_device_bodies *b) {
    const double f = static_cast<scale_args *>(user)->factor;
    if (b->n == 0) return 0;
    scale_velocities_kernel<<<(unsigned)((b->n + 255) / 256), 256, 0, (cudaStream_t)b->stream>>>(b->n, b->vel, f);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 1;
}

struct count_args {
    unsigned long long *counter;  // device
    unsigned long long limit;
};

int hook_count_steps(void *user, const gtd_device_bodies *b) {
    auto *a = static_cast<count_args *>(user);
    count_steps_kernel<<<1, 1, 0, (cudaStream_t)b->stream>>>(a->counter, a->limit, b->cont);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 1;
}

// A hook that reports a failure (the evolve must stop with GTD_ERR_CALLBACK).
int hook_fail(void *, const gtd_device_bodies *) { return 7; }

// Host-side helpers for the test: the argument blocks, with the counter in device memory.
void *make_scale_args(double factor) { return new scale_args{factor}; }
void *make_count_args(unsigned long long limit) {
    auto *a = new count_args{nullptr, limit};
    if (cudaMalloc(&a->counter, sizeof(unsigned long long)) != cudaSuccess) return nullptr;
    cudaMemset(a->counter, 0, sizeof(unsigned long long));
    cudaDeviceSynchronize();
    return a;
}
int reset_count_args(void *p) {
    auto *a = static_cast<count_args *>(p);
    cudaMemset(a->counter, 0, sizeof(unsigned long long));
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}
void free_args(void *p, int is_count) {
    if (is_count) {
        cudaFree(static_cast<count_args *>(p)->counter);
        delete static_cast<count_args *>(p);
    } else {
        delete static_cast<scale_args *>(p);
    }
}

}  // extern "C"
