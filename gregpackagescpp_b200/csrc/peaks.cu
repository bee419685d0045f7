// Roofline denominators measured on the device itself: a dependent-FMA microkernel with enough
// independent chains per thread and enough warps per SM to saturate the FP32 (FFMA and packed
// FFMA2) or FP64 (DFMA) pipes.  2 flops per FMA.  No counterpart in the reference.
#include <cuda_runtime.h>

#include <algorithm>

#include "gtd_internal.cuh"

namespace {

constexpr int kChains = 8;

__global__ void ffma_kernel(float *out, int iters, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-3f + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void ffma2_kernel(float *out, int iters, float a, float b) {
    float2 x[kChains / 2];
#pragma unroll
    for (int k = 0; k < kChains / 2; ++k) x[k] = make_float2(threadIdx.x * 1e-3f + k, k + 0.5f);
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains / 2; ++k) x[k] = __ffma2_rn(x[k], a2, b2);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kChains / 2; ++k) s += x[k].x + x[k].y;
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void dfma_kernel(double *out, int iters, double a, double b) {
    double x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = threadIdx.x * 1e-3 + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s == 1234.5) out[threadIdx.x] = s;
}

}  // namespace

extern "C" int gtd_measure_fma_peak(int device, int precision, double *flops_per_s) {
    using namespace gtd;
    if (!flops_per_s) return fail(GTD_ERR_INVALID_ARGUMENT, "flops_per_s is NULL");
    *flops_per_s = 0.0;
    int prev = 0;
    cudaGetDevice(&prev);
    GTD_CUDA(cudaSetDevice(device));
    int sms = 0;
    GTD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int threads = 256, blocks = sms * 8;
    void *buf = nullptr;
    GTD_CUDA(cudaMalloc(&buf, 1024 * sizeof(double)));
    cudaEvent_t e0, e1;
    GTD_CUDA(cudaEventCreate(&e0));
    GTD_CUDA(cudaEventCreate(&e1));
    double best = 0.0;
    const int variants = precision == GTD_PREC_F64 ? 1 : 2;
    for (int var = 0; var < variants; ++var) {
        int iters = precision == GTD_PREC_F64 ? 4096 : 16384;
        for (int rep = 0; rep < 4; ++rep) {
            GTD_CUDA(cudaEventRecord(e0));
            if (precision == GTD_PREC_F64)
                dfma_kernel<<<blocks, threads>>>((double *)buf, iters, 0.999999, 1e-7);
            else if (var == 0)
                ffma_kernel<<<blocks, threads>>>((float *)buf, iters, 0.9999f, 1e-4f);
            else
                ffma2_kernel<<<blocks, threads>>>((float *)buf, iters, 0.9999f, 1e-4f);
            GTD_CHECK_LAUNCH();
            GTD_CUDA(cudaEventRecord(e1));
            GTD_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            GTD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            const double flops = 2.0 * kChains * (double)iters * threads * blocks;
            if (rep > 0) best = std::max(best, flops / (ms * 1e-3));
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    cudaSetDevice(prev);
    *flops_per_s = best;
    return GTD_OK;
}
