// Internal declarations shared by the CUDA translation units of libgtd_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>

#include "gtd_b200.h"

namespace gtd {

// ---- error plumbing: every C entry point returns a status and leaves a thread-local message ----
void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define GTD_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t _e = (call);                                              \
        if (_e != cudaSuccess) return ::gtd::cuda_fail(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define GTD_CHECK_LAUNCH() GTD_CUDA(cudaPeekAtLastError())

// ---- direct-summation work decomposition (stream-K over (i-block, j-tile) pairs) --------------
//
// The N x N interaction square is cut into R = ceil(N/BI) rows of i-bodies and J = ceil(N/BJ)
// j-tiles.  The T = R*J (row, tile) pairs are split into G equal contiguous ranges, one per CTA
// of a grid sized to exactly fill the GPU, so every SM gets the same number of pair-tiles
// whatever N is.  A CTA writes one partial sum per row segment it touches, into slot (g + r);
// the integrate kernel adds the partials of each row in CTA order (deterministic).
struct ForcePlan {
    int64_t n = 0;
    int bi = 0, bj = 0;      // bodies per i-block, per j-tile
    int64_t rows = 0, tiles = 0, total = 0;
    int grid = 0;            // CTAs of the force kernel
    int64_t slots = 0;       // partial-sum slots: grid + rows (stream-K), rows * segs (work queue)
    // Work queue (mixed kernel): each row's tiles are cut into segs segments of seg_tiles tiles; the
    // rows * segs units are taken in turn from a counter by the CTAs, each unit writing its own slot.
    // segs == 0: the stream-K split above.
    int64_t segs = 0, seg_tiles = 0, units = 0;
    int variant = 0;         // kernel variant (i-bodies per thread, fold length)
    float near2 = 0.f;       // mixed kernel: precise-path threshold, near2_of(near factor)
};

// Mixed kernel: a fold that holds a pair closer than 2 |X_i| / (K - 1) to one of its i-bodies (X_i:
// the body's coordinates in its row's FP32 frame) is recomputed on the precise path, so that the
// FP32 rounding of the coordinates costs no pair more than K 2^-24 of its relative accuracy.
// K <= 1 turns the check off.
constexpr double kDefaultNearFactor = 8.0;
inline float near2_of(double k) { return k > 1.0 ? (float)((2.0 / (k - 1.0)) * (2.0 / (k - 1.0))) : 0.f; }

// Per-thread launch shape of the two force kernels.
constexpr int kThreads = 256;

enum Epilogue : int {
    EPI_ACC = 0,         // acc = a
    EPI_KDK = 1,         // v += h/2 a (end of step); if !last: v += h/2 a, x_dst = x + h v
    EPI_DKD = 2,         // v += h a; x = x_half + h/2 v; if !last: x_dst = x + h/2 v (next half drift)
    EPI_EULER = 3,       // x_dst = x + h v; v += h a
    EPI_PREDICT = 4,     // acc = a; pred_x = x + hp v; pred_v = v + hp a
    EPI_CORR_MEULER = 5, // x_dst = x + h/2 (v + pred_v); v += h/2 (acc + a)
    EPI_CORR_MIDPOINT = 6,  // x_dst = x + h pred_v; v += h a
};

struct StepArgs {
    int64_t n;
    const double4 *src;   // positions (x,y,z) + mass (w) the force is evaluated at
    const double4 *cur;   // state positions + mass the update starts from
    double4 *dst;         // updated positions + mass
    double4 *vel;
    double4 *acc;
    double4 *pred_pos;    // predictor positions (modified Euler / midpoint)
    double4 *pred_vel;
    double h, hp;         // step, predictor step
    int last;             // KDK/DKD: leave the state synchronised
};

ForcePlan make_plan(int64_t n, int precision, int device, int variant);
int variant_count(int precision);
int variant_info(int precision, int variant, int *i_per_thread, int *fold);
// Process-wide autotune results: a handle without a pinned variant takes the variant last tuned on
// its device for its precision and size class (the bit length of N), else default_variant.
int default_variant(int precision, int64_t n);
// Up to this many bodies an FP64 force evaluation and its update run as one fused launch.
constexpr int64_t kFusedMaxN = 4096;
int launch_fused_small(int64_t n, const double4 *src, double G, int epi, const StepArgs &st, cudaStream_t s);
void remember_variant(int device, int precision, int64_t n, int variant);
int tuned_variant(int device, int precision, int64_t n);
size_t partial_bytes(const ForcePlan &p);
// Shrinks the plan's partial-sum footprint to at most max_bytes (fewer queue segments, or a smaller
// stream-K grid); GTD_ERR_CAPACITY when even the smallest split does not fit.
int fit_plan_partials(ForcePlan &p, size_t max_bytes);
// acc3[3 i + d] = the summed partials of body i (the force alone, in the bodies' order).
int launch_sum_partials(const ForcePlan &p, const double *partials, double *acc3, cudaStream_t s);
// Force on every body of `src` (positions + G-free masses), written as partial sums.
int launch_force(int precision, const ForcePlan &p, const double4 *src, double G, double *partials,
                 cudaStream_t s);
// Combines the partials of each body and applies the integrator epilogue.
int launch_integrate(const ForcePlan &p, const double *partials, int epi, const StepArgs &a, cudaStream_t s);
// Kick-drift (KDK start) and half drift (DKD start) on a synchronised state.
int launch_kick_drift(int64_t n, const double4 *cur, double4 *dst, double4 *vel, const double4 *acc, double h,
                      cudaStream_t s);
int launch_half_drift(int64_t n, const double4 *cur, double4 *dst, const double4 *vel, double h, cudaStream_t s);

// FP64 diagnostics: out[0]=KE, out[1]=PE, out[2..4]=momentum, out[5..7]=sum m x, out[8]=sum m.
int launch_energy(int64_t n, const double4 *pm, const double4 *vel, double G, double *scratch, int64_t scratch_n,
                  cudaStream_t s);
int64_t energy_scratch_doubles(int64_t n);
int finish_energy(const double *scratch_host, int64_t n, double *out9);

}  // namespace gtd
