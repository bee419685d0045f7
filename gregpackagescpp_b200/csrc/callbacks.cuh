// Device side of the callback-driven evolve (callbacks.cu), shared with the collision pass
// (collide.cu), whose resolving CTA can take over random_comet's for_all_bods and the predicate
// that follows the pass.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

namespace gtd {

// Device control block of one callback-driven evolve.
struct CbCtl {
    unsigned cont;                // verdict written by a user continue_ev_if hook
    unsigned go;                  // last verdict
    unsigned done;                // the predicate returned false
    unsigned capped;              // max_steps reached (predicate not evaluated)
    int status;                   // first collision-pass error
    unsigned iter;                // WHILE iterations in this graph launch
    unsigned long long steps;     // steps taken in this evolve
    unsigned long long chunk;     // steps taken in this graph launch
    unsigned long long count;     // the rest-below predicate's probing counter (random_comet's _count)
    unsigned long long max_steps; // 0: no guard
    unsigned long long iterations;
    double com[3];                // carried centre of the rest-from-COM functor
    double divisor;               // N or total mass, fixed when the functor is set
};

constexpr unsigned kChunkSteps = 64;        // steps per graph launch; even (two steps per iteration)
constexpr unsigned kMaxIter = kChunkSteps;  // WHILE iterations per launch, whatever the inner nodes do

// Fixed-order block reductions (the result does not depend on timing): a shuffle tree inside each
// warp, then one over the warps' results.  sh: 32 doubles of shared memory.
__device__ __forceinline__ double cb_block_sum(double v, double *sh) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < nw ? sh[lane] : 0.0;
        for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
        if (lane == 0) sh[0] = v;
    }
    __syncthreads();
    const double r = sh[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double cb_block_min(double v, double *sh) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
    for (int d = 16; d > 0; d >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, d));
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = lane < nw ? sh[lane] : INFINITY;
        for (int d = 16; d > 0; d >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, d));
        if (lane == 0) sh[0] = v;
    }
    __syncthreads();
    const double r = sh[0];
    __syncthreads();
    return r;
}

// Smallest restitution coefficient (NaN never compares below, as in the reference).  Block-wide.
__device__ __forceinline__ double cb_min_rest(const double *rest, int64_t n, double *sh) {
    double lo = INFINITY;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) lo = fmin(lo, rest[i]);
    return cb_block_min(lo, sh);
}

// continue_ev_if's verdict, evaluated before every step (thread 0).  mode 0: steps < iterations
// (no predicate, gregsys.hpp:2948); 1: the user hook's verdict; 2: random_comet's predicate
// (gregsys.hpp:1956-1963): true (and the counter reset) while some body has rest < bound (lo: the
// smallest rest), else `count++ < probing`.  A collision-pass error or max_steps ends the loop
// without evaluating the predicate.
__device__ __forceinline__ bool cb_verdict(CbCtl *c, int mode, double lo, double bound, unsigned long long probing,
                                           const int *coll_status) {
    if (coll_status && *coll_status && !c->status) c->status = *coll_status;
    bool go;
    if (c->status) {
        go = false;
    } else if (c->max_steps && c->steps >= c->max_steps) {
        go = false;
        c->capped = 1;
    } else if (mode == 0) {
        go = c->steps < c->iterations;
    } else if (mode == 1) {
        go = c->cont != 0;
    } else if (lo < bound) {
        c->count = 0;
        go = true;
    } else {
        go = c->count++ < probing;
    }
    if (go) {
        c->steps += 1;
        c->chunk += 1;
    } else if (!c->status && !c->capped) {
        c->done = 1;
    }
    c->go = go ? 1u : 0u;
    return go;
}

__device__ __forceinline__ double cb_rest_from_distance(const double4 &p, const double *com, double min_cor,
                                                        double max_cor, double scale, double n_exp) {
    const double dx = p.x - com[0], dy = p.y - com[1], dz = p.z - com[2];
    const double de = pow(sqrt(dx * dx + dy * dy + dz * dz), n_exp);
    return max_cor - (max_cor - min_cor) * (de / (de + scale));
}

// random_comet's for_all_bods (gregsys.hpp:1971-1983), block-wide: the centre is NOT reset before
// the sum, so it carries: com = (com + sum x) / N, or (com + sum m x) / M with GREGSYS_MERGERS;
// then, with set_rest, every body takes its restitution from the distance to it.  The sum is
// strided over kForAllLanes threads whatever the block size (512 or more), so every caller gets the
// same bits.  sh: 32 doubles, com: 3 doubles of shared memory.
constexpr int kForAllLanes = 512;

__device__ __forceinline__ void cb_for_all_block(int64_t n, const double4 *pm, double *rest, CbCtl *c, int weighted,
                                                 int set_rest, double min_cor, double max_cor, double scale,
                                                 double n_exp, double *sh, double *com) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int64_t i = threadIdx.x; threadIdx.x < kForAllLanes && i < n; i += kForAllLanes) {
        const double4 p = pm[i];
        if (weighted) {
            sx += p.w * p.x;
            sy += p.w * p.y;
            sz += p.w * p.z;
        } else {
            sx += p.x;
            sy += p.y;
            sz += p.z;
        }
    }
    sx = cb_block_sum(sx, sh);
    sy = cb_block_sum(sy, sh);
    sz = cb_block_sum(sz, sh);
    if (threadIdx.x == 0) {
        com[0] = c->com[0] = (c->com[0] + sx) / c->divisor;
        com[1] = c->com[1] = (c->com[1] + sy) / c->divisor;
        com[2] = c->com[2] = (c->com[2] + sz) / c->divisor;
    }
    __syncthreads();
    if (!set_rest) return;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
        rest[i] = cb_rest_from_distance(pm[i], com, min_cor, max_cor, scale, n_exp);
    __syncthreads();
}

// What a collision pass's resolving CTA takes over inside the callback loop: random_comet's
// for_all_bods before resolving (restitution is the only thing it changes, and only the resolution
// reads it), and the predicate after the pass, which opens or closes the next step's IF node.
struct PassHooks {
    CbCtl *ctl = nullptr;
    int for_all = 0, weighted = 0;
    double min_cor = 0.0, max_cor = 1.0, scale = 1.0, n_exp = 1.0;
    int decide = 0, mode = 0;
    double bound = 0.0;
    unsigned long long probing = 0;
    cudaGraphConditionalHandle handle = 0;
};

}  // namespace gtd
