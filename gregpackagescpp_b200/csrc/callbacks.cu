// Callback-driven evolve: gtd::system::evolve(method, continue_ev_if, for_each_bod, for_all_bods)
// (gregsys.hpp:2593-3071) with the callbacks on the GPU.
//
// Per step the reference runs: continue_ev_if(); the method's update; for_all_bods(bodies); the
// collision pass (s_coll); for_each_bod(body) on every body (FUNC_TEMPL_SELECT, gregsys.hpp:16-106,
// and the loops at 2691-2712, 2762-2801, 2849-2889, 2970-2987, 3019-3036).  Here each callback is
// device work: the built-ins of random_comet (gregsys.hpp:1935-1984) or hooks that enqueue the
// caller's own kernels.  The predicate's verdict stays on the device: the loop is a CUDA graph whose
// WHILE node runs up to kChunkSteps steps, each behind IF nodes that the predicate kernel opens or
// closes, so the host waits once per chunk.  Cases the graph cannot hold (merging collisions, the
// periodic spatial reorder of the mixed path, force timing, memFreq recording) run the same kernels
// eagerly with one 64-byte read of the verdict per step; the bodies never cross PCIe in either form
// (a recorded frame is read back when it is made, every memFreq-th step).
#include <cuda_runtime.h>

#include <cmath>

#include "callbacks.cuh"
#include "gtd_internal.cuh"
#include "gtd_system.cuh"

namespace gtd {

constexpr int kCbThreads = 1024;

__global__ void cb_begin_kernel(CbCtl *c, unsigned long long max_steps, unsigned long long iterations) {
    c->cont = 0;
    c->go = c->done = c->capped = 0;
    c->status = 0;
    c->iter = 0;
    c->steps = c->chunk = c->count = 0;
    c->max_steps = max_steps;
    c->iterations = iterations;
}

__global__ void cb_reset_chunk_kernel(CbCtl *c) {
    c->iter = 0;
    c->chunk = 0;
}

// continue_ev_if as its own kernel (cb_verdict); with set_handle its verdict opens or closes the
// next step's IF node.
constexpr int kDecideThreads = 256;

__global__ void __launch_bounds__(kDecideThreads) cb_decide_kernel(CbCtl *c, int mode, const double *rest, int64_t n,
                                                                   double bound, unsigned long long probing,
                                                                   const int *coll_status,
                                                                   cudaGraphConditionalHandle h, int set_handle) {
    __shared__ double sh[32];
    const double lo = mode == 2 ? cb_min_rest(rest, n, sh) : INFINITY;
    if (threadIdx.x != 0) return;
    const bool go = cb_verdict(c, mode, lo, bound, probing, coll_status);
    if (set_handle) cudaGraphSetConditional(h, go ? 1u : 0u);
}

// First node of every WHILE iteration: ends the loop when the evolve is over, the chunk is full or
// the iteration bound is reached (this kernel alone sets the loop's handle, so the loop ends after
// at most kMaxIter iterations whatever the nested nodes do), else opens the iteration's body.
__global__ void cb_gate_kernel(CbCtl *c, const int *coll_status, cudaGraphConditionalHandle hw,
                               cudaGraphConditionalHandle hbody) {
    if (coll_status && *coll_status && !c->status) c->status = *coll_status;
    const unsigned it = ++c->iter;
    const bool stop = c->done || c->capped || c->status || c->chunk >= kChunkSteps || it > kMaxIter;
    cudaGraphSetConditional(hbody, stop ? 0u : 1u);
    if (stop) cudaGraphSetConditional(hw, 0u);
}

// The same first node for a built-in predicate (mode 0 or 2), which it also evaluates: the body
// opens only for a true verdict, and a false one ends the loop.  A stop for a full chunk evaluates
// nothing (the next launch's first node does).
__global__ void __launch_bounds__(kDecideThreads) cb_gate_decide_kernel(CbCtl *c, const int *coll_status, int mode,
                                                                        const double *rest, int64_t n, double bound,
                                                                        unsigned long long probing,
                                                                        cudaGraphConditionalHandle hw,
                                                                        cudaGraphConditionalHandle hbody) {
    __shared__ double sh[32];
    const double lo = mode == 2 ? cb_min_rest(rest, n, sh) : INFINITY;
    if (threadIdx.x != 0) return;
    if (coll_status && *coll_status && !c->status) c->status = *coll_status;
    const unsigned it = ++c->iter;
    const bool stop = c->done || c->capped || c->status || c->chunk >= kChunkSteps || it > kMaxIter;
    const bool go = !stop && cb_verdict(c, mode, lo, bound, probing, nullptr);
    cudaGraphSetConditional(hbody, go ? 1u : 0u);
    if (!go) cudaGraphSetConditional(hw, 0u);
}

// N (body count) or M (total mass) of the rest-from-COM functor.
__global__ void __launch_bounds__(kCbThreads) cb_divisor_kernel(int64_t n, const double4 *pm, CbCtl *c, int weighted) {
    __shared__ double sh[32];
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += pm[i].w;
    s = cb_block_sum(s, sh);
    if (threadIdx.x == 0) c->divisor = weighted ? s : (double)n;
}

// random_comet's for_all_bods as its own kernels: one CTA up to kForAllOneBlock bodies; above that
// the CTA only carries the centre and a body-parallel kernel sets the restitution.
constexpr int64_t kForAllOneBlock = 16384;

__global__ void __launch_bounds__(kCbThreads) cb_for_all_kernel(int64_t n, const double4 *pm, double *rest, CbCtl *c,
                                                                int weighted, int set_rest, double min_cor,
                                                                double max_cor, double scale, double n_exp) {
    __shared__ double sh[32];
    __shared__ double com[3];
    cb_for_all_block(n, pm, rest, c, weighted, set_rest, min_cor, max_cor, scale, n_exp, sh, com);
}

__global__ void cb_rest_kernel(int64_t n, const double4 *pm, double *rest, const CbCtl *c, double min_cor,
                               double max_cor, double scale, double n_exp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rest[i] = cb_rest_from_distance(pm[i], c->com, min_cor, max_cor, scale, n_exp);
}

}  // namespace gtd

using namespace gtd;

static CbCtl *ctl_of(gtd_system *s) { return static_cast<CbCtl *>(s->cb_ctl); }

static int ensure_ctl(gtd_system *s) {
    if (s->cb_ctl) return GTD_OK;
    GTD_CUDA(cudaMalloc(&s->cb_ctl, sizeof(CbCtl)));
    GTD_CUDA(cudaMemsetAsync(s->cb_ctl, 0, sizeof(CbCtl), s->stream));
    GTD_CUDA(cudaMallocHost(&s->cb_host, sizeof(CbCtl)));
    return GTD_OK;
}

void release_callbacks(gtd_system *s) {
    cudaFree(s->cb_ctl);
    cudaFreeHost(s->cb_host);
    s->cb_ctl = nullptr;
    s->cb_host = nullptr;
}

static gtd_device_bodies bodies_view(gtd_system *s) {
    gtd_device_bodies b;
    b.n = s->n;
    b.pos_mass = reinterpret_cast<double *>(s->pm[s->cur]);
    b.vel = reinterpret_cast<double *>(s->vel);
    b.acc = reinterpret_cast<double *>(s->acc);
    b.radius = s->rad;
    b.rest = s->rest;
    b.upload_index = s->ids;
    b.cont = &ctl_of(s)->cont;
    b.stream = s->stream;
    return b;
}

static int run_hook(gtd_system *s, gtd_device_hook fn, void *user, const char *which) {
    const gtd_device_bodies b = bodies_view(s);
    const int rc = fn(user, &b);
    if (rc) return fail(GTD_ERR_CALLBACK, "device %s hook returned %d", which, rc);
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}

static int enqueue_predicate(gtd_system *s, const int *coll_status, cudaGraphConditionalHandle h, bool set_handle) {
    if (s->cb.cont_kind == 1) {
        int rc = run_hook(s, s->cb.cont_fn, s->cb.cont_user, "continue_ev_if");
        if (rc) return rc;
    }
    cb_decide_kernel<<<1, kDecideThreads, 0, s->stream>>>(ctl_of(s), s->cb.cont_kind, s->rest, s->n, s->cb.min_max_cor,
                                                      s->cb.probing_iters, coll_status, h, set_handle ? 1 : 0);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    return GTD_OK;
}

static int enqueue_for_all(gtd_system *s) {
    if (s->cb.all_kind == 1) return run_hook(s, s->cb.all_fn, s->cb.all_user, "for_all_bods");
    if (s->cb.all_kind != 2 || s->n == 0) return GTD_OK;
    const double4 *pm = s->pm[s->cur];
    const bool one = s->n <= kForAllOneBlock;
    cb_for_all_kernel<<<1, kCbThreads, 0, s->stream>>>(s->n, pm, s->rest, ctl_of(s), s->cb.mass_weighted, one ? 1 : 0,
                                                       s->cb.min_cor, s->cb.max_cor, s->cb.scale_factor, s->cb.n_exp);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    if (one) return GTD_OK;
    cb_rest_kernel<<<(unsigned)((s->n + 255) / 256), 256, 0, s->stream>>>(
        s->n, pm, s->rest, ctl_of(s), s->cb.min_cor, s->cb.max_cor, s->cb.scale_factor, s->cb.n_exp);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    return GTD_OK;
}

// One step of the loop body: update, for_all_bods, collision pass, for_each_bod.  In a capture the
// collision pass is enqueued without its read-back (its status reaches the next verdict); its
// resolving CTA also takes over the built-in for_all_bods and, when `decide` is given and nothing
// runs between the pass and the next verdict, that verdict too (*decided).
static int callback_step(gtd_system *s, bool capture, const cudaGraphConditionalHandle *decide, bool *decided) {
    if (decided) *decided = false;
    int rc = cb_direct_step(s);
    if (rc) return rc;
    if (!(capture && s->coll == GTD_OVERLAP_COLL && s->n >= 2)) {
        rc = enqueue_for_all(s);
        if (rc) return rc;
        if (s->coll != GTD_NO_COLL) {
            rc = capture ? enqueue_collisions(s, nullptr) : run_collisions(s);
            if (rc) return rc;
        }
    } else {
        PassHooks hk;
        hk.ctl = ctl_of(s);
        if (s->cb.all_kind == 2 && s->n <= kForAllOneBlock) {
            hk.for_all = 1;
            hk.weighted = s->cb.mass_weighted;
            hk.min_cor = s->cb.min_cor;
            hk.max_cor = s->cb.max_cor;
            hk.scale = s->cb.scale_factor;
            hk.n_exp = s->cb.n_exp;
        } else {
            rc = enqueue_for_all(s);
            if (rc) return rc;
        }
        if (decide && s->cb.cont_kind != 1 && !s->cb.each_fn) {
            hk.decide = 1;
            hk.mode = s->cb.cont_kind;
            hk.bound = s->cb.min_max_cor;
            hk.probing = s->cb.probing_iters;
            hk.handle = *decide;
            if (decided) *decided = true;
        }
        rc = enqueue_collisions(s, &hk);
        if (rc) return rc;
    }
    if (!capture && s->rec_every) {  // s_coll<true> records after the collision pass, before for_each_bod
        s->rec_step += 1;
        if (s->rec_step % s->rec_every == 0 && (rc = record_frame(s, s->rec_step))) return rc;
    }
    if (s->cb.each_fn) return run_hook(s, s->cb.each_fn, s->cb.each_user, "for_each_bod");
    return GTD_OK;
}

// Adds a conditional node after the current capture point of `st` and makes it the new one.
static int add_conditional(cudaStream_t st, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                           cudaGraph_t *body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    GTD_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) return fail(GTD_ERR_CUDA, "stream is not capturing");
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    GTD_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
    *body = p.conditional.phGraph_out[0];
    GTD_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return GTD_OK;
}

// Runs `fill` with `st` capturing into `g`; always ends the capture.
template <typename F>
static int capture_into(cudaStream_t st, cudaGraph_t g, F &&fill) {
    GTD_CUDA(cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const int rc = fill();
    cudaGraph_t out = g;
    const cudaError_t e = cudaStreamEndCapture(st, &out);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    return GTD_OK;
}

// The loop graph.  Two steps per iteration bring the double-buffered positions back to the buffer
// they started in, so one graph serves every launch.  With a built-in predicate (none, or
// random_comet's) the iteration's first node evaluates it:
//   reset; WHILE(hw) { gate+verdict -> IF(h1) { step A (+ verdict) -> IF(h3) { step B } } }
// where step A's collision pass evaluates the verdict when it is the last node of the step; with a
// user predicate its hook's kernels precede each verdict:
//   reset; WHILE(hw) { gate -> IF(h1) { hook, verdict -> IF(h2) { step A; hook, verdict -> IF(h3) { step B } } } }
// *flips: position-buffer flips per step (parity of the end); *launches_per_step: kernels of one
// step; *verdicts_apart: whether verdicts run as kernels of their own (for the launch count).
static int build_loop_graph(gtd_system *s, const int *coll_status, cudaGraphExec_t *exec, int *flips,
                            uint64_t *launches_per_step, int *verdicts_apart) {
    *exec = nullptr;
    cudaGraph_t G = nullptr;
    GTD_CUDA(cudaGraphCreate(&G, 0));
    const int cur0 = s->cur;
    const uint64_t launches0 = s->launches;
    cudaStream_t st = s->stream;
    CbCtl *c = ctl_of(s);
    int cur_a = cur0;
    uint64_t per_step = 0;
    bool fused = false;
    const bool builtin = s->cb.cont_kind != 1;
    int rc = [&]() -> int {
        cudaGraphConditionalHandle hw, h1, h2, h3;
        GTD_CUDA(cudaGraphConditionalHandleCreate(&hw, G, 1, cudaGraphCondAssignDefault));
        cudaGraph_t wb = nullptr, b1 = nullptr, b2 = nullptr, b3 = nullptr;
        int r = capture_into(st, G, [&]() -> int {
            cb_reset_chunk_kernel<<<1, 1, 0, st>>>(c);
            GTD_CHECK_LAUNCH();
            return add_conditional(st, hw, cudaGraphCondTypeWhile, &wb);
        });
        if (r) return r;
        GTD_CUDA(cudaGraphConditionalHandleCreate(&h1, wb, 0, cudaGraphCondAssignDefault));
        r = capture_into(st, wb, [&]() -> int {
            if (builtin)
                cb_gate_decide_kernel<<<1, kDecideThreads, 0, st>>>(c, coll_status, s->cb.cont_kind, s->rest, s->n,
                                                                    s->cb.min_max_cor, s->cb.probing_iters, hw, h1);
            else
                cb_gate_kernel<<<1, 1, 0, st>>>(c, coll_status, hw, h1);
            GTD_CHECK_LAUNCH();
            return add_conditional(st, h1, cudaGraphCondTypeIf, &b1);
        });
        if (r) return r;
        cudaGraph_t step_a = b1;
        if (!builtin) {
            GTD_CUDA(cudaGraphConditionalHandleCreate(&h2, b1, 0, cudaGraphCondAssignDefault));
            r = capture_into(st, b1, [&]() -> int {
                int q = enqueue_predicate(s, coll_status, h2, true);
                if (q) return q;
                return add_conditional(st, h2, cudaGraphCondTypeIf, &b2);
            });
            if (r) return r;
            step_a = b2;
        }
        GTD_CUDA(cudaGraphConditionalHandleCreate(&h3, step_a, 0, cudaGraphCondAssignDefault));
        r = capture_into(st, step_a, [&]() -> int {
            const uint64_t l0 = s->launches;
            int q = callback_step(s, true, &h3, &fused);
            if (q) return q;
            cur_a = s->cur;
            if (!fused) {
                per_step = s->launches - l0;
                q = enqueue_predicate(s, coll_status, h3, true);
                if (q) return q;
            } else {
                per_step = s->launches - l0;
            }
            return add_conditional(st, h3, cudaGraphCondTypeIf, &b3);
        });
        if (r) return r;
        r = capture_into(st, b3, [&]() -> int { return callback_step(s, true, nullptr, nullptr); });
        if (r) return r;
        if (s->cur != cur0) return fail(GTD_ERR_CUDA, "loop body does not return to its position buffer");
        GTD_CUDA(cudaGraphInstantiate(exec, G, 0));
        return GTD_OK;
    }();
    cudaGraphDestroy(G);
    s->cur = cur0;
    s->synced = true;
    s->launches = launches0;  // captured, not yet run
    if (rc) {
        if (*exec) cudaGraphExecDestroy(*exec);
        *exec = nullptr;
        cudaGetLastError();
        return rc;
    }
    *flips = cur_a != cur0 ? 1 : 0;
    *launches_per_step = per_step;
    *verdicts_apart = builtin ? (fused ? 0 : 1) : 2;
    return GTD_OK;
}

static int read_ctl(gtd_system *s, CbCtl *h) {
    GTD_CUDA(cudaMemcpyAsync(s->cb_host, s->cb_ctl, sizeof(CbCtl), cudaMemcpyDeviceToHost, s->stream));
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    *h = *static_cast<CbCtl *>(s->cb_host);
    return GTD_OK;
}

static int status_error(int status) {
    if (status == GTD_ERR_CAPACITY)
        return fail(GTD_ERR_CAPACITY, "overlapping pairs in one step exceeded what the collision pass holds");
    return fail(status, "collision pass failed with status %d", status);
}

// The eager form: the same kernels, one read of the verdict per step.
static int eager_loop(gtd_system *s, uint64_t *waits) {
    const bool reorder = s->precision == GTD_PREC_MIXED && s->coll == GTD_NO_COLL;
    for (;;) {
        int rc = enqueue_predicate(s, nullptr, 0, false);
        if (rc) return rc;
        CbCtl h;
        rc = read_ctl(s, &h);
        if (rc) return rc;
        *waits += 1;
        if (!h.go) return GTD_OK;
        if (reorder && (rc = cb_maybe_reorder(s))) return rc;
        rc = callback_step(s, false, nullptr, nullptr);
        if (rc) return rc;
    }
}

static int graph_loop(gtd_system *s, cudaGraphExec_t exec, int flips, uint64_t per_step, int verdicts_apart,
                      uint64_t *waits) {
    const int cur0 = s->cur;
    CbCtl h{};
    for (;;) {
        GTD_CUDA(cudaGraphLaunch(exec, s->stream));
        int rc = read_ctl(s, &h);
        if (rc) return rc;
        *waits += 1;
        // reset, first nodes, steps, and the verdicts that run as kernels of their own
        s->launches += 1 + h.iter + h.chunk * per_step +
                       (verdicts_apart == 2 ? h.chunk + 1 : verdicts_apart == 1 ? (h.chunk + 1) / 2 : 0);
        if (h.status) return status_error(h.status);
        if (h.done || h.capped) break;
        if (h.chunk < kChunkSteps) return fail(GTD_ERR_CUDA, "callback loop chunk ended early (%llu steps)", h.chunk);
    }
    s->cur = cur0 ^ (int)((flips * h.chunk) & 1);  // every chunk but the last is even
    return GTD_OK;
}

extern "C" {

int gtd_system_set_step_hook(gtd_system *s, gtd_step_hook hook, void *user) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    s->step_hook = hook;
    s->step_hook_user = hook ? user : nullptr;
    return GTD_OK;
}

int gtd_system_update_bodies(gtd_system *s, const double *m, const double *r, const double *rest, const double *x3,
                             const double *v3) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    DeviceGuard g(s->device);
    return device_update(s, m, r, rest, x3, v3);
}

int gtd_system_set_device_callbacks(gtd_system *s, gtd_device_hook continue_ev_if, void *cont_user,
                                    gtd_device_hook for_each_bod, void *each_user, gtd_device_hook for_all_bods,
                                    void *all_user) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    s->cb.cont_kind = continue_ev_if ? 1 : 0;
    s->cb.cont_fn = continue_ev_if;
    s->cb.cont_user = cont_user;
    s->cb.each_fn = for_each_bod;
    s->cb.each_user = each_user;
    s->cb.all_kind = for_all_bods ? 1 : 0;
    s->cb.all_fn = for_all_bods;
    s->cb.all_user = all_user;
    return GTD_OK;
}

int gtd_system_set_rest_from_com(gtd_system *s, double min_cor, double max_cor, double scale_factor, double n_exp,
                                 const double com[3], int mass_weighted) {
    if (!s || !com) return fail(GTD_ERR_INVALID_ARGUMENT, "system or com is NULL");
    DeviceGuard g(s->device);
    int rc = ensure_ctl(s);
    if (rc) return rc;
    s->cb.all_kind = 2;
    s->cb.all_fn = nullptr;
    s->cb.all_user = nullptr;
    s->cb.min_cor = min_cor;
    s->cb.max_cor = max_cor;
    s->cb.scale_factor = scale_factor;
    s->cb.n_exp = n_exp;
    s->cb.mass_weighted = mass_weighted ? 1 : 0;
    CbCtl *c = ctl_of(s);
    GTD_CUDA(cudaMemcpyAsync(c->com, com, 3 * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    cb_divisor_kernel<<<1, kCbThreads, 0, s->stream>>>(s->n, s->pm[s->cur], c, s->cb.mass_weighted);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    return GTD_OK;
}

int gtd_system_rest_from_com_centre(gtd_system *s, double com[3]) {
    if (!s || !com) return fail(GTD_ERR_INVALID_ARGUMENT, "system or com is NULL");
    if (!s->cb_ctl) return fail(GTD_ERR_INVALID_ARGUMENT, "no rest-from-COM functor was set");
    DeviceGuard g(s->device);
    GTD_CUDA(cudaMemcpyAsync(com, ctl_of(s)->com, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    return GTD_OK;
}

int gtd_system_set_continue_while_rest_below(gtd_system *s, double min_max_cor, uint64_t probing_iters) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    s->cb.cont_kind = 2;
    s->cb.cont_fn = nullptr;
    s->cb.cont_user = nullptr;
    s->cb.min_max_cor = min_max_cor;
    s->cb.probing_iters = probing_iters;
    return GTD_OK;
}

int gtd_system_callback_stats(const gtd_system *s, uint64_t *host_waits, int *graph_loop) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (host_waits) *host_waits = s->cb_waits;
    if (graph_loop) *graph_loop = s->cb_graph ? 1 : 0;
    return GTD_OK;
}

int gtd_system_evolve_callbacks(gtd_system *s, int method, uint64_t max_steps, uint64_t *steps_taken,
                                int64_t *elapsed_ns) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (steps_taken) *steps_taken = 0;
    if (elapsed_ns) *elapsed_ns = 0;
    s->cb_waits = 0;
    s->cb_graph = false;
    const int branch = cb_select_branch(method);
    if (s->n == 0 || branch == 0) return GTD_OK;  // gregsys.hpp:2611-2612, empty branches
    if ((method & GTD_BARNES_HUT) == GTD_BARNES_HUT) {
        // the Barnes-Hut branch ignores the callbacks and runs `iterations` steps (gregsys.hpp:2913)
        int rc = gtd_system_evolve(s, method, elapsed_ns);
        if (!rc && steps_taken && (branch == GTD_LEAPFROG_KDK)) *steps_taken = s->iterations;
        return rc;
    }
    if (branch == GTD_TWO_BODY || branch == GTD_RK4 || branch == GTD_RK3_8) return gtd_system_evolve(s, method, elapsed_ns);
    DeviceGuard g(s->device);
    int rc = ensure_ctl(s);
    if (rc) return rc;
    GTD_CUDA(cudaEventRecord(s->ev0, s->stream));
    rc = cb_evolve_begin(s, branch);
    if (rc) return rc;
    cb_begin_kernel<<<1, 1, 0, s->stream>>>(ctl_of(s), max_steps, s->iterations);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    uint64_t waits = 0;
    // recorded frames are read back as they are made: a recording evolve runs eagerly
    const bool graphable = s->coll != GTD_MERGE_COLL && !(s->precision == GTD_PREC_MIXED && s->coll == GTD_NO_COLL) &&
                           !s->time_force && !s->rec_every;
    cudaGraphExec_t exec = nullptr;
    int flips = 0, verdicts_apart = 0;
    uint64_t per_step = 0;
    if (graphable) {
        // everything the captured steps need exists before the capture
        int *coll_status = nullptr;
        if (s->coll != GTD_NO_COLL) rc = prepare_collisions(s, &coll_status);
        if (!rc) rc = cb_prepare_steps(s);
        if (rc) return rc;
        if (build_loop_graph(s, coll_status, &exec, &flips, &per_step, &verdicts_apart) != GTD_OK)
            exec = nullptr;  // eager below
    }
    if (exec) {
        s->cb_graph = true;
        rc = graph_loop(s, exec, flips, per_step, verdicts_apart, &waits);
        cudaGraphExecDestroy(exec);
    } else {
        rc = eager_loop(s, &waits);
    }
    s->cb_waits = waits;
    if (rc) return rc;
    CbCtl h;
    rc = read_ctl(s, &h);
    if (rc) return rc;
    if (steps_taken) *steps_taken = h.steps;
    GTD_CUDA(cudaEventRecord(s->ev1, s->stream));
    GTD_CUDA(cudaEventSynchronize(s->ev1));
    float ms = 0.f;
    GTD_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    if (elapsed_ns) *elapsed_ns = (int64_t)((double)ms * 1e6);
    return GTD_OK;
}

}  // extern "C"
