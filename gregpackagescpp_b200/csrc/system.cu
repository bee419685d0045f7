// C ABI of the device-resident gtd::system (include/gtd_b200.h): handle lifetime, gather/scatter
// of the AoS bodies, and the evolve() loop of gregsys.hpp:2593-3071 driven on one CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "gtd_internal.cuh"
#include "gtd_system.cuh"

namespace gtd {

static thread_local char g_err[1024];

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
    set_error("CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e), what, file, line);
    return e == cudaErrorMemoryAllocation ? GTD_ERR_OUT_OF_MEMORY : GTD_ERR_CUDA;
}

const char *last_error() { return g_err; }

}  // namespace gtd

using namespace gtd;

// ---------------------------------------------------------------------------------------------
// buffers
// ---------------------------------------------------------------------------------------------
static int ensure_capacity(gtd_system *s, int64_t n) {
    if (n <= s->cap) return GTD_OK;
    release_bodies(s);
    const size_t b4 = sizeof(double4) * (size_t)n;
    GTD_CUDA(cudaMalloc(&s->pm[0], b4));
    GTD_CUDA(cudaMalloc(&s->pm[1], b4));
    GTD_CUDA(cudaMalloc(&s->vel, b4));
    GTD_CUDA(cudaMalloc(&s->acc, b4));
    GTD_CUDA(cudaMalloc(&s->rad, sizeof(double) * (size_t)n));
    GTD_CUDA(cudaMalloc(&s->rest, sizeof(double) * (size_t)n));
    GTD_CUDA(cudaMalloc(&s->ids, sizeof(int32_t) * (size_t)n));
    GTD_CUDA(cudaMallocHost(&s->stage, 4 * b4));
    s->cap = n;
    return GTD_OK;
}

int ensure_body_capacity(gtd_system *s, int64_t n) { return ensure_capacity(s, n); }

// State after n bodies were written straight into the device arrays in upload order.
int set_loaded_bodies(gtd_system *s, int64_t n) {
    s->n = n;
    s->n_uploaded = n;
    s->cur = 0;
    s->begun = false;
    s->synced = true;
    s->tree_valid = false;
    s->ordered = false;
    s->steps_since_reorder = 0;
    return GTD_OK;
}

void release_bodies(gtd_system *s) {
    cudaFree(s->pm[0]);
    cudaFree(s->pm[1]);
    cudaFree(s->vel);
    cudaFree(s->acc);
    cudaFree(s->pred_pos);
    cudaFree(s->pred_vel);
    cudaFree(s->rad);
    cudaFree(s->rest);
    cudaFree(s->ids);
    cudaFree(s->partials);
    cudaFree(s->escratch);
    cudaFree(s->sc4);
    cudaFree(s->sc1);
    cudaFree(s->sci);
    cudaFree(s->bh_ninter);
    s->sc4 = nullptr;
    s->sc1 = nullptr;
    s->sci = nullptr;
    s->bh_ninter = nullptr;
    cudaFreeHost(s->stage);
    s->pm[0] = s->pm[1] = s->vel = s->acc = s->pred_pos = s->pred_vel = nullptr;
    s->rad = s->rest = nullptr;
    s->ids = nullptr;
    s->partials = nullptr;
    s->escratch = nullptr;
    s->stage = nullptr;
    s->part_bytes = 0;
    s->escratch_n = 0;
    s->cap = 0;
}

int ensure_plan(gtd_system *s) {
    if (!s->variant_pinned) s->variant = tuned_variant(s->device, s->precision, s->n);
    if (s->plan.n == s->n && s->plan_prec == s->precision && s->plan.variant == s->variant && s->partials) {
        s->plan.near2 = near2_of(s->near_factor);
        return GTD_OK;
    }
    s->plan = make_plan(s->n, s->precision, s->device, s->variant);
    s->plan.near2 = near2_of(s->near_factor);
    s->plan_prec = s->precision;
    const size_t need = partial_bytes(s->plan);
    if (need > s->part_bytes) {
        cudaFree(s->partials);
        s->partials = nullptr;
        GTD_CUDA(cudaMalloc(&s->partials, need));
        s->part_bytes = need;
    }
    return GTD_OK;
}

static int ensure_pred(gtd_system *s) {
    if (s->pred_pos) return GTD_OK;
    GTD_CUDA(cudaMalloc(&s->pred_pos, sizeof(double4) * (size_t)s->cap));
    GTD_CUDA(cudaMalloc(&s->pred_vel, sizeof(double4) * (size_t)s->cap));
    return GTD_OK;
}

// Force at `src` into acc (and the integrator epilogue); counts launches.
static int collect_force_timing(gtd_system *s) {
    if (s->ev_used == 0) return GTD_OK;
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    for (size_t k = 0; k + 1 < s->ev_used; k += 2) {
        float ms = 0.f;
        GTD_CUDA(cudaEventElapsedTime(&ms, s->ev_pool[k], s->ev_pool[k + 1]));
        s->force_ms += ms;
        s->force_launches += 1;
    }
    s->ev_used = 0;
    return GTD_OK;
}

static int timed_event(gtd_system *s) {
    if (s->ev_used == s->ev_pool.size()) {
        if (s->ev_pool.size() >= 4096) {
            int rc = collect_force_timing(s);
            if (rc) return rc;
        } else {
            cudaEvent_t e;
            GTD_CUDA(cudaEventCreate(&e));
            s->ev_pool.push_back(e);
        }
    }
    GTD_CUDA(cudaEventRecord(s->ev_pool[s->ev_used++], s->stream));
    return GTD_OK;
}

int force_and_integrate(gtd_system *s, const double4 *src, int epi, const StepArgs &st) {
    int rc;
    if (s->precision == GTD_PREC_F64 && s->n <= kFusedMaxN) {
        if (s->time_force && (rc = timed_event(s))) return rc;
        rc = launch_fused_small(s->n, src, s->G, epi, st, s->stream);
        if (rc) return rc;
        if (s->time_force && (rc = timed_event(s))) return rc;
        s->launches += 1;
        return GTD_OK;
    }
    rc = ensure_plan(s);
    if (rc) return rc;
    if (s->time_force && (rc = timed_event(s))) return rc;
    rc = launch_force(s->precision, s->plan, src, s->G, s->partials, s->stream);
    if (rc) return rc;
    if (s->time_force && (rc = timed_event(s))) return rc;
    rc = launch_integrate(s->plan, s->partials, epi, st, s->stream);
    if (rc) return rc;
    s->launches += 2;
    return GTD_OK;
}

static StepArgs step_args(gtd_system *s, const double4 *src, bool last) {
    StepArgs a{};
    a.n = s->n;
    a.src = src;
    a.cur = s->pm[s->cur];
    a.dst = s->pm[s->cur ^ 1];
    a.vel = s->vel;
    a.acc = s->acc;
    a.pred_pos = s->pred_pos;
    a.pred_vel = s->pred_vel;
    a.h = s->dt;
    a.hp = s->dt;
    a.last = last ? 1 : 0;
    return a;
}

// One direct-summation step of `method` (the bodies of the evolve loops, gregsys.hpp:2666-3039).
static int direct_step(gtd_system *s, int method, bool last) {
    int rc = GTD_OK;
    switch (method) {
        case GTD_LEAPFROG_KDK: {
            if (s->synced) {
                rc = launch_kick_drift(s->n, s->pm[s->cur], s->pm[s->cur ^ 1], s->vel, s->acc, s->dt, s->stream);
                if (rc) return rc;
                s->launches += 1;
                s->cur ^= 1;
            }
            StepArgs a = step_args(s, s->pm[s->cur], last);
            rc = force_and_integrate(s, s->pm[s->cur], EPI_KDK, a);
            if (rc) return rc;
            if (!last) s->cur ^= 1;
            s->synced = last;
            return GTD_OK;
        }
        case GTD_LEAPFROG_DKD: {
            if (s->synced) {
                rc = launch_half_drift(s->n, s->pm[s->cur], s->pm[s->cur ^ 1], s->vel, s->dt, s->stream);
                if (rc) return rc;
                s->launches += 1;
                s->cur ^= 1;
            }
            StepArgs a = step_args(s, s->pm[s->cur], last);
            rc = force_and_integrate(s, s->pm[s->cur], EPI_DKD, a);
            if (rc) return rc;
            s->cur ^= 1;
            s->synced = last;
            return GTD_OK;
        }
        case GTD_EULER: {
            StepArgs a = step_args(s, s->pm[s->cur], true);
            rc = force_and_integrate(s, s->pm[s->cur], EPI_EULER, a);
            if (rc) return rc;
            s->cur ^= 1;
            return GTD_OK;
        }
        case GTD_MODIFIED_EULER:
        case GTD_MIDPOINT: {
            rc = ensure_pred(s);
            if (rc) return rc;
            StepArgs a = step_args(s, s->pm[s->cur], true);
            a.hp = method == GTD_MIDPOINT ? 0.5 * s->dt : s->dt;
            rc = force_and_integrate(s, s->pm[s->cur], EPI_PREDICT, a);
            if (rc) return rc;
            StepArgs b = step_args(s, s->pred_pos, true);
            rc = force_and_integrate(s, s->pred_pos, method == GTD_MIDPOINT ? EPI_CORR_MIDPOINT : EPI_CORR_MEULER, b);
            if (rc) return rc;
            s->cur ^= 1;
            return GTD_OK;
        }
        default:
            return fail(GTD_ERR_UNSUPPORTED, "method %d has no direct-summation step", method);
    }
}

// gtd::system::check_option, gregsys.hpp:1406-1411 (accepts nearly every value, like the original).
static bool check_option(int option) {
    const uint16_t lo = (uint16_t)(option & 0x0000ffff);
    const uint16_t hi = (uint16_t)((unsigned)option >> 16);
    return !(lo & (lo - 1)) || !lo || lo > GTD_RK4 || !(hi & (hi - 1)) || hi > 2;
}

// The branch of evolve() a method value selects, in the reference's if/else order
// (gregsys.hpp:2626-3059).  Returns 0 when no branch does any work.
static int select_branch(int method) {
    if ((method & GTD_TWO_BODY) == GTD_TWO_BODY) return GTD_TWO_BODY;
    if ((method & GTD_EULER) == GTD_EULER) return GTD_EULER;
    if ((method & GTD_MODIFIED_EULER) == GTD_MODIFIED_EULER) return GTD_MODIFIED_EULER;
    if ((method & GTD_MIDPOINT) == GTD_MIDPOINT) return GTD_MIDPOINT;
    if ((method & GTD_LEAPFROG_KDK) == GTD_LEAPFROG_KDK) return GTD_LEAPFROG_KDK;
    if ((method & GTD_LEAPFROG_DKD) == GTD_LEAPFROG_DKD) return GTD_LEAPFROG_DKD;
    if ((method & GTD_RK4) == GTD_RK4) return GTD_RK4;
    if ((method & GTD_RK3_8) == GTD_RK3_8) return GTD_RK3_8;
    return 0;
}

int run_collisions(gtd_system *s);  // collide.cu
int bh_evolve_kdk(gtd_system *s, uint64_t steps);  // octree.cu
int bh_accelerations(gtd_system *s, double *a3, uint32_t *n_inter);  // octree.cu

int output_rows(gtd_system *s, std::vector<int64_t> &row) {
    const int64_t n = s->n;
    row.resize((size_t)n);
    if (!s->ordered && n == s->n_uploaded) {
        for (int64_t i = 0; i < n; ++i) row[(size_t)i] = i;
        return GTD_OK;
    }
    std::vector<int32_t> ids((size_t)n);
    GTD_CUDA(cudaMemcpyAsync(ids.data(), s->ids, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    if (n == s->n_uploaded) {
        for (int64_t i = 0; i < n; ++i) row[(size_t)i] = ids[(size_t)i];
        return GTD_OK;
    }
    std::vector<int64_t> idx((size_t)n);
    for (int64_t i = 0; i < n; ++i) idx[(size_t)i] = i;
    std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return ids[(size_t)a] < ids[(size_t)b]; });
    for (int64_t k = 0; k < n; ++k) row[(size_t)idx[(size_t)k]] = k;
    return GTD_OK;
}

// The mixed kernel centres each row's FP32 frame on the row; Hilbert-ordered bodies keep rows
// compact, so the mixed path reorders at the start of an evolve and every reorder_interval steps.
static int maybe_reorder(gtd_system *s, bool force) {
    // collisions scan the bodies in upload order (as the reference scans its vector): no reordering
    if (s->precision != GTD_PREC_MIXED || s->n < 2 || s->coll != GTD_NO_COLL) return GTD_OK;
    if (!force && s->steps_since_reorder < (uint64_t)s->reorder_interval) return GTD_OK;
    s->steps_since_reorder = 0;
    return reorder_bodies(s);
}

static int evolve_begin(gtd_system *s, int method) {
    s->method = method;
    s->begun = true;
    s->synced = true;
    s->rec_step = 0;
    s->rec_frames.clear();
    s->rec_states.clear();
    if (s->n == 0) return GTD_OK;
    if (s->rec_every && s->coll == GTD_MERGE_COLL)
        return fail(GTD_ERR_UNSUPPORTED, "trajectory recording with merging collisions is not supported");
    int rc = maybe_reorder(s, true);
    if (rc) return rc;
    if (s->rec_every) {
        rc = record_frame(s, 0);
        if (rc) return rc;
    }
    if (method == GTD_LEAPFROG_KDK) {
        StepArgs a = step_args(s, s->pm[s->cur], true);
        return force_and_integrate(s, s->pm[s->cur], EPI_ACC, a);
    }
    return GTD_OK;
}

// Steady-state steps with no host logic between them (FP64, no collisions, recording or force
// timing) are replayed from a CUDA graph of kGraphSteps steps: at small N the launches, not the
// arithmetic, set the step time.  kGraphSteps is even, so the position double buffer ends where it
// started and one graph per (method, buffer parity, parameters) serves every replay.
constexpr int kGraphSteps = 16;

static bool graph_eligible(const gtd_system *s) {
    if (s->precision != GTD_PREC_F64 || s->coll != GTD_NO_COLL || s->rec_every || s->time_force || s->step_hook)
        return false;
    if ((s->method == GTD_LEAPFROG_KDK || s->method == GTD_LEAPFROG_DKD) && s->synced) return false;
    return true;
}

void release_graph(gtd_system *s) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
}

static int run_graph_chunk(gtd_system *s) {
    int rc = ensure_plan(s);  // no allocation inside the capture
    if (rc) return rc;
    if (s->method == GTD_MODIFIED_EULER || s->method == GTD_MIDPOINT) {
        rc = ensure_pred(s);
        if (rc) return rc;
    }
    const GraphKey key{s->method, s->cur, s->n, s->variant, s->G, s->dt, s->pm[0], s->pm[1], s->partials,
                       s->pred_pos};
    if (!s->graph || !(key == s->graph_key)) {
        release_graph(s);
        const int cur0 = s->cur;
        const bool synced0 = s->synced;
        const uint64_t launches0 = s->launches;
        GTD_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        for (int c = 0; c < kGraphSteps && !rc; ++c) rc = direct_step(s, s->method, false);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
        s->graph_launches = s->launches - launches0;
        s->launches = launches0;  // captured, not yet run
        s->cur = cur0;
        s->synced = synced0;
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
        const cudaError_t ie = cudaGraphInstantiate(&s->graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            s->graph = nullptr;
            return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
        }
        s->graph_key = key;
    }
    GTD_CUDA(cudaGraphLaunch(s->graph, s->stream));
    s->launches += s->graph_launches;
    // the state after kGraphSteps steps: same buffer parity, still unsynchronised
    return GTD_OK;
}

static int evolve_steps(gtd_system *s, uint64_t k) {
    if (!s->begun) return fail(GTD_ERR_INVALID_ARGUMENT, "gtd_system_evolve_steps before gtd_system_evolve_begin");
    if (s->n == 0 || k == 0) return GTD_OK;
    for (uint64_t i = 0; i < k; ++i) {
        // whole graph chunks while more than one chunk's worth of steps remains (the final step
        // runs on its own, with `last` set)
        while (k - i > (uint64_t)kGraphSteps && graph_eligible(s)) {
            int rc = run_graph_chunk(s);
            if (rc) return rc;
            i += kGraphSteps;
            s->rec_step += kGraphSteps;
            s->steps_since_reorder += kGraphSteps;
        }
        const bool rec = s->rec_every && (s->rec_step + 1) % s->rec_every == 0;
        const bool last = (i + 1 == k) || s->coll != GTD_NO_COLL || rec || s->step_hook;
        int rc = maybe_reorder(s, false);
        if (rc) return rc;
        rc = direct_step(s, s->method, last);
        if (rc) return rc;
        s->steps_since_reorder += 1;
        s->rec_step += 1;
        if (s->step_hook) {  // for_all_bods' place: after the update, before the collision pass
            rc = s->step_hook(s->step_hook_user);
            if (rc) return rc < 0 ? fail(GTD_ERR_INVALID_ARGUMENT, "step hook returned %d", rc) : rc;
        }
        if (s->coll != GTD_NO_COLL) {
            rc = run_collisions(s);
            if (rc) return rc;
        }
        if (rec) {
            rc = record_frame(s, s->rec_step);
            if (rc) return rc;
        }
    }
    return GTD_OK;
}

// Entry points for the callback-driven evolve (callbacks.cu).
int cb_evolve_begin(gtd_system *s, int method) { return evolve_begin(s, method); }
int cb_direct_step(gtd_system *s) { return direct_step(s, s->method, true); }
int cb_maybe_reorder(gtd_system *s) {
    const int rc = maybe_reorder(s, false);
    s->steps_since_reorder += 1;
    return rc;
}
int cb_select_branch(int method) { return check_option(method) ? select_branch(method) : 0; }
// Allocates what the steps of s->method use, so that they can be captured.
int cb_prepare_steps(gtd_system *s) {
    int rc = GTD_OK;
    if (!(s->precision == GTD_PREC_F64 && s->n <= kFusedMaxN)) rc = ensure_plan(s);
    if (!rc && (s->method == GTD_MODIFIED_EULER || s->method == GTD_MIDPOINT)) rc = ensure_pred(s);
    return rc;
}

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------
extern "C" {

const char *gtd_last_error(void) { return gtd::last_error(); }

int gtd_abi_version(void) { return GTD_ABI_VERSION; }

int gtd_check_option(int option, int *accepted) {
    if (!accepted) return fail(GTD_ERR_INVALID_ARGUMENT, "accepted is NULL");
    *accepted = check_option(option) ? 1 : 0;
    return GTD_OK;
}

int gtd_device_count(int *count) {
    if (!count) return fail(GTD_ERR_INVALID_ARGUMENT, "count is NULL");
    *count = 0;
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        return fail(GTD_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    }
    return GTD_OK;
}

int gtd_system_create(gtd_system **out, int device, int precision) {
    if (!out) return fail(GTD_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (precision != GTD_PREC_F64 && precision != GTD_PREC_MIXED)
        return fail(GTD_ERR_INVALID_ARGUMENT, "unknown precision %d", precision);
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) {
        cudaGetLastError();
        return fail(GTD_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= nd) return fail(GTD_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    DeviceGuard g(device);
    gtd_system *s = new (std::nothrow) gtd_system();
    if (!s) return fail(GTD_ERR_OUT_OF_MEMORY, "host allocation failed");
    s->device = device;
    s->precision = precision;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
    if (e != cudaSuccess) {
        int rc = cuda_fail(e, "stream/event creation", __FILE__, __LINE__);
        delete s;
        return rc;
    }
    *out = s;
    return GTD_OK;
}

int gtd_system_destroy(gtd_system *s) {
    if (!s) return GTD_OK;
    DeviceGuard g(s->device);
    cudaStreamSynchronize(s->stream);
    release_bodies(s);
    release_tree(s);
    release_collide(s);
    release_nsys(s);
    release_record(s);
    release_io(s);
    release_graph(s);
    release_callbacks(s);
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    cudaEventDestroy(s->ev0);
    cudaEventDestroy(s->ev1);
    cudaStreamDestroy(s->stream);
    delete s;
    return GTD_OK;
}

int gtd_system_set_params(gtd_system *s, double G, double dt, uint64_t iterations, double softening,
                          double bh_theta) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (!(dt > 0)) return fail(GTD_ERR_INVALID_ARGUMENT, "Time-step cannot be zero or negative.");
    if (iterations == 0) return fail(GTD_ERR_INVALID_ARGUMENT, "iterations cannot be zero");
    if (!(bh_theta >= 0) || bh_theta >= M_PI)
        return fail(GTD_ERR_INVALID_ARGUMENT,
                    "Error: opening angle cannot be negative or equal to or larger than PI radians.");
    if (!(softening >= 0)) return fail(GTD_ERR_INVALID_ARGUMENT, "softening cannot be negative");
    s->G = G;
    s->dt = dt;
    s->iterations = iterations;
    s->eps = softening;
    s->theta = bh_theta;
    return GTD_OK;
}

int gtd_system_set_collisions(gtd_system *s, int mode) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (mode != GTD_NO_COLL && mode != GTD_OVERLAP_COLL && mode != GTD_MERGE_COLL)
        return fail(GTD_ERR_INVALID_ARGUMENT, "unknown collision mode %d", mode);
    s->coll = mode;
    return GTD_OK;
}

int gtd_system_upload(gtd_system *s, int64_t n, const double *m, const double *r, const double *rest,
                      const double *x3, const double *v3) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (n < 0 || n > (int64_t)INT32_MAX) return fail(GTD_ERR_CAPACITY, "body count %lld not supported", (long long)n);
    if (n > 0 && (!m || !x3)) return fail(GTD_ERR_INVALID_ARGUMENT, "masses and positions are required");
    DeviceGuard g(s->device);
    int rc = ensure_capacity(s, n);
    if (rc) return rc;
    s->n = n;
    s->n_uploaded = n;
    s->cur = 0;
    s->begun = false;
    s->synced = true;
    s->tree_valid = false;
    s->ordered = false;
    s->steps_since_reorder = 0;
    s->rec_frames.clear();  // recordings belong to the bodies they were made from
    s->rec_states.clear();
    if (n == 0) return GTD_OK;
    rc = device_upload(s, n, m, r, rest, x3, v3);
    if (rc) {  // a negative mass or radius: leave the handle empty
        s->n = s->n_uploaded = 0;
        return rc;
    }
    return GTD_OK;
}

int gtd_system_survivors(gtd_system *s, int64_t *upload_index) {
    if (!s || !upload_index) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(s->device);
    const int64_t n = s->n;
    if (n == 0) return GTD_OK;
    std::vector<int32_t> ids((size_t)n);
    GTD_CUDA(cudaMemcpyAsync(ids.data(), s->ids, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    std::sort(ids.begin(), ids.end());
    for (int64_t i = 0; i < n; ++i) upload_index[i] = ids[(size_t)i];
    return GTD_OK;
}

int gtd_system_num_bodies(const gtd_system *s, int64_t *n) {
    if (!s || !n) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    *n = s->n;
    return GTD_OK;
}

int gtd_system_download(gtd_system *s, int64_t *n_out, double *m, double *r, double *rest, double *x3, double *v3,
                        double *a3) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    DeviceGuard g(s->device);
    const int64_t n = s->n;
    if (n_out) *n_out = n;
    if (n == 0) return GTD_OK;
    return device_download(s, m, r, rest, x3, v3, a3);
}

}  // extern "C"

// Device acceleration array -> host triples in host row order.
int copy_acc_out(gtd_system *s, double *a3) { return device_download(s, nullptr, nullptr, nullptr, nullptr, nullptr, a3); }

extern "C" {

int gtd_system_evolve_begin(gtd_system *s, int method) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    DeviceGuard g(s->device);
    return evolve_begin(s, method);
}

int gtd_system_evolve_steps(gtd_system *s, uint64_t k) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    DeviceGuard g(s->device);
    int rc = evolve_steps(s, k);
    if (rc) return rc;
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    return GTD_OK;
}

int gtd_system_evolve(gtd_system *s, int method, int64_t *elapsed_ns) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (elapsed_ns) *elapsed_ns = 0;
    if (s->n == 0 || !check_option(method)) return GTD_OK;  // gregsys.hpp:2611-2612
    DeviceGuard g(s->device);
    const int branch = select_branch(method);
    const bool bh = (method & GTD_BARNES_HUT) == GTD_BARNES_HUT;
    if (branch == GTD_TWO_BODY) {
        if (s->n != 2) return fail(GTD_ERR_TWO_BODY, "two-body integration requires exactly two bodies");
        return GTD_OK;  // the reference performs no integration in this branch
    }
    if (branch == 0 || branch == GTD_RK4 || branch == GTD_RK3_8) return GTD_OK;  // empty branches
    if (bh && branch == GTD_EULER)
        return fail(GTD_ERR_UNSUPPORTED, "Barnes-Hut Euler never advances in the reference (steps is not "
                                         "incremented, gregsys.hpp:2631-2665); refusing to loop forever");
    if (bh && branch != GTD_LEAPFROG_KDK) return GTD_OK;  // empty Barnes-Hut branches
    GTD_CUDA(cudaEventRecord(s->ev0, s->stream));
    int rc;
    if (bh) {
        s->rec_frames.clear();  // the reference records nothing in its Barnes-Hut branches
        s->rec_states.clear();
        rc = bh_evolve_kdk(s, s->iterations);
    } else {
        rc = evolve_begin(s, branch);
        if (!rc) rc = evolve_steps(s, s->iterations);
    }
    if (rc) return rc;
    GTD_CUDA(cudaEventRecord(s->ev1, s->stream));
    GTD_CUDA(cudaEventSynchronize(s->ev1));
    float ms = 0.f;
    GTD_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    if (elapsed_ns) *elapsed_ns = (int64_t)((double)ms * 1e6);
    return GTD_OK;
}

int gtd_system_accelerations(gtd_system *s, int method, double *a3) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    DeviceGuard g(s->device);
    if (s->n == 0) return GTD_OK;
    if ((method & GTD_BARNES_HUT) == GTD_BARNES_HUT) return bh_accelerations(s, a3, nullptr);
    int rc = maybe_reorder(s, true);
    if (rc) return rc;
    StepArgs a = step_args(s, s->pm[s->cur], true);
    rc = force_and_integrate(s, s->pm[s->cur], EPI_ACC, a);
    if (rc) return rc;
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    if (a3) return copy_acc_out(s, a3);
    return GTD_OK;
}

int gtd_system_energy(gtd_system *s, double *ke, double *pe, double *p3, double *com3) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    DeviceGuard g(s->device);
    double out[9] = {0};
    if (s->n > 0) {
        const int64_t need = energy_scratch_doubles(s->n);
        if (need > s->escratch_n) {
            cudaFree(s->escratch);
            s->escratch = nullptr;
            GTD_CUDA(cudaMalloc(&s->escratch, sizeof(double) * (size_t)need));
            s->escratch_n = need;
        }
        int rc = launch_energy(s->n, s->pm[s->cur], s->vel, s->G, s->escratch, s->escratch_n, s->stream);
        if (rc) return rc;
        s->launches += 1;
        std::vector<double> h((size_t)need);
        GTD_CUDA(cudaMemcpyAsync(h.data(), s->escratch, sizeof(double) * (size_t)need, cudaMemcpyDeviceToHost,
                                 s->stream));
        GTD_CUDA(cudaStreamSynchronize(s->stream));
        finish_energy(h.data(), s->n, out);
    }
    if (ke) *ke = out[0];
    if (pe) *pe = out[1];
    if (p3) { p3[0] = out[2]; p3[1] = out[3]; p3[2] = out[4]; }
    if (com3) {
        for (int k = 0; k < 3; ++k) com3[k] = out[8] > 0 ? out[5 + k] / out[8] : 0.0;
    }
    return GTD_OK;
}

int gtd_system_launch_count(const gtd_system *s, uint64_t *count) {
    if (!s || !count) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    *count = s->launches;
    return GTD_OK;
}

int gtd_direct_variant_count(int precision, int *count) {
    if (!count) return fail(GTD_ERR_INVALID_ARGUMENT, "count is NULL");
    *count = variant_count(precision);
    return GTD_OK;
}

int gtd_direct_variant_info(int precision, int variant, int *i_per_thread, int *fold) {
    return variant_info(precision, variant, i_per_thread, fold);
}

int gtd_system_set_direct_variant(gtd_system *s, int variant) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (variant >= variant_count(s->precision)) return fail(GTD_ERR_INVALID_ARGUMENT, "variant %d out of range", variant);
    s->variant_pinned = variant >= 0;
    if (variant >= 0) s->variant = variant;
    return GTD_OK;
}

int gtd_system_direct_plan_info(gtd_system *s, int64_t *units, int64_t *partial_bytes_out) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (s->n == 0) return fail(GTD_ERR_INVALID_ARGUMENT, "no bodies");
    DeviceGuard g(s->device);
    int rc = ensure_plan(s);
    if (rc) return rc;
    if (units) *units = s->plan.segs > 0 ? s->plan.units : s->plan.total;
    if (partial_bytes_out) *partial_bytes_out = (int64_t)partial_bytes(s->plan);
    return GTD_OK;
}

int gtd_system_set_mixed_near_factor(gtd_system *s, double k) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (!(k == k)) return fail(GTD_ERR_INVALID_ARGUMENT, "near factor is NaN");
    s->near_factor = k;
    s->plan.near2 = near2_of(k);
    return GTD_OK;
}

int gtd_system_autotune_direct(gtd_system *s, int reps, int *best, double *best_ms) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (s->n == 0) return fail(GTD_ERR_INVALID_ARGUMENT, "autotune needs bodies");
    DeviceGuard g(s->device);
    if (reps < 1) reps = 1;
    int rc = maybe_reorder(s, true);
    if (rc) return rc;
    struct RestorePin {
        gtd_system *s;
        bool pinned;
        ~RestorePin() { s->variant_pinned = pinned; }
    } restore{s, s->variant_pinned};
    s->variant_pinned = true;  // while timing, ensure_plan keeps the variant under test
    int arg = s->variant;
    double bestv = 1e300;
    for (int v = 0; v < variant_count(s->precision); ++v) {
        s->variant = v;
        rc = ensure_plan(s);
        if (rc) return rc;
        // warm-up launch, then the median of `reps` timed force launches
        rc = launch_force(s->precision, s->plan, s->pm[s->cur], s->G, s->partials, s->stream);
        if (rc) return rc;
        std::vector<float> t(reps);
        for (int k = 0; k < reps; ++k) {
            GTD_CUDA(cudaEventRecord(s->ev0, s->stream));
            rc = launch_force(s->precision, s->plan, s->pm[s->cur], s->G, s->partials, s->stream);
            if (rc) return rc;
            GTD_CUDA(cudaEventRecord(s->ev1, s->stream));
            GTD_CUDA(cudaEventSynchronize(s->ev1));
            GTD_CUDA(cudaEventElapsedTime(&t[k], s->ev0, s->ev1));
        }
        s->launches += (uint64_t)reps + 1;
        std::sort(t.begin(), t.end());
        const double med = t[reps / 2];
        if (med < bestv) {
            bestv = med;
            arg = v;
        }
    }
    s->variant = arg;
    remember_variant(s->device, s->precision, s->n, arg);
    s->variant_pinned = restore.pinned;
    rc = ensure_plan(s);
    if (rc) return rc;
    if (best) *best = arg;
    if (best_ms) *best_ms = bestv;
    return GTD_OK;
}

int gtd_system_stream(const gtd_system *s, void **stream) {
    if (!s || !stream) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    *stream = (void *)s->stream;
    return GTD_OK;
}

int gtd_system_time_force_kernels(gtd_system *s, int enable) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    DeviceGuard g(s->device);
    int rc = collect_force_timing(s);
    if (rc) return rc;
    s->time_force = enable != 0;
    return GTD_OK;
}

int gtd_system_force_timing(gtd_system *s, double *total_ms, uint64_t *launches, int reset) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    DeviceGuard g(s->device);
    int rc = collect_force_timing(s);
    if (rc) return rc;
    if (total_ms) *total_ms = s->force_ms;
    if (launches) *launches = s->force_launches;
    if (reset) {
        s->force_ms = 0.0;
        s->force_launches = 0;
    }
    return GTD_OK;
}

}  // extern "C"
