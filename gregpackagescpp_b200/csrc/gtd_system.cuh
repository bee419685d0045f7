// The device-resident state behind a gtd_system handle (include/gtd_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <future>
#include <string>
#include <vector>

#include "gtd_internal.cuh"

// What a captured step graph depends on.
struct GraphKey {
    int method = 0, cur = 0;
    int64_t n = 0;
    int variant = 0;
    double G = 0, dt = 0;
    const void *p0 = nullptr, *p1 = nullptr, *part = nullptr, *pred = nullptr;
    bool operator==(const GraphKey &o) const {
        return method == o.method && cur == o.cur && n == o.n && variant == o.variant && G == o.G && dt == o.dt &&
               p0 == o.p0 && p1 == o.p1 && part == o.part && pred == o.pred;
    }
};

struct gtd_system {
    int device = 0;
    int precision = GTD_PREC_F64;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    // gtd::system scalars (gregsys.hpp:171-213); G defaults to G_SI
    double G = 6.6743e-11;
    double dt = 1.0;
    uint64_t iterations = 1000;
    double eps = 0.0;
    double theta = 1.0471975511965976;  // pi/3, gregsys.hpp:212
    int coll = GTD_NO_COLL;

    // bodies: position + mass double-buffered, velocity, acceleration, radius, restitution
    int64_t n = 0, cap = 0;
    int64_t n_uploaded = 0;  // bodies at upload (n shrinks after merges)
    double4 *pm[2] = {nullptr, nullptr};
    int cur = 0;
    double4 *vel = nullptr, *acc = nullptr;
    double4 *pred_pos = nullptr, *pred_vel = nullptr;
    double *rad = nullptr, *rest = nullptr;
    int32_t *ids = nullptr;  // upload index of the body in each slot
    double4 *stage = nullptr;  // pinned host staging (4 double4 per body)

    // direct summation
    gtd::ForcePlan plan;
    int plan_prec = -1;
    int variant = 0;              // force-kernel variant in use
    bool variant_pinned = false;  // set by gtd_system_set_direct_variant; else the process-wide choice
    double near_factor = gtd::kDefaultNearFactor;  // mixed kernel's precise-path factor K
    double *partials = nullptr;
    size_t part_bytes = 0;
    double *escratch = nullptr;
    int64_t escratch_n = 0;

    // evolve() state
    int method = 0;
    bool begun = false;
    bool synced = true;
    uint64_t launches = 0;

    // optional per-launch timing of the force kernel (instrumentation)
    bool time_force = false;
    std::vector<cudaEvent_t> ev_pool;  // pairs (start, stop), reused
    size_t ev_used = 0;
    double force_ms = 0.0;
    uint64_t force_launches = 0;

    // Barnes-Hut linear octree (octree.cu); arrays indexed by sorted slot [n] or by node [cap]
    bool tree_valid = false;
    int tree_float = 1;
    int64_t tree_n = 0;                 // bodies the n-sized arrays were sized for
    int64_t node_cap = 0;               // nodes the node-sized arrays hold
    int64_t n_nodes = 0, n_leaves = 0;
    void *tree_nbuf = nullptr, *tree_kbuf = nullptr;
    unsigned long long *codes = nullptr, *codes_alt = nullptr;
    int32_t *perm = nullptr, *perm_alt = nullptr;  // slot -> body index
    int32_t *lcp = nullptr;
    uint32_t *node_start = nullptr;     // [n+1] exclusive scan of nodes started per slot
    int32_t *own_leaf = nullptr;
    void *slot_pos = nullptr;           // float4 or double4 (x, y, z, G m) per slot
    void *slot_acc = nullptr;           // float4 or double4 per slot
    uint32_t *slot_cnt = nullptr;       // interactions per slot
    uint32_t *scratch = nullptr;        // radix / scan scratch
    size_t scratch_words = 0;
    double *bbox_part = nullptr;        // per-block min/max partials
    double *box_dev = nullptr;          // btm xyz, top xyz
    int *status = nullptr;              // device error word
    uint32_t *host_total = nullptr;     // pinned: node total, status
    int8_t *ndepth = nullptr, *nleaf = nullptr;
    int32_t *nfirst = nullptr, *ncount = nullptr, *nskip = nullptr;
    double4 *ncom = nullptr;            // FP64 centre of mass xyz + mass
    double *nwidth = nullptr;           // top.x - btm.x in T
    void *nwalk_a = nullptr;            // walk record: com xyz + G M (float4 / double4)
    int4 *nwalk_b = nullptr;            // walk record: skip, first, count | leaf<<31, width^2 bits
    double *nwalk_w2 = nullptr;         // width^2 for the FP64 walk
    int walk_variant = -1;              // float walk records: -1 default (interleaved), 0 split, 1 interleaved
    int walk_interleaved = 0;           // layout of the built float tree's records (1: A,B adjacent, 32 B)
    int32_t *depth_list = nullptr;      // internal nodes grouped by depth
    uint32_t *depth_off = nullptr;      // [22] offsets + [22] cursors
    double box[6] = {0, 0, 0, 0, 0, 0};
    uint32_t *bh_ninter = nullptr;      // interactions per body (body order)

    // spatial reordering of the bodies for the mixed-precision direct sum
    int reorder_interval = 16;
    uint64_t steps_since_reorder = 0;
    bool ordered = false;
    double4 *sc4 = nullptr;
    double *sc1 = nullptr;
    int32_t *sci = nullptr;

    // collisions (collide.cu)
    void *coll_buf = nullptr;
    size_t coll_bytes = 0;
    double *coll_nbox = nullptr;  // Barnes-Hut cell bounds, 6 per node (bh_s_coll)
    int64_t coll_nbox_cap = 0;

    // .nsys chunk staging (nsys.cu)
    void *nsys_dev = nullptr, *nsys_host = nullptr;
    size_t nsys_dev_bytes = 0, nsys_host_bytes = 0;
    // snapshot writes in flight: pinned buffer, copy-done event and host writer per slot
    struct NsysWrite {
        void *buf = nullptr;
        size_t bytes = 0;
        cudaEvent_t done = nullptr;
        std::future<std::pair<int, std::string>> job;  // status, message (bytes written on success)
        int64_t written = 0;
    } nsys_w[2];
    int nsys_next = 0, nsys_last = -1;

    // captured steady-state steps (system.cu)
    cudaGraphExec_t graph = nullptr;
    GraphKey graph_key;
    uint64_t graph_launches = 0;

    // host-array staging on the device (io.cu)
    void *io_dev = nullptr;
    size_t io_bytes = 0;

    // evolve callbacks (callbacks.cu).  Host: a hook called inside every step of evolve_steps at
    // for_all_bods' place.  Device: continue_ev_if / for_each_bod / for_all_bods as GPU work.
    gtd_step_hook step_hook = nullptr;
    void *step_hook_user = nullptr;
    struct DeviceCallbacks {
        int cont_kind = 0;  // 0 none (run `iterations` steps), 1 user hook, 2 rest below a bound
        gtd_device_hook cont_fn = nullptr;
        void *cont_user = nullptr;
        double min_max_cor = 0.0;
        uint64_t probing_iters = 0;
        int all_kind = 0;   // 0 none, 1 user hook, 2 restitution from the distance to the carried COM
        gtd_device_hook all_fn = nullptr;
        void *all_user = nullptr;
        double min_cor = 0.0, max_cor = 1.0, scale_factor = 1.0, n_exp = 1.0;
        int mass_weighted = 0;
        gtd_device_hook each_fn = nullptr;
        void *each_user = nullptr;
    } cb;
    void *cb_ctl = nullptr;   // device control block of the device-driven loop
    void *cb_host = nullptr;  // pinned mirror of it
    uint64_t cb_waits = 0;    // host waits of the last callback-driven evolve
    bool cb_graph = false;    // whether it ran as graph chunks

    // trajectory frames (record.cu): every rec_every-th state of a direct-summation evolve
    uint64_t rec_every = 0;
    uint64_t rec_step = 0;               // steps since evolve_begin
    std::vector<double> rec_frames;      // [frames][rec_n][8]: x y z vx vy vz ke pe
    std::vector<int64_t> rec_states;     // step index of each frame
    int64_t rec_n = 0;
    double *rec_dev = nullptr;
    int64_t rec_dev_n = 0;
};

// Makes the handle's device current for the scope of an entry point.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        cudaGetDevice(&prev);
        if (prev != d) cudaSetDevice(d);
    }
    ~DeviceGuard() {
        int now = -1;
        cudaGetDevice(&now);
        if (prev >= 0 && now != prev) cudaSetDevice(prev);
    }
};

void release_bodies(gtd_system *s);
void release_tree(gtd_system *s);
// bh_s_coll on the current tree (collide.cu); the tree must have been built at the current positions
int run_bh_collisions(gtd_system *s);
int reorder_bodies(gtd_system *s);
int restore_upload_order(gtd_system *s);
// row[s] = host row of device slot s: ascending upload index among the live bodies
int output_rows(gtd_system *s, std::vector<int64_t> &row);
// device accelerations -> host triples in host row order (synchronises the stream)
int copy_acc_out(gtd_system *s, double *a3);
void release_collide(gtd_system *s);
void release_nsys(gtd_system *s);
void release_record(gtd_system *s);
void release_io(gtd_system *s);
void release_graph(gtd_system *s);
void release_callbacks(gtd_system *s);
// overwrite live bodies in download order, keeping accelerations and the evolve state (io.cu)
int device_update(gtd_system *s, const double *m, const double *r, const double *rest, const double *x3,
                  const double *v3);
// overlap collision pass split for capture (collide.cu); hooks: work of the callback loop that the
// pass's resolving CTA takes over (callbacks.cuh), or nullptr
namespace gtd {
struct PassHooks;
}
int prepare_collisions(gtd_system *s, int **status);
int enqueue_collisions(gtd_system *s, const gtd::PassHooks *hooks);
int run_collisions(gtd_system *s);
// pieces of evolve for the callback-driven loop (system.cu)
int cb_evolve_begin(gtd_system *s, int method);
int cb_direct_step(gtd_system *s);
int cb_maybe_reorder(gtd_system *s);
int cb_select_branch(int method);
int cb_prepare_steps(gtd_system *s);
// caller's arrays (upload order) <-> device bodies, converted on the device (io.cu)
int device_upload(gtd_system *s, int64_t n, const double *m, const double *r, const double *rest, const double *x3,
                  const double *v3);
int device_download(gtd_system *s, double *m, double *r, double *rest, double *x3, double *v3, double *a3);
int record_frame(gtd_system *s, uint64_t state);
int ensure_body_capacity(gtd_system *s, int64_t n);
int set_loaded_bodies(gtd_system *s, int64_t n);
int ensure_plan(gtd_system *s);
int force_and_integrate(gtd_system *s, const double4 *src, int epi, const gtd::StepArgs &st);
