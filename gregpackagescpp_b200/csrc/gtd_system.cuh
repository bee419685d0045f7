// The device-resident state behind a gtd_system handle (include/gtd_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "gtd_internal.cuh"

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

    // Barnes-Hut tree (octree.cu)
    bool tree_valid = false;
    int tree_float = 1;
    int64_t tree_cap_n = 0, tree_cap_nodes = 0;
    int64_t n_nodes = 0, n_leaves = 0;
    double box[6] = {0, 0, 0, 0, 0, 0};
    void *tree_buf = nullptr;  // one allocation carved into the arrays below
    size_t tree_bytes = 0;
    unsigned long long *codes = nullptr, *codes_alt = nullptr;
    int32_t *perm = nullptr, *perm_alt = nullptr;
    int32_t *lcp = nullptr, *node_start = nullptr;
    int8_t *ndepth = nullptr, *nleaf = nullptr;
    int32_t *nfirst = nullptr, *ncount = nullptr, *nskip = nullptr, *own_leaf = nullptr;
    double4 *ncom = nullptr;      // com xyz + mass (FP64)
    double *nwidth = nullptr;
    float4 *nwalk = nullptr;      // walk record: com xyz (FP32) + G M
    float *nwidth2 = nullptr;     // width^2 / theta^2 (FP32 criterion)
    float4 *sorted_pos = nullptr; // bodies in slot order: x y z (FP32) + G m
    uint32_t *scan_tmp = nullptr; // radix histograms / scan scratch
    int32_t *depth_list = nullptr, *depth_off = nullptr;
    int *status = nullptr;        // device error word (placement / indistinguishable)
    int64_t *counters = nullptr;  // device scalars: node total, etc.
    double *box_dev = nullptr;

    // collisions (collide.cu)
    void *coll_buf = nullptr;
    size_t coll_bytes = 0;
};

void release_bodies(gtd_system *s);
void release_tree(gtd_system *s);
void release_collide(gtd_system *s);
int ensure_plan(gtd_system *s);
int force_and_integrate(gtd_system *s, const double4 *src, int epi, const gtd::StepArgs &st);
