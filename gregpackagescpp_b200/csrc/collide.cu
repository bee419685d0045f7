// Radius-overlap collisions of gtd::system on the device.
//
//  * GTD_OVERLAP_COLL - s_coll without GREGSYS_MERGERS (gregsys.hpp:690-914): for each body o in
//    order, the later bodies i overlapping it (|x_i - x_o| < r_o + r_i) are taken in ascending
//    distance (a std::map keyed by distance keeps the first of equal keys), their momenta along
//    the unit separation are snapshotted for the whole group, and each pair that is approaching
//    gets the restitution impulse with the mean coefficient of the two bodies.
//  * GTD_MERGE_COLL   - overlap merges in the scan order of check_overlap (gregsys.hpp:307-342)
//    as that routine intends it: a merged body is re-checked against every body from index 0;
//    the merge itself is body::operator+= (gregbod.hpp:1066-1082): mass-weighted position,
//    velocity and acceleration, summed mass, r = cbrt(r1^3 + r2^3), mean restitution.
//
// Detection of all overlapping pairs is a tiled O(N^2) kernel (FP64); the order-dependent
// resolution runs on one thread (restitution) or one block (merges), as the reference's
// sequential loops define the result.
#include <cuda_runtime.h>

#include <algorithm>

#include "gtd_internal.cuh"
#include "gtd_system.cuh"

namespace gtd {

constexpr int kCT = 256;
constexpr int kMaxCand = 1 << 16;

struct Cand {
    int32_t o, i;
    double dist;
};

// All pairs o < i with dist < r_o + r_i; appends (o, i, dist) to the candidate list.
__global__ void __launch_bounds__(kCT) overlap_pairs_kernel(int64_t n, const double4 *pm, const double *rad,
                                                            Cand *cand, int *count, int cap) {
    __shared__ double4 tp[kCT];
    __shared__ double tr[kCT];
    const int64_t o = (int64_t)blockIdx.x * kCT + threadIdx.x;
    const double4 po = o < n ? pm[o] : make_double4(0, 0, 0, 0);
    const double ro = o < n ? rad[o] : 0.0;
    const int64_t first_tile = (int64_t)blockIdx.x * kCT;
    for (int64_t j0 = first_tile; j0 < n; j0 += kCT) {
        const int64_t j = j0 + threadIdx.x;
        tp[threadIdx.x] = j < n ? pm[j] : make_double4(0, 0, 0, 0);
        tr[threadIdx.x] = j < n ? rad[j] : 0.0;
        __syncthreads();
        if (o < n) {
            const int lim = (int)min((int64_t)kCT, n - j0);
            for (int jj = 0; jj < lim; ++jj) {
                const int64_t i = j0 + jj;
                if (i <= o) continue;
                const double4 q = tp[jj];
                const double dx = __dsub_rn(q.x, po.x), dy = __dsub_rn(q.y, po.y), dz = __dsub_rn(q.z, po.z);
                const double d = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
                const double rsum = __dadd_rn(ro, tr[jj]);
                if (rsum > d) {
                    const int k = atomicAdd(count, 1);
                    if (k < cap) cand[k] = Cand{(int32_t)o, (int32_t)i, d};
                }
            }
        }
        __syncthreads();
    }
}

__device__ __forceinline__ bool cand_less(const Cand &a, const Cand &b) {
    if (a.o != b.o) return a.o < b.o;
    if (a.dist != b.dist) return a.dist < b.dist;
    return a.i < b.i;
}

// One thread: heap sort of the candidates by (o, dist, i), then the sequential s_coll response.
// With perm != nullptr the candidates hold Barnes-Hut slots (the order of the reference's leaf and
// neighbour iteration) and perm maps them to bodies.
__global__ void restitution_kernel(Cand *cand, const int *count, int cap, const int32_t *perm, const double4 *pm,
                                   const double *rest, double4 *vel, int *status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int c = *count;
    if (c > cap) {
        *status = GTD_ERR_CAPACITY;
        return;
    }
    // heap sort
    for (int start = c / 2 - 1; start >= 0; --start) {
        int root = start;
        while (true) {
            int child = 2 * root + 1;
            if (child >= c) break;
            if (child + 1 < c && cand_less(cand[child], cand[child + 1])) ++child;
            if (!cand_less(cand[root], cand[child])) break;
            Cand t = cand[root]; cand[root] = cand[child]; cand[child] = t;
            root = child;
        }
    }
    for (int end = c - 1; end > 0; --end) {
        Cand t = cand[0]; cand[0] = cand[end]; cand[end] = t;
        int root = 0;
        while (true) {
            int child = 2 * root + 1;
            if (child >= end) break;
            if (child + 1 < end && cand_less(cand[child], cand[child + 1])) ++child;
            if (!cand_less(cand[root], cand[child])) break;
            Cand u = cand[root]; cand[root] = cand[child]; cand[child] = u;
            root = child;
        }
    }
    auto body = [&](int32_t q) { return perm ? perm[q] : q; };
    int g = 0;
    while (g < c) {
        const int og = cand[g].o;
        const int o = body(og);
        int e = g;
        while (e < c && cand[e].o == og) ++e;
        // momenta along r12 snapshotted for the whole group before any update (gregsys.hpp:740-742)
        const double4 xo = pm[o];
        for (int k = g; k < e; ++k) {
            const int i = body(cand[k].i);
            const double4 xi = pm[i];
            const double d = cand[k].dist;
            const double ux = (xi.x - xo.x) / d, uy = (xi.y - xo.y) / d, uz = (xi.z - xo.z) / d;
            const double4 vo = vel[o], vi = vel[i];
            const double po = xo.w * vo.x * ux + xo.w * vo.y * uy + xo.w * vo.z * uz;
            const double pi = xi.w * vi.x * ux + xi.w * vi.y * uy + xi.w * vi.z * uz;
            // reuse the record: dist keeps the key, o/i the bodies; stash momenta in a side slot
            cand[k].dist = d;
            reinterpret_cast<double2 *>(cand + cap)[k] = make_double2(po, pi);
        }
        double prev = -1.0;
        for (int k = g; k < e; ++k) {
            const double d = cand[k].dist;
            if (k > g && d == prev) continue;  // std::map::emplace keeps the first equal key
            prev = d;
            const int i = body(cand[k].i);
            const double4 xi = pm[i];
            const double ux = (xi.x - xo.x) / d, uy = (xi.y - xo.y) / d, uz = (xi.z - xo.z) / d;
            const double2 pp = reinterpret_cast<double2 *>(cand + cap)[k];
            const double mo = xo.w, mi = xi.w;
            const double o_vel = pp.x / mo, i_vel = pp.y / mi;
            const double o_minus_i = o_vel - i_vel;
            const double avg_rest = 0.5 * (rest[o] + rest[i]);
            if (o_vel > 0 || i_vel < 0) {
                if (o_vel <= 0 && i_vel < 0 && o_vel < i_vel) continue;
                if (o_vel > 0 && i_vel >= 0 && o_vel < i_vel) continue;
                const double psum = pp.x + pp.y, msum = mo + mi;
                const double new_o = (psum - mi * avg_rest * o_minus_i) / msum;
                const double new_i = (psum + mo * avg_rest * o_minus_i) / msum;
                const double d_o = new_o - o_vel, d_i = new_i - i_vel;
                double4 vo = vel[o], vi = vel[i];
                vo.x += d_o * ux; vo.y += d_o * uy; vo.z += d_o * uz;
                vi.x += d_i * ux; vi.y += d_i * uy; vi.z += d_i * uz;
                vel[o] = vo;
                vel[i] = vi;
            }
        }
        g = e;
    }
}

// ---- Barnes-Hut path: bh_s_coll (gregsys.hpp:631-688) ----------------------------------------
// Bounds of every node's cell: the set_corners splits (greg8tree.hpp:81-131) of the root box along
// the node's code prefix, in T (float trees round every midpoint to float).
template <bool F>
__global__ void node_box_kernel(int64_t n_nodes, const unsigned long long *codes, const int32_t *first,
                                const int8_t *depth, const double *box, double *nbox) {
    const int64_t nd = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (nd >= n_nodes) return;
    const unsigned long long c = codes[first[nd]];
    double lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = box[k];
        hi[k] = box[3 + k];
    }
    const int dl = depth[nd];
    for (int l = 0; l < dl; ++l) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double mid = F ? (double)__fmul_rn(__fadd_rn((float)lo[k], (float)hi[k]), 0.5f)
                                 : __dmul_rn(__dadd_rn(lo[k], hi[k]), 0.5);
            if ((c >> (3 * (20 - l) + k)) & 1ull) lo[k] = mid;
            else hi[k] = mid;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        nbox[6 * nd + k] = lo[k];
        nbox[6 * nd + 3 + k] = hi[k];
    }
}

// One thread per slot a: the nn_iterator neighbours of a's leaf (greg8tree.hpp:615-701: depth-first
// from the root's children, descending only into cells that touch the leaf's cell, closed-interval
// test of :624-628, the own leaf skipped), keeping the bodies that overlap a's body.  A depth-21
// bucket leaf counts its other bodies as neighbours.  Candidates are (slot a, slot q, distance).
__global__ void __launch_bounds__(kCT) bh_touch_pairs_kernel(int64_t n, int64_t n_nodes, const int32_t *own,
                                                             const int32_t *perm, const int8_t *leaf,
                                                             const int32_t *first, const int32_t *count,
                                                             const int32_t *skip, const double *nbox,
                                                             const double4 *pm, const double *rad, Cand *cand,
                                                             int *cand_count, int cap) {
    const int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const int32_t L = own[a];
    const int32_t o = perm[a];
    const double4 po = pm[o];
    const double ro = rad[o];
    const double bx0 = nbox[6 * L], by0 = nbox[6 * L + 1], bz0 = nbox[6 * L + 2];
    const double bx1 = nbox[6 * L + 3], by1 = nbox[6 * L + 4], bz1 = nbox[6 * L + 5];
    int64_t k = 1;
    while (k < n_nodes) {
        bool take;
        if (k == L) {
            take = count[k] > 1;
        } else {
            const double *C = nbox + 6 * k;
            const bool touch = !(bx1 < C[0] || bx0 > C[3] || by1 < C[1] || by0 > C[4] || bz1 < C[2] || bz0 > C[5]);
            if (!touch) {
                k = skip[k];
                continue;
            }
            if (!leaf[k]) {
                ++k;
                continue;
            }
            take = true;
        }
        if (take) {
            const int32_t q0 = first[k], q1 = first[k] + count[k];
            for (int32_t q = q0; q < q1; ++q) {
                if (q == a) continue;
                const int32_t i = perm[q];
                const double4 pi = pm[i];
                const double dx = __dsub_rn(pi.x, po.x), dy = __dsub_rn(pi.y, po.y), dz = __dsub_rn(pi.z, po.z);
                const double d =
                    sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
                if (__dadd_rn(ro, rad[i]) > d) {
                    const int slot = atomicAdd(cand_count, 1);
                    if (slot < cap) cand[slot] = Cand{(int32_t)a, q, d};
                }
            }
        }
        k = skip[k];
    }
}

// body::operator+= (gregbod.hpp:1066-1082), FP64 with the reference's rounding order.
__device__ void merge_into(double4 &po, double4 &vo, double4 &ao, double &ro, double &eo, const double4 &pi,
                           const double4 &vi, const double4 &ai, double ri, double ei) {
    const double ma = po.w, mb = pi.w, ms = __dadd_rn(ma, mb);
    auto mix = [&](double a, double b) { return __ddiv_rn(__dadd_rn(__dmul_rn(ma, a), __dmul_rn(mb, b)), ms); };
    const double4 np = make_double4(mix(po.x, pi.x), mix(po.y, pi.y), mix(po.z, pi.z), ms);
    const double4 nv = make_double4(mix(vo.x, vi.x), mix(vo.y, vi.y), mix(vo.z, vi.z), 0.0);
    const double4 na = make_double4(mix(ao.x, ai.x), mix(ao.y, ai.y), mix(ao.z, ai.z), 0.0);
    eo = 0.5 * (eo + ei);
    ro = cbrt(__dadd_rn(__dmul_rn(__dmul_rn(ro, ro), ro), __dmul_rn(__dmul_rn(ri, ri), ri)));
    po = np;
    vo = nv;
    ao = na;
}

__device__ __forceinline__ bool overlaps(const double4 &a, double ra, const double4 &b, double rb) {
    const double dx = __dsub_rn(b.x, a.x), dy = __dsub_rn(b.y, a.y), dz = __dsub_rn(b.z, a.z);
    const double d = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    return d < __dadd_rn(ra, rb);
}

// One block: the check_overlap scan with merges.  For the current outer body the block finds the
// first overlapping body in scan order (a min-reduction over indices), merges it, compacts the
// arrays and restarts the scan from index 0, exactly as the sequential loop would.
constexpr int kMT = 1024;

__global__ void __launch_bounds__(kMT) merge_scan_kernel(int64_t *n_io, double4 *pm, double4 *vel, double4 *acc,
                                                         double *rad, double *rest, int32_t *ids, int only_check,
                                                         int *status, int32_t *pair) {
    __shared__ int best;
    __shared__ int num_s, o_s;
    const int t = threadIdx.x;
    if (t == 0) {
        num_s = (int)*n_io;
        o_s = 0;
    }
    __syncthreads();
    bool restarted = false;
    while (true) {
        const int num = num_s, o = o_s;
        if (o >= num) break;
        const int lo = restarted ? 0 : o + 1;
        if (t == 0) best = INT32_MAX;
        __syncthreads();
        const double4 po = pm[o];
        const double ro = rad[o];
        for (int i = lo + t; i < num; i += kMT) {
            if (i == o) continue;
            if (overlaps(po, ro, pm[i], rad[i])) atomicMin(&best, i);
        }
        __syncthreads();
        const int i = best;
        if (i == INT32_MAX) {
            if (t == 0) o_s = o + 1;
            restarted = false;
            __syncthreads();
            continue;
        }
        if (only_check) {
            if (t == 0) {
                *status = GTD_ERR_OVERLAPPING_BODIES;
                pair[0] = ids[o] < ids[i] ? ids[o] : ids[i];
                pair[1] = ids[o] < ids[i] ? ids[i] : ids[o];
            }
            return;
        }
        if (t == 0) {
            double4 p = pm[o], v = vel[o], a = acc[o];
            double r = rad[o], e = rest[o];
            merge_into(p, v, a, r, e, pm[i], vel[i], acc[i], rad[i], rest[i]);
            pm[o] = p; vel[o] = v; acc[o] = a; rad[o] = r; rest[o] = e;
        }
        __syncthreads();
        // erase body i: shift [i+1, num) down by one (in chunks so no element is read after overwrite)
        for (int base = i; base < num - 1; base += kMT) {
            const int k = base + t;
            double4 p, v, a;
            double r = 0, e = 0;
            int32_t id = 0;
            const bool act = k < num - 1;
            if (act) {
                p = pm[k + 1]; v = vel[k + 1]; a = acc[k + 1]; r = rad[k + 1]; e = rest[k + 1]; id = ids[k + 1];
            }
            __syncthreads();
            if (act) {
                pm[k] = p; vel[k] = v; acc[k] = a; rad[k] = r; rest[k] = e; ids[k] = id;
            }
            __syncthreads();
        }
        if (t == 0) {
            num_s = num - 1;
            o_s = i < o ? o - 1 : o;
        }
        restarted = true;
        __syncthreads();
    }
    if (t == 0) *n_io = num_s;
}

}  // namespace gtd

using namespace gtd;

void release_collide(gtd_system *s) {
    cudaFree(s->coll_buf);
    s->coll_buf = nullptr;
    s->coll_bytes = 0;
    cudaFree(s->coll_nbox);
    s->coll_nbox = nullptr;
    s->coll_nbox_cap = 0;
}

static int ensure_coll(gtd_system *s) {
    const size_t need = sizeof(Cand) * kMaxCand + sizeof(double2) * kMaxCand + 256;
    if (s->coll_buf && s->coll_bytes >= need) return GTD_OK;
    release_collide(s);
    GTD_CUDA(cudaMalloc(&s->coll_buf, need));
    s->coll_bytes = need;
    return GTD_OK;
}

struct CollPtrs {
    Cand *cand;
    int *count, *status;
    int32_t *pair;
    int64_t *n_dev;
};

static CollPtrs coll_ptrs(gtd_system *s) {
    char *b = reinterpret_cast<char *>(s->coll_buf);
    CollPtrs p;
    p.cand = reinterpret_cast<Cand *>(b);
    char *tail = b + sizeof(Cand) * kMaxCand + sizeof(double2) * kMaxCand;
    p.count = reinterpret_cast<int *>(tail);
    p.status = p.count + 1;
    p.pair = p.count + 2;
    p.n_dev = reinterpret_cast<int64_t *>(tail + 64);
    return p;
}

// Merge scan on the device; updates s->n.  only_check: report the first overlapping pair.
static int merge_scan(gtd_system *s, bool only_check, int32_t *pair_out) {
    int rc = restore_upload_order(s);
    if (rc) return rc;
    rc = ensure_coll(s);
    if (rc) return rc;
    CollPtrs p = coll_ptrs(s);
    cudaStream_t st = s->stream;
    GTD_CUDA(cudaMemsetAsync(p.count, 0, 64, st));
    GTD_CUDA(cudaMemcpyAsync(p.n_dev, &s->n, sizeof(int64_t), cudaMemcpyHostToDevice, st));
    merge_scan_kernel<<<1, kMT, 0, st>>>(p.n_dev, s->pm[s->cur], s->vel, s->acc, s->rad, s->rest, s->ids,
                                         only_check ? 1 : 0, p.status, p.pair);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    int host[4] = {0, 0, 0, 0};
    int64_t n_new = s->n;
    GTD_CUDA(cudaMemcpyAsync(host, p.count, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    GTD_CUDA(cudaMemcpyAsync(&n_new, p.n_dev, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    GTD_CUDA(cudaStreamSynchronize(st));
    if (host[1] == GTD_ERR_OVERLAPPING_BODIES) {
        if (pair_out) { pair_out[0] = host[2]; pair_out[1] = host[3]; }
        return fail(GTD_ERR_OVERLAPPING_BODIES,
                    "The bodies with id=%d and id=%d that were added to this system object overlap.", host[2],
                    host[3]);
    }
    if (n_new != s->n) {
        s->n = n_new;
        s->tree_valid = false;
        s->plan.n = -1;  // force a new force plan for the smaller N
    }
    return GTD_OK;
}

// Upload order and the candidate buffer for overlap passes; *status: the pass's device error word
// (GTD_ERR_CAPACITY when the candidates overflowed), cleared by every pass.
int prepare_collisions(gtd_system *s, int **status) {
    int rc = restore_upload_order(s);
    if (rc) return rc;
    rc = ensure_coll(s);
    if (rc) return rc;
    if (status) *status = coll_ptrs(s).status;
    return GTD_OK;
}

// One s_coll pass (overlap restitution) enqueued on the stream, without reading its status back;
// prepare_collisions must have run since the last reorder.  Capturable.
int enqueue_collisions(gtd_system *s) {
    if (s->n < 2) return GTD_OK;
    CollPtrs p = coll_ptrs(s);
    cudaStream_t st = s->stream;
    GTD_CUDA(cudaMemsetAsync(p.count, 0, 64, st));
    overlap_pairs_kernel<<<(unsigned)((s->n + kCT - 1) / kCT), kCT, 0, st>>>(s->n, s->pm[s->cur], s->rad, p.cand,
                                                                           p.count, kMaxCand);
    GTD_CHECK_LAUNCH();
    restitution_kernel<<<1, 32, 0, st>>>(p.cand, p.count, kMaxCand, nullptr, s->pm[s->cur], s->rest, s->vel,
                                         p.status);
    GTD_CHECK_LAUNCH();
    s->launches += 2;
    return GTD_OK;
}

int run_collisions(gtd_system *s) {
    if (s->n < 2) return GTD_OK;
    if (s->coll == GTD_MERGE_COLL) return merge_scan(s, false, nullptr);
    int rc = prepare_collisions(s, nullptr);
    if (rc) return rc;
    rc = enqueue_collisions(s);
    if (rc) return rc;
    CollPtrs p = coll_ptrs(s);
    cudaStream_t st = s->stream;
    int host[2] = {0, 0};
    GTD_CUDA(cudaMemcpyAsync(host, p.count, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    GTD_CUDA(cudaStreamSynchronize(st));
    if (host[1] == GTD_ERR_CAPACITY)
        return fail(GTD_ERR_CAPACITY, "%d overlapping pairs in one step exceed the %d the collision pass holds",
                    host[0], kMaxCand);
    return GTD_OK;
}

// bh_s_coll after a Barnes-Hut kick, on the tree of the current positions (gregsys.hpp:2936-2938).
int run_bh_collisions(gtd_system *s) {
    if (s->n < 2 || !s->tree_valid) return GTD_OK;
    int rc = ensure_coll(s);
    if (rc) return rc;
    const int64_t nn = s->n_nodes;
    if (nn > s->coll_nbox_cap) {
        cudaFree(s->coll_nbox);
        s->coll_nbox = nullptr;
        s->coll_nbox_cap = 0;
        GTD_CUDA(cudaMalloc(&s->coll_nbox, sizeof(double) * 6 * (size_t)nn));
        s->coll_nbox_cap = nn;
    }
    CollPtrs p = coll_ptrs(s);
    cudaStream_t st = s->stream;
    GTD_CUDA(cudaMemsetAsync(p.count, 0, 64, st));
    const unsigned gn = (unsigned)((nn + kCT - 1) / kCT), gb = (unsigned)((s->n + kCT - 1) / kCT);
    if (s->tree_float)
        node_box_kernel<true><<<gn, kCT, 0, st>>>(nn, s->codes, s->nfirst, s->ndepth, s->box_dev, s->coll_nbox);
    else
        node_box_kernel<false><<<gn, kCT, 0, st>>>(nn, s->codes, s->nfirst, s->ndepth, s->box_dev, s->coll_nbox);
    GTD_CHECK_LAUNCH();
    bh_touch_pairs_kernel<<<gb, kCT, 0, st>>>(s->n, nn, s->own_leaf, s->perm, s->nleaf, s->nfirst, s->ncount,
                                              s->nskip, s->coll_nbox, s->pm[s->cur], s->rad, p.cand, p.count,
                                              kMaxCand);
    GTD_CHECK_LAUNCH();
    restitution_kernel<<<1, 32, 0, st>>>(p.cand, p.count, kMaxCand, s->perm, s->pm[s->cur], s->rest, s->vel,
                                         p.status);
    GTD_CHECK_LAUNCH();
    s->launches += 3;
    int host[2] = {0, 0};
    GTD_CUDA(cudaMemcpyAsync(host, p.count, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    GTD_CUDA(cudaStreamSynchronize(st));
    if (host[1] == GTD_ERR_CAPACITY)
        return fail(GTD_ERR_CAPACITY, "%d overlapping neighbour pairs in one step exceed the %d the collision pass holds",
                    host[0], kMaxCand);
    return GTD_OK;
}

extern "C" int gtd_system_check_overlap(gtd_system *s, int merge, int32_t *pair) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (s->n < 2) return GTD_OK;
    return merge_scan(s, merge == 0, pair);
}
