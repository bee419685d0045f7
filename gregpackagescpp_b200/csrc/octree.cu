// Barnes-Hut on the device: the greg8tree octree rebuilt as a linear octree, and the reference
// walk, plus the Morton ordering the mixed-precision direct sum uses.
//
// Reference semantics (greg8tree.hpp) and how they map here:
//  * root box: bh_tree::find_min_max (:1012-1047) - min/max, longest edge, pad = edge/20, a cube
//    anchored at min - pad - computed in T (float or double) exactly as the reference rounds.
//  * octant splits: set_corners (:81-131) splits at (btm + top)/2 with the sum rounded to T; a
//    coordinate >= the split goes to the upper child (half-open cells, gregvec.hpp:2115-2120);
//    octant index bit0 = x, bit1 = y, bit2 = z (:74-76).  The 63-bit Morton code of a body is that
//    descent repeated 21 times, so the codes reproduce the reference's cell assignment bit for bit.
//  * topology: the reference octree (one body per leaf, a cell for every shared prefix) is the set
//    of octal prefixes shared by >= 2 bodies plus one leaf per body; emitted here in DFS pre-order
//    (children in octant order = ascending code = the leaf order of bh_cube::iterator :502-614)
//    with skip links.  Depth is capped at 21: bodies sharing a full code form one bucket leaf.
//  * centres of mass: calc_com (:213-281) in FP64 moments (the float moments of the reference
//    overflow in SI units), children summed in octant order, deepest level first.
//  * walk: cell_iterator (:702-833) - DFS from the root's children, leaves always accepted
//    except the body's own, cells accepted when width/|x - com| < theta, otherwise descended.
//    A warp walks 32 consecutive (Morton-adjacent) bodies together.  walk_kernel: each lane keeps
//    its own next node, the warp fetches the minimum of those (one broadcast load for all lanes at
//    that node), so every lane visits exactly its reference sequence of cells.  list_walk_kernel:
//    the warp classifies 32 nodes at a time for all its lanes (exactly, by the monotonicity of
//    rounding), collects each lane's accepted cells in a shared interaction list and sums them in a
//    dense pass; every lane takes exactly its reference set of cells, in another order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "gtd_internal.cuh"
#include "gtd_math.cuh"
#include "gtd_sort.cuh"
#include "gtd_system.cuh"

namespace gtd {

constexpr int kMaxDepth = 21;
constexpr int kBBoxBlocks = 296;
constexpr int kTT = 256;

template <bool F>
struct TreeT;
template <>
struct TreeT<true> {
    using T = float;
    __device__ static float rnd(double v) { return __double2float_rn(v); }
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ static float div(float a, float b) { return __fdiv_rn(a, b); }
};
template <>
struct TreeT<false> {
    using T = double;
    __device__ static double rnd(double v) { return v; }
    __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ static double sub(double a, double b) { return __dsub_rn(a, b); }
    __device__ static double div(double a, double b) { return __ddiv_rn(a, b); }
};

// ---- root box (find_min_max) ---------------------------------------------------------------
template <bool F>
__global__ void bbox_partial_kernel(const double4 *pm, int64_t n, double *part) {
    using TT = TreeT<F>;
    __shared__ double red[6][kTT];
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double4 p = pm[i];
        const double c[3] = {(double)TT::rnd(p.x), (double)TT::rnd(p.y), (double)TT::rnd(p.z)};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = fmin(mn[k], c[k]);
            mx[k] = fmax(mx[k], c[k]);
        }
    }
    const int t = threadIdx.x;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        red[k][t] = mn[k];
        red[3 + k][t] = mx[k];
    }
    __syncthreads();
    for (int w = kTT / 2; w > 0; w >>= 1) {
        if (t < w) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                red[k][t] = fmin(red[k][t], red[k][t + w]);
                red[3 + k][t] = fmax(red[3 + k][t], red[3 + k][t + w]);
            }
        }
        __syncthreads();
    }
    if (t < 6) part[(size_t)blockIdx.x * 6 + t] = red[t][0];
}

// One warp folds the block partials (min and max are exact, so the lane split does not change the
// result); then one thread does the reference's arithmetic for the cube, greg8tree.hpp:1037-1046, in T.
template <bool F>
__global__ void bbox_final_kernel(const double *part, int blocks, double *box, int *status) {
    using TT = TreeT<F>;
    using T = typename TT::T;
    const int lane = threadIdx.x & 31;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int b = lane; b < blocks; b += 32)
        for (int k = 0; k < 3; ++k) {
            mn[k] = fmin(mn[k], part[b * 6 + k]);
            mx[k] = fmax(mx[k], part[b * 6 + 3 + k]);
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = fmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    if (threadIdx.x != 0) return;
    const T xr = TT::sub((T)mx[0], (T)mn[0]), yr = TT::sub((T)mx[1], (T)mn[1]), zr = TT::sub((T)mx[2], (T)mn[2]);
    T edge = xr > yr ? (xr > zr ? xr : zr) : (yr > zr ? yr : zr);
    // pad = edge / 20.0l: the long-double quotient rounded to T equals the correctly rounded T
    // quotient (a division by 20 never lands on a rounding tie at 64 -> 53 or 24 bits)
    const T pad = TT::div(edge, (T)20);
    T btm[3];
    for (int k = 0; k < 3; ++k) btm[k] = TT::sub((T)mn[k], pad);
    edge = TT::add(edge, (T)2 * pad);
    for (int k = 0; k < 3; ++k) {
        box[k] = (double)btm[k];
        box[3 + k] = (double)TT::add(btm[k], edge);
    }
    if (!(edge > (T)0) || !isfinite((double)edge)) atomicExch(status, GTD_ERR_INVALID_BODY_PLACEMENT);
}

// ---- Morton codes: 21 levels of the reference's octant descent -------------------------------
template <bool F>
__device__ __forceinline__ bool morton_of(double x, double y, double z, const double *box, unsigned long long &code) {
    using TT = TreeT<F>;
    using T = typename TT::T;
    const T p[3] = {TT::rnd(x), TT::rnd(y), TT::rnd(z)};
    T lo[3], hi[3];
    bool inside = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = (T)box[k];
        hi[k] = (T)box[3 + k];
        inside = inside && lo[k] <= p[k] && p[k] < hi[k];
    }
    unsigned long long c = 0;
#pragma unroll 1
    for (int l = 0; l < kMaxDepth; ++l) {
        unsigned oct = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const T mid = TT::add(lo[k], hi[k]) * (T)0.5;
            if (p[k] >= mid) {
                oct |= 1u << k;
                lo[k] = mid;
            } else {
                hi[k] = mid;
            }
        }
        c = (c << 3) | oct;
    }
    code = c;
    return inside;
}

template <bool F>
__global__ void morton_kernel(const double4 *pm, int64_t n, const double *box_g, unsigned long long *keys,
                              int32_t *vals, int *status) {
    __shared__ double box[6];
    if (threadIdx.x < 6) box[threadIdx.x] = box_g[threadIdx.x];
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = pm[i];
    unsigned long long c;
    if (!morton_of<F>(p.x, p.y, p.z, box, c)) atomicExch(status, GTD_ERR_INVALID_BODY_PLACEMENT);
    keys[i] = c;
    vals[i] = (int32_t)i;
}

// Hilbert key of a position quantised to 21 bits per axis over the box (btm, top): the axes are
// mapped to the transposed Hilbert index with Skilling's procedure (J. Skilling, "Programming the
// Hilbert curve", AIP Conf. Proc. 707, 381-387, 2004) and the three transposed words interleaved,
// most significant bit first.  Consecutive keys are adjacent cells (no jumps as in Morton order), so
// runs of bodies in key order are spatially compact; the direct sum's reorder uses them.
__device__ __forceinline__ unsigned long long hilbert_key21(uint32_t x0, uint32_t x1, uint32_t x2) {
    uint32_t X[3] = {x0, x1, x2};
    constexpr uint32_t kTop = 1u << 20;
    for (uint32_t q = kTop; q > 1; q >>= 1) {  // undo excess work, level by level
        const uint32_t p = q - 1;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (X[i] & q) {
                X[0] ^= p;  // invert
            } else {
                const uint32_t t = (X[0] ^ X[i]) & p;  // exchange
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    X[1] ^= X[0];  // Gray encode
    X[2] ^= X[1];
    uint32_t t = 0;
    for (uint32_t q = kTop; q > 1; q >>= 1)
        if (X[2] & q) t ^= q - 1;
    X[0] ^= t;
    X[1] ^= t;
    X[2] ^= t;
    unsigned long long key = 0;
    for (int lev = 20; lev >= 0; --lev)
        key = (key << 3) | (((X[0] >> lev) & 1u) << 2) | (((X[1] >> lev) & 1u) << 1) | ((X[2] >> lev) & 1u);
    return key;
}

__global__ void hilbert_kernel(const double4 *pm, int64_t n, const double *box_g, unsigned long long *keys,
                               int32_t *vals) {
    __shared__ double box[6];
    if (threadIdx.x < 6) box[threadIdx.x] = box_g[threadIdx.x];
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 p = pm[i];
    const double c[3] = {p.x, p.y, p.z};
    uint32_t q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double w = box[3 + d] - box[d];
        double f = w > 0.0 ? (c[d] - box[d]) / w * 2097152.0 : 0.0;
        f = f == f ? fmin(fmax(f, 0.0), 2097151.0) : 0.0;  // clamped; a NaN coordinate goes to cell 0
        q[d] = (uint32_t)f;
    }
    keys[i] = hilbert_key21(q[0], q[1], q[2]);
    vals[i] = (int32_t)i;
}

// ---- topology ---------------------------------------------------------------------------------
__device__ __forceinline__ int lcp_digits(unsigned long long a, unsigned long long b) {
    const unsigned long long x = a ^ b;
    if (!x) return kMaxDepth;
    return (__clzll((long long)x) - 1) / 3;
}

// Per slot: common octal prefix with the next slot and the number of nodes the slot opens.
template <bool F>
__global__ void lcp_count_kernel(const unsigned long long *codes, const int32_t *perm, const double4 *pm, int64_t n,
                                 int32_t *lcp, uint32_t *cnt, int *status) {
    using TT = TreeT<F>;
    const int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (a > n) return;
    if (a == n) {
        cnt[n] = 0;
        return;
    }
    int la = -1;
    if (a + 1 < n) {
        la = lcp_digits(codes[a], codes[a + 1]);
        if (la == kMaxDepth) {
            const double4 p = pm[perm[a]], q = pm[perm[a + 1]];
            if (TT::rnd(p.x) == TT::rnd(q.x) && TT::rnd(p.y) == TT::rnd(q.y) && TT::rnd(p.z) == TT::rnd(q.z))
                atomicExch(status, GTD_ERR_INDISTINGUISHABLE);
        }
        lcp[a] = la;
    }
    const int lm = a > 0 ? lcp_digits(codes[a - 1], codes[a]) : -1;
    const int lim = la < kMaxDepth - 1 ? la : kMaxDepth - 1;
    const int ni = lim - lm > 0 ? lim - lm : 0;
    cnt[a] = (uint32_t)(ni + (lm < kMaxDepth ? 1 : 0));
}

// last slot sharing the first d octal digits with slot a (galloping then binary search)
__device__ __forceinline__ int64_t range_end(const unsigned long long *code, int64_t n, int64_t a, int d) {
    if (d == 0) return n - 1;
    const int shift = 63 - 3 * d;
    const unsigned long long pre = code[a] >> shift;
    int64_t lo = a, step = 1;
    while (true) {
        const int64_t nx = lo + step;
        if (nx >= n || (code[nx] >> shift) != pre) break;
        lo = nx;
        step <<= 1;
    }
    int64_t hi = min(lo + step, n) - 1;
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo + 1) / 2;
        if ((code[mid] >> shift) == pre) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

struct EmitArgs {
    int64_t n;
    const unsigned long long *codes;
    const int32_t *perm, *lcp;
    const uint32_t *node_start;
    const double4 *pm;
    const double *box;
    int8_t *depth, *leaf;
    int32_t *first, *count, *skip, *own;
    double4 *com;
    double *width;
};

template <bool F>
__device__ double cell_width(unsigned long long code, int depth, const double *box) {
    using TT = TreeT<F>;
    using T = typename TT::T;
    T lo = (T)box[0], hi = (T)box[3];
    for (int l = 0; l < depth; ++l) {
        const T mid = TT::add(lo, hi) * (T)0.5;
        if ((code >> (3 * (kMaxDepth - 1 - l))) & 1ull) lo = mid;
        else hi = mid;
    }
    return (double)TT::sub(hi, lo);
}

template <bool F>
__global__ void emit_kernel(EmitArgs e) {
    using TT = TreeT<F>;
    const int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= e.n) return;
    const int lm = a > 0 ? e.lcp[a - 1] : -1;
    const int la = a + 1 < e.n ? e.lcp[a] : -1;
    const int lim = la < kMaxDepth - 1 ? la : kMaxDepth - 1;
    int64_t node = e.node_start[a];
    const unsigned long long ca = e.codes[a];
    for (int d = lm + 1; d <= lim; ++d, ++node) {
        const int64_t last = range_end(e.codes, e.n, a, d);
        e.depth[node] = (int8_t)d;
        e.leaf[node] = 0;
        e.first[node] = (int32_t)a;
        e.count[node] = (int32_t)(last - a + 1);
        e.skip[node] = (int32_t)e.node_start[last + 1];
        e.width[node] = cell_width<F>(ca, d, e.box);
    }
    if (lm < kMaxDepth) {
        const int64_t last = la == kMaxDepth ? range_end(e.codes, e.n, a, kMaxDepth) : a;
        const int lb = last + 1 < e.n ? e.lcp[last] : -1;
        const int dl = last > a ? kMaxDepth : (lm > lb ? lm : lb) + 1;
        e.depth[node] = (int8_t)dl;
        e.leaf[node] = 1;
        e.first[node] = (int32_t)a;
        e.count[node] = (int32_t)(last - a + 1);
        e.skip[node] = (int32_t)e.node_start[last + 1];
        e.width[node] = cell_width<F>(ca, dl, e.box);
        if (last == a) {
            const double4 p = e.pm[e.perm[a]];
            e.com[node] = make_double4((double)TT::rnd(p.x), (double)TT::rnd(p.y), (double)TT::rnd(p.z),
                                       (double)TT::rnd(p.w));
        } else {
            double ms = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
            for (int64_t q = a; q <= last; ++q) {
                const double4 p = e.pm[e.perm[q]];
                const double mb = (double)TT::rnd(p.w);
                ms = __dadd_rn(ms, mb);
                mx = __dadd_rn(mx, __dmul_rn(mb, (double)TT::rnd(p.x)));
                my = __dadd_rn(my, __dmul_rn(mb, (double)TT::rnd(p.y)));
                mz = __dadd_rn(mz, __dmul_rn(mb, (double)TT::rnd(p.z)));
            }
            e.com[node] = make_double4(__ddiv_rn(mx, ms), __ddiv_rn(my, ms), __ddiv_rn(mz, ms), ms);
        }
        for (int64_t q = a; q <= last; ++q) e.own[q] = (int32_t)node;
    }
}

__global__ void depth_offsets_kernel(uint32_t *depth_off) {
    // depth_off[0..20]: counts in, exclusive offsets out; depth_off[22..42]: cursors
    if (threadIdx.x != 0) return;
    uint32_t run = 0;
    for (int d = 0; d < kMaxDepth; ++d) {
        const uint32_t c = depth_off[d];
        depth_off[d] = run;
        depth_off[22 + d] = run;
        run += c;
    }
    depth_off[kMaxDepth] = run;
}

// Internal nodes per depth.  Each CTA counts a chunk of kDepthChunk nodes in shared memory and adds
// its counts with one global atomic per depth: a global atomic per node would serialise ~N atomics
// on 21 addresses (about 1 ms at N = 4194304).
constexpr int kDepthChunk = 16 * kTT;

__global__ void __launch_bounds__(kTT) depth_count_kernel(const int8_t *depth, const int8_t *leaf, int64_t n_nodes,
                                                          uint32_t *depth_off) {
    __shared__ uint32_t cnt[kMaxDepth];
    const int t = threadIdx.x;
    if (t < kMaxDepth) cnt[t] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kDepthChunk;
    for (int k = 0; k < kDepthChunk / kTT; ++k) {
        const int64_t nd = base + (int64_t)k * kTT + t;
        if (nd < n_nodes && !leaf[nd]) atomicAdd(&cnt[depth[nd]], 1u);
    }
    __syncthreads();
    if (t < kMaxDepth && cnt[t]) atomicAdd(&depth_off[t], cnt[t]);
}

// Lists the internal nodes by depth (the order inside a depth is free: each node's moments are
// computed from its own children alone).  A CTA ranks its chunk's nodes per depth in shared memory
// and reserves one range per depth with a single global atomic.
__global__ void __launch_bounds__(kTT) depth_scatter_kernel(const int8_t *depth, const int8_t *leaf, int64_t n_nodes,
                                                            uint32_t *depth_off, int32_t *list) {
    constexpr int kItems = kDepthChunk / kTT;
    __shared__ uint32_t cnt[kMaxDepth], start[kMaxDepth];
    const int t = threadIdx.x;
    if (t < kMaxDepth) cnt[t] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kDepthChunk;
    int8_t d[kItems];
    uint32_t r[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const int64_t nd = base + (int64_t)k * kTT + t;
        d[k] = -1;
        r[k] = 0;
        if (nd < n_nodes && !leaf[nd]) {
            d[k] = depth[nd];
            r[k] = atomicAdd(&cnt[d[k]], 1u);
        }
    }
    __syncthreads();
    if (t < kMaxDepth && cnt[t]) start[t] = atomicAdd(&depth_off[22 + t], cnt[t]);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kItems; ++k)
        if (d[k] >= 0) list[start[d[k]] + r[k]] = (int32_t)(base + (int64_t)k * kTT + t);
}

// Internal nodes of one depth: FP64 moments of the children in octant order.
__global__ void com_level_kernel(const int32_t *list, const uint32_t *depth_off, int d, const int32_t *skip,
                                 double4 *com) {
    const uint32_t b = depth_off[d], e = depth_off[d + 1];
    for (uint32_t k = b + blockIdx.x * blockDim.x + threadIdx.x; k < e; k += gridDim.x * blockDim.x) {
        const int32_t nd = list[k];
        const int32_t end = skip[nd];
        double ms = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
        for (int32_t c = nd + 1; c < end; c = skip[c]) {
            const double4 q = com[c];
            ms = __dadd_rn(ms, q.w);
            mx = __dadd_rn(mx, __dmul_rn(q.w, q.x));
            my = __dadd_rn(my, __dmul_rn(q.w, q.y));
            mz = __dadd_rn(mz, __dmul_rn(q.w, q.z));
        }
        com[nd] = make_double4(__ddiv_rn(mx, ms), __ddiv_rn(my, ms), __ddiv_rn(mz, ms), ms);
    }
}

// Walk records (one 16-byte A + one 16-byte B load per visited node) and slot-ordered bodies.  With
// IL (float trees only) A and B of a node sit side by side in rec_a, so both loads hit one 32-byte
// sector.
template <bool F, bool IL = false>
__global__ void walk_records_kernel(int64_t n_nodes, const double4 *com, const double *width, const int8_t *leaf,
                                    const int32_t *first, const int32_t *count, const int32_t *skip, double G,
                                    void *rec_a, int4 *rec_b, double *w2_64) {
    const int64_t nd = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (nd >= n_nodes) return;
    const double4 c = com[nd];
    const double w = width[nd];
    int4 b;
    b.x = skip[nd];
    b.y = first[nd];
    b.z = count[nd] | (leaf[nd] ? (int)0x80000000u : 0);
    if (F) {
        const float4 A =
            make_float4(__double2float_rn(c.x), __double2float_rn(c.y), __double2float_rn(c.z), (float)(G * c.w));
        const float wf = (float)w;
        b.w = __float_as_int(__fmul_rn(wf, wf));
        if (IL) {
            reinterpret_cast<float4 *>(rec_a)[2 * nd] = A;
            reinterpret_cast<int4 *>(rec_a)[2 * nd + 1] = b;
            return;
        }
        reinterpret_cast<float4 *>(rec_a)[nd] = A;
    } else {
        reinterpret_cast<double4 *>(rec_a)[nd] = make_double4(c.x, c.y, c.z, G * c.w);
        b.w = 0;
        w2_64[nd] = w * w;
    }
    rec_b[nd] = b;
}

template <bool F>
__global__ void slot_bodies_kernel(const double4 *pm, const int32_t *perm, int64_t n, double G, void *slot_pos) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double4 p = pm[perm[s]];
    if (F) {
        reinterpret_cast<float4 *>(slot_pos)[s] = make_float4(__double2float_rn(p.x), __double2float_rn(p.y),
                                                              __double2float_rn(p.z), (float)(G * (double)(float)p.w));
    } else {
        reinterpret_cast<double4 *>(slot_pos)[s] = make_double4(p.x, p.y, p.z, G * p.w);
    }
}

// ---- warp-cooperative walk ---------------------------------------------------------------------
template <typename T>
struct V4;
template <>
struct V4<float> {
    using type = float4;
};
template <>
struct V4<double> {
    using type = double4;
};

// 1/sqrt(r2) of a walk term.  FP32: the MUFU approximation with subnormal inputs flushed (a
// separation whose square is below 2^-126 does not occur in a tree of distinct bodies; the
// non-flushing form spends extra instructions per term on that range).  FP64: the MUFU seed and its
// binomial correction (inv_r).
__device__ __forceinline__ float rsqrt_t(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ double rsqrt_t(double x) { return inv_r(x); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul_t(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_t(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float sub_t(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_t(double a, double b) { return __dsub_rn(a, b); }

// One warp walks 32 consecutive slots (Morton-adjacent bodies).  Every body follows its own pre-order
// walk (accept a leaf, or a cell with width^2 < theta^2 r^2, then jump to the skip link; otherwise
// step into the first child); the warp visits the smallest next node of its lanes, so a node record
// is loaded once for the lanes that need it and each body meets exactly the nodes of its own walk,
// in its own order.  IL: the float tree's A and B halves of a node are interleaved in rec_a, so the
// two 16-byte loads hit one 32-byte sector (measured 23.2 -> 21.5 ms at N = 4194304, theta = 0.5).
// SOFT = false drops the + eps^2 of an unsoftened walk (eps = 0, the reference's default; adding 0
// changes no value); COUNT = false skips the per-body interaction count nobody reads.
template <typename T, bool IL = false, bool SOFT = true, bool COUNT = true>
__global__ void __launch_bounds__(kTT, sizeof(T) == 4 ? 6 : 1) walk_kernel(int64_t n, int64_t n_nodes, const void *rec_a_v, const int4 *rec_b,
                                                   const double *w2_64, const void *slot_pos_v, const int32_t *own,
                                                   T th2, T eps2, void *slot_acc_v, uint32_t *slot_cnt) {
    using V = typename V4<T>::type;
    const V *rec_a = reinterpret_cast<const V *>(rec_a_v);
    const V *bodies = reinterpret_cast<const V *>(slot_pos_v);
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = s < n;
    V p;
    p.x = p.y = p.z = p.w = (T)0;
    int32_t ol = -1;
    uint32_t next = 0x7fffffffu;
    if (active) {
        p = bodies[s];
        ol = own[s];
        next = n_nodes > 1 ? 1u : (uint32_t)n_nodes;
    }
    T ax = 0, ay = 0, az = 0;
    uint32_t cnt = 0;
    const uint32_t nn = (uint32_t)n_nodes;
    while (true) {
        const uint32_t node = __reduce_min_sync(0xffffffffu, next);
        if (node >= nn) break;
        if (next != node) continue;
        V A;
        int4 B;
        if constexpr (IL) {
            A = rec_a[2 * (size_t)node];
            B = reinterpret_cast<const int4 *>(rec_a_v)[2 * (size_t)node + 1];
        } else {
            A = rec_a[node];
            B = rec_b[node];
        }
        const bool leaf = B.z < 0;
        const int count = B.z & 0x7fffffff;
        if (leaf) {
            if (count == 1) {
                if ((int32_t)node != ol) {
                    const T dx = sub_t(A.x, p.x), dy = sub_t(A.y, p.y), dz = sub_t(A.z, p.z);
                    const T r2 = fma_t(dz, dz, fma_t(dy, dy, mul_t(dx, dx)));
                    const T inv = rsqrt_t(SOFT ? r2 + eps2 : r2);
                    const T sc = mul_t(mul_t(mul_t(A.w, inv), inv), inv);
                    ax = fma_t(sc, dx, ax);
                    ay = fma_t(sc, dy, ay);
                    az = fma_t(sc, dz, az);
                    if constexpr (COUNT) ++cnt;
                }
            } else {
                for (int q = B.y; q < B.y + count; ++q) {
                    if (q == (int)s) continue;
                    const V Q = bodies[q];
                    const T dx = sub_t(Q.x, p.x), dy = sub_t(Q.y, p.y), dz = sub_t(Q.z, p.z);
                    const T r2 = fma_t(dz, dz, fma_t(dy, dy, mul_t(dx, dx)));
                    const T inv = rsqrt_t(SOFT ? r2 + eps2 : r2);
                    const T sc = mul_t(mul_t(mul_t(Q.w, inv), inv), inv);
                    ax = fma_t(sc, dx, ax);
                    ay = fma_t(sc, dy, ay);
                    az = fma_t(sc, dz, az);
                    if constexpr (COUNT) ++cnt;
                }
            }
            next = (uint32_t)B.x;
        } else {
            const T dx = sub_t(A.x, p.x), dy = sub_t(A.y, p.y), dz = sub_t(A.z, p.z);
            const T r2 = fma_t(dz, dz, fma_t(dy, dy, mul_t(dx, dx)));
            const T w2 = sizeof(T) == 4 ? (T)__int_as_float(B.w) : (T)w2_64[node];
            if (w2 < mul_t(th2, r2)) {
                const T inv = rsqrt_t(SOFT ? r2 + eps2 : r2);
                const T sc = mul_t(mul_t(mul_t(A.w, inv), inv), inv);
                ax = fma_t(sc, dx, ax);
                ay = fma_t(sc, dy, ay);
                az = fma_t(sc, dz, az);
                if constexpr (COUNT) ++cnt;
                next = (uint32_t)B.x;
            } else {
                next = node + 1;
            }
        }
    }
    if (active) {
        V o;
        o.x = ax; o.y = ay; o.z = az; o.w = (T)0;
        reinterpret_cast<V *>(slot_acc_v)[s] = o;
        if constexpr (COUNT) slot_cnt[s] = cnt;
    }
}

// ---- list walk (float trees) ------------------------------------------------------------------
// The same per-body cell sets as walk_kernel, computed in two phases per warp of 32 consecutive
// slots.  Traversal: the warp pops up to 32 (sibling chain, lane mask) entries from a stack in
// shared memory - one node per lane - and classifies each node for all lanes of its mask at once
// against the box of the warp's bodies.  Rounding is monotone, so the FP32 separation a lane
// computes, fl(fma(dz,dz,fma(dy,dy,dx*dx))) with dx = fl(com.x - p.x), lies between the same
// expression evaluated at the box's nearest and farthest offsets: a node accepted at the nearest
// offset (w^2 < th2 * r2min) is accepted by every lane, one refused at the farthest is refused by
// every lane, and only the nodes in between take the per-lane test (one broadcast per node).
// Leaves are accepted by every lane but their own body.  Accepted (node, lanes) pairs go to an
// interaction list; a refused node's children go back on the stack as one sibling chain with the
// lanes that refused it.  Evaluation: every lane runs down the list (three broadcast shared-memory
// reads per two entries, stored as interleaved pairs) and keeps the terms its mask bit selects, with
// walk_kernel's arithmetic per term; only the order of the sum differs.
// Resident warps hide the traversal's dependent loads: 4 warps per CTA with 6.25 KB of shared
// memory each and at most 64 registers give 8 CTAs (32 warps) per SM (13.1 ms per walk at
// N = 4194304, against 15.2 ms with a 512-entry stack at 24 warps per SM).
constexpr int kLwWarps = 4;      // warps per CTA
constexpr int kLwStack = 320;    // stack entries per warp (a walk of 2M bodies peaks near 220)
constexpr int kLwDfs = kLwStack - 64;  // above this many entries the warp pops one entry at a time
constexpr int kLwList = 128;     // list entries per warp before an evaluation pass

struct LwWarp {
    int st[kLwStack], en[kLwStack];  // sibling chain: nodes st, skip[st], ... below en
    unsigned mk[kLwStack];           // lanes still walking below the chain's parent
    // accepted node: centre of mass and G M (or a bucket leaf's body), stored by pairs of entries:
    // pxy[q] = (x, x', y, y') and pzw[q] = (z, z', w, w') of entries 2q and 2q + 1, so that the
    // evaluation reads two entries with two float4 loads whose halves are its FP32x2 operands
    float4 pxy[kLwList / 2], pzw[kLwList / 2];
    unsigned lm[kLwList];            // lanes that take it
};
static_assert(kLwList % 2 == 0 && (3 * kLwStack * sizeof(int)) % 16 == 0, "float4 pairs of list entries");

// writes list entry `at`
__device__ __forceinline__ void lw_put(LwWarp &W, int at, float x, float y, float z, float w, unsigned m) {
    float *a = reinterpret_cast<float *>(&W.pxy[at >> 1]) + (at & 1);
    float *b = reinterpret_cast<float *>(&W.pzw[at >> 1]) + (at & 1);
    a[0] = x;
    a[2] = y;
    b[0] = z;
    b[2] = w;
    W.lm[at] = m;
}
constexpr size_t kLwSmem = sizeof(LwWarp) * kLwWarps;

__device__ __forceinline__ float lw_r2(float dx, float dy, float dz) {
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// distance from a box [lo, hi] to c along one axis: nearest and farthest offsets as the lanes
// round them (c - hi <= fl(c - p) <= c - lo for every lane p in the box)
__device__ __forceinline__ void lw_axis(float c, float lo, float hi, float &dmin, float &dmax) {
    const float a = __fsub_rn(c, hi), b = __fsub_rn(c, lo);
    dmin = a > 0.f ? a : (b < 0.f ? -b : 0.f);
    dmax = fmaxf(fabsf(a), fabsf(b));
}

// Evaluation pass over the list: two entries per step in packed FP32x2 arithmetic (per lane of the
// pair the same correctly rounded operations as the scalar walk: x + (-p) = x - p exactly as
// rounded), summed in two partial sums.
template <bool SOFT, bool COUNT>
__device__ __forceinline__ void lw_eval(const LwWarp &W, int len, unsigned lane, float4 p, float eps2, float &ax,
                                        float &ay, float &az, uint32_t &cnt) {
    const float2 npx = make_float2(-p.x, -p.x), npy = make_float2(-p.y, -p.y), npz = make_float2(-p.z, -p.z);
    const float2 zero = make_float2(0.f, 0.f);
    const unsigned lbit = 1u << lane;
    float2 fx = zero, fy = zero, fz = zero, gx = zero, gy = zero, gz = zero;
    auto pair = [&](int e, float2 &ox, float2 &oy, float2 &oz) {  // entries e, e + 1 (e even)
        const float4 P = W.pxy[e >> 1], Q = W.pzw[e >> 1];
        const float2 X = make_float2(P.x, P.y), Y = make_float2(P.z, P.w);
        const float2 Z = make_float2(Q.x, Q.y), M = make_float2(Q.z, Q.w);
        const uint2 mk = *reinterpret_cast<const uint2 *>(&W.lm[e]);
        const bool b0 = (mk.x & lbit) != 0u, b1 = (mk.y & lbit) != 0u;
        const float2 dx = __fadd2_rn(X, npx), dy = __fadd2_rn(Y, npy), dz = __fadd2_rn(Z, npz);
        float2 r2 = __fmul2_rn(dx, dx);
        r2 = __ffma2_rn(dy, dy, r2);
        r2 = __ffma2_rn(dz, dz, r2);
        const float2 inv = make_float2(rsqrt_t(SOFT ? r2.x + eps2 : r2.x), rsqrt_t(SOFT ? r2.y + eps2 : r2.y));
        float2 sc = __fmul2_rn(__fmul2_rn(__fmul2_rn(M, inv), inv), inv);
        sc.x = b0 ? sc.x : 0.f;
        sc.y = b1 ? sc.y : 0.f;
        ox = __ffma2_rn(sc, dx, ox);
        oy = __ffma2_rn(sc, dy, oy);
        oz = __ffma2_rn(sc, dz, oz);
        if constexpr (COUNT) cnt += (b0 ? 1u : 0u) + (b1 ? 1u : 0u);
    };
    int e = 0;
    for (; e + 3 < len; e += 4) {  // two independent pairs per step
        pair(e, fx, fy, fz);
        pair(e + 2, gx, gy, gz);
    }
    if (e + 1 < len) {
        pair(e, fx, fy, fz);
        e += 2;
    }
    fx = __fadd2_rn(fx, gx);
    fy = __fadd2_rn(fy, gy);
    fz = __fadd2_rn(fz, gz);
    if (e < len) {  // e even: the first half of its pair
        const float4 P = W.pxy[e >> 1], Q = W.pzw[e >> 1];
        const float X = P.x, Y = P.z, Z = Q.x, M = Q.z;
        const bool bit = (W.lm[e] & lbit) != 0u;
        const float dx = __fsub_rn(X, p.x), dy = __fsub_rn(Y, p.y), dz = __fsub_rn(Z, p.z);
        const float r2 = lw_r2(dx, dy, dz);
        const float inv = rsqrt_t(SOFT ? r2 + eps2 : r2);
        float sc = __fmul_rn(__fmul_rn(__fmul_rn(M, inv), inv), inv);
        sc = bit ? sc : 0.f;
        fx.x = __fmaf_rn(sc, dx, fx.x);
        fy.x = __fmaf_rn(sc, dy, fy.x);
        fz.x = __fmaf_rn(sc, dz, fz.x);
        if constexpr (COUNT) cnt += bit ? 1u : 0u;
    }
    ax += fx.x + fx.y;
    ay += fy.x + fy.y;
    az += fz.x + fz.y;
}

template <bool SOFT, bool COUNT>
__global__ void __launch_bounds__(kLwWarps * 32, 8) list_walk_kernel(int64_t n, int64_t n_nodes, const float4 *rec,
                                                                  const float4 *bodies, float th2, float eps2,
                                                                  float4 *slot_acc, uint32_t *slot_cnt, int *status) {
    extern __shared__ __align__(16) unsigned char lw_smem[];
    LwWarp &W = reinterpret_cast<LwWarp *>(lw_smem)[threadIdx.x >> 5];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt = (1u << lane) - 1u;  // lanes below this one
    const int64_t base = ((int64_t)blockIdx.x * kLwWarps + (threadIdx.x >> 5)) * 32;
    if (base >= n) return;  // whole warps only
    const int64_t s = base + lane;
    const bool active = s < n;
    const unsigned full = __ballot_sync(0xffffffffu, active);
    float4 p = bodies[active ? s : base];  // lanes past n stand on lane 0's body (in no mask)
    float lox = p.x, hix = p.x, loy = p.y, hiy = p.y, loz = p.z, hiz = p.z;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lox = fminf(lox, __shfl_xor_sync(0xffffffffu, lox, o));
        hix = fmaxf(hix, __shfl_xor_sync(0xffffffffu, hix, o));
        loy = fminf(loy, __shfl_xor_sync(0xffffffffu, loy, o));
        hiy = fmaxf(hiy, __shfl_xor_sync(0xffffffffu, hiy, o));
        loz = fminf(loz, __shfl_xor_sync(0xffffffffu, loz, o));
        hiz = fmaxf(hiz, __shfl_xor_sync(0xffffffffu, hiz, o));
    }
    const int4 *recb = reinterpret_cast<const int4 *>(rec);
    float ax = 0.f, ay = 0.f, az = 0.f;
    uint32_t cnt = 0;
    int top = 0, len = 0;  // warp-uniform stack and list sizes
    const int nn = (int)n_nodes;
    if (nn > 1) {  // the root's children: nodes 1, skip[1], ... below nn
        if (lane == 0) {
            W.st[0] = 1;
            W.en[0] = nn;
            W.mk[0] = full;
        }
        top = 1;
    }
    __syncwarp();
    // every pop takes one (node, warp) pair and each node enters the stack once per warp: at most
    // n_nodes batches
    for (int64_t batch = 0; top > 0; ++batch) {
        if (batch > n_nodes) {
            if (lane == 0) atomicExch(status, 2);
            break;
        }
        if (len > kLwList - 32) {  // room for this batch's appends (at most one per popped entry)
            __syncwarp();
            lw_eval<SOFT, COUNT>(W, len, lane, p, eps2, ax, ay, az, cnt);
            len = 0;
            __syncwarp();
        }
        // Pop k entries; their pushes (a sibling remainder and a child chain each) need top + k <= cap.
        // Up to kLwDfs entries the warp pops 32 at a time (so at most kLwDfs + 32 after a batch);
        // above, one at a time: depth first from there, the stack grows by at most one entry per
        // tree level (21) before it shrinks, so it stays below the capacity.
        const int k = min(top > kLwDfs ? 1 : min(32, top), kLwStack - top);
        if (k <= 0) {
            if (lane == 0) atomicExch(status, 3);
            break;
        }
        const bool have = (int)lane < k;
        int st = 0, en = 0;
        unsigned mk = 0;
        if (have) {
            const int idx = top - 1 - (int)lane;
            st = W.st[idx];
            en = W.en[idx];
            mk = W.mk[idx];
        }
        top -= k;
        __syncwarp();
        float4 A = make_float4(0.f, 0.f, 0.f, 0.f);
        int4 B = make_int4(0, 0, 0, 0);
        if (have) {
            A = rec[2 * (size_t)st];
            B = recb[2 * (size_t)st + 1];
        }
        const bool leaf = have && B.z < 0;
        const int count = B.z & 0x7fffffff;
        const float w2 = __int_as_float(B.w);
        bool far = false, near = false, mixed = false;
        if (have && !leaf) {
            float nx, fx, ny, fy, nz, fz;
            lw_axis(A.x, lox, hix, nx, fx);
            lw_axis(A.y, loy, hiy, ny, fy);
            lw_axis(A.z, loz, hiz, nz, fz);
            far = w2 < __fmul_rn(th2, lw_r2(nx, ny, nz));
            near = !far && !(w2 < __fmul_rn(th2, lw_r2(fx, fy, fz)));
            mixed = !far && !near;
        }
        // the in-between nodes: each lane of the node's mask applies walk_kernel's test
        unsigned acc = 0;
        unsigned mm = __ballot_sync(0xffffffffu, mixed);
        while (mm) {
            const int j = __ffs(mm) - 1;
            mm &= mm - 1;
            const float cx = __shfl_sync(0xffffffffu, A.x, j), cy = __shfl_sync(0xffffffffu, A.y, j);
            const float cz = __shfl_sync(0xffffffffu, A.z, j), cw = __shfl_sync(0xffffffffu, w2, j);
            const float dx = __fsub_rn(cx, p.x), dy = __fsub_rn(cy, p.y), dz = __fsub_rn(cz, p.z);
            // every lane tests; lane j keeps the answers of the lanes in its node's mask
            const unsigned a = __ballot_sync(0xffffffffu, cw < __fmul_rn(th2, lw_r2(dx, dy, dz)));
            if ((int)lane == j) acc = a & mk;
        }
        unsigned em = 0;
        if (leaf && count == 1) {
            const int64_t own = (int64_t)B.y - base;  // the lane whose body this leaf holds
            em = mk & ~((own >= 0 && own < 32) ? (1u << own) : 0u);
        } else if (far) {
            em = mk;
        } else if (mixed) {
            em = acc;
        }
        const bool app = em != 0u;
        const unsigned ab = __ballot_sync(0xffffffffu, app);
        if (app) lw_put(W, len + __popc(ab & lt), A.x, A.y, A.z, A.w, em);
        len += __popc(ab);
        const bool rem = have && B.x < en;
        const unsigned rb = __ballot_sync(0xffffffffu, rem);
        if (rem) {
            const int at = top + __popc(rb & lt);
            W.st[at] = B.x;
            W.en[at] = en;
            W.mk[at] = mk;
        }
        top += __popc(rb);
        const unsigned cm = near ? mk : (mixed ? (mk & ~acc) : 0u);
        const bool ch = cm != 0u;
        const unsigned cb = __ballot_sync(0xffffffffu, ch);
        if (ch) {
            const int at = top + __popc(cb & lt);
            W.st[at] = st + 1;
            W.en[at] = B.x;
            W.mk[at] = cm;
        }
        top += __popc(cb);
        // bucket leaves (bodies sharing a full-depth code): one entry per body, its own lane left out
        unsigned ml = __ballot_sync(0xffffffffu, leaf && count > 1);
        while (ml) {
            const int j = __ffs(ml) - 1;
            ml &= ml - 1;
            const int f = __shfl_sync(0xffffffffu, B.y, j), c = __shfl_sync(0xffffffffu, count, j);
            const unsigned bm = __shfl_sync(0xffffffffu, mk, j);
            for (int q0 = 0; q0 < c; q0 += 32) {
                if (len > kLwList - 32) {
                    __syncwarp();
                    lw_eval<SOFT, COUNT>(W, len, lane, p, eps2, ax, ay, az, cnt);
                    len = 0;
                    __syncwarp();
                }
                const int q = f + q0 + (int)lane;
                const int64_t own = (int64_t)q - base;
                const unsigned m1 = bm & ~((own >= 0 && own < 32) ? (1u << own) : 0u);
                const bool ap = q0 + (int)lane < c && m1 != 0u;
                const unsigned b2 = __ballot_sync(0xffffffffu, ap);
                if (ap) {
                    const float4 Q = bodies[q];
                    lw_put(W, len + __popc(b2 & lt), Q.x, Q.y, Q.z, Q.w, m1);
                }
                len += __popc(b2);
            }
        }
        __syncwarp();
    }
    __syncwarp();
    lw_eval<SOFT, COUNT>(W, len, lane, p, eps2, ax, ay, az, cnt);
    if (active) {
        slot_acc[s] = make_float4(ax, ay, az, 0.f);
        if constexpr (COUNT) slot_cnt[s] = cnt;
    }
}

// slot order -> body order, optionally kicking the velocities with the new acceleration
template <typename T>
__global__ void scatter_acc_kernel(int64_t n, const int32_t *perm, const void *slot_acc_v, const uint32_t *slot_cnt,
                                   double4 *acc, uint32_t *ninter, double4 *vel, double kick) {
    using V = typename V4<T>::type;
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const V a = reinterpret_cast<const V *>(slot_acc_v)[s];
    const int32_t b = perm[s];
    const double4 ad = make_double4((double)a.x, (double)a.y, (double)a.z, 0.0);
    acc[b] = ad;
    if (ninter) ninter[b] = slot_cnt[s];
    if (vel) {
        double4 v = vel[b];
        v.x = fma(kick, ad.x, v.x);
        v.y = fma(kick, ad.y, v.y);
        v.z = fma(kick, ad.z, v.z);
        vel[b] = v;
    }
}

__global__ void drift_kernel(int64_t n, double4 *pm, const double4 *vel, double h) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = pm[i];
    const double4 v = vel[i];
    p.x = fma(h, v.x, p.x);
    p.y = fma(h, v.y, p.y);
    p.z = fma(h, v.z, p.z);
    pm[i] = p;
}

__global__ void ids_to_keys_kernel(int64_t n, const int32_t *ids, unsigned long long *keys, int32_t *vals) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    keys[s] = (unsigned long long)(uint32_t)ids[s];
    vals[s] = (int32_t)s;
}

// gather for the spatial reorder
template <typename V>
__global__ void gather_kernel(int64_t n, const int32_t *perm, const V *in, V *out) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) out[s] = in[perm[s]];
}

}  // namespace gtd

using namespace gtd;

static unsigned blocks_for(int64_t n, int t = kTT) { return (unsigned)((n + t - 1) / t); }

// Float walk: 0 = walk_kernel with A and B in separate arrays, 1 = walk_kernel with interleaved
// records, 2 = list_walk_kernel (interleaved records; the default: 13.1 ms against 21.0 ms for 1 at
// N = 4194304, theta = 0.5).  Double trees take walk_kernel.
constexpr int kDefaultWalkVariant = 2;
constexpr int kNumWalkVariants = 3;
static int walk_variant_of(const gtd_system *s) { return s->walk_variant < 0 ? kDefaultWalkVariant : s->walk_variant; }

void release_tree(gtd_system *s) {
    cudaFree(s->tree_nbuf);
    cudaFree(s->tree_kbuf);
    cudaFreeHost(s->host_total);
    cudaFree(s->sc4);
    cudaFree(s->sc1);
    cudaFree(s->sci);
    cudaFree(s->bh_ninter);
    s->tree_nbuf = s->tree_kbuf = nullptr;
    s->host_total = nullptr;
    s->sc4 = nullptr;
    s->sc1 = nullptr;
    s->sci = nullptr;
    s->bh_ninter = nullptr;
    s->tree_n = s->node_cap = 0;
    s->tree_valid = false;
}

template <typename P>
static P *carve(char *&cur, size_t count) {
    const size_t bytes = ((sizeof(P) * count) + 255) & ~(size_t)255;
    P *p = reinterpret_cast<P *>(cur);
    cur += bytes;
    return p;
}

static size_t carve_size(size_t bytes) { return (bytes + 255) & ~(size_t)255; }

static int ensure_tree_n(gtd_system *s, int64_t n) {
    if (n <= s->tree_n && s->tree_nbuf) return GTD_OK;
    cudaFree(s->tree_nbuf);
    s->tree_nbuf = nullptr;
    const size_t nn = (size_t)n + 1;
    s->scratch_words = radix_scratch_words(n) + scan_scratch_words((int64_t)nn) + 64;
    size_t total = 0;
    total += 2 * carve_size(8 * nn);            // codes, codes_alt
    total += 2 * carve_size(4 * nn);            // perm, perm_alt
    total += carve_size(4 * nn);                // lcp
    total += carve_size(4 * nn);                // node_start
    total += carve_size(4 * nn);                // own_leaf
    total += 2 * carve_size(32 * nn);           // slot_pos, slot_acc (double4 worst case)
    total += carve_size(4 * nn);                // slot_cnt
    total += carve_size(4 * s->scratch_words);  // scratch
    total += carve_size(8 * 6 * kBBoxBlocks);   // bbox partials
    total += carve_size(8 * 6) + carve_size(64) + carve_size(4 * 64);
    GTD_CUDA(cudaMalloc(&s->tree_nbuf, total));
    char *c = reinterpret_cast<char *>(s->tree_nbuf);
    s->codes = carve<unsigned long long>(c, nn);
    s->codes_alt = carve<unsigned long long>(c, nn);
    s->perm = carve<int32_t>(c, nn);
    s->perm_alt = carve<int32_t>(c, nn);
    s->lcp = carve<int32_t>(c, nn);
    s->node_start = carve<uint32_t>(c, nn);
    s->own_leaf = carve<int32_t>(c, nn);
    s->slot_pos = carve<double4>(c, nn);
    s->slot_acc = carve<double4>(c, nn);
    s->slot_cnt = carve<uint32_t>(c, nn);
    s->scratch = carve<uint32_t>(c, s->scratch_words);
    s->bbox_part = carve<double>(c, 6 * kBBoxBlocks);
    s->box_dev = carve<double>(c, 6);
    s->status = carve<int>(c, 16);
    s->depth_off = carve<uint32_t>(c, 64);
    GTD_CUDA(cudaMemsetAsync(s->status, 0, 16 * sizeof(int), s->stream));  // [0] build, [1] walk
    if (!s->host_total) GTD_CUDA(cudaMallocHost(&s->host_total, 16 * sizeof(uint32_t)));
    s->tree_n = n;
    return GTD_OK;
}

static int ensure_tree_nodes(gtd_system *s, int64_t nodes) {
    if (nodes <= s->node_cap && s->tree_kbuf) return GTD_OK;
    cudaFree(s->tree_kbuf);
    s->tree_kbuf = nullptr;
    const size_t k = (size_t)(nodes + nodes / 4 + 1024);
    size_t total = 2 * carve_size(k) + 3 * carve_size(4 * k) + carve_size(32 * k) + carve_size(8 * k) +
                   carve_size(32 * k) + carve_size(16 * k) + carve_size(8 * k) + carve_size(4 * k);
    GTD_CUDA(cudaMalloc(&s->tree_kbuf, total));
    char *c = reinterpret_cast<char *>(s->tree_kbuf);
    s->ndepth = carve<int8_t>(c, k);
    s->nleaf = carve<int8_t>(c, k);
    s->nfirst = carve<int32_t>(c, k);
    s->ncount = carve<int32_t>(c, k);
    s->nskip = carve<int32_t>(c, k);
    s->ncom = carve<double4>(c, k);
    s->nwidth = carve<double>(c, k);
    s->nwalk_a = carve<double4>(c, k);
    s->nwalk_b = carve<int4>(c, k);
    s->nwalk_w2 = carve<double>(c, k);
    s->depth_list = carve<int32_t>(c, k);
    s->node_cap = (int64_t)k;
    return GTD_OK;
}

// Morton codes of the current positions, sorted (codes, perm).  Leaves the box in s->box_dev.
static int morton_sort(gtd_system *s, bool tree_float) {
    const int64_t n = s->n;
    int rc = ensure_tree_n(s, n);
    if (rc) return rc;
    const double4 *pm = s->pm[s->cur];
    cudaStream_t st = s->stream;
    GTD_CUDA(cudaMemsetAsync(s->status, 0, sizeof(int), st));
    const int bb = (int)std::min<int64_t>(kBBoxBlocks, std::max<int64_t>(1, (n + kTT - 1) / kTT));
    if (tree_float) {
        bbox_partial_kernel<true><<<bb, kTT, 0, st>>>(pm, n, s->bbox_part);
        bbox_final_kernel<true><<<1, 32, 0, st>>>(s->bbox_part, bb, s->box_dev, s->status);
        morton_kernel<true><<<blocks_for(n), kTT, 0, st>>>(pm, n, s->box_dev, s->codes, s->perm, s->status);
    } else {
        bbox_partial_kernel<false><<<bb, kTT, 0, st>>>(pm, n, s->bbox_part);
        bbox_final_kernel<false><<<1, 32, 0, st>>>(s->bbox_part, bb, s->box_dev, s->status);
        morton_kernel<false><<<blocks_for(n), kTT, 0, st>>>(pm, n, s->box_dev, s->codes, s->perm, s->status);
    }
    GTD_CHECK_LAUNCH();
    s->launches += 3;
    return radix_sort_u64(s->codes, s->perm, s->codes_alt, s->perm_alt, n, 63, s->scratch, st, &s->launches);
}

// Hilbert order of the current positions in s->perm (slot -> body), over the root box of the T=double
// tree (any box holding the bodies would do: the order only has to be spatially compact).
static int hilbert_sort(gtd_system *s) {
    const int64_t n = s->n;
    int rc = ensure_tree_n(s, n);
    if (rc) return rc;
    const double4 *pm = s->pm[s->cur];
    cudaStream_t st = s->stream;
    GTD_CUDA(cudaMemsetAsync(s->status, 0, sizeof(int), st));
    const int bb = (int)std::min<int64_t>(kBBoxBlocks, std::max<int64_t>(1, (n + kTT - 1) / kTT));
    bbox_partial_kernel<false><<<bb, kTT, 0, st>>>(pm, n, s->bbox_part);
    bbox_final_kernel<false><<<1, 32, 0, st>>>(s->bbox_part, bb, s->box_dev, s->status);
    hilbert_kernel<<<blocks_for(n), kTT, 0, st>>>(pm, n, s->box_dev, s->codes, s->perm);
    GTD_CHECK_LAUNCH();
    s->launches += 3;
    return radix_sort_u64(s->codes, s->perm, s->codes_alt, s->perm_alt, n, 63, s->scratch, st, &s->launches);
}

static int read_status(gtd_system *s) {
    GTD_CUDA(cudaMemcpyAsync(s->host_total + 1, s->status, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    const int st = (int)s->host_total[1];
    if (st == GTD_ERR_INVALID_BODY_PLACEMENT)
        return fail(st, "Error: a body does not lie within the Barnes-Hut root cube (non-finite position?).");
    if (st == GTD_ERR_INDISTINGUISHABLE)
        return fail(st, "Error: two bodies have positions that are either equal or so close together that they "
                        "cannot be told apart.");
    if (st) return fail(st, "device status %d", st);
    return GTD_OK;
}

static int bh_build_impl(gtd_system *s, int tree_float) {
    const int64_t n = s->n;
    s->tree_valid = false;
    if (n < 2) {
        // the reference's root cube of a single body has zero size and rejects its own body
        return fail(GTD_ERR_INVALID_BODY_PLACEMENT, "Error: body with ID = 0 is not contained within the current "
                                                    "Barnes-Hut cube.");
    }
    s->tree_float = tree_float ? 1 : 0;
    int rc = morton_sort(s, tree_float != 0);
    if (rc) return rc;
    cudaStream_t st = s->stream;
    const double4 *pm = s->pm[s->cur];
    if (tree_float)
        lcp_count_kernel<true><<<blocks_for(n + 1), kTT, 0, st>>>(s->codes, s->perm, pm, n, s->lcp, s->node_start,
                                                                  s->status);
    else
        lcp_count_kernel<false><<<blocks_for(n + 1), kTT, 0, st>>>(s->codes, s->perm, pm, n, s->lcp, s->node_start,
                                                                   s->status);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    rc = exclusive_scan_u32(s->node_start, s->node_start, n + 1, s->scratch, st, &s->launches);
    if (rc) return rc;
    GTD_CUDA(cudaMemcpyAsync(s->host_total, s->node_start + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    GTD_CUDA(cudaMemcpyAsync(s->host_total + 1, s->status, sizeof(int), cudaMemcpyDeviceToHost, st));
    GTD_CUDA(cudaStreamSynchronize(st));
    rc = read_status(s);
    if (rc) return rc;
    const int64_t nodes = s->host_total[0];
    rc = ensure_tree_nodes(s, nodes);
    if (rc) return rc;
    GTD_CUDA(cudaMemsetAsync(s->depth_off, 0, 64 * sizeof(uint32_t), st));
    EmitArgs e{n, s->codes, s->perm, s->lcp, s->node_start, pm, s->box_dev, s->ndepth, s->nleaf, s->nfirst,
               s->ncount, s->nskip, s->own_leaf, s->ncom, s->nwidth};
    if (tree_float) emit_kernel<true><<<blocks_for(n), kTT, 0, st>>>(e);
    else emit_kernel<false><<<blocks_for(n), kTT, 0, st>>>(e);
    GTD_CHECK_LAUNCH();
    const unsigned depth_blocks = (unsigned)((nodes + kDepthChunk - 1) / kDepthChunk);
    depth_count_kernel<<<depth_blocks, kTT, 0, st>>>(s->ndepth, s->nleaf, nodes, s->depth_off);
    depth_offsets_kernel<<<1, 32, 0, st>>>(s->depth_off);
    depth_scatter_kernel<<<depth_blocks, kTT, 0, st>>>(s->ndepth, s->nleaf, nodes, s->depth_off, s->depth_list);
    GTD_CHECK_LAUNCH();
    s->launches += 4;
    for (int d = kMaxDepth - 1; d >= 0; --d) {
        com_level_kernel<<<4 * 148, kTT, 0, st>>>(s->depth_list, s->depth_off, d, s->nskip, s->ncom);
        s->launches += 1;
    }
    GTD_CHECK_LAUNCH();
    s->walk_interleaved = (tree_float && walk_variant_of(s) >= 1) ? 1 : 0;
    if (s->walk_interleaved)
        walk_records_kernel<true, true><<<blocks_for(nodes), kTT, 0, st>>>(nodes, s->ncom, s->nwidth, s->nleaf,
                                                                            s->nfirst, s->ncount, s->nskip, s->G,
                                                                            s->nwalk_a, s->nwalk_b, s->nwalk_w2);
    else if (tree_float)
        walk_records_kernel<true><<<blocks_for(nodes), kTT, 0, st>>>(nodes, s->ncom, s->nwidth, s->nleaf, s->nfirst,
                                                                      s->ncount, s->nskip, s->G, s->nwalk_a,
                                                                      s->nwalk_b, s->nwalk_w2);
    else
        walk_records_kernel<false><<<blocks_for(nodes), kTT, 0, st>>>(nodes, s->ncom, s->nwidth, s->nleaf, s->nfirst,
                                                                       s->ncount, s->nskip, s->G, s->nwalk_a,
                                                                       s->nwalk_b, s->nwalk_w2);
    GTD_CHECK_LAUNCH();
    if (tree_float) slot_bodies_kernel<true><<<blocks_for(n), kTT, 0, st>>>(pm, s->perm, n, s->G, s->slot_pos);
    else slot_bodies_kernel<false><<<blocks_for(n), kTT, 0, st>>>(pm, s->perm, n, s->G, s->slot_pos);
    GTD_CHECK_LAUNCH();
    s->launches += 2;
    s->n_nodes = nodes;
    s->tree_valid = true;
    return GTD_OK;
}

// Launches the walk form for (softened?, counted?) on the handle's stream.
template <typename T, bool IL>
static void launch_walk(gtd_system *s, T th2, T e2, bool count) {
    const int64_t n = s->n;
    const bool soft = e2 != (T)0;
    auto go = [&](auto kern) {
        kern<<<blocks_for(n), kTT, 0, s->stream>>>(n, s->n_nodes, s->nwalk_a, s->nwalk_b, s->nwalk_w2, s->slot_pos,
                                                   s->own_leaf, th2, e2, s->slot_acc, s->slot_cnt);
    };
    if (soft) {
        if (count) go(walk_kernel<T, IL, true, true>);
        else go(walk_kernel<T, IL, true, false>);
    } else {
        if (count) go(walk_kernel<T, IL, false, true>);
        else go(walk_kernel<T, IL, false, false>);
    }
}

// The list walk (float trees, interleaved records); errors go to status[1].
static int launch_list_walk(gtd_system *s, float th2, float e2, bool count) {
    const int64_t n = s->n;
    const bool soft = e2 != 0.f;
    const unsigned blocks = (unsigned)((n + kLwWarps * 32 - 1) / (kLwWarps * 32));
    cudaError_t ce = cudaSuccess;
    auto go = [&](auto kern) {
        ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLwSmem);
        if (ce != cudaSuccess) return;
        kern<<<blocks, kLwWarps * 32, kLwSmem, s->stream>>>(
            n, s->n_nodes, reinterpret_cast<const float4 *>(s->nwalk_a), reinterpret_cast<const float4 *>(s->slot_pos),
            th2, e2, reinterpret_cast<float4 *>(s->slot_acc), s->slot_cnt, s->status + 1);
    };
    if (soft) {
        if (count) go(list_walk_kernel<true, true>);
        else go(list_walk_kernel<true, false>);
    } else {
        if (count) go(list_walk_kernel<false, true>);
        else go(list_walk_kernel<false, false>);
    }
    GTD_CUDA(ce);
    return GTD_OK;
}

// Reads and clears the walk's error word (status[1]); call after the stream has the walks queued.
static int walk_status(gtd_system *s) {
    int h = 0;
    GTD_CUDA(cudaMemcpyAsync(&h, s->status + 1, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    if (h == 0) return GTD_OK;
    GTD_CUDA(cudaMemsetAsync(s->status + 1, 0, sizeof(int), s->stream));
    return fail(GTD_ERR_CAPACITY, "Barnes-Hut list walk: %s", h == 3 ? "stack capacity exceeded" : "walk did not end");
}

// Walk for every body; accelerations in body order, optionally kicking v by kick * a, and with
// `count` the interactions each body took (for gtd_bh_accelerations' n_inter).
static int bh_walk_impl(gtd_system *s, double kick, bool do_kick, bool count) {
    if (!s->tree_valid) return fail(GTD_ERR_INVALID_ARGUMENT, "no Barnes-Hut tree: call gtd_bh_build first");
    const int64_t n = s->n;
    cudaStream_t st = s->stream;
    if (!s->bh_ninter) GTD_CUDA(cudaMalloc(&s->bh_ninter, sizeof(uint32_t) * (size_t)s->cap));
    uint32_t *ninter = count ? s->bh_ninter : nullptr;
    if (s->tree_float) {
        const float th2 = (float)(s->theta * s->theta), e2 = (float)(s->eps * s->eps);
        if (s->walk_interleaved && walk_variant_of(s) == 2) {
            int rc = launch_list_walk(s, th2, e2, count);
            if (rc) return rc;
        } else if (s->walk_interleaved) {
            launch_walk<float, true>(s, th2, e2, count);
        } else {
            launch_walk<float, false>(s, th2, e2, count);
        }
        GTD_CHECK_LAUNCH();
        scatter_acc_kernel<float><<<blocks_for(n), kTT, 0, st>>>(n, s->perm, s->slot_acc, s->slot_cnt, s->acc,
                                                                 ninter, do_kick ? s->vel : nullptr, kick);
    } else {
        const double th2 = s->theta * s->theta, e2 = s->eps * s->eps;
        launch_walk<double, false>(s, th2, e2, count);
        GTD_CHECK_LAUNCH();
        scatter_acc_kernel<double><<<blocks_for(n), kTT, 0, st>>>(n, s->perm, s->slot_acc, s->slot_cnt, s->acc,
                                                                  ninter, do_kick ? s->vel : nullptr, kick);
    }
    GTD_CHECK_LAUNCH();
    s->launches += 2;
    return GTD_OK;
}

// Leapfrog KDK with Barnes-Hut forces in the reference's schedule (gregsys.hpp:2893-2945):
// initial walk and half kick, then per step a full drift, a rebuild, a walk and a full kick
// (the velocities end half a step ahead of the positions, as in the reference).
int bh_evolve_kdk(gtd_system *s, uint64_t steps) {
    if (s->n == 0) return GTD_OK;
    const int tf = s->tree_float;
    int rc = bh_build_impl(s, tf);
    if (rc) return rc;
    rc = bh_walk_impl(s, 0.5 * s->dt, true, false);
    if (rc) return rc;
    for (uint64_t k = 0; k < steps; ++k) {
        drift_kernel<<<blocks_for(s->n), kTT, 0, s->stream>>>(s->n, s->pm[s->cur], s->vel, s->dt);
        GTD_CHECK_LAUNCH();
        s->launches += 1;
        rc = bh_build_impl(s, tf);
        if (rc) return rc;
        rc = bh_walk_impl(s, s->dt, true, false);
        if (rc) return rc;
        if (s->coll != GTD_NO_COLL) {
            rc = run_bh_collisions(s);
            if (rc) return rc;
        }
    }
    return walk_status(s);
}

static int copy_bh_out(gtd_system *s, double *a3, uint32_t *n_inter) {
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    if (a3) {
        int rc = copy_acc_out(s, a3);
        if (rc) return rc;
    }
    if (n_inter) {
        const int64_t n = s->n;
        std::vector<uint32_t> h((size_t)n);
        GTD_CUDA(cudaMemcpy(h.data(), s->bh_ninter, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToHost));
        std::vector<int64_t> row;
        int rc = output_rows(s, row);
        if (rc) return rc;
        for (int64_t i = 0; i < n; ++i) n_inter[row[(size_t)i]] = h[(size_t)i];
    }
    return GTD_OK;
}

int bh_accelerations(gtd_system *s, double *a3, uint32_t *n_inter) {
    int rc = bh_build_impl(s, s->tree_float);
    if (rc) return rc;
    rc = bh_walk_impl(s, 0.0, false, n_inter != nullptr);
    if (rc) return rc;
    rc = walk_status(s);
    if (rc) return rc;
    return copy_bh_out(s, a3, n_inter);
}

// Spatial (Hilbert) reordering of every per-body array, so that the direct-sum rows and warps are
// compact: the mixed kernel's per-row FP32 frame stays close to its bodies and fewer folds need its
// precise path (2.9 % of warp-folds against 6.4 % in Morton order at N = 262144).
int reorder_bodies(gtd_system *s) {
    const int64_t n = s->n;
    if (n < 2) return GTD_OK;
    int rc = hilbert_sort(s);
    if (rc) return rc;
    cudaStream_t st = s->stream;
    if (!s->sc4) {
        GTD_CUDA(cudaMalloc(&s->sc4, sizeof(double4) * (size_t)s->cap));
        GTD_CUDA(cudaMalloc(&s->sc1, sizeof(double) * (size_t)s->cap));
        GTD_CUDA(cudaMalloc(&s->sci, sizeof(int32_t) * (size_t)s->cap));
    }
    const unsigned g = blocks_for(n);
    gather_kernel<double4><<<g, kTT, 0, st>>>(n, s->perm, s->pm[s->cur], s->pm[s->cur ^ 1]);
    s->cur ^= 1;
    gather_kernel<double4><<<g, kTT, 0, st>>>(n, s->perm, s->vel, s->sc4);
    std::swap(s->vel, s->sc4);
    gather_kernel<double4><<<g, kTT, 0, st>>>(n, s->perm, s->acc, s->sc4);
    std::swap(s->acc, s->sc4);
    gather_kernel<double><<<g, kTT, 0, st>>>(n, s->perm, s->rad, s->sc1);
    std::swap(s->rad, s->sc1);
    gather_kernel<double><<<g, kTT, 0, st>>>(n, s->perm, s->rest, s->sc1);
    std::swap(s->rest, s->sc1);
    gather_kernel<int32_t><<<g, kTT, 0, st>>>(n, s->perm, s->ids, s->sci);
    std::swap(s->ids, s->sci);
    GTD_CHECK_LAUNCH();
    s->launches += 6;
    s->ordered = true;
    s->tree_valid = false;
    return GTD_OK;
}

// Puts the bodies back in upload order (ascending ids), undoing reorder_bodies; the order-dependent
// collision passes scan in this order, as the reference scans its std::vector.
int restore_upload_order(gtd_system *s) {
    if (!s->ordered) return GTD_OK;
    const int64_t n = s->n;
    s->ordered = false;
    if (n < 2) return GTD_OK;
    int rc = ensure_tree_n(s, n);
    if (rc) return rc;
    cudaStream_t st = s->stream;
    const unsigned g = blocks_for(n);
    ids_to_keys_kernel<<<g, kTT, 0, st>>>(n, s->ids, s->codes, s->perm);
    GTD_CHECK_LAUNCH();
    s->launches += 1;
    rc = radix_sort_u64(s->codes, s->perm, s->codes_alt, s->perm_alt, n, 32, s->scratch, st, &s->launches);
    if (rc) return rc;
    gather_kernel<double4><<<g, kTT, 0, st>>>(n, s->perm, s->pm[s->cur], s->pm[s->cur ^ 1]);
    s->cur ^= 1;
    gather_kernel<double4><<<g, kTT, 0, st>>>(n, s->perm, s->vel, s->sc4);
    std::swap(s->vel, s->sc4);
    gather_kernel<double4><<<g, kTT, 0, st>>>(n, s->perm, s->acc, s->sc4);
    std::swap(s->acc, s->sc4);
    gather_kernel<double><<<g, kTT, 0, st>>>(n, s->perm, s->rad, s->sc1);
    std::swap(s->rad, s->sc1);
    gather_kernel<double><<<g, kTT, 0, st>>>(n, s->perm, s->rest, s->sc1);
    std::swap(s->rest, s->sc1);
    gather_kernel<int32_t><<<g, kTT, 0, st>>>(n, s->perm, s->ids, s->sci);
    std::swap(s->ids, s->sci);
    GTD_CHECK_LAUNCH();
    s->launches += 6;
    s->tree_valid = false;
    return GTD_OK;
}

extern "C" {

int gtd_bh_build(gtd_system *s, int tree_float) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    int rc = bh_build_impl(s, tree_float);
    if (rc) return rc;
    GTD_CUDA(cudaStreamSynchronize(s->stream));
    return GTD_OK;
}

int gtd_bh_set_tree_float(gtd_system *s, int tree_float) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    s->tree_float = tree_float ? 1 : 0;
    s->tree_valid = false;
    return GTD_OK;
}

int gtd_bh_set_walk_variant(gtd_system *s, int variant) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (variant < -1 || variant >= kNumWalkVariants)
        return fail(GTD_ERR_INVALID_ARGUMENT, "walk variant %d out of range", variant);
    s->walk_variant = variant;
    s->tree_valid = false;  // the record layout is chosen at build time
    return GTD_OK;
}

int gtd_bh_tree_size(gtd_system *s, int64_t *n_nodes, int64_t *n_leaves, double *box6) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (!s->tree_valid) return fail(GTD_ERR_INVALID_ARGUMENT, "no Barnes-Hut tree: call gtd_bh_build first");
    if (n_nodes) *n_nodes = s->n_nodes;
    if (n_leaves) {
        std::vector<int8_t> lf((size_t)s->n_nodes);
        GTD_CUDA(cudaMemcpy(lf.data(), s->nleaf, (size_t)s->n_nodes, cudaMemcpyDeviceToHost));
        int64_t c = 0;
        for (int8_t v : lf) c += v ? 1 : 0;
        *n_leaves = c;
    }
    if (box6) GTD_CUDA(cudaMemcpy(box6, s->box_dev, 6 * sizeof(double), cudaMemcpyDeviceToHost));
    return GTD_OK;
}

int gtd_bh_tree_download(gtd_system *s, uint64_t *codes, int32_t *perm, int8_t *depth, int8_t *is_leaf,
                         int32_t *first, int32_t *count, int32_t *skip, double *mass, double *com3, double *width) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (!s->tree_valid) return fail(GTD_ERR_INVALID_ARGUMENT, "no Barnes-Hut tree: call gtd_bh_build first");
    const size_t n = (size_t)s->n, k = (size_t)s->n_nodes;
    if (codes) GTD_CUDA(cudaMemcpy(codes, s->codes, 8 * n, cudaMemcpyDeviceToHost));
    if (perm) {
        // slot -> upload index of the body
        std::vector<int32_t> p(n), ids(n);
        GTD_CUDA(cudaMemcpy(p.data(), s->perm, 4 * n, cudaMemcpyDeviceToHost));
        GTD_CUDA(cudaMemcpy(ids.data(), s->ids, 4 * n, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) perm[i] = ids[(size_t)p[i]];
    }
    if (depth) GTD_CUDA(cudaMemcpy(depth, s->ndepth, k, cudaMemcpyDeviceToHost));
    if (is_leaf) GTD_CUDA(cudaMemcpy(is_leaf, s->nleaf, k, cudaMemcpyDeviceToHost));
    if (first) GTD_CUDA(cudaMemcpy(first, s->nfirst, 4 * k, cudaMemcpyDeviceToHost));
    if (count) GTD_CUDA(cudaMemcpy(count, s->ncount, 4 * k, cudaMemcpyDeviceToHost));
    if (skip) GTD_CUDA(cudaMemcpy(skip, s->nskip, 4 * k, cudaMemcpyDeviceToHost));
    if (width) GTD_CUDA(cudaMemcpy(width, s->nwidth, 8 * k, cudaMemcpyDeviceToHost));
    if (mass || com3) {
        std::vector<double4> c(k);
        GTD_CUDA(cudaMemcpy(c.data(), s->ncom, sizeof(double4) * k, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < k; ++i) {
            if (mass) mass[i] = c[i].w;
            if (com3) { com3[3 * i] = c[i].x; com3[3 * i + 1] = c[i].y; com3[3 * i + 2] = c[i].z; }
        }
    }
    return GTD_OK;
}

int gtd_bh_accelerations(gtd_system *s, double *a3, uint32_t *n_inter) {
    if (!s) return fail(GTD_ERR_INVALID_ARGUMENT, "system is NULL");
    if (!s->tree_valid) return fail(GTD_ERR_INVALID_ARGUMENT, "no Barnes-Hut tree: call gtd_bh_build first");
    int rc = bh_walk_impl(s, 0.0, false, n_inter != nullptr);
    if (rc) return rc;
    return copy_bh_out(s, a3, n_inter);
}

}  // extern "C"
