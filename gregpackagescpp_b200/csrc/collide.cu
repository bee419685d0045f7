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
// Detection of all overlapping pairs is a tiled O(N^2) kernel (FP64).  The order-dependent
// restitution is resolved by one CTA that orders the outer bodies' groups by their data
// dependencies and applies independent groups in parallel, reproducing the sequential loop's
// result (a single thread takes over above kFastCand pairs); merges run on one block, as the
// reference's sequential scan defines the result.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "callbacks.cuh"
#include "gtd_internal.cuh"
#include "gtd_system.cuh"

namespace gtd {

constexpr int kCT = 256;
constexpr int kMaxCand = 1 << 16;

struct Cand {
    int32_t o, i;
    double dist;
};

// All pairs o < i with dist < r_o + r_i; appends (o, i, dist) to the candidate list.  One CTA per
// (o-tile, j-tile) pair of the upper triangle of TW x TW tiles, so that small systems still spread
// over the SMs; the pair tests of a thread are independent, so the loop keeps several in flight.
// The square root is taken only for pairs whose squared distance is not clearly above
// (r_o + r_i)^2; the overlap decision is the one of the exact test.
template <int TW>
__global__ void __launch_bounds__(TW) overlap_pairs_kernel(int64_t n, int64_t tiles, const double4 *pm,
                                                           const double *rad, Cand *cand, int *count, int cap) {
    __shared__ double4 tp[TW];
    __shared__ double tr[TW];
    // block -> (to, tj), to <= tj: row r of the triangle starts at r*T - r(r-1)/2
    const int64_t b = blockIdx.x, T = tiles;
    auto row_start = [&](int64_t r) { return r * T - r * (r - 1) / 2; };
    const double q = (double)(2 * T + 1);
    int64_t to = (int64_t)floor((q - sqrt(q * q - 8.0 * (double)b)) * 0.5);
    if (to < 0) to = 0;
    if (to > T - 1) to = T - 1;
    while (to > 0 && row_start(to) > b) --to;
    while (to + 1 < T && row_start(to + 1) <= b) ++to;
    const int64_t tj = to + (b - row_start(to));
    const int t = threadIdx.x;
    const int64_t j = tj * TW + t;
    tp[t] = j < n ? pm[j] : make_double4(0, 0, 0, 0);
    tr[t] = j < n ? rad[j] : 0.0;
    __syncthreads();
    const int64_t o = to * TW + t;
    if (o >= n) return;
    const double4 po = pm[o];
    const double ro = rad[o];
    const int lim = (int)min((int64_t)TW, n - tj * TW);
    const int first = tj == to ? t + 1 : 0;  // i > o
#pragma unroll 8
    for (int jj = first; jj < lim; ++jj) {
        const double4 qj = tp[jj];
        const double dx = __dsub_rn(qj.x, po.x), dy = __dsub_rn(qj.y, po.y), dz = __dsub_rn(qj.z, po.z);
        const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        const double rsum = __dadd_rn(ro, tr[jj]);
        // d2 > rsum^2 (1 + 2^-40) implies sqrt(d2) > rsum whatever the roundings: no overlap
        if (d2 > __dmul_rn(__dmul_rn(rsum, rsum), 1.0 + 0x1p-40)) continue;
        const double d = sqrt(d2);
        if (rsum > d) {
            const int k = atomicAdd(count, 1);
            if (k < cap) cand[k] = Cand{(int32_t)o, (int32_t)(tj * TW + jj), d};
        }
    }
}

// Tile width of the detection grid: narrow tiles for small systems (more CTAs, shorter loops).
constexpr int kDTSmall = 32, kDTLarge = 64;
int overlap_tile(int64_t n) { return n <= 32768 ? kDTSmall : kDTLarge; }
int64_t overlap_tiles(int64_t n) { return (n + overlap_tile(n) - 1) / overlap_tile(n); }

static void launch_overlap_pairs(int64_t n, const double4 *pm, const double *rad, Cand *cand, int *count, int cap,
                                 cudaStream_t st) {
    const int64_t tiles = overlap_tiles(n);
    const unsigned blocks = (unsigned)(tiles * (tiles + 1) / 2);
    if (overlap_tile(n) == kDTSmall)
        overlap_pairs_kernel<kDTSmall><<<blocks, kDTSmall, 0, st>>>(n, tiles, pm, rad, cand, count, cap);
    else
        overlap_pairs_kernel<kDTLarge><<<blocks, kDTLarge, 0, st>>>(n, tiles, pm, rad, cand, count, cap);
}

__device__ __forceinline__ bool cand_less(const Cand &a, const Cand &b) {
    if (a.o != b.o) return a.o < b.o;
    if (a.dist != b.dist) return a.dist < b.dist;
    return a.i < b.i;
}

// The s_coll response to one candidate k of outer body o (gregsys.hpp:808-836): the momenta along
// the unit separation were snapshotted for the whole group (pp); returns whether the pair gets the
// impulse, with o's velocity change d_o along u and i's velocity vi updated.
__device__ __forceinline__ bool pair_impulse(const double4 &xo, double rest_o, const double4 &xi, double rest_i,
                                             double d, double2 pp, double4 &vi, double &d_o, double &ux,
                                             double &uy, double &uz) {
    ux = (xi.x - xo.x) / d;
    uy = (xi.y - xo.y) / d;
    uz = (xi.z - xo.z) / d;
    const double mo = xo.w, mi = xi.w;
    const double o_vel = pp.x / mo, i_vel = pp.y / mi;
    const double o_minus_i = o_vel - i_vel;
    const double avg_rest = 0.5 * (rest_o + rest_i);
    if (!(o_vel > 0 || i_vel < 0)) return false;
    if (o_vel <= 0 && i_vel < 0 && o_vel < i_vel) return false;  // already separating
    if (o_vel > 0 && i_vel >= 0 && o_vel < i_vel) return false;
    const double psum = pp.x + pp.y, msum = mo + mi;
    const double new_o = (psum - mi * avg_rest * o_minus_i) / msum;
    const double new_i = (psum + mo * avg_rest * o_minus_i) / msum;
    d_o = new_o - o_vel;
    const double d_i = new_i - i_vel;
    vi.x += d_i * ux;
    vi.y += d_i * uy;
    vi.z += d_i * uz;
    return true;
}

// Momentum of a body along u, as bod->momentum()*r12 (gregbod.hpp:595-597, dot gregvec.hpp:3742).
__device__ __forceinline__ double axis_momentum(const double4 &x, const double4 &v, double ux, double uy, double uz) {
    return x.w * v.x * ux + x.w * v.y * uy + x.w * v.z * uz;
}

// The sequential form (one thread): heap sort of the candidates by (o, dist, i), then the groups in
// order.  Used above kFastCand candidates.
__device__ void resolve_serial(Cand *cand, int c, int cap, const int32_t *perm, const double4 *pm,
                               const double *rest, double4 *vel) {
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
    double2 *mom = reinterpret_cast<double2 *>(cand + cap);
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
            mom[k] = make_double2(axis_momentum(xo, vel[o], ux, uy, uz), axis_momentum(xi, vel[i], ux, uy, uz));
        }
        for (int k = g; k < e; ++k) {
            if (k > g && cand[k].dist == cand[k - 1].dist) continue;  // std::map::emplace keeps the first key
            const int i = body(cand[k].i);
            double d_o, ux, uy, uz;
            double4 vi = vel[i];
            if (pair_impulse(xo, rest[o], pm[i], rest[i], cand[k].dist, mom[k], vi, d_o, ux, uy, uz)) {
                vel[i] = vi;
                double4 vo = vel[o];
                vo.x += d_o * ux;
                vo.y += d_o * uy;
                vo.z += d_o * uz;
                vel[o] = vo;
            }
        }
        g = e;
    }
}

// ---- the parallel resolution ------------------------------------------------------------------
// The reference resolves the outer bodies' groups in order; a group reads and writes the
// velocities of its outer body and of its partners only.  So a group depends on the earlier groups
// that share a body with it, and groups at the same depth of that dependency order touch disjoint
// bodies.  One CTA: sorts the candidates by outer body (bitonic on 64-bit keys in shared memory)
// and each group by (distance, partner); gives every group its depth (the longest chain of earlier
// groups sharing a body, found by relaxing over each body's groups in order); lists the groups of
// each depth; then applies the depths one after another, a warp per group and a lane per pair.
// Every velocity sees exactly the updates, in the order, that the sequential loop gives it.
constexpr int kResolveThreads = 512;
constexpr int kFastCand = 4096;

// Shared-memory layout of restitution_kernel, sized for kFastCand candidates.
struct ResolveSmem {
    static constexpr size_t F = kFastCand;
    static constexpr size_t ck = 0;                      // u64 [F + 2]: (o, k) keys; later depth lists
    static constexpr size_t sd = ck + 8 * (F + 2);       // double [F]: distances (sorted order)
    static constexpr size_t si = sd + 8 * F;             // int [F]: partners (sorted order)
    static constexpr size_t go = si + 4 * F;             // int [F]: outer body of each group
    static constexpr size_t gstart = go + 4 * F;         // int [F + 1]
    static constexpr size_t aux = gstart + 4 * (F + 1);  // int [F]: scan, group ids, cursors
    static constexpr size_t key = aux + 4 * F + 12;      // u64 [2F] (16-aligned): (body, group); later momenta
    static constexpr size_t lev = key + 16 * F;          // int [F]: depths
    static constexpr size_t scratch = lev + 4 * F;       // int [64]
    static constexpr size_t bytes = scratch + 4 * 64;
};
static_assert(ResolveSmem::key % 16 == 0, "momenta alias the key array as double2");

size_t resolve_smem_bytes() { return ResolveSmem::bytes; }

template <typename Less, typename Swap>
__device__ void bitonic_sort(int P, Less less, Swap swp) {
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int x = threadIdx.x; x < P / 2; x += blockDim.x) {
                const int i = (x / j) * 2 * j + (x % j);
                const int l = i + j;
                const bool up = (i & k) == 0;
                if (up ? less(l, i) : less(i, l)) swp(i, l);
            }
            __syncthreads();
        }
}

__device__ void bitonic_sort_u64(unsigned long long *a, int P) {
    bitonic_sort(
        P, [&](int x, int y) { return a[x] < a[y]; },
        [&](int x, int y) {
            const unsigned long long v = a[x];
            a[x] = a[y];
            a[y] = v;
        });
}

// Exclusive prefix sum of a[0..len) in place; returns the total.  scratch: 33 ints.
__device__ int block_exclusive_scan(int *a, int len, int *scratch) {
    const int t = threadIdx.x, nt = blockDim.x, lane = t & 31;
    const int per = (len + nt - 1) / nt;
    const int b0 = min(len, t * per), b1 = min(len, b0 + per);
    int s = 0;
    for (int k = b0; k < b1; ++k) s += a[k];
    int x = s;
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) scratch[t >> 5] = x;
    __syncthreads();
    if (t < 32) {
        const int w = t < (nt >> 5) ? scratch[t] : 0;
        int z = w;
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, z, d);
            if (t >= d) z += y;
        }
        scratch[t] = z - w;
        if (t == 31) scratch[32] = z;
    }
    __syncthreads();
    int run = scratch[t >> 5] + (x - s);
    for (int k = b0; k < b1; ++k) {
        const int v = a[k];
        a[k] = run;
        run += v;
    }
    __syncthreads();
    const int total = scratch[32];
    __syncthreads();
    return total;
}

// With perm != nullptr the candidates hold Barnes-Hut slots (the order of the reference's leaf and
// neighbour iteration) and perm maps them to bodies.
__device__ __forceinline__ void resolve_groups(unsigned char *smem, const Cand *cand, int c, const int32_t *perm,
                                               const double4 *pm, const double *rest, double4 *vel) {
    using L = ResolveSmem;
    const int t = threadIdx.x, nt = blockDim.x, lane = t & 31, warp = t >> 5, nw = nt >> 5;
    unsigned long long *ck = reinterpret_cast<unsigned long long *>(smem + L::ck);
    double *sd = reinterpret_cast<double *>(smem + L::sd);
    int *si = reinterpret_cast<int *>(smem + L::si);
    int *go = reinterpret_cast<int *>(smem + L::go);
    int *gstart = reinterpret_cast<int *>(smem + L::gstart);
    int *aux = reinterpret_cast<int *>(smem + L::aux);
    unsigned long long *key = reinterpret_cast<unsigned long long *>(smem + L::key);
    int *lev = reinterpret_cast<int *>(smem + L::lev);
    int *scratch = reinterpret_cast<int *>(smem + L::scratch);
    int *flag = scratch + 40;
    auto body = [&](int q) { return perm ? perm[q] : q; };
    constexpr unsigned long long kNone = ~0ull;

    int P = 2;
    while (P < c) P <<= 1;
    // (outer body, arrival index) keys; distances and partners stay in arrival order for now
    for (int k = t; k < P; k += nt) {
        if (k < c) {
            const Cand cd = cand[k];
            ck[k] = ((unsigned long long)(unsigned)cd.o << 32) | (unsigned)k;
            sd[k] = cd.dist;
            si[k] = cd.i;
        } else {
            ck[k] = kNone;
        }
    }
    __syncthreads();
    bitonic_sort_u64(ck, P);
    // groups: heads where the outer body changes
    for (int p = t; p < P; p += nt) aux[p] = (p < c && (p == 0 || (ck[p] >> 32) != (ck[p - 1] >> 32))) ? 1 : 0;
    __syncthreads();
    const int G = block_exclusive_scan(aux, P, scratch);
    for (int p = t; p < c; p += nt) {
        const bool head = p == 0 || (ck[p] >> 32) != (ck[p - 1] >> 32);
        const int g = aux[p] + (head ? 1 : 0) - 1;
        if (head) {
            gstart[g] = p;
            go[g] = (int)(ck[p] >> 32);
        }
        aux[p] = g;
    }
    if (t == 0) gstart[G] = c;
    __syncthreads();
    // each group by (distance, partner): the std::map order, the first of equal keys kept
    for (int g = t; g < G; g += nt) {
        const int b0 = gstart[g], b1 = gstart[g + 1];
        for (int p = b0 + 1; p < b1; ++p) {
            const unsigned long long v = ck[p];
            const int kv = (int)(v & 0xffffffffu);
            int q = p - 1;
            while (q >= b0) {
                const int kq = (int)(ck[q] & 0xffffffffu);
                if (sd[kq] < sd[kv] || (sd[kq] == sd[kv] && si[kq] < si[kv])) break;
                ck[q + 1] = ck[q];
                --q;
            }
            ck[q + 1] = v;
        }
    }
    __syncthreads();
    // distances and partners into sorted order (the key array is free scratch until its keys)
    {
        double *td = reinterpret_cast<double *>(key);
        int *ti = reinterpret_cast<int *>(td + kFastCand);
        for (int p = t; p < c; p += nt) {
            const int k = (int)(ck[p] & 0xffffffffu);
            td[p] = sd[k];
            ti[p] = si[k];
        }
        __syncthreads();
        for (int p = t; p < c; p += nt) {
            sd[p] = td[p];
            si[p] = ti[p];
        }
        __syncthreads();
    }
    // (body, group) keys: every group's outer body and every kept partner
    const int E = G + c;
    int E2 = 2;
    while (E2 < E) E2 <<= 1;
    for (int e = t; e < E2; e += nt) {
        unsigned long long kv = kNone;
        if (e < G) {
            kv = ((unsigned long long)(unsigned)go[e] << 32) | (unsigned)e;
        } else if (e < E) {
            const int p = e - G, g = aux[p];
            const bool dup = p > gstart[g] && sd[p] == sd[p - 1];
            if (!dup) kv = ((unsigned long long)(unsigned)si[p] << 32) | (unsigned)g;
        }
        key[e] = kv;
    }
    for (int g = t; g < G; g += nt) lev[g] = 0;
    __syncthreads();
    bitonic_sort_u64(key, E2);
    // depths: a group is one deeper than the last earlier group that shares a body with it
    for (int it = 0; it <= G; ++it) {
        if (t == 0) flag[0] = 0;
        __syncthreads();
        for (int e = t + 1; e < E; e += nt) {
            const unsigned long long ke = key[e], kp = key[e - 1];
            if (ke == kNone || (ke >> 32) != (kp >> 32)) continue;
            const int g = (int)(ke & 0xffffffffu), q = (int)(kp & 0xffffffffu);
            const int need = lev[q] + 1;
            if (lev[g] < need) {
                atomicMax(&lev[g], need);
                flag[0] = 1;
            }
        }
        __syncthreads();
        if (!flag[0]) break;
        __syncthreads();
    }
    if (t == 0) flag[1] = 0;
    __syncthreads();
    for (int g = t; g < G; g += nt) atomicMax(&flag[1], lev[g]);
    __syncthreads();
    const int D = flag[1] + 1;
    // the groups of each depth: lorder[lstart[d] .. lstart[d + 1])
    int *lorder = reinterpret_cast<int *>(ck);
    int *lstart = lorder + kFastCand;
    for (int d = t; d <= D; d += nt) lstart[d] = 0;
    for (int d = t; d < D; d += nt) aux[d] = 0;
    __syncthreads();
    for (int g = t; g < G; g += nt) atomicAdd(&lstart[lev[g]], 1);
    __syncthreads();
    block_exclusive_scan(lstart, D + 1, scratch);
    for (int g = t; g < G; g += nt) {
        const int d = lev[g];
        lorder[lstart[d] + atomicAdd(&aux[d], 1)] = g;
    }
    __syncthreads();
    // apply the depths in order; a warp per group, a lane per pair
    double2 *mom = reinterpret_cast<double2 *>(key);
    for (int d = 0; d < D; ++d) {
        const int q1 = lstart[d + 1];
        for (int q = lstart[d] + warp; q < q1; q += nw) {
            const int g = lorder[q];
            const int k0 = gstart[g], k1 = gstart[g + 1];
            const int o = body(go[g]);
            const double4 xo = pm[o];
            const double4 vo0 = vel[o];
            const double rest_o = rest[o];
            // momenta along r12 snapshotted for the whole group before any update
            // (gregsys.hpp:740-742); the first 32 partners stay in registers
            int i0 = 0;
            double4 xi0 = make_double4(0, 0, 0, 0), vi0 = xi0;
            double ri0 = 0.0;
            for (int kb = k0; kb < k1; kb += 32) {
                const int k = kb + lane;
                if (k < k1) {
                    const int i = body(si[k]);
                    const double4 xi = pm[i], vi = vel[i];
                    const double dd = sd[k];
                    const double ux = (xi.x - xo.x) / dd, uy = (xi.y - xo.y) / dd, uz = (xi.z - xo.z) / dd;
                    mom[k] = make_double2(axis_momentum(xo, vo0, ux, uy, uz), axis_momentum(xi, vi, ux, uy, uz));
                    if (kb == k0) {
                        i0 = i;
                        xi0 = xi;
                        vi0 = vi;
                        ri0 = rest[i];
                    }
                }
            }
            __syncwarp();
            double4 vo = vo0;
            for (int kb = k0; kb < k1; kb += 32) {
                const int k = kb + lane;
                double d_o = 0.0, ux = 0.0, uy = 0.0, uz = 0.0;
                int hit = 0;
                if (k < k1 && !(k > k0 && sd[k] == sd[k - 1])) {  // std::map keeps the first equal key
                    int i = i0;
                    double4 xi = xi0, vi = vi0;
                    double ri = ri0;
                    if (kb != k0) {
                        i = body(si[k]);
                        xi = pm[i];
                        vi = vel[i];
                        ri = rest[i];
                    }
                    if (pair_impulse(xo, rest_o, xi, ri, sd[k], mom[k], vi, d_o, ux, uy, uz)) {
                        vel[i] = vi;
                        hit = 1;
                    }
                }
                // o's velocity takes the changes in candidate order, as the sequential loop adds them
                const int m = min(32, k1 - kb);
                for (int j = 0; j < m; ++j) {
                    const int h = __shfl_sync(0xffffffffu, hit, j);
                    const double a = __shfl_sync(0xffffffffu, d_o, j);
                    const double bx = __shfl_sync(0xffffffffu, ux, j);
                    const double by = __shfl_sync(0xffffffffu, uy, j);
                    const double bz = __shfl_sync(0xffffffffu, uz, j);
                    if (h) {
                        vo.x += a * bx;
                        vo.y += a * by;
                        vo.z += a * bz;
                    }
                }
            }
            if (lane == 0) vel[o] = vo;
            __syncwarp();
        }
        __syncthreads();
    }
}

// One CTA.  The candidate count is reset to zero at the end (for the next pass) unless it overflowed.
// hk (callback loop only): random_comet's for_all_bods first, the predicate after the pass.
__global__ void __launch_bounds__(kResolveThreads, 1) restitution_kernel(int64_t n, Cand *cand, int *count, int cap,
                                                                         const int32_t *perm, const double4 *pm,
                                                                         double *rest, double4 *vel, int *status,
                                                                         PassHooks hk) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double hsh[32];
    __shared__ double hcom[3];
    const int c = *count;
    if (hk.for_all)
        cb_for_all_block(n, pm, rest, hk.ctl, hk.weighted, 1, hk.min_cor, hk.max_cor, hk.scale, hk.n_exp, hsh, hcom);
    if (c > cap) {
        if (threadIdx.x == 0) *status = GTD_ERR_CAPACITY;
    } else if (c > kFastCand) {
        if (threadIdx.x == 0) resolve_serial(cand, c, cap, perm, pm, rest, vel);
    } else if (c > 0) {
        resolve_groups(smem, cand, c, perm, pm, rest, vel);
    }
    __syncthreads();
    if (threadIdx.x == 0 && c <= cap) *count = 0;
    if (hk.decide) {
        __syncthreads();
        const double lo = hk.mode == 2 ? cb_min_rest(rest, n, hsh) : INFINITY;
        if (threadIdx.x == 0) {
            const bool go = cb_verdict(hk.ctl, hk.mode, lo, hk.bound, hk.probing, status);
            cudaGraphSetConditional(hk.handle, go ? 1u : 0u);
        }
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
    GTD_CUDA(cudaFuncSetAttribute(restitution_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)resolve_smem_bytes()));
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

// Upload order, the candidate buffer and a cleared candidate count and status for overlap passes;
// *status: the passes' device error word (GTD_ERR_CAPACITY when the candidates overflowed; it stays
// set until the next prepare).  Every pass that fits leaves the count at zero for the next one.
int prepare_collisions(gtd_system *s, int **status) {
    int rc = restore_upload_order(s);
    if (rc) return rc;
    rc = ensure_coll(s);
    if (rc) return rc;
    CollPtrs p = coll_ptrs(s);
    GTD_CUDA(cudaMemsetAsync(p.count, 0, 64, s->stream));
    if (status) *status = p.status;
    return GTD_OK;
}

// One s_coll pass (overlap restitution) enqueued on the stream, without reading its status back;
// prepare_collisions must have run since the last reorder.  Capturable.
int enqueue_collisions(gtd_system *s, const PassHooks *hooks) {
    if (s->n < 2) return GTD_OK;
    const PassHooks hk = hooks ? *hooks : PassHooks{};
    CollPtrs p = coll_ptrs(s);
    cudaStream_t st = s->stream;
    launch_overlap_pairs(s->n, s->pm[s->cur], s->rad, p.cand, p.count, kMaxCand, st);
    GTD_CHECK_LAUNCH();
    restitution_kernel<<<1, kResolveThreads, resolve_smem_bytes(), st>>>(s->n, p.cand, p.count, kMaxCand, nullptr,
                                                                         s->pm[s->cur], s->rest, s->vel, p.status,
                                                                         hk);
    GTD_CHECK_LAUNCH();
    s->launches += 2;
    return GTD_OK;
}

int run_collisions(gtd_system *s) {
    if (s->n < 2) return GTD_OK;
    if (s->coll == GTD_MERGE_COLL) return merge_scan(s, false, nullptr);
    int rc = prepare_collisions(s, nullptr);
    if (rc) return rc;
    rc = enqueue_collisions(s, nullptr);
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
    restitution_kernel<<<1, kResolveThreads, resolve_smem_bytes(), st>>>(s->n, p.cand, p.count, kMaxCand, s->perm,
                                                                         s->pm[s->cur], s->rest, s->vel, p.status,
                                                                         PassHooks{});
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
