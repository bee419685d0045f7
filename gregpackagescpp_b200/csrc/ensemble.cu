// Batched ensemble of independent few-body systems: one persistent launch advances every system
// by one leapfrog KDK step (gregsys.hpp:2946-2990 per system), the step loop is captured in a CUDA
// graph, and overlap merges (body::operator+=, the check_overlap scan) run inside the same launch.
//
// This is the device form of the reference drivers' ensemble pattern - one gtd::system per
// std::thread (bdsim.cpp:82-113) - with FP64 state and FP32 pair forces.
//
// Work decomposition: one CTA owns one system at a time.  Systems are handed out largest first
// from an atomic work counter (longest-processing-time order), so the spread in per-system work
// (N = 3 .. 2048: 4.7e5x in pairs) balances across the persistent grid.  A system's bodies are staged once per
// step in shared memory as FP32 coordinates relative to the system's mean position, with G m and
// the radius; the rows are spread over the CTA in passes of IB rows per thread (IB = 1, 2 or 4),
// and each thread sums its rows' forces two j-bodies per packed FP32x2 instruction, folding every
// 64 j-bodies into FP64.  Alongside the force it keeps the smallest separation to any other body (a
// 3-input float minimum; the one fold holding the row's own body excludes the self pair by its bit
// pattern); a body closer to another than its radius plus the system's largest radius, plus a
// bound on the FP32 staging error, flags the row; only systems with flagged rows run the exact FP64
// merge scan, over those rows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <numeric>
#include <vector>

#include "gtd_internal.cuh"

struct gtd_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double G = 6.6743e-11, dt = 1.0;
    int merge = 1;
    int threads = 256;   // CTA size (autotuned)
    int ib = 1;          // bodies per thread in the force loop (autotuned; 2 and 4 need threads <= 256)
    int blocks_per_sm = 0;
    int64_t n_sys = 0, n_bodies = 0;
    int max_n = 0;
    std::vector<int64_t> off_h;       // [n_sys+1]
    int64_t *off = nullptr;           // [n_sys+1]
    int32_t *cnt = nullptr;           // live bodies per system
    int32_t *order = nullptr;         // systems, largest first
    double4 *pos = nullptr, *vel = nullptr, *acc = nullptr;
    double *rad = nullptr, *rest = nullptr;
    int32_t *ids = nullptr;
    unsigned *work = nullptr;         // [2]: work counter, merges this launch
    int *status = nullptr;
    bool begun = false;
    uint64_t launches = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    int graph_threads = 0;
};

namespace gtd {

constexpr int kEnsMaxN = 8192;
constexpr int kEnsFold = 64;

struct EnsArgs {
    int n_sys;
    const int64_t *off;
    int32_t *cnt;
    const int32_t *order;
    double4 *pos, *vel, *acc;
    double *rad, *rest;
    int32_t *ids;
    double G, h;
    int kdk;     // 0: force only (initial acceleration); 1: kick-drift, force, kick
    int merge;
    int stride;  // floats per staged coordinate array (largest system, rounded up to even)
    unsigned *work;
    int *status;
};

__device__ __forceinline__ float ens_rsqrt(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Smallest r2 floor that keeps the self pair's G m / r^3 finite in FP32 for every body of a system
// whose largest G m is Gm: floor^(3/2) >= Gm * 2^-120, and at least 2^-100 (a normal float whose
// 1/r^2 = 2^100 stays finite).  For G m = 6.7e20 (1e31 kg, SI) that is 6.3e-11 m^2: it changes r2
// only for pairs closer than ~5 cm, far inside the FP32 resolution of the staged coordinates.
__device__ __forceinline__ float ens_r2_floor(float Gm) {
    const double c = cbrt((double)Gm * 0x1p-120);
    const double f = c * c;
    return f > 0x1p-100 ? (float)f : 0x1p-100f;
}

__device__ void ens_merge_into(double4 &po, double4 &vo, double4 &ao, double &ro, double &eo, const double4 &pi,
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

__device__ __forceinline__ bool ens_overlaps(const double4 &a, double ra, const double4 &b, double rb) {
    const double dx = __dsub_rn(b.x, a.x), dy = __dsub_rn(b.y, a.y), dz = __dsub_rn(b.z, a.z);
    const double d = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    return d < __dadd_rn(ra, rb);
}

// Removes row i of a system of num rows (the vector erase of the reference's scan): rows i+1 .. num-1
// move down by one, in passes of T rows.
__device__ __noinline__ void ens_erase_row(int i, int num, double4 *pos, double4 *vel, double4 *acc, double *rad, double *rest,
                              int32_t *ids) {
    const int t = threadIdx.x, T = blockDim.x;
    for (int base = i; base < num - 1; base += T) {
        const int k = base + t;
        const bool act = k < num - 1;
        double4 p, v, a;
        double r = 0, e = 0;
        int32_t id = 0;
        if (act) { p = pos[k + 1]; v = vel[k + 1]; a = acc[k + 1]; r = rad[k + 1]; e = rest[k + 1]; id = ids[k + 1]; }
        __syncthreads();
        if (act) { pos[k] = p; vel[k] = v; acc[k] = a; rad[k] = r; rest[k] = e; ids[k] = id; }
        __syncthreads();
    }
}

// The check_overlap scan (merges, restart from index 0 after each) over one system, by one CTA,
// from scan state (n rows, at row o0, restarted0: the last step merged into o0).
__device__ __noinline__ int ens_merge_scan(int n, int o0, bool restarted0, double4 *pos, double4 *vel, double4 *acc, double *rad,
                              double *rest, int32_t *ids, int *sh) {
    // sh[0] = best, sh[1] = num, sh[2] = o
    const int t = threadIdx.x, T = blockDim.x;
    if (t == 0) {
        sh[1] = n;
        sh[2] = o0;
    }
    __syncthreads();
    bool restarted = restarted0;
    while (true) {
        const int num = sh[1], o = sh[2];
        if (o >= num) break;
        const int lo = restarted ? 0 : o + 1;
        if (t == 0) sh[0] = INT32_MAX;
        __syncthreads();
        const double4 po = pos[o];
        const double ro = rad[o];
        for (int i = lo + t; i < num; i += T)
            if (i != o && ens_overlaps(po, ro, pos[i], rad[i])) atomicMin(&sh[0], i);
        __syncthreads();
        const int i = sh[0];
        if (i == INT32_MAX) {
            if (t == 0) sh[2] = o + 1;
            restarted = false;
            __syncthreads();
            continue;
        }
        if (t == 0) {
            double4 p = pos[o], v = vel[o], a = acc[o];
            double r = rad[o], e = rest[o];
            ens_merge_into(p, v, a, r, e, pos[i], vel[i], acc[i], rad[i], rest[i]);
            pos[o] = p; vel[o] = v; acc[o] = a; rad[o] = r; rest[o] = e;
        }
        __syncthreads();
        ens_erase_row(i, num, pos, vel, acc, rad, rest, ids);
        if (t == 0) {
            sh[1] = num - 1;
            sh[2] = i < o ? o - 1 : o;
        }
        restarted = true;
        __syncthreads();
    }
    const int out = sh[1];
    __syncthreads();
    return out;
}

constexpr int kEnsCand = 256;  // candidate rows a system's scan tracks before it falls back to the full scan

struct EnsCand {
    int n;                 // candidates listed (may exceed kEnsCand: then the list is incomplete)
    int o, num, next;      // scan state: current row, rows, the partner found (-1: none, -2: done)
    int restarted;
    int row[kEnsCand];
};

// One step of the candidate scan, by one thread: sorts and de-duplicates the list, finds the next
// (row, partner) pair in scan order from the state in c and merges the partner into the row
// (c.next = the partner), or ends the scan (c.next = -2).
__device__ __noinline__ void ens_cand_next(double4 *pos, double4 *vel, double4 *acc, double *rad, double *rest,
                                           EnsCand &c) {
    // sort the list (few entries; insertion sort) and drop duplicates
    int k = 0;
    for (int a = 0; a < c.n; ++a) {
        const int v = c.row[a];
        int b = k;
        while (b > 0 && c.row[b - 1] > v) { c.row[b] = c.row[b - 1]; --b; }
        c.row[b] = v;
        ++k;
    }
    int u = 0;
    for (int a = 0; a < k; ++a)
        if (u == 0 || c.row[u - 1] != c.row[a]) c.row[u++] = c.row[a];
    c.n = u;
    int o = c.o;
    bool restarted = c.restarted != 0;
    int found = -2;
    while (true) {
        if (!restarted) {  // jump to the first candidate at or after o
            int a = 0;
            while (a < c.n && c.row[a] < o) ++a;
            if (a == c.n) break;
            o = c.row[a];
        }
        const int lo = restarted ? 0 : o + 1;
        const double4 po = pos[o];
        const double ro = rad[o];
        int best = -1;
        for (int a = 0; a < c.n; ++a) {
            const int i = c.row[a];
            if (i >= lo && i != o && ens_overlaps(po, ro, pos[i], rad[i])) {
                best = i;  // the list is sorted: the first partner is the smallest
                break;
            }
        }
        if (best >= 0) {
            found = best;
            break;
        }
        ++o;
        restarted = false;
    }
    c.o = o;
    c.next = found;
    if (found >= 0) {
        double4 p = pos[o], v = vel[o], a = acc[o];
        double r = rad[o], e = rest[o];
        ens_merge_into(p, v, a, r, e, pos[found], vel[found], acc[found], rad[found], rest[found]);
        pos[o] = p; vel[o] = v; acc[o] = a; rad[o] = r; rest[o] = e;
    }
}

// The same scan restricted to candidate rows.  Every row with an FP64 overlap partner was flagged
// by the force loop's FP32 separation test (a bound that covers the staging error), and overlap is
// symmetric, so a row outside the list overlaps nothing and its partners are all listed: the scan
// can jump from candidate to candidate and search the list alone, taking the same merges in the same
// order as the full scan.  After a merge only the merged row has moved; it is tested against every
// row and its new partners join the list.  Returns the rows left; if the list overflows, the full
// scan continues from the state reached.
__device__ __noinline__ int ens_merge_scan_cand(int n, double4 *pos, double4 *vel, double4 *acc, double *rad, double *rest,
                                   int32_t *ids, EnsCand &c, int *sh) {
    const int t = threadIdx.x;
    if (t == 0) {
        c.o = 0;
        c.num = n;
        c.restarted = 0;
    }
    while (true) {
        if (t == 0) ens_cand_next(pos, vel, acc, rad, rest, c);
        __syncthreads();
        const int i = c.next, num = c.num;
        __syncthreads();  // every thread has read the state before thread 0 changes it
        if (i < 0) break;
        ens_erase_row(i, num, pos, vel, acc, rad, rest, ids);
        if (t == 0) {
            // the list after the erase: i leaves, later rows move down by one
            int u = 0;
            for (int a = 0; a < c.n; ++a) {
                const int r = c.row[a];
                if (r != i) c.row[u++] = r > i ? r - 1 : r;
            }
            c.n = u;
            c.o = i < c.o ? c.o - 1 : c.o;
            c.num = num - 1;
            c.restarted = 1;
        }
        __syncthreads();
        // the merged row's partners join the list (with the merged row itself)
        const int o = c.o, nm = c.num;
        const double4 po = pos[o];
        const double ro = rad[o];
        bool any = false;
        for (int k = t; k < nm; k += blockDim.x)
            if (k != o && ens_overlaps(po, ro, pos[k], rad[k])) {
                const int s = atomicAdd(&c.n, 1);
                if (s < kEnsCand) c.row[s] = k;
                any = true;
            }
        if (__syncthreads_or(any) && t == 0) {
            const int s = atomicAdd(&c.n, 1);
            if (s < kEnsCand) c.row[s] = o;
        }
        __syncthreads();
        const bool overflow = c.n > kEnsCand;
        const int o1 = c.o, n1 = c.num;
        __syncthreads();
        if (overflow)  // too many to track: the full scan from here
            return ens_merge_scan(n1, o1, true, pos, vel, acc, rad, rest, ids, sh);
    }
    const int out = c.num;
    __syncthreads();
    return out;
}

__device__ __forceinline__ float ens_min3(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// One fold (j pairs q0 .. q1-1) of the force loop for IB rows.  kOwn: the fold holds one of the
// rows' own bodies, whose self pair (r2 = floor2 exactly) must stay out of the minimum: the
// separation minimum is then taken on the integer bits offset past floor2 (2 ALU operations per
// value); every other fold takes a plain 3-input float minimum (1 operation per two values).
template <int IB, bool kOwn>
__device__ __forceinline__ void ens_fold(int q0, int q1, const float2 *X2, const float2 *Y2, const float2 *Z2,
                                         const float2 *M2, const float2 (&nx)[IB], const float2 (&ny)[IB],
                                         const float2 (&nz)[IB], float2 fl2, unsigned fbits, float2 (&fx)[IB],
                                         float2 (&fy)[IB], float2 (&fz)[IB], float (&mnf)[IB], unsigned (&mnr)[IB]) {
#pragma unroll 4
    for (int q = q0; q < q1; ++q) {
        const float2 X = X2[q], Y = Y2[q], Z = Z2[q], M = M2[q];
#pragma unroll
        for (int b = 0; b < IB; ++b) {
            const float2 dx = __fadd2_rn(X, nx[b]), dy = __fadd2_rn(Y, ny[b]), dz = __fadd2_rn(Z, nz[b]);
            float2 r2 = __ffma2_rn(dx, dx, fl2);
            r2 = __ffma2_rn(dy, dy, r2);
            r2 = __ffma2_rn(dz, dz, r2);
            if constexpr (kOwn) {
                mnr[b] = min(mnr[b], (unsigned)__float_as_int(r2.x) - fbits);
                mnr[b] = min(mnr[b], (unsigned)__float_as_int(r2.y) - fbits);
            } else {
                mnf[b] = ens_min3(mnf[b], r2.x, r2.y);
            }
            const float2 inv = make_float2(ens_rsqrt(r2.x), ens_rsqrt(r2.y));
            const float2 inv2 = __fmul2_rn(inv, inv);
            float2 sc = __fmul2_rn(M, inv);
            sc = __fmul2_rn(sc, inv2);
            fx[b] = __ffma2_rn(dx, sc, fx[b]);
            fy[b] = __ffma2_rn(dy, sc, fy[b]);
            fz[b] = __ffma2_rn(dz, sc, fz[b]);
        }
    }
}

// Forces on the IB rows r0, r0 + s, ..., r0 + (IB-1) s (those below nc) of a staged system: each
// staged j pair is read from shared memory once for all IB rows.  Returns whether any of them may
// overlap another body.  floor2 is added to every r2 inside its first FMA (no extra instruction):
// the self pair gets r2 = floor2 exactly, a finite 1/r and a zero term (dx = 0).  floor2 is far
// below the staged coordinates' resolution (ens_r2_floor).  r0 - t and s are multiples of 32, so
// the 32 rows of a warp share one fold of kEnsFold j-bodies for each b, and the choice of fold form
// (ens_fold's kOwn) is uniform across the warp.
template <int IB>
__device__ __forceinline__ int ens_force_rows(int r0, int s, int nc, int npad, const float *sx, const float *sy,
                                              const float *sz, const float *sm, double4 *pos, double4 *vel,
                                              double4 *acc, const double *rad, float rmx, float slack, bool kick,
                                              double h2, float floor2, EnsCand &cand) {
    const float2 *X2 = reinterpret_cast<const float2 *>(sx);
    const float2 *Y2 = reinterpret_cast<const float2 *>(sy);
    const float2 *Z2 = reinterpret_cast<const float2 *>(sz);
    const float2 *M2 = reinterpret_cast<const float2 *>(sm);
    float2 nx[IB], ny[IB], nz[IB];
    double ax[IB], ay[IB], az[IB];
    float mnf[IB];      // min r2 over the folds without the row's own body
    unsigned mnr[IB];   // min over the own fold's j != i of r2 bits, offset past floor2
    int own[IB];        // fold of the row's own body
#pragma unroll
    for (int b = 0; b < IB; ++b) {
        const int i = r0 + b * s;
        const int ic = i < nc ? i : r0;  // a missing row repeats the first; its result is dropped
        nx[b] = make_float2(-sx[ic], -sx[ic]);
        ny[b] = make_float2(-sy[ic], -sy[ic]);
        nz[b] = make_float2(-sz[ic], -sz[ic]);
        ax[b] = ay[b] = az[b] = 0.0;
        mnf[b] = INFINITY;
        mnr[b] = 0xffffffffu;
        own[b] = ic / kEnsFold;
    }
    const float2 fl2 = make_float2(floor2, floor2);
    const unsigned fbits = (unsigned)__float_as_int(floor2) + 1u;
    for (int q0 = 0; q0 < npad / 2; q0 += kEnsFold / 2) {
        const int q1 = min(q0 + kEnsFold / 2, npad / 2);
        const int fold = q0 / (kEnsFold / 2);
        float2 fx[IB], fy[IB], fz[IB];
#pragma unroll
        for (int b = 0; b < IB; ++b) fx[b] = fy[b] = fz[b] = make_float2(0.f, 0.f);
        bool mine = false;
#pragma unroll
        for (int b = 0; b < IB; ++b) mine |= own[b] == fold;
        if (__any_sync(0xffffffffu, mine))
            ens_fold<IB, true>(q0, q1, X2, Y2, Z2, M2, nx, ny, nz, fl2, fbits, fx, fy, fz, mnf, mnr);
        else
            ens_fold<IB, false>(q0, q1, X2, Y2, Z2, M2, nx, ny, nz, fl2, fbits, fx, fy, fz, mnf, mnr);
#pragma unroll
        for (int b = 0; b < IB; ++b) {
            ax[b] += (double)fx[b].x + (double)fx[b].y;
            ay[b] += (double)fy[b].x + (double)fy[b].y;
            az[b] += (double)fz[b].x + (double)fz[b].y;
        }
    }
    int flagged = 0;
#pragma unroll
    for (int b = 0; b < IB; ++b) {
        const int i = r0 + b * s;
        if (i >= nc) continue;
        float mind2 = mnf[b];
        if (mnr[b] != 0xffffffffu) mind2 = fminf(mind2, __int_as_float((int)(mnr[b] + fbits)));
        if (mind2 < INFINITY) {  // some other body exists
            const float reach = ((float)rad[i] + rmx) * 1.00001f + slack;
            if (mind2 < reach * reach * 1.0001f + floor2) {
                flagged = 1;
                const int k = atomicAdd(&cand.n, 1);
                if (k < kEnsCand) cand.row[k] = i;
            }
        }
        if (kick) {
            double4 v = vel[i];
            v.x = fma(h2, ax[b], v.x); v.y = fma(h2, ay[b], v.y); v.z = fma(h2, az[b], v.z);
            vel[i] = v;
        }
        acc[i] = make_double4(ax[b], ay[b], az[b], 0.0);
    }
    return flagged;
}

// One launch = one KDK step (or the initial force) for every system.  IB bodies per thread (1, 2 or 4;
// each staged j pair feeds IB bodies, dividing the shared-memory reads per interaction by IB).
template <int IB>
__global__ void __launch_bounds__(IB == 1 ? 512 : 256) ensemble_step_kernel(EnsArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *sx = reinterpret_cast<float *>(smem_raw);
    float *sy = sx + a.stride;
    float *sz = sy + a.stride;
    float *sm = sz + a.stride;
    __shared__ double red[3][32];
    __shared__ double cen[3];
    __shared__ float redr[32], redg[32];
    __shared__ int sh[8];
    __shared__ float rmax_s, floor_s;
    __shared__ int xmax_bits;  // largest staged |coordinate| (non-negative float bits)
    __shared__ EnsCand cand;   // rows the separation test flagged
    const int t = threadIdx.x, T = blockDim.x, lane = t & 31, warp = t >> 5, nw = (T + 31) >> 5;
    const double h = a.h, h2 = 0.5 * a.h;
    while (true) {
        if (t == 0) sh[3] = (int)atomicAdd(&a.work[0], 1u);
        __syncthreads();
        const int item = sh[3];
        __syncthreads();
        if (item >= a.n_sys) break;
        const int s = a.order[item];
        const int64_t b0 = a.off[s];
        const int n = a.cnt[s];
        double4 *pos = a.pos + b0, *vel = a.vel + b0, *acc = a.acc + b0;
        double *rad = a.rad + b0;
        // pass 0: kick-drift, force, kick, merge check; pass 1 (only after merges): the force at the
        // merged state, so the next step's first half kick uses a(x) of the bodies that remain
        int nc = n;
        for (int pass = 0; pass < 2; ++pass) {
            const bool first = pass == 0;
            double cx = 0.0, cy = 0.0, cz = 0.0;
            float rmax = 0.f, gmax = 0.f;
            for (int i = t; i < nc; i += T) {
                double4 p = pos[i];
                if (a.kdk && first) {
                    double4 v = vel[i];
                    const double4 ac = acc[i];
                    v.x = fma(h2, ac.x, v.x); v.y = fma(h2, ac.y, v.y); v.z = fma(h2, ac.z, v.z);
                    p.x = fma(h, v.x, p.x); p.y = fma(h, v.y, p.y); p.z = fma(h, v.z, p.z);
                    vel[i] = v;
                    pos[i] = p;
                }
                cx += p.x; cy += p.y; cz += p.z;
                rmax = fmaxf(rmax, (float)rad[i]);
                gmax = fmaxf(gmax, (float)(a.G * p.w));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                cx += __shfl_xor_sync(0xffffffffu, cx, o);
                cy += __shfl_xor_sync(0xffffffffu, cy, o);
                cz += __shfl_xor_sync(0xffffffffu, cz, o);
                rmax = fmaxf(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
                gmax = fmaxf(gmax, __shfl_xor_sync(0xffffffffu, gmax, o));
            }
            if (lane == 0) {
                red[0][warp] = cx; red[1][warp] = cy; red[2][warp] = cz;
                redr[warp] = rmax;
                redg[warp] = gmax;
            }
            __syncthreads();
            if (t == 0) {
                double X = 0, Y = 0, Z = 0;
                float R = 0.f, Gm = 0.f;
                for (int w = 0; w < nw; ++w) {
                    X += red[0][w]; Y += red[1][w]; Z += red[2][w];
                    R = fmaxf(R, redr[w]);
                    Gm = fmaxf(Gm, redg[w]);
                }
                cen[0] = X / nc; cen[1] = Y / nc; cen[2] = Z / nc;
                rmax_s = R;
                floor_s = ens_r2_floor(Gm);
                xmax_bits = 0;
                cand.n = 0;
            }
            __syncthreads();
            const double mx = cen[0], my = cen[1], mz = cen[2];
            const float rmx = rmax_s, floor2 = floor_s;
            // stage the system: FP32 relative positions and G m (pad to an even count, far and massless)
            const int npad = (nc + 1) & ~1;
            float xm = 0.f;
            for (int i = t; i < npad; i += T) {
                if (i < nc) {
                    const double4 p = pos[i];
                    const float X = (float)(p.x - mx), Y = (float)(p.y - my), Z = (float)(p.z - mz);
                    sx[i] = X; sy[i] = Y; sz[i] = Z;
                    sm[i] = (float)(a.G * p.w);
                    xm = fmaxf(xm, fmaxf(fabsf(X), fmaxf(fabsf(Y), fabsf(Z))));
                } else {
                    sx[i] = 1e30f; sy[i] = 1e30f; sz[i] = 1e30f; sm[i] = 0.f;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) xm = fmaxf(xm, __shfl_xor_sync(0xffffffffu, xm, o));
            if (lane == 0) atomicMax(&xmax_bits, __float_as_int(xm));
            __syncthreads();
            // Bound on the FP32 error of a staged separation: each staged coordinate is within
            // 2^-24 |X| of its FP64 value, so a separation is off by at most sqrt(3) 2^-23 xmax
            // (plus its own relative rounding, covered by the factor on the reach); 2^-21 xmax
            // keeps a factor 2 of room.  Every pair the FP64 overlap test would merge is flagged.
            const float slack = __int_as_float(xmax_bits) * 0x1p-21f;
            // rows in passes of up to IB*T; a pass of c rows gives each of its first s threads (s the
            // smallest multiple of 32 with IB*s >= c) the rows t, t + s, ...: threads hold IB valid
            // rows except in the last warp, and whole warps past s sit the pass out
            int flagged = 0;
            for (int base = 0; base < nc; base += IB * T) {
                const int c = min(IB * T, nc - base);
                const int sw = ((c + IB - 1) / IB + 31) & ~31;
                if (t < sw)
                    flagged |= ens_force_rows<IB>(base + t, sw, nc, npad, sx, sy, sz, sm, pos, vel, acc, rad, rmx,
                                                  slack, a.kdk && first, h2, floor2, cand);
            }
            flagged = __syncthreads_or(flagged);
            if (!first || !flagged || !a.merge) break;
            const int nn = cand.n <= kEnsCand
                               ? ens_merge_scan_cand(nc, pos, vel, acc, rad, a.rest + b0, a.ids + b0, cand, sh)
                               : ens_merge_scan(nc, 0, false, pos, vel, acc, rad, a.rest + b0, a.ids + b0, sh);
            if (nn == nc) break;
            if (t == 0) {
                a.cnt[s] = nn;
                atomicAdd(&a.work[1], (unsigned)(nc - nn));
            }
            nc = nn;
            __syncthreads();
        }
        __syncthreads();
    }
}

// The kernel for ib bodies per thread (1, 2 or 4).
template <typename F>
void with_ens_kernel(int ib, F &&f) {
    if (ib == 4) f(ensemble_step_kernel<4>);
    else if (ib == 2) f(ensemble_step_kernel<2>);
    else f(ensemble_step_kernel<1>);
}

int ens_stride(int max_n) { return std::max(2, (max_n + 1) & ~1); }
int ens_smem_bytes(int max_n) { return 4 * ens_stride(max_n) * (int)sizeof(float); }

}  // namespace gtd

using namespace gtd;

static void ens_release(gtd_ensemble *e) {
    if (e->graph) cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
    cudaFree(e->off); cudaFree(e->cnt); cudaFree(e->order); cudaFree(e->pos); cudaFree(e->vel); cudaFree(e->acc);
    cudaFree(e->rad); cudaFree(e->rest); cudaFree(e->ids); cudaFree(e->work); cudaFree(e->status);
    e->off = nullptr; e->cnt = nullptr; e->order = nullptr; e->pos = e->vel = e->acc = nullptr;
    e->rad = e->rest = nullptr; e->ids = nullptr; e->work = nullptr; e->status = nullptr;
}

static int ens_launch(gtd_ensemble *e, int kdk) {
    EnsArgs a{(int)e->n_sys, e->off, e->cnt, e->order, e->pos, e->vel, e->acc, e->rad, e->rest, e->ids,
              e->G, e->dt, kdk, e->merge, ens_stride(e->max_n), e->work, e->status};
    const int smem = ens_smem_bytes(e->max_n);
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, e->device);
    int per_sm = 1;
    with_ens_kernel(e->ib, [&](auto k) { cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, e->threads, smem); });
    if (per_sm < 1) per_sm = 1;
    const int grid = (int)std::min<int64_t>((int64_t)dev_sms * per_sm, std::max<int64_t>(e->n_sys, 1));
    GTD_CUDA(cudaMemsetAsync(e->work, 0, sizeof(unsigned), e->stream));
    with_ens_kernel(e->ib, [&](auto k) { k<<<grid, e->threads, smem, e->stream>>>(a); });
    GTD_CHECK_LAUNCH();
    e->launches += 1;
    return GTD_OK;
}

// Captures `steps` KDK steps (a memset and one persistent launch each) into a CUDA graph.
static int ens_build_graph(gtd_ensemble *e, int steps) {
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    cudaGraph_t g;
    GTD_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int rc = GTD_OK;
    const uint64_t before = e->launches;
    for (int k = 0; k < steps && !rc; ++k) rc = ens_launch(e, 1);
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    e->launches = before;  // captured, not launched
    if (rc) return rc;
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
    ce = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate", __FILE__, __LINE__);
    e->graph_steps = steps;
    e->graph_threads = e->threads * 4 + e->ib;
    return GTD_OK;
}

static int ens_steps(gtd_ensemble *e, uint64_t steps) {
    if (!e->begun) {
        int rc = ens_launch(e, 0);  // initial accelerations (and add-time merges)
        if (rc) return rc;
        e->begun = true;
    }
    const int chunk = 16;
    if (steps >= (uint64_t)chunk) {
        if (!e->graph || e->graph_steps != chunk || e->graph_threads != e->threads * 4 + e->ib) {
            int rc = ens_build_graph(e, chunk);
            if (rc) return rc;
        }
        while (steps >= (uint64_t)chunk) {
            GTD_CUDA(cudaGraphLaunch(e->graph, e->stream));
            e->launches += chunk;
            steps -= chunk;
        }
    }
    for (uint64_t k = 0; k < steps; ++k) {
        int rc = ens_launch(e, 1);
        if (rc) return rc;
    }
    return GTD_OK;
}

extern "C" {

int gtd_ensemble_create(gtd_ensemble **out, int device) {
    if (!out) return fail(GTD_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) {
        cudaGetLastError();
        return fail(GTD_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= nd) return fail(GTD_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    GTD_CUDA(cudaSetDevice(device));
    gtd_ensemble *e = new (std::nothrow) gtd_ensemble();
    if (!e) return fail(GTD_ERR_OUT_OF_MEMORY, "host allocation failed");
    e->device = device;
    GTD_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    GTD_CUDA(cudaEventCreate(&e->ev0));
    GTD_CUDA(cudaEventCreate(&e->ev1));
    for (int ib : {1, 2, 4}) {
        cudaError_t c = cudaSuccess;
        with_ens_kernel(ib, [&](auto k) {
            c = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, ens_smem_bytes(kEnsMaxN));
        });
        GTD_CUDA(c);
    }
    *out = e;
    return GTD_OK;
}

int gtd_ensemble_destroy(gtd_ensemble *e) {
    if (!e) return GTD_OK;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    ens_release(e);
    cudaEventDestroy(e->ev0);
    cudaEventDestroy(e->ev1);
    cudaStreamDestroy(e->stream);
    delete e;
    return GTD_OK;
}

int gtd_ensemble_set_params(gtd_ensemble *e, double G, double dt, int merge) {
    if (!e) return fail(GTD_ERR_INVALID_ARGUMENT, "ensemble is NULL");
    if (!(dt > 0)) return fail(GTD_ERR_INVALID_ARGUMENT, "Time-step cannot be zero or negative.");
    e->G = G;
    e->dt = dt;
    e->merge = merge ? 1 : 0;
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    return GTD_OK;
}

int gtd_ensemble_upload(gtd_ensemble *e, int64_t n_systems, const int64_t *offsets, const double *m,
                        const double *r, const double *rest, const double *x3, const double *v3) {
    if (!e) return fail(GTD_ERR_INVALID_ARGUMENT, "ensemble is NULL");
    if (n_systems < 0 || (n_systems > 0 && (!offsets || !m || !x3)))
        return fail(GTD_ERR_INVALID_ARGUMENT, "bad ensemble description");
    cudaSetDevice(e->device);
    ens_release(e);
    e->n_sys = n_systems;
    e->off_h.assign(offsets, offsets + n_systems + 1);
    const int64_t nb = n_systems ? offsets[n_systems] : 0;
    e->n_bodies = nb;
    e->max_n = 0;
    std::vector<int32_t> cnt((size_t)n_systems), order((size_t)n_systems);
    for (int64_t s = 0; s < n_systems; ++s) {
        const int64_t k = offsets[s + 1] - offsets[s];
        if (k < 0 || offsets[s] < 0) return fail(GTD_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing from 0");
        if (k > kEnsMaxN) return fail(GTD_ERR_CAPACITY, "system %lld has %lld bodies; the ensemble kernel holds %d",
                                      (long long)s, (long long)k, kEnsMaxN);
        cnt[(size_t)s] = (int32_t)k;
        e->max_n = std::max(e->max_n, (int)k);
    }
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return cnt[a] > cnt[b]; });
    std::vector<double4> hp((size_t)nb), hv((size_t)nb);
    std::vector<double> hr((size_t)nb), he((size_t)nb);
    std::vector<int32_t> hid((size_t)nb);
    for (int64_t s = 0; s < n_systems; ++s)
        for (int64_t i = offsets[s]; i < offsets[s + 1]; ++i) {
            if (m[i] < 0) return fail(GTD_ERR_INVALID_ARGUMENT, "negative mass at body %lld", (long long)i);
            hp[(size_t)i] = make_double4(x3[3 * i], x3[3 * i + 1], x3[3 * i + 2], m[i]);
            hv[(size_t)i] = v3 ? make_double4(v3[3 * i], v3[3 * i + 1], v3[3 * i + 2], 0.0) : make_double4(0, 0, 0, 0);
            hr[(size_t)i] = r ? r[i] : 0.0;
            he[(size_t)i] = rest ? rest[i] : 1.0;
            hid[(size_t)i] = (int32_t)(i - offsets[s]);
        }
    const size_t b4 = sizeof(double4) * (size_t)std::max<int64_t>(nb, 1);
    GTD_CUDA(cudaMalloc(&e->off, sizeof(int64_t) * (size_t)(n_systems + 1)));
    GTD_CUDA(cudaMalloc(&e->cnt, sizeof(int32_t) * (size_t)std::max<int64_t>(n_systems, 1)));
    GTD_CUDA(cudaMalloc(&e->order, sizeof(int32_t) * (size_t)std::max<int64_t>(n_systems, 1)));
    GTD_CUDA(cudaMalloc(&e->pos, b4));
    GTD_CUDA(cudaMalloc(&e->vel, b4));
    GTD_CUDA(cudaMalloc(&e->acc, b4));
    GTD_CUDA(cudaMalloc(&e->rad, sizeof(double) * (size_t)std::max<int64_t>(nb, 1)));
    GTD_CUDA(cudaMalloc(&e->rest, sizeof(double) * (size_t)std::max<int64_t>(nb, 1)));
    GTD_CUDA(cudaMalloc(&e->ids, sizeof(int32_t) * (size_t)std::max<int64_t>(nb, 1)));
    GTD_CUDA(cudaMalloc(&e->work, 4 * sizeof(unsigned)));
    GTD_CUDA(cudaMalloc(&e->status, sizeof(int)));
    GTD_CUDA(cudaMemcpy(e->off, offsets, sizeof(int64_t) * (size_t)(n_systems + 1), cudaMemcpyHostToDevice));
    if (n_systems) {
        GTD_CUDA(cudaMemcpy(e->cnt, cnt.data(), sizeof(int32_t) * cnt.size(), cudaMemcpyHostToDevice));
        GTD_CUDA(cudaMemcpy(e->order, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice));
    }
    if (nb) {
        GTD_CUDA(cudaMemcpy(e->pos, hp.data(), b4, cudaMemcpyHostToDevice));
        GTD_CUDA(cudaMemcpy(e->vel, hv.data(), b4, cudaMemcpyHostToDevice));
        GTD_CUDA(cudaMemset(e->acc, 0, b4));
        GTD_CUDA(cudaMemcpy(e->rad, hr.data(), sizeof(double) * (size_t)nb, cudaMemcpyHostToDevice));
        GTD_CUDA(cudaMemcpy(e->rest, he.data(), sizeof(double) * (size_t)nb, cudaMemcpyHostToDevice));
        GTD_CUDA(cudaMemcpy(e->ids, hid.data(), sizeof(int32_t) * (size_t)nb, cudaMemcpyHostToDevice));
    }
    GTD_CUDA(cudaMemset(e->work, 0, 4 * sizeof(unsigned)));
    GTD_CUDA(cudaMemset(e->status, 0, sizeof(int)));
    e->begun = false;
    return GTD_OK;
}

int gtd_ensemble_evolve(gtd_ensemble *e, uint64_t steps, int64_t *elapsed_ns) {
    if (!e) return fail(GTD_ERR_INVALID_ARGUMENT, "ensemble is NULL");
    if (elapsed_ns) *elapsed_ns = 0;
    if (e->n_sys == 0 || steps == 0) return GTD_OK;
    cudaSetDevice(e->device);
    GTD_CUDA(cudaEventRecord(e->ev0, e->stream));
    int rc = ens_steps(e, steps);
    if (rc) return rc;
    GTD_CUDA(cudaEventRecord(e->ev1, e->stream));
    GTD_CUDA(cudaEventSynchronize(e->ev1));
    float ms = 0.f;
    GTD_CUDA(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
    if (elapsed_ns) *elapsed_ns = (int64_t)((double)ms * 1e6);
    return GTD_OK;
}

int gtd_ensemble_counts(gtd_ensemble *e, int64_t *counts, uint64_t *merges, uint64_t *launches) {
    if (!e) return fail(GTD_ERR_INVALID_ARGUMENT, "ensemble is NULL");
    cudaSetDevice(e->device);
    GTD_CUDA(cudaStreamSynchronize(e->stream));
    if (counts && e->n_sys) {
        std::vector<int32_t> c((size_t)e->n_sys);
        GTD_CUDA(cudaMemcpy(c.data(), e->cnt, sizeof(int32_t) * c.size(), cudaMemcpyDeviceToHost));
        for (int64_t s = 0; s < e->n_sys; ++s) counts[s] = c[(size_t)s];
    }
    if (merges) {
        unsigned w[2] = {0, 0};
        GTD_CUDA(cudaMemcpy(w, e->work, sizeof(w), cudaMemcpyDeviceToHost));
        *merges = w[1];
    }
    if (launches) *launches = e->launches;
    return GTD_OK;
}

int gtd_ensemble_download(gtd_ensemble *e, double *m, double *r, double *rest, double *x3, double *v3,
                          double *a3) {
    if (!e) return fail(GTD_ERR_INVALID_ARGUMENT, "ensemble is NULL");
    cudaSetDevice(e->device);
    GTD_CUDA(cudaStreamSynchronize(e->stream));
    const int64_t nb = e->n_bodies;
    if (!nb) return GTD_OK;
    std::vector<double4> hp((size_t)nb), hv((size_t)nb), ha((size_t)nb);
    std::vector<double> hr((size_t)nb), he((size_t)nb);
    GTD_CUDA(cudaMemcpy(hp.data(), e->pos, sizeof(double4) * (size_t)nb, cudaMemcpyDeviceToHost));
    GTD_CUDA(cudaMemcpy(hv.data(), e->vel, sizeof(double4) * (size_t)nb, cudaMemcpyDeviceToHost));
    GTD_CUDA(cudaMemcpy(ha.data(), e->acc, sizeof(double4) * (size_t)nb, cudaMemcpyDeviceToHost));
    GTD_CUDA(cudaMemcpy(hr.data(), e->rad, sizeof(double) * (size_t)nb, cudaMemcpyDeviceToHost));
    GTD_CUDA(cudaMemcpy(he.data(), e->rest, sizeof(double) * (size_t)nb, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nb; ++i) {
        if (m) m[i] = hp[(size_t)i].w;
        if (x3) { x3[3 * i] = hp[(size_t)i].x; x3[3 * i + 1] = hp[(size_t)i].y; x3[3 * i + 2] = hp[(size_t)i].z; }
        if (v3) { v3[3 * i] = hv[(size_t)i].x; v3[3 * i + 1] = hv[(size_t)i].y; v3[3 * i + 2] = hv[(size_t)i].z; }
        if (a3) { a3[3 * i] = ha[(size_t)i].x; a3[3 * i + 1] = ha[(size_t)i].y; a3[3 * i + 2] = ha[(size_t)i].z; }
        if (r) r[i] = hr[(size_t)i];
        if (rest) rest[i] = he[(size_t)i];
    }
    return GTD_OK;
}

int gtd_ensemble_set_threads(gtd_ensemble *e, int threads) {
    if (!e) return fail(GTD_ERR_INVALID_ARGUMENT, "ensemble is NULL");
    if (threads != 64 && threads != 128 && threads != 256 && threads != 512)
        return fail(GTD_ERR_INVALID_ARGUMENT, "threads must be 64, 128, 256 or 512");
    if (e->ib > 1 && threads > 256) e->ib = 1;
    e->threads = threads;
    return GTD_OK;
}

int gtd_ensemble_set_bodies_per_thread(gtd_ensemble *e, int bodies) {
    if (!e) return fail(GTD_ERR_INVALID_ARGUMENT, "ensemble is NULL");
    if (bodies != 1 && bodies != 2 && bodies != 4)
        return fail(GTD_ERR_INVALID_ARGUMENT, "bodies per thread must be 1, 2 or 4");
    if (bodies > 1 && e->threads > 256)
        return fail(GTD_ERR_INVALID_ARGUMENT, "%d bodies per thread need a CTA of at most 256 threads", bodies);
    e->ib = bodies;
    return GTD_OK;
}

int gtd_ensemble_config(const gtd_ensemble *e, int *threads, int *bodies_per_thread) {
    if (!e) return fail(GTD_ERR_INVALID_ARGUMENT, "ensemble is NULL");
    if (threads) *threads = e->threads;
    if (bodies_per_thread) *bodies_per_thread = e->ib;
    return GTD_OK;
}

// Times a few steps for each CTA size and bodies-per-thread choice on a copy of the current state
// (restored afterwards) and keeps the fastest: the project's tile autotuner for the ensemble.
int gtd_ensemble_autotune(gtd_ensemble *e, int *best_threads, double *best_ms) {
    if (!e) return fail(GTD_ERR_INVALID_ARGUMENT, "ensemble is NULL");
    if (e->n_sys == 0) return fail(GTD_ERR_INVALID_ARGUMENT, "autotune needs systems");
    cudaSetDevice(e->device);
    const int64_t nb = e->n_bodies;
    const size_t b4 = sizeof(double4) * (size_t)nb;
    // copies of the state, freed on every return path
    struct Saved {
        double4 *sp = nullptr, *sv = nullptr, *sa = nullptr;
        double *sr = nullptr, *se = nullptr;
        int32_t *si = nullptr, *sc = nullptr;
        ~Saved() {
            cudaFree(sp); cudaFree(sv); cudaFree(sa); cudaFree(sr); cudaFree(se); cudaFree(si); cudaFree(sc);
        }
    } S;
    GTD_CUDA(cudaMalloc(&S.sp, b4)); GTD_CUDA(cudaMalloc(&S.sv, b4)); GTD_CUDA(cudaMalloc(&S.sa, b4));
    GTD_CUDA(cudaMalloc(&S.sr, 8 * (size_t)nb)); GTD_CUDA(cudaMalloc(&S.se, 8 * (size_t)nb));
    GTD_CUDA(cudaMalloc(&S.si, 4 * (size_t)nb)); GTD_CUDA(cudaMalloc(&S.sc, 4 * (size_t)e->n_sys));
    double4 *sp = S.sp, *sv = S.sv, *sa = S.sa;
    double *sr = S.sr, *se = S.se;
    int32_t *si = S.si, *sc = S.sc;
    auto save = [&](bool back) -> int {
        auto cp = [&](void *dst, void *src, size_t bytes) { return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, e->stream); };
        cudaError_t c = cudaSuccess;
        if (!back) {
            c = cp(sp, e->pos, b4); if (!c) c = cp(sv, e->vel, b4); if (!c) c = cp(sa, e->acc, b4);
            if (!c) c = cp(sr, e->rad, 8 * nb); if (!c) c = cp(se, e->rest, 8 * nb); if (!c) c = cp(si, e->ids, 4 * nb);
            if (!c) c = cp(sc, e->cnt, 4 * e->n_sys);
        } else {
            c = cp(e->pos, sp, b4); if (!c) c = cp(e->vel, sv, b4); if (!c) c = cp(e->acc, sa, b4);
            if (!c) c = cp(e->rad, sr, 8 * nb); if (!c) c = cp(e->rest, se, 8 * nb); if (!c) c = cp(e->ids, si, 4 * nb);
            if (!c) c = cp(e->cnt, sc, 4 * e->n_sys);
        }
        return c == cudaSuccess ? GTD_OK : cuda_fail(c, "autotune state copy", __FILE__, __LINE__);
    };
    int rc = save(false);
    const bool was_begun = e->begun;
    const int orig_threads = e->threads, orig_ib = e->ib;
    const int cands[][2] = {{128, 1}, {256, 1}, {512, 1}, {128, 2}, {256, 2}, {128, 4}, {256, 4}};
    constexpr int kCands = sizeof(cands) / sizeof(cands[0]);
    // Each timing runs kTuneSteps consecutive steps from the saved state, so a candidate is judged on
    // steady stepping rather than on one launch.  The candidates take turns (round robin) so that a
    // clock still ramping up after the upload favours none of them; the first round only warms up.
    constexpr int kTuneSteps = 4, kRounds = 3;
    double per[kCands];
    for (int k = 0; k < kCands; ++k) per[k] = 1e300;
    for (int round = 0; round < kRounds && !rc; ++round) {
        for (int k = 0; k < kCands && !rc; ++k) {
            e->threads = cands[k][0];
            e->ib = cands[k][1];
            if ((rc = cudaEventRecord(e->ev0, e->stream) ? GTD_ERR_CUDA : GTD_OK)) break;
            for (int q = 0; q < kTuneSteps && !rc; ++q) rc = ens_launch(e, 1);
            if (rc) break;
            cudaEventRecord(e->ev1, e->stream);
            cudaEventSynchronize(e->ev1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e->ev0, e->ev1);
            if (round > 0) per[k] = std::min(per[k], (double)ms / kTuneSteps);
            rc = save(true);
        }
    }
    if (rc) {  // a failed copy or launch: leave the configuration as it was
        e->threads = orig_threads;
        e->ib = orig_ib;
        e->begun = was_begun;
        cudaStreamSynchronize(e->stream);
        return rc;
    }
    int best = orig_threads, best_ib = orig_ib;  // kept if no timing completed
    double bestv = 1e300;
    for (int k = 0; k < kCands; ++k)
        if (per[k] < bestv) {
            bestv = per[k];
            best = cands[k][0];
            best_ib = cands[k][1];
        }
    e->threads = best;
    e->ib = best_ib;
    e->begun = was_begun;
    GTD_CUDA(cudaStreamSynchronize(e->stream));
    GTD_CUDA(cudaMemset(e->work, 0, 4 * sizeof(unsigned)));
    if (best_threads) *best_threads = best;
    if (best_ms) *best_ms = bestv;
    return GTD_OK;
}

}  // extern "C"
