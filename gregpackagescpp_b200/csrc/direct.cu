// Direct-summation force kernels and the integrator epilogues of gtd::system::evolve.
//
// Replaces, on the device: cumulative_acc / calc_acc_and_e (gregsys.hpp:352-357, 439-476), the
// kick/drift updates of loop_kdk / loop_dkd and the KDK/DKD drivers (gregsys.hpp:477-607,
// 2946-3039), take_euler_step (:380-391), the modified-Euler and midpoint predictors and steps
// (:392-419, 2714-2891), and calc_energy (:608-630).
//
// Layout in HBM: one double4 per body for position + mass (x, y, z, m), double4 velocity and
// acceleration (w unused), all coalesced 32-byte loads.  The force kernels stream j-tiles of 256
// bodies through shared memory; every CTA of a grid sized to fill all SMs exactly processes an
// equal contiguous range of (i-block, j-tile) pairs (stream-K), writing per-row partial sums that
// the integrate kernel combines in a fixed order, so results are bit-reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "gtd_internal.cuh"
#include "gtd_math.cuh"

namespace gtd {

struct ForceKArgs {
    int64_t n, rows, tiles, total;
    int grid, bi;
    const double4 *src;
    double G;
    double *part;
    float near2;  // mixed kernel: a pair with r^2 < near2 |X_i|^2 sends its fold to the precise path
    int64_t segs, seg_tiles, units;  // mixed kernel's work queue (ForcePlan)
    unsigned *queue;                 // its counter, zeroed before each launch
};

__device__ __forceinline__ void cta_range(const ForceKArgs &a, int g, int64_t &s, int64_t &e) {
    s = (int64_t)g * a.total / a.grid;
    e = (int64_t)(g + 1) * a.total / a.grid;
}

// -------------------------------------------------------------------------------------------
// FP64: a_i = sum_j G m_j (x_j - x_i) / |x_j - x_i|^3, no softening (the reference's direct path
// ignores eps).  |r|^-3 comes from inv_r3 (a MUFU seed and a second-order binomial correction,
// gtd_math.cuh): 16 FP64 operations per pair in all.  Tiles that hold the self pair (i == j,
// r2 == 0) or padding bodies take the guarded loop, which selects their terms away; all others
// run without a compare.
// -------------------------------------------------------------------------------------------
template <int I, int BJ, bool kGuard>
__device__ __forceinline__ void f64_tile(const double4 *__restrict__ tile, const double (&xi)[I],
                                         const double (&yi)[I], const double (&zi)[I], double (&ax)[I],
                                         double (&ay)[I], double (&az)[I]) {
#pragma unroll 4
    for (int jj = 0; jj < BJ; ++jj) {
        const double4 q = tile[jj];
#pragma unroll
        for (int k = 0; k < I; ++k) {
            const double dx = q.x - xi[k], dy = q.y - yi[k], dz = q.z - zi[k];
            const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
            double sc = q.w * inv_r3(r2);
            if (kGuard) sc = r2 > 0.0 ? sc : 0.0;
            ax[k] = fma(sc, dx, ax[k]);
            ay[k] = fma(sc, dy, ay[k]);
            az[k] = fma(sc, dz, az[k]);
        }
    }
}

// BJ: j-bodies per work unit (a row of bi = 256 I bodies against BJ j-bodies).  Narrow units (BJ 32
// or 64) let a small system spread over every SM: at N = 1024 the 256-wide units give 8 CTAs.
template <int I, int BJ = kThreads>
__global__ void __launch_bounds__(kThreads) force_f64_kernel(ForceKArgs a) {
    static_assert(BJ <= kThreads && kThreads % BJ == 0, "BJ divides the CTA size");
    __shared__ double4 tile[2][BJ];
    const int t = threadIdx.x;
    int64_t s, e;
    cta_range(a, blockIdx.x, s, e);
    const double4 zero = make_double4(0.0, 0.0, 0.0, 0.0);
    while (s < e) {
        const int64_t r = s / a.tiles;
        const int64_t jt0 = s - r * a.tiles;
        const int64_t row_end = min(e, (r + 1) * a.tiles);
        const int64_t jt1 = row_end - r * a.tiles;
        const int64_t row0 = r * a.bi;
        double xi[I], yi[I], zi[I], ax[I], ay[I], az[I];
#pragma unroll
        for (int k = 0; k < I; ++k) {
            const int64_t i = row0 + k * kThreads + t;
            const double4 p = i < a.n ? a.src[i] : zero;
            xi[k] = p.x; yi[k] = p.y; zi[k] = p.z;
            ax[k] = 0.0; ay[k] = 0.0; az[k] = 0.0;
        }
        if (t < BJ) {
            const int64_t j = jt0 * BJ + t;
            double4 q = j < a.n ? a.src[j] : zero;
            q.w *= a.G;
            tile[0][t] = q;
        }
        __syncthreads();
        int cur = 0;
        for (int64_t jt = jt0; jt < jt1; ++jt) {
            const bool more = jt + 1 < jt1;
            double4 qn = zero;
            if (more && t < BJ) {
                const int64_t j = (jt + 1) * BJ + t;
                if (j < a.n) qn = a.src[j];
            }
            const int64_t j0 = jt * BJ;
            // the self pair lies in this tile, or the tile ends in padding bodies (mass 0 at the origin)
            const bool guard = (j0 < row0 + a.bi && row0 < j0 + BJ) || j0 + BJ > a.n;
            if (guard)
                f64_tile<I, BJ, true>(tile[cur], xi, yi, zi, ax, ay, az);
            else
                f64_tile<I, BJ, false>(tile[cur], xi, yi, zi, ax, ay, az);
            if (more && t < BJ) {
                qn.w *= a.G;
                tile[cur ^ 1][t] = qn;
            }
            __syncthreads();
            cur ^= 1;
        }
        double *slot = a.part + (size_t)(blockIdx.x + r) * 3 * a.bi;
#pragma unroll
        for (int k = 0; k < I; ++k) {
            const int l = k * kThreads + t;
            slot[l] = ax[k];
            slot[a.bi + l] = ay[k];
            slot[2 * a.bi + l] = az[k];
        }
        s = row_end;
        __syncthreads();
    }
}

// -------------------------------------------------------------------------------------------
// Mixed precision.  Each j-tile is staged in shared memory as FP32 coordinates relative to the
// row's centre c (the FP64 mean position of the row's bodies, which the Hilbert reordering keeps
// compact), with G m_j in FP32.  Pair arithmetic runs two j-bodies per instruction on the packed
// FP32x2 pipe (add/mul/fma .f32x2) with one MUFU rsqrt per pair; each i keeps FP32 partial sums
// for FOLD j-bodies, then folds them into FP64 Kahan-compensated accumulators.  Tiles that
// overlap the row (where i == j occurs) take the guarded path; all others run without a compare.
//
// Close pairs far from the frame centre.  Rounding X = x - c to FP32 moves each body by up to
// 2^-24 |X|, so a pair at distance r gets a relative error of up to 2^-24 (|X_i| + |X_j|) / r
// <= 2^-24 (2 |X_i| + r) / r: a pair 0.002 AU apart in a row whose centre is 1.3 AU away loses
// ~5e-5 of its force.  Every staged tile therefore carries the FP32 remainders lo = X - hi of its
// coordinates and the bounding box of each warp's 32 bodies; each warp of i-bodies (32 I bodies
// consecutive in the spatial order) knows its box and its largest threshold near2 |X_i|^2.  A fold
// whose j-box comes closer to the warp's i-box than that threshold is summed on the precise path,
// dx = (hi_j - hi_i) + (lo_j - lo_i), which carries only the rounding of dx itself; every other
// fold provably holds no pair with r^2 < near2 |X_i|^2.  With near2 = (2 / (K - 1))^2 every pair
// on the fast path keeps its coordinate error below K 2^-24 relative.
// -------------------------------------------------------------------------------------------
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void kahan_add(double &sum, double &comp, double v) {
    const double y = v - comp;
    const double t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

// FP64 Kahan accumulators of the I i-bodies of a thread: in registers, or (SMEM) in shared memory,
// which they only touch once per fold; the latter frees 12 registers per i-body for occupancy.
template <int I, bool SMEM>
struct KahanAcc;

template <int I>
struct KahanAcc<I, false> {
    double s[3][I], c[3][I];
    __device__ __forceinline__ void init(int) {
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int k = 0; k < I; ++k) s[d][k] = c[d][k] = 0.0;
    }
    __device__ __forceinline__ void add(int d, int k, double v) { kahan_add(s[d][k], c[d][k], v); }
    __device__ __forceinline__ double result(int d, int k) const { return s[d][k] - c[d][k]; }
};

template <int I>
struct KahanAcc<I, true> {
    double (*sm)[I][kThreads];  // [6][I][kThreads]: sums x y z, compensations x y z
    int t;
    __device__ __forceinline__ void init(int tid) {
        t = tid;
#pragma unroll
        for (int d = 0; d < 6; ++d)
#pragma unroll
            for (int k = 0; k < I; ++k) sm[d][k][t] = 0.0;
    }
    __device__ __forceinline__ void add(int d, int k, double v) {
        double s = sm[d][k][t], c = sm[3 + d][k][t];
        kahan_add(s, c, v);
        sm[d][k][t] = s;
        sm[3 + d][k][t] = c;
    }
    __device__ __forceinline__ double result(int d, int k) const { return sm[d][k][t] - sm[3 + d][k][t]; }
};

// The staged j-tile: FP32 coordinates relative to the row centre (hi), their FP32 remainders (lo,
// read only on the precise path), G m, and the bounding box of each warp's 32 staged bodies.
struct MixedTile {
    const float *x, *y, *z, *m, *lx, *ly, *lz;
    const float *box;  // [kThreads / 32][6]: lo xyz, hi xyz
};

// Order-preserving map of a float onto an unsigned int, so that warp minima and maxima of floats
// are single REDUX operations (__reduce_min_sync / __reduce_max_sync).
__device__ __forceinline__ unsigned f2key(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key2f(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
__device__ __forceinline__ float warp_minf(float v) { return key2f(__reduce_min_sync(0xffffffffu, f2key(v))); }
__device__ __forceinline__ float warp_maxf(float v) { return key2f(__reduce_max_sync(0xffffffffu, f2key(v))); }

// The loop over j-pairs [u0, u0 + LEN) of a staged tile.  kPrecise: the coordinate differences are
// taken from the hi/lo splits, dx = (hi_j - hi_i) + (lo_j - lo_i), which carries only the rounding
// of dx itself (three more packed adds per coordinate and pair of j-bodies); otherwise dx = hi_j -
// hi_i.  Padding bodies (hi = 1e30, r2 = inf) contribute 0 on both paths.
template <int I, int LEN, int U, bool kGuard, bool kPrecise>
__device__ __forceinline__ void mixed_span(const MixedTile &T, int u0, const float2 (&nx)[I], const float2 (&ny)[I],
                                           const float2 (&nz)[I], const float *__restrict__ ilo, float2 (&fx)[I],
                                           float2 (&fy)[I], float2 (&fz)[I]) {
    const float2 *X = reinterpret_cast<const float2 *>(T.x) + u0;
    const float2 *Y = reinterpret_cast<const float2 *>(T.y) + u0;
    const float2 *Z = reinterpret_cast<const float2 *>(T.z) + u0;
    const float2 *M = reinterpret_cast<const float2 *>(T.m) + u0;
    const float2 *LX = reinterpret_cast<const float2 *>(T.lx) + u0;
    const float2 *LY = reinterpret_cast<const float2 *>(T.ly) + u0;
    const float2 *LZ = reinterpret_cast<const float2 *>(T.lz) + u0;
    float2 lx[I], ly[I], lz[I];
    if (kPrecise) {
        const int t = threadIdx.x;
#pragma unroll
        for (int k = 0; k < I; ++k) {
            const float a = -ilo[(0 * I + k) * kThreads + t], b = -ilo[(1 * I + k) * kThreads + t],
                        c = -ilo[(2 * I + k) * kThreads + t];
            lx[k] = make_float2(a, a);
            ly[k] = make_float2(b, b);
            lz[k] = make_float2(c, c);
        }
    }
#pragma unroll U
    for (int u = 0; u < LEN; ++u) {
        const float2 xj = X[u], yj = Y[u], zj = Z[u], mj = M[u];
        float2 lxj, lyj, lzj;
        if (kPrecise) {
            lxj = LX[u];
            lyj = LY[u];
            lzj = LZ[u];
        }
#pragma unroll
        for (int k = 0; k < I; ++k) {
            float2 dx = __fadd2_rn(xj, nx[k]);
            float2 dy = __fadd2_rn(yj, ny[k]);
            float2 dz = __fadd2_rn(zj, nz[k]);
            if (kPrecise) {
                dx = __fadd2_rn(dx, __fadd2_rn(lxj, lx[k]));
                dy = __fadd2_rn(dy, __fadd2_rn(lyj, ly[k]));
                dz = __fadd2_rn(dz, __fadd2_rn(lzj, lz[k]));
            }
            float2 r2 = __fmul2_rn(dx, dx);
            r2 = __ffma2_rn(dy, dy, r2);
            r2 = __ffma2_rn(dz, dz, r2);
            float2 inv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
            if (kGuard) {
                inv.x = r2.x > 0.f ? inv.x : 0.f;
                inv.y = r2.y > 0.f ? inv.y : 0.f;
            }
            const float2 inv2 = __fmul2_rn(inv, inv);
            float2 sc = __fmul2_rn(mj, inv);
            sc = __fmul2_rn(sc, inv2);
            fx[k] = __ffma2_rn(dx, sc, fx[k]);
            fy[k] = __ffma2_rn(dy, sc, fy[k]);
            fz[k] = __ffma2_rn(dz, sc, fz[k]);
        }
    }
}

// One staged tile against the thread's I i-bodies, in folds of FOLD j-bodies.  Before each fold,
// the bounding boxes of the warp's i-bodies (iw: lo xyz, hi xyz, and the warp's largest threshold
// near2 |X_i|^2) and of the fold's j-bodies decide whether any pair of the two can be closer than
// its threshold; such a fold runs on the precise path, every other one on the fast path.
template <int I, int FOLD, int U, bool kGuard, class Acc>
__device__ __forceinline__ void mixed_tile(const MixedTile &T, const float2 (&nx)[I], const float2 (&ny)[I],
                                           const float2 (&nz)[I], const float *__restrict__ ilo,
                                           const float *__restrict__ iw, Acc &acc) {
    constexpr int kFoldWarps = FOLD / 32;
#pragma unroll 1
    for (int q0 = 0; q0 < kThreads / 2; q0 += FOLD / 2) {
        float2 fx[I], fy[I], fz[I];
#pragma unroll
        for (int k = 0; k < I; ++k) fx[k] = fy[k] = fz[k] = make_float2(0.f, 0.f);
        // smallest possible squared distance between the warp's i-bodies and the fold's j-bodies
        const float *cb = T.box + (q0 / (FOLD / 2)) * kFoldWarps * 6;
        float g2 = 0.f;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            float lo = cb[d], hi = cb[3 + d];
#pragma unroll
            for (int w = 1; w < kFoldWarps; ++w) {
                lo = fminf(lo, cb[w * 6 + d]);
                hi = fmaxf(hi, cb[w * 6 + 3 + d]);
            }
            const float g = fmaxf(0.f, fmaxf(lo - iw[3 + d], iw[d] - hi));
            g2 = fmaf(g, g, g2);
        }
        if (g2 < iw[6])
            mixed_span<I, FOLD / 2, U, kGuard, true>(T, q0, nx, ny, nz, ilo, fx, fy, fz);
        else
            mixed_span<I, FOLD / 2, U, kGuard, false>(T, q0, nx, ny, nz, ilo, fx, fy, fz);
#pragma unroll
        for (int k = 0; k < I; ++k) {
            acc.add(0, k, (double)fx[k].x + (double)fx[k].y);
            acc.add(1, k, (double)fy[k].x + (double)fy[k].y);
            acc.add(2, k, (double)fz[k].x + (double)fz[k].y);
        }
    }
}

// One staged body: FP32 hi part of x - c, its FP32 remainder lo, and G m.  Padding bodies are far
// away and massless, so their terms are exactly 0 on both paths.
__device__ __forceinline__ void stage_body(bool have, const double4 &q, const double3 &c, double G, int slot,
                                           float *hx, float *hy, float *hz, float *hm, float *lx, float *ly,
                                           float *lz) {
    if (have) {
        const double ex = q.x - c.x, ey = q.y - c.y, ez = q.z - c.z;
        const float fx = (float)ex, fy = (float)ey, fz = (float)ez;
        hx[slot] = fx;
        hy[slot] = fy;
        hz[slot] = fz;
        lx[slot] = (float)(ex - (double)fx);
        ly[slot] = (float)(ey - (double)fy);
        lz[slot] = (float)(ez - (double)fz);
        hm[slot] = (float)(G * q.w);
    } else {
        const float kFar = 1e30f;
        hx[slot] = hy[slot] = hz[slot] = kFar;
        lx[slot] = ly[slot] = lz[slot] = 0.f;
        hm[slot] = 0.f;
    }
}

// Bounding box of the 32 bodies a warp just staged (padding bodies left out), written by lane 0 to
// box[warp][6] of the buffer.  Every lane of the warp calls it.
__device__ __forceinline__ void stage_box(bool have, const float *hx, const float *hy, const float *hz, int slot,
                                          float *box) {
    const float kInf = __int_as_float(0x7f800000);
    const float x = hx[slot], y = hy[slot], z = hz[slot];
    const float lx = warp_minf(have ? x : kInf), ly = warp_minf(have ? y : kInf), lz = warp_minf(have ? z : kInf);
    const float ux = warp_maxf(have ? x : -kInf), uy = warp_maxf(have ? y : -kInf), uz = warp_maxf(have ? z : -kInf);
    if ((threadIdx.x & 31) == 0) {
        float *b = box + (threadIdx.x >> 5) * 6;
        b[0] = lx; b[1] = ly; b[2] = lz;
        b[3] = ux; b[4] = uy; b[5] = uz;
    }
}

template <int I, int FOLD, int MINB, bool SMK, int U>
__global__ void __launch_bounds__(kThreads, MINB) force_mixed_kernel(ForceKArgs a) {
    __shared__ __align__(16) float tx[2][kThreads];
    __shared__ __align__(16) float ty[2][kThreads];
    __shared__ __align__(16) float tz[2][kThreads];
    __shared__ __align__(16) float tm[2][kThreads];
    __shared__ __align__(16) float tlx[2][kThreads];
    __shared__ __align__(16) float tly[2][kThreads];
    __shared__ __align__(16) float tlz[2][kThreads];
    __shared__ float ilo[3 * I * kThreads];  // lo parts of the row's bodies, [dim][k][thread]
    __shared__ float jbox[2][kThreads / 32 * 6];  // per staged warp of j-bodies: lo xyz, hi xyz
    __shared__ float ibox[kThreads / 32][7];      // per warp of i-bodies: lo xyz, hi xyz, max threshold
    __shared__ double cred[3][kThreads / 32];
    __shared__ double kah[SMK ? 6 : 1][SMK ? I : 1][SMK ? kThreads : 1];
    __shared__ int64_t unit_sh;
    const int t = threadIdx.x;
    // Work queue: units (row r, segment) are taken in turn, so that CTAs whose rows hold more
    // precise-path folds take fewer units; each unit writes its own partial-sum slot.
    for (;;) {
        if (t == 0) unit_sh = (int64_t)atomicAdd(a.queue, 1u);
        __syncthreads();
        const int64_t unit = unit_sh;
        if (unit >= a.units) break;
        const int64_t r = unit / a.segs;
        const int64_t jt0 = (unit - r * a.segs) * a.seg_tiles;
        const int64_t jt1 = min(jt0 + a.seg_tiles, a.tiles);
        const int64_t row0 = r * a.bi;
        // the row's FP32 frame is centred on the mean position of its bodies
        double px[I], py[I], pz[I];
        double msx = 0.0, msy = 0.0, msz = 0.0;
#pragma unroll
        for (int k = 0; k < I; ++k) {
            const int64_t i = row0 + t * I + k;  // a warp holds 32 I consecutive bodies
            px[k] = py[k] = pz[k] = 0.0;
            if (i < a.n) {
                const double4 p = a.src[i];
                px[k] = p.x; py[k] = p.y; pz[k] = p.z;
                msx += p.x; msy += p.y; msz += p.z;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            msx += __shfl_xor_sync(0xffffffffu, msx, o);
            msy += __shfl_xor_sync(0xffffffffu, msy, o);
            msz += __shfl_xor_sync(0xffffffffu, msz, o);
        }
        if ((t & 31) == 0) {
            cred[0][t >> 5] = msx;
            cred[1][t >> 5] = msy;
            cred[2][t >> 5] = msz;
        }
        __syncthreads();
        double3 c = make_double3(0.0, 0.0, 0.0);
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) {
            c.x += cred[0][w];
            c.y += cred[1][w];
            c.z += cred[2][w];
        }
        const double inv_rows = 1.0 / (double)min((int64_t)a.bi, a.n - row0);
        c.x *= inv_rows;
        c.y *= inv_rows;
        c.z *= inv_rows;
        __syncthreads();
        float2 nx[I], ny[I], nz[I];
        const float kInf = __int_as_float(0x7f800000);
        float blo[3] = {kInf, kInf, kInf}, bhi[3] = {-kInf, -kInf, -kInf}, bth = 0.f;
        KahanAcc<I, SMK> acc;
        if constexpr (SMK) acc.sm = kah;
        acc.init(t);
#pragma unroll
        for (int k = 0; k < I; ++k) {
            const int64_t i = row0 + t * I + k;  // a warp holds 32 I consecutive bodies
            float fx = 0.f, fy = 0.f, fz = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
            if (i < a.n) {  // padding i-bodies sit at the centre with a zero threshold
                const double ex = px[k] - c.x, ey = py[k] - c.y, ez = pz[k] - c.z;
                fx = (float)ex;
                fy = (float)ey;
                fz = (float)ez;
                lx = (float)(ex - (double)fx);
                ly = (float)(ey - (double)fy);
                lz = (float)(ez - (double)fz);
            }
            nx[k] = make_float2(-fx, -fx);
            ny[k] = make_float2(-fy, -fy);
            nz[k] = make_float2(-fz, -fz);
            ilo[(0 * I + k) * kThreads + t] = lx;
            ilo[(1 * I + k) * kThreads + t] = ly;
            ilo[(2 * I + k) * kThreads + t] = lz;
            const bool real = i < a.n;
            blo[0] = fminf(blo[0], real ? fx : kInf);
            blo[1] = fminf(blo[1], real ? fy : kInf);
            blo[2] = fminf(blo[2], real ? fz : kInf);
            bhi[0] = fmaxf(bhi[0], real ? fx : -kInf);
            bhi[1] = fmaxf(bhi[1], real ? fy : -kInf);
            bhi[2] = fmaxf(bhi[2], real ? fz : -kInf);
            bth = fmaxf(bth, a.near2 * fmaf(fz, fz, fmaf(fy, fy, fx * fx)));
        }
        {
            const float v0 = warp_minf(blo[0]), v1 = warp_minf(blo[1]), v2 = warp_minf(blo[2]);
            const float v3 = warp_maxf(bhi[0]), v4 = warp_maxf(bhi[1]), v5 = warp_maxf(bhi[2]);
            const float v6 = warp_maxf(bth);
            if ((t & 31) == 0) {
                float *b = ibox[t >> 5];
                b[0] = v0; b[1] = v1; b[2] = v2; b[3] = v3; b[4] = v4; b[5] = v5; b[6] = v6;
            }
        }
        {
            const int64_t j = jt0 * kThreads + t;
            const bool have = j < a.n;
            stage_body(have, have ? a.src[j] : make_double4(0.0, 0.0, 0.0, 0.0), c, a.G, t, tx[0], ty[0], tz[0],
                       tm[0], tlx[0], tly[0], tlz[0]);
            stage_box(have, tx[0], ty[0], tz[0], t, jbox[0]);
        }
        __syncthreads();
        int cur = 0;
        for (int64_t jt = jt0; jt < jt1; ++jt) {
            const bool more = jt + 1 < jt1;
            double4 qn = make_double4(0.0, 0.0, 0.0, 0.0);
            bool have = false;
            if (more) {
                const int64_t j = (jt + 1) * kThreads + t;
                if (j < a.n) {
                    qn = a.src[j];
                    have = true;
                }
            }
            const int64_t j0 = jt * kThreads;
            const bool diag = j0 < row0 + a.bi && row0 < j0 + kThreads;
            const MixedTile T{tx[cur], ty[cur], tz[cur], tm[cur], tlx[cur], tly[cur], tlz[cur], jbox[cur]};
            const float *iw = ibox[t >> 5];
            if (diag)
                mixed_tile<I, FOLD, U, true>(T, nx, ny, nz, ilo, iw, acc);
            else
                mixed_tile<I, FOLD, U, false>(T, nx, ny, nz, ilo, iw, acc);
            if (more) {
                const int nb = cur ^ 1;
                stage_body(have, qn, c, a.G, t, tx[nb], ty[nb], tz[nb], tm[nb], tlx[nb], tly[nb], tlz[nb]);
                stage_box(have, tx[nb], ty[nb], tz[nb], t, jbox[nb]);
            }
            __syncthreads();
            cur ^= 1;
        }
        double *slot = a.part + (size_t)unit * 3 * a.bi;
#pragma unroll
        for (int k = 0; k < I; ++k) {
            const int l = t * I + k;
            slot[l] = acc.result(0, k);
            slot[a.bi + l] = acc.result(1, k);
            slot[2 * a.bi + l] = acc.result(2, k);
        }
        __syncthreads();  // also orders every read of unit_sh before thread 0 takes the next unit
    }
}

// -------------------------------------------------------------------------------------------
// Plan and launch
// -------------------------------------------------------------------------------------------
// Kernel variants: i-bodies per thread (I) and, for the mixed kernel, the j-bodies summed in FP32
// between FP64 folds (FOLD).  Index 0 of each table is the default; gtd_system_autotune_direct
// times them all on the caller's bodies and keeps the fastest.
struct VariantInfo {
    int i, fold;
    int bj = kThreads;  // j-bodies per work unit
};
// mixed: {I, FOLD}; the launch bound (blocks per SM) and where the Kahan sums live are in with_mixed
static const VariantInfo kMixedVariants[] = {{2, 64}, {4, 128}, {2, 128}, {2, 128}, {1, 64},
                                             {4, 64}, {2, 64},  {2, 64},  {4, 128}};
static const VariantInfo kF64Variants[] = {{2, 0}, {1, 0}, {4, 0}, {1, 0, 64}, {1, 0, 32}};
constexpr int kNumMixed = sizeof(kMixedVariants) / sizeof(kMixedVariants[0]);
constexpr int kNumF64 = sizeof(kF64Variants) / sizeof(kF64Variants[0]);

int variant_count(int precision) { return precision == GTD_PREC_MIXED ? kNumMixed : kNumF64; }

// Variant for a handle nobody tuned.  From N ~ 32768 up the mixed kernel is fastest with 4 i-bodies
// per thread at 1 CTA/SM (<4,128,1,regs,U4>, variant 8: 27.4 ms against 29.1 ms for variant 0 at
// N = 262144 on B200); below that the 2-per-thread variants keep more CTAs busy.  Small FP64
// systems take the 32-wide work units so that every SM has work; up to N = 32768 one i-body per
// thread (0.37 against 0.41 ms per force at N = 16384), above that four (4.50 against 4.64 ms at
// N = 65536).
int default_variant(int precision, int64_t n) {
    if (precision == GTD_PREC_MIXED) return n >= 32768 ? 8 : 0;
    if (n <= 4096) return 4;  // FP64: 32-wide units up to N = 4096 (at least 512 units on 148 SMs)
    return n <= 32768 ? 1 : 2;
}

namespace {
std::mutex g_tuned_mu;
std::map<std::tuple<int, int, int>, int> g_tuned;  // (device, precision, bit length of N) -> variant
int size_class(int64_t n) {
    int b = 0;
    while (n > 0) { ++b; n >>= 1; }
    return b;
}
}  // namespace

void remember_variant(int device, int precision, int64_t n, int variant) {
    std::lock_guard<std::mutex> lock(g_tuned_mu);
    g_tuned[std::make_tuple(device, precision, size_class(n))] = variant;
}

int tuned_variant(int device, int precision, int64_t n) {
    std::lock_guard<std::mutex> lock(g_tuned_mu);
    auto it = g_tuned.find(std::make_tuple(device, precision, size_class(n)));
    return it != g_tuned.end() ? it->second : default_variant(precision, n);
}

int variant_info(int precision, int v, int *i, int *fold) {
    if (v < 0 || v >= variant_count(precision)) return fail(GTD_ERR_INVALID_ARGUMENT, "variant %d out of range", v);
    const VariantInfo &vi = precision == GTD_PREC_MIXED ? kMixedVariants[v] : kF64Variants[v];
    if (i) *i = vi.i;
    if (fold) *fold = vi.fold;
    return GTD_OK;
}

template <typename F>
static void with_mixed(int v, F &&f) {
    switch (v) {
        case 1: f(force_mixed_kernel<4, 128, 1, false, 8>); break;
        case 2: f(force_mixed_kernel<2, 128, 2, false, 4>); break;
        case 3: f(force_mixed_kernel<2, 128, 2, false, 8>); break;
        case 4: f(force_mixed_kernel<1, 64, 3, false, 4>); break;
        case 5: f(force_mixed_kernel<4, 64, 1, false, 4>); break;
        case 6: f(force_mixed_kernel<2, 64, 2, true, 4>); break;
        case 7: f(force_mixed_kernel<2, 64, 2, false, 4>); break;
        case 8: f(force_mixed_kernel<4, 128, 1, false, 4>); break;
        default: f(force_mixed_kernel<2, 64, 2, false, 8>); break;
    }
}

template <typename F>
static void with_f64(int v, F &&f) {
    switch (v) {
        case 1: f(force_f64_kernel<1>); break;
        case 2: f(force_f64_kernel<4>); break;
        case 3: f(force_f64_kernel<1, 64>); break;
        case 4: f(force_f64_kernel<1, 32>); break;
        default: f(force_f64_kernel<2>); break;
    }
}

// Cuts each row's tiles into at most `segs` segments of equal tile count.
static void set_segments(ForcePlan &p, int64_t segs) {
    p.seg_tiles = (p.tiles + segs - 1) / segs;
    p.segs = (p.tiles + p.seg_tiles - 1) / p.seg_tiles;
    p.units = p.rows * p.segs;
    p.slots = p.units;
}

ForcePlan make_plan(int64_t n, int precision, int device, int variant) {
    ForcePlan p;
    p.n = n;
    p.variant = (variant >= 0 && variant < variant_count(precision)) ? variant : 0;
    const VariantInfo &vi = precision == GTD_PREC_MIXED ? kMixedVariants[p.variant] : kF64Variants[p.variant];
    p.bi = kThreads * vi.i;
    p.bj = vi.bj;
    p.rows = (n + p.bi - 1) / p.bi;
    p.tiles = (n + p.bj - 1) / p.bj;
    p.total = p.rows * p.tiles;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (precision == GTD_PREC_MIXED)
        with_mixed(p.variant, [&](auto k) { cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, 0); });
    else
        with_f64(p.variant, [&](auto k) { cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, 0); });
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)sms * per_sm;
    if (precision == GTD_PREC_MIXED) {
        // about 64 units per CTA, so that the last units to finish leave a short tail (measured at
        // N = 262144: 29.4 ms per launch against 29.8 with 32 units per CTA and 30.2 with 16)
        const int64_t target = 64 * grid;
        int64_t segs = std::max<int64_t>(1, std::min<int64_t>(p.tiles, (target + p.rows - 1) / p.rows));
        set_segments(p, segs);
        if (grid > p.units) grid = p.units > 0 ? p.units : 1;
        p.grid = (int)grid;
    } else {
        if (grid > p.total) grid = p.total > 0 ? p.total : 1;
        p.grid = (int)grid;
        p.slots = p.grid + p.rows;
    }
    p.near2 = near2_of(kDefaultNearFactor);
    return p;
}

// The queue counter sits after the partial sums, on its own 256-byte line.
static size_t queue_offset(const ForcePlan &p) {
    return ((size_t)p.slots * 3 * p.bi * sizeof(double) + 255) / 256 * 256;
}

size_t partial_bytes(const ForcePlan &p) { return queue_offset(p) + (p.segs > 0 ? 256 : 0); }

int fit_plan_partials(ForcePlan &p, size_t max_bytes) {
    if (partial_bytes(p) <= max_bytes) return GTD_OK;
    const size_t per_slot = (size_t)3 * p.bi * sizeof(double);
    const int64_t max_slots = max_bytes > 512 ? (int64_t)((max_bytes - 512) / per_slot) : 0;
    if (p.segs > 0) {
        const int64_t segs = max_slots / std::max<int64_t>(p.rows, 1);
        if (segs < 1) return fail(GTD_ERR_CAPACITY, "%lld rows need more partial sums than %zu bytes hold",
                                  (long long)p.rows, max_bytes);
        set_segments(p, segs);
        if (p.grid > p.units) p.grid = (int)p.units;
    } else {
        const int64_t grid = max_slots - p.rows;
        if (grid < 1) return fail(GTD_ERR_CAPACITY, "%lld rows need more partial sums than %zu bytes hold",
                                  (long long)p.rows, max_bytes);
        if (p.grid > grid) p.grid = (int)grid;
        p.slots = p.grid + p.rows;
    }
    return partial_bytes(p) <= max_bytes ? GTD_OK : fail(GTD_ERR_CAPACITY, "partial sums do not fit %zu bytes", max_bytes);
}

int launch_force(int precision, const ForcePlan &p, const double4 *src, double G, double *partials,
                 cudaStream_t s) {
    if (p.n == 0) return GTD_OK;
    unsigned *queue = p.segs > 0 ? reinterpret_cast<unsigned *>(reinterpret_cast<char *>(partials) + queue_offset(p))
                                 : nullptr;
    ForceKArgs a{p.n, p.rows, p.tiles, p.total, p.grid, p.bi, src, G, partials, p.near2, p.segs, p.seg_tiles,
                 p.units, queue};
    if (precision == GTD_PREC_MIXED) {
        if (!queue) return fail(GTD_ERR_INVALID_ARGUMENT, "mixed-precision plan without a work queue");
        GTD_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned), s));
        with_mixed(p.variant, [&](auto k) { k<<<p.grid, kThreads, 0, s>>>(a); });
    }
    else
        with_f64(p.variant, [&](auto k) { k<<<p.grid, kThreads, 0, s>>>(a); });
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}

// -------------------------------------------------------------------------------------------
// Integrate: sum the partials of body i (CTA order) and apply the method's update in FP64.
// -------------------------------------------------------------------------------------------
struct IntArgs {
    int64_t n, tiles, total;
    int grid, bi, epi;
    const double *part;
    StepArgs st;
    int64_t segs;  // > 0: work-queue slots r * segs .. r * segs + segs - 1
};

__device__ __forceinline__ int64_t cta_of(int64_t pos, int grid, int64_t total) {
    return ((pos + 1) * (int64_t)grid - 1) / total;
}

// The partial-sum slots of row r, first to last (fixed order: the sums are reproducible).
__device__ __forceinline__ void row_slots(const IntArgs &a, int64_t r, int64_t &first, int64_t &last) {
    if (a.segs > 0) {
        first = r * a.segs;
        last = first + a.segs - 1;
    } else {
        first = cta_of(r * a.tiles, a.grid, a.total) + r;
        last = cta_of((r + 1) * a.tiles - 1, a.grid, a.total) + r;
    }
}

// The method's update of body i from its summed force (ax, ay, az), in FP64.
__device__ __forceinline__ void apply_epilogue(const IntArgs &a, int64_t i, double ax, double ay, double az) {
    const StepArgs &st = a.st;
    const double h = st.h, h2 = 0.5 * st.h;
    if (a.epi == EPI_ACC) {  // the force alone: position and velocity are not read
        st.acc[i] = make_double4(ax, ay, az, 0.0);
        return;
    }
    const double4 x = st.cur[i];
    double4 v = st.vel[i];
    switch (a.epi) {
        case EPI_KDK: {
            st.acc[i] = make_double4(ax, ay, az, 0.0);
            v.x = fma(h2, ax, v.x); v.y = fma(h2, ay, v.y); v.z = fma(h2, az, v.z);
            if (!st.last) {
                v.x = fma(h2, ax, v.x); v.y = fma(h2, ay, v.y); v.z = fma(h2, az, v.z);
                st.dst[i] = make_double4(fma(h, v.x, x.x), fma(h, v.y, x.y), fma(h, v.z, x.z), x.w);
            }
            st.vel[i] = v;
            break;
        }
        case EPI_DKD: {
            st.acc[i] = make_double4(ax, ay, az, 0.0);
            v.x = fma(h, ax, v.x); v.y = fma(h, ay, v.y); v.z = fma(h, az, v.z);
            double4 y = make_double4(fma(h2, v.x, x.x), fma(h2, v.y, x.y), fma(h2, v.z, x.z), x.w);
            if (!st.last) y = make_double4(fma(h2, v.x, y.x), fma(h2, v.y, y.y), fma(h2, v.z, y.z), x.w);
            st.dst[i] = y;
            st.vel[i] = v;
            break;
        }
        case EPI_EULER: {
            st.acc[i] = make_double4(ax, ay, az, 0.0);
            st.dst[i] = make_double4(fma(h, v.x, x.x), fma(h, v.y, x.y), fma(h, v.z, x.z), x.w);
            v.x = fma(h, ax, v.x); v.y = fma(h, ay, v.y); v.z = fma(h, az, v.z);
            st.vel[i] = v;
            break;
        }
        case EPI_PREDICT: {
            const double hp = st.hp;
            st.acc[i] = make_double4(ax, ay, az, 0.0);
            st.pred_pos[i] = make_double4(fma(hp, v.x, x.x), fma(hp, v.y, x.y), fma(hp, v.z, x.z), x.w);
            st.pred_vel[i] = make_double4(fma(hp, ax, v.x), fma(hp, ay, v.y), fma(hp, az, v.z), 0.0);
            break;
        }
        case EPI_CORR_MEULER: {
            const double4 pv = st.pred_vel[i], a0 = st.acc[i];
            st.dst[i] = make_double4(fma(h2, v.x + pv.x, x.x), fma(h2, v.y + pv.y, x.y), fma(h2, v.z + pv.z, x.z),
                                     x.w);
            v.x = fma(h2, a0.x + ax, v.x); v.y = fma(h2, a0.y + ay, v.y); v.z = fma(h2, a0.z + az, v.z);
            st.vel[i] = v;
            break;
        }
        case EPI_CORR_MIDPOINT: {
            const double4 pv = st.pred_vel[i];
            st.dst[i] = make_double4(fma(h, pv.x, x.x), fma(h, pv.y, x.y), fma(h, pv.z, x.z), x.w);
            v.x = fma(h, ax, v.x); v.y = fma(h, ay, v.y); v.z = fma(h, az, v.z);
            st.vel[i] = v;
            break;
        }
        default:
            break;
    }
}

// Thread per body: the partial sums of body i in CTA order, one after another.
__global__ void integrate_kernel(IntArgs a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t r = i / a.bi;
    const int l = (int)(i - r * a.bi);
    int64_t g0, g1;
    row_slots(a, r, g0, g1);
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int64_t g = g0; g <= g1; ++g) {
        const double *slot = a.part + (size_t)g * 3 * a.bi;
        ax += slot[l];
        ay += slot[a.bi + l];
        az += slot[2 * a.bi + l];
    }
    apply_epilogue(a, i, ax, ay, az);
}

// Warp per body, for rows spread over many CTAs (small N with narrow work units): the lanes load
// the partial sums in parallel and reduce them with shuffles, lane 0 applies the update.
__global__ void integrate_warp_kernel(IntArgs a) {
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= a.n) return;  // whole warps leave together
    const int64_t r = i / a.bi;
    const int l = (int)(i - r * a.bi);
    int64_t g0, g1;
    row_slots(a, r, g0, g1);
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int64_t g = g0 + lane; g <= g1; g += 32) {
        const double *slot = a.part + (size_t)g * 3 * a.bi;
        ax += slot[l];
        ay += slot[a.bi + l];
        az += slot[2 * a.bi + l];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    if (lane == 0) apply_epilogue(a, i, ax, ay, az);
}

// Small FP64 systems, one launch per force evaluation.  kFusedSlices warps share a body: warp s sums
// the j in the 32-wide chunks s, s + S, s + 2S, ... (loads straight from the L1/L2-resident
// positions, several in flight), reduces with shuffles, and the body's first warp adds the slices
// in order and applies the method's update.  No partial sums in memory, no second kernel; the short
// per-warp loops keep the latency of a step low when there are few bodies.
constexpr int kFusedBodies = 4;  // bodies per CTA
constexpr int kFusedSlices = 4;  // warps per body

__global__ void __launch_bounds__(kFusedBodies * kFusedSlices * 32)
    fused_small_kernel(IntArgs a, const double4 *__restrict__ src, double G) {
    __shared__ double part[kFusedSlices][kFusedBodies][3];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bl = w % kFusedBodies, slice = w / kFusedBodies;
    const int64_t i = (int64_t)blockIdx.x * kFusedBodies + bl;
    double ax = 0.0, ay = 0.0, az = 0.0;
    if (i < a.n) {
        const double4 p = src[i];
#pragma unroll 4
        for (int64_t j = (int64_t)slice * 32 + lane; j < a.n; j += 32 * kFusedSlices) {
            const double4 q = src[j];
            const double gm = q.w * G;
            const double dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
            const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
            const double sc = r2 > 0.0 ? gm * inv_r3(r2) : 0.0;
            ax = fma(sc, dx, ax);
            ay = fma(sc, dy, ay);
            az = fma(sc, dz, az);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    if (lane == 0) {
        part[slice][bl][0] = ax;
        part[slice][bl][1] = ay;
        part[slice][bl][2] = az;
    }
    __syncthreads();
    if (slice == 0 && lane == 0 && i < a.n) {
        double sx = part[0][bl][0], sy = part[0][bl][1], sz = part[0][bl][2];
#pragma unroll
        for (int k = 1; k < kFusedSlices; ++k) {
            sx += part[k][bl][0];
            sy += part[k][bl][1];
            sz += part[k][bl][2];
        }
        apply_epilogue(a, i, sx, sy, sz);
    }
}

int launch_fused_small(int64_t n, const double4 *src, double G, int epi, const StepArgs &st, cudaStream_t s) {
    if (n == 0) return GTD_OK;
    IntArgs a{n, 0, 0, 0, 0, epi, nullptr, st, 0};
    fused_small_kernel<<<(unsigned)((n + kFusedBodies - 1) / kFusedBodies), kFusedBodies * kFusedSlices * 32, 0, s>>>(
        a, src, G);
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}

int launch_integrate(const ForcePlan &p, const double *partials, int epi, const StepArgs &st, cudaStream_t s) {
    if (p.n == 0) return GTD_OK;
    IntArgs a{p.n, p.tiles, p.total, p.grid, p.bi, epi, partials, st, p.segs};
    const int threads = 256;
    // A row's force spread over more than ~4 slots, with too few bodies for a thread each to keep
    // the loads in flight: a warp per body.  From 2^17 bodies the thread-per-body form has the
    // parallelism, and its loads of 32 neighbouring bodies' slots are coalesced where the warp form
    // reads one 8-byte value per sector (0.196 ms per step at N = 262144 with 37 slots per row).
    if (p.slots > 4 * p.rows && p.n < ((int64_t)1 << 17))
        integrate_warp_kernel<<<(unsigned)((p.n * 32 + threads - 1) / threads), threads, 0, s>>>(a);
    else
        integrate_kernel<<<(unsigned)((p.n + threads - 1) / threads), threads, 0, s>>>(a);
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}

// Thread per body: the summed partials written as a triple (the force alone).
__global__ void sum_partials_kernel(IntArgs a, double *acc3) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int64_t r = i / a.bi;
    const int l = (int)(i - r * a.bi);
    int64_t g0, g1;
    row_slots(a, r, g0, g1);
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int64_t g = g0; g <= g1; ++g) {
        const double *slot = a.part + (size_t)g * 3 * a.bi;
        ax += slot[l];
        ay += slot[a.bi + l];
        az += slot[2 * a.bi + l];
    }
    acc3[3 * i] = ax;
    acc3[3 * i + 1] = ay;
    acc3[3 * i + 2] = az;
}

int launch_sum_partials(const ForcePlan &p, const double *partials, double *acc3, cudaStream_t s) {
    if (p.n == 0) return GTD_OK;
    IntArgs a{p.n, p.tiles, p.total, p.grid, p.bi, EPI_ACC, partials, StepArgs{}, p.segs};
    sum_partials_kernel<<<(unsigned)((p.n + 255) / 256), 256, 0, s>>>(a, acc3);
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}

__global__ void kick_drift_kernel(int64_t n, const double4 *cur, double4 *dst, double4 *vel, const double4 *acc,
                                  double h) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h2 = 0.5 * h;
    const double4 x = cur[i], a = acc[i];
    double4 v = vel[i];
    v.x = fma(h2, a.x, v.x); v.y = fma(h2, a.y, v.y); v.z = fma(h2, a.z, v.z);
    vel[i] = v;
    dst[i] = make_double4(fma(h, v.x, x.x), fma(h, v.y, x.y), fma(h, v.z, x.z), x.w);
}

__global__ void half_drift_kernel(int64_t n, const double4 *cur, double4 *dst, const double4 *vel, double h) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h2 = 0.5 * h;
    const double4 x = cur[i], v = vel[i];
    dst[i] = make_double4(fma(h2, v.x, x.x), fma(h2, v.y, x.y), fma(h2, v.z, x.z), x.w);
}

int launch_kick_drift(int64_t n, const double4 *cur, double4 *dst, double4 *vel, const double4 *acc, double h,
                      cudaStream_t s) {
    if (n == 0) return GTD_OK;
    kick_drift_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, cur, dst, vel, acc, h);
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}

int launch_half_drift(int64_t n, const double4 *cur, double4 *dst, const double4 *vel, double h, cudaStream_t s) {
    if (n == 0) return GTD_OK;
    half_drift_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, cur, dst, vel, h);
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}

// -------------------------------------------------------------------------------------------
// FP64 energy / momentum diagnostics.  One thread per i sums G m_j / r_ij over all j != i
// (j-tiles through shared memory); each block reduces its 9 sums in a fixed tree order and the
// host adds the block partials in block order, so the result is reproducible run to run.
// -------------------------------------------------------------------------------------------
constexpr int kEThreads = 256;

__global__ void __launch_bounds__(kEThreads) energy_kernel(int64_t n, const double4 *pm, const double4 *vel,
                                                           double G, double *out) {
    __shared__ double4 tile[kEThreads];
    __shared__ double red[9][kEThreads];
    const int t = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * kEThreads + t;
    double4 p = make_double4(0.0, 0.0, 0.0, 0.0), v = p;
    if (i < n) {
        p = pm[i];
        v = vel[i];
    }
    double phi = 0.0;
    for (int64_t j0 = 0; j0 < n; j0 += kEThreads) {
        const int64_t j = j0 + t;
        tile[t] = j < n ? pm[j] : make_double4(0.0, 0.0, 0.0, 0.0);
        __syncthreads();
        const int lim = (int)min((int64_t)kEThreads, n - j0);
        for (int jj = 0; jj < lim; ++jj) {
            const double4 q = tile[jj];
            const double dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
            const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
            if (r2 > 0.0) phi += q.w / sqrt(r2);
        }
        __syncthreads();
    }
    double val[9];
    val[0] = 0.5 * p.w * (v.x * v.x + v.y * v.y + v.z * v.z);
    val[1] = -0.5 * G * p.w * phi;
    val[2] = p.w * v.x; val[3] = p.w * v.y; val[4] = p.w * v.z;
    val[5] = p.w * p.x; val[6] = p.w * p.y; val[7] = p.w * p.z;
    val[8] = p.w;
#pragma unroll
    for (int k = 0; k < 9; ++k) red[k][t] = i < n ? val[k] : 0.0;
    __syncthreads();
    for (int w = kEThreads / 2; w > 0; w >>= 1) {
        if (t < w)
            for (int k = 0; k < 9; ++k) red[k][t] += red[k][t + w];
        __syncthreads();
    }
    if (t < 9) out[(size_t)blockIdx.x * 9 + t] = red[t][0];
}

int64_t energy_scratch_doubles(int64_t n) { return ((n + kEThreads - 1) / kEThreads) * 9 + 9; }

int launch_energy(int64_t n, const double4 *pm, const double4 *vel, double G, double *scratch, int64_t scratch_n,
                  cudaStream_t s) {
    if (n == 0) return GTD_OK;
    const int64_t blocks = (n + kEThreads - 1) / kEThreads;
    if (blocks * 9 > scratch_n) return fail(GTD_ERR_CAPACITY, "energy scratch too small");
    energy_kernel<<<(unsigned)blocks, kEThreads, 0, s>>>(n, pm, vel, G, scratch);
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}

int finish_energy(const double *h, int64_t n, double *out9) {
    const int64_t blocks = (n + kEThreads - 1) / kEThreads;
    long double acc[9] = {0};
    for (int64_t b = 0; b < blocks; ++b)
        for (int k = 0; k < 9; ++k) acc[k] += h[b * 9 + k];
    for (int k = 0; k < 9; ++k) out9[k] = (double)acc[k];
    return GTD_OK;
}

}  // namespace gtd
