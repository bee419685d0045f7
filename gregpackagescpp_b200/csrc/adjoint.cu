// Hand-written adjoint of the FP64 leapfrog KDK direct-summation evolve: gradients of a loss on
// the final state with respect to the initial positions, velocities and masses.  There is no
// counterpart in the reference; the forward it differentiates is gtd::system::evolve(leapfrog_kdk)
// (gregsys.hpp:2946-2990, force gregsys.hpp:352-357).
//
// Forward, as a sequence of kicks K(c, x): v += c a(x) and drifts D: x += h v:
//     K(h/2, x0) D K(h, x1) D ... D K(h, x_{T-1}) D K(h/2, xT)
// (a step's closing half kick and the next step's opening half kick act at the same positions and
// merge into one full kick).  Reverse sweep from (lx, lv) = (dL/dxT, dL/dvT), mu = 0:
//     for k = T .. 0:   lx += c_k J(x_k)^T lv ;  mu += c_k (da/dm)^T lv ;  if k > 0: lv += h lx
// with, for a_i = sum_j G m_j d_ij / r^3 (d_ij = x_j - x_i),
//     (J^T w)_k = sum_j G [ u / r^3 - 3 d (d . u) / r^5 ],  u = m_k w_j - m_j w_k,  d = x_j - x_k
//     (dL/dm)_k += sum_j G (w_j . (x_k - x_j)) / r^3.
// Memory: sqrt(T)-step checkpointing.  The forward keeps (x, v_{k-1/2}, a) every C steps; the
// reverse sweep recomputes one segment of positions at a time from its checkpoint, then runs the
// segment's VJPs backwards.  The force uses the stream-K FP64 decomposition of direct.cu; the VJP
// takes each unordered pair once (vjp_sym_kernel: the J^T w term is antisymmetric in the pair),
// or, where that kernel's partial sums would not fit, every ordered pair (vjp_kernel).
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <type_traits>
#include <vector>

#include "gtd_internal.cuh"
#include "gtd_math.cuh"

namespace gtd {

struct VjpArgs {
    int64_t n, rows, tiles, total;
    int grid, bi;
    const double4 *x;   // positions + mass
    const double4 *w;   // c_k * lambda_v (xyz)
    double G;
    double *part;       // 4 doubles per body per slot
};

constexpr int kVT = 256;

// One staged j-tile against body k.  The J^T w sum is kept as two parts, sum u / r^3 (j*) and
// sum (d . u) d / r^5 (k*), combined as j - 3 k by the caller, so that the factor 3 costs no
// operation per pair; with the |r|^-1 correction that is 34 FP64 operations per pair.  kGuard: the
// tile holds k itself or padding bodies (r2 = 0 or a zero mass), whose terms are selected away; every
// other tile runs without the compare.
template <bool kGuard>
__device__ __forceinline__ void vjp_tile(const double4 *__restrict__ tx, const double4 *__restrict__ tw,
                                         const double4 &xk, const double4 &wk, double &jx, double &jy, double &jz,
                                         double &kx, double &ky, double &kz, double &mu) {
#pragma unroll 2
    for (int jj = 0; jj < kVT; ++jj) {
        const double4 xj = tx[jj], wj = tw[jj];
        const double dx = xj.x - xk.x, dy = xj.y - xk.y, dz = xj.z - xk.z;
        const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
        double inv = inv_r(r2);
        if (kGuard) inv = r2 > 0.0 ? inv : 0.0;  // j == k and padding contribute nothing
        const double inv2 = inv * inv, inv3 = inv2 * inv, inv5 = inv3 * inv2;
        const double ux = xk.w * wj.x - xj.w * wk.x;
        const double uy = xk.w * wj.y - xj.w * wk.y;
        const double uz = xk.w * wj.z - xj.w * wk.z;
        const double c5 = fma(dz, uz, fma(dy, uy, dx * ux)) * inv5;
        jx = fma(inv3, ux, jx);
        jy = fma(inv3, uy, jy);
        jz = fma(inv3, uz, jz);
        kx = fma(c5, dx, kx);
        ky = fma(c5, dy, ky);
        kz = fma(c5, dz, kz);
        const double wd = fma(wj.z, dz, fma(wj.y, dy, wj.x * dx));
        mu = fma(-wd, inv3, mu);
    }
}

// Partial VJP sums over j-tiles; same (row, tile) stream-K split as the force kernel, I = 1.
__global__ void __launch_bounds__(kVT) vjp_kernel(VjpArgs a) {
    __shared__ double4 tx[kVT];
    __shared__ double4 tw[kVT];
    const int t = threadIdx.x;
    int64_t s = (int64_t)blockIdx.x * a.total / a.grid;
    const int64_t e = (int64_t)(blockIdx.x + 1) * a.total / a.grid;
    while (s < e) {
        const int64_t r = s / a.tiles;
        const int64_t jt0 = s - r * a.tiles;
        const int64_t row_end = min(e, (r + 1) * a.tiles);
        const int64_t jt1 = row_end - r * a.tiles;
        const int64_t k = r * a.bi + t;
        double4 xk = make_double4(0, 0, 0, 0), wk = xk;
        if (k < a.n) {
            xk = a.x[k];
            wk = a.w[k];
        }
        double jx = 0, jy = 0, jz = 0, kx = 0, ky = 0, kz = 0, mu = 0;
        for (int64_t jt = jt0; jt < jt1; ++jt) {
            const int64_t j = jt * kVT + t;
            __syncthreads();
            tx[t] = j < a.n ? a.x[j] : make_double4(0, 0, 0, 0);
            tw[t] = j < a.n ? a.w[j] : make_double4(0, 0, 0, 0);
            __syncthreads();
            // rows and tiles are both kVT bodies wide (bi == kVT): tile r holds the row's own bodies
            const bool guard = jt == r || (jt + 1) * kVT > a.n;
            if (guard)
                vjp_tile<true>(tx, tw, xk, wk, jx, jy, jz, kx, ky, kz, mu);
            else
                vjp_tile<false>(tx, tw, xk, wk, jx, jy, jz, kx, ky, kz, mu);
        }
        double *slot = a.part + (size_t)(blockIdx.x + r) * 4 * a.bi;
        slot[t] = fma(-3.0, kx, jx);
        slot[a.bi + t] = fma(-3.0, ky, jy);
        slot[2 * a.bi + t] = fma(-3.0, kz, jz);
        slot[3 * a.bi + t] = mu;
        s = row_end;
    }
}

// ---- symmetric VJP ---------------------------------------------------------------------------
// The J^T w term of a pair is antisymmetric: with d = x_j - x_k and u = m_k w_j - m_j w_k, body k
// receives T = u / r^3 - 3 d (d . u) / r^5 and body j receives -T.  So each unordered pair of
// 256-body blocks (r < c) is evaluated once, 47 FP64 operations per pair for both bodies' J^T w
// and mass terms and their sums (two ordered pairs cost 68 in vjp_kernel); a diagonal block
// (r == c) sums its ordered pairs for its own rows only.  Work: items (r, c), c >= r, in row-major
// order, each cut into 8 units of 32 columns; CTA g takes the contiguous units
// [g U / grid, (g + 1) U / grid), so a CTA touches consecutive items and every CTA has the same
// number of units.
//   Rows: summed in registers over the units of an item, written to slot g + item (unique per
//   (CTA, item), as in the stream-K split of the force kernel).
//   Columns: inside a unit a warp's lane l pairs its rows with column (l + s) mod 32 at step s and
//   carries that column's running sum, passed on to lane l - 1 after each step by one shuffle, so
//   lane l ends holding column l; the warps' sums are added in warp order and written per unit.
// Every sum is taken in a fixed order: the results are bit-reproducible.
constexpr int kSymChunks = kVT / 32;  // units per item

struct SymArgs {
    int64_t n;
    int nb;          // 256-body blocks
    int64_t items;   // nb (nb + 1) / 2
    int64_t units;   // items * kSymChunks
    int grid;
    const int2 *item_rc;  // item -> (r, c)
    const double4 *x;     // positions + mass
    const double4 *w;     // c_k * lambda_v
    double *rowpart;      // (grid + items) slots of 4 x kVT doubles
    double *colpart;      // units slots of 4 x 32 doubles
};

// The pair terms of body k against body j (d = x_j - x_k): T (for k; -T for j) and the two mass
// terms, mk_term for k's mass sum and mj_term for j's.
template <bool kGuard>
__device__ __forceinline__ void sym_pair(const double4 &xk, const double4 &wk, const double4 &xj, const double4 &wj,
                                         double &tx, double &ty, double &tz, double &mk_term, double &mj_term) {
    const double dx = xj.x - xk.x, dy = xj.y - xk.y, dz = xj.z - xk.z;
    const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
    double inv = inv_r(r2);
    if (kGuard) inv = r2 > 0.0 ? inv : 0.0;  // the self pair and padding contribute nothing
    const double inv2 = inv * inv, inv3 = inv2 * inv, inv5 = inv3 * inv2;
    const double ux = xk.w * wj.x - xj.w * wk.x;
    const double uy = xk.w * wj.y - xj.w * wk.y;
    const double uz = xk.w * wj.z - xj.w * wk.z;
    const double c5 = 3.0 * (fma(dz, uz, fma(dy, uy, dx * ux)) * inv5);
    tx = fma(inv3, ux, -c5 * dx);
    ty = fma(inv3, uy, -c5 * dy);
    tz = fma(inv3, uz, -c5 * dz);
    mk_term = -fma(wj.z, dz, fma(wj.y, dy, wj.x * dx)) * inv3;
    mj_term = fma(wk.z, dz, fma(wk.y, dy, wk.x * dx)) * inv3;
}

// Two rows per thread (k and k + 128 of the row block): each rotated column read and each shuffle
// of the column sums serves two pairs.
constexpr int kSymRows = 2;
constexpr int kSymThreads = kVT / kSymRows;
static_assert(kSymThreads >= 128 && kSymThreads % 32 == 0, "the column reduction uses 128 threads");

__global__ void __launch_bounds__(kSymThreads, 3) vjp_sym_kernel(SymArgs a) {
    // the column block, one array per component: a warp reads 32 different bodies per step (lane l
    // the body (l + s) mod 32), which as 8-byte words fall in distinct banks
    __shared__ double cxx[kVT], cxy[kVT], cxz[kVT], cxm[kVT], cwx[kVT], cwy[kVT], cwz[kVT];
    __shared__ double red[kSymThreads / 32][4][32];
    auto col_x = [&](int i) { return make_double4(cxx[i], cxy[i], cxz[i], cxm[i]); };
    auto col_w = [&](int i) { return make_double4(cwx[i], cwy[i], cwz[i], 0.0); };
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t u0 = (int64_t)blockIdx.x * a.units / a.grid;
    const int64_t u1 = (int64_t)(blockIdx.x + 1) * a.units / a.grid;
    int64_t cur = -1;
    int r = 0, c = 0;
    double4 xk[kSymRows], wk[kSymRows];
    double rx[kSymRows], ry[kSymRows], rz[kSymRows], rm[kSymRows];
#pragma unroll
    for (int q = 0; q < kSymRows; ++q) {
        xk[q] = wk[q] = make_double4(0, 0, 0, 0);
        rx[q] = ry[q] = rz[q] = rm[q] = 0;
    }
    auto flush_rows = [&]() {
        double *slot = a.rowpart + (size_t)(blockIdx.x + cur) * 4 * kVT;
#pragma unroll
        for (int q = 0; q < kSymRows; ++q) {
            const int l = t + q * kSymThreads;
            slot[l] = rx[q];
            slot[kVT + l] = ry[q];
            slot[2 * kVT + l] = rz[q];
            slot[3 * kVT + l] = rm[q];
            rx[q] = ry[q] = rz[q] = rm[q] = 0;
        }
    };
    for (int64_t u = u0; u < u1; ++u) {
        const int64_t it = u / kSymChunks;
        const int chunk = (int)(u - it * kSymChunks);
        if (it != cur) {
            if (cur >= 0) flush_rows();
            cur = it;
            const int2 rc = a.item_rc[it];
            r = rc.x;
            c = rc.y;
            double4 qx[kSymRows], qw[kSymRows];
#pragma unroll
            for (int q = 0; q < kSymRows; ++q) {
                const int64_t k = (int64_t)r * kVT + t + q * kSymThreads;
                xk[q] = k < a.n ? a.x[k] : make_double4(0, 0, 0, 0);
                wk[q] = k < a.n ? a.w[k] : make_double4(0, 0, 0, 0);
                const int64_t j = (int64_t)c * kVT + t + q * kSymThreads;
                qx[q] = j < a.n ? a.x[j] : make_double4(0, 0, 0, 0);
                qw[q] = j < a.n ? a.w[j] : make_double4(0, 0, 0, 0);
            }
            __syncthreads();  // the previous item's columns are no longer read
#pragma unroll
            for (int q = 0; q < kSymRows; ++q) {
                const int l = t + q * kSymThreads;
                cxx[l] = qx[q].x;
                cxy[l] = qx[q].y;
                cxz[l] = qx[q].z;
                cxm[l] = qx[q].w;
                cwx[l] = qw[q].x;
                cwy[l] = qw[q].y;
                cwz[l] = qw[q].z;
            }
            __syncthreads();
        }
        const int jb = chunk * 32;
        if (r == c) {
            // diagonal block: the rows' ordered pairs with this chunk's columns, self pairs excluded
            for (int i = 0; i < 32; ++i) {
                const double4 xj = col_x(jb + i), wj = col_w(jb + i);
#pragma unroll
                for (int q = 0; q < kSymRows; ++q) {
                    double tx, ty, tz, mk, mj;
                    sym_pair<true>(xk[q], wk[q], xj, wj, tx, ty, tz, mk, mj);
                    rx[q] += tx;
                    ry[q] += ty;
                    rz[q] += tz;
                    rm[q] += mk;
                }
            }
        } else {
            double cx = 0, cy = 0, cz = 0, cm = 0;  // running sums of column (lane + s) mod 32
            const bool guard = (int64_t)(c + 1) * kVT > a.n;  // padding columns in the last block
            auto step = [&](auto gd, int s) {
                const int i = jb + ((lane + s) & 31);
                const double4 xj = col_x(i), wj = col_w(i);
#pragma unroll
                for (int q = 0; q < kSymRows; ++q) {
                    double tx, ty, tz, mk, mj;
                    sym_pair<decltype(gd)::value>(xk[q], wk[q], xj, wj, tx, ty, tz, mk, mj);
                    rx[q] += tx;
                    ry[q] += ty;
                    rz[q] += tz;
                    rm[q] += mk;
                    cx -= tx;
                    cy -= ty;
                    cz -= tz;
                    cm += mj;
                }
                const int from = (lane + 1) & 31;
                cx = __shfl_sync(0xffffffffu, cx, from);
                cy = __shfl_sync(0xffffffffu, cy, from);
                cz = __shfl_sync(0xffffffffu, cz, from);
                cm = __shfl_sync(0xffffffffu, cm, from);
            };
            if (guard) {
                for (int s2 = 0; s2 < 32; ++s2) step(std::true_type{}, s2);
            } else {
#pragma unroll 2
                for (int s2 = 0; s2 < 32; ++s2) step(std::false_type{}, s2);
            }
            // after 32 steps and 32 passes lane l holds column l's sum over this warp's rows
            red[warp][0][lane] = cx;
            red[warp][1][lane] = cy;
            red[warp][2][lane] = cz;
            red[warp][3][lane] = cm;
            __syncthreads();
            if (t < 128) {
                const int comp = t >> 5;
                double sum = 0;
#pragma unroll
                for (int w2 = 0; w2 < kSymThreads / 32; ++w2) sum += red[w2][comp][lane];
                a.colpart[((size_t)u * 4 + comp) * 32 + lane] = sum;
            }
            __syncthreads();
        }
    }
    if (cur >= 0) flush_rows();
}

// The combine of vjp_sym_kernel's sums for body i of block b (fixed order: its row slots over the
// items (b, c), c = b .. nb-1, then its column sums over the items (r, b), r < b), then the same
// update as vjp_combine_kernel.
__global__ void vjp_sym_combine_kernel(SymArgs a, double G, double4 *lx, double4 *lv, double *mu, double h,
                                       int drift) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int b = (int)(i / kVT);
    const int t = (int)(i - (int64_t)b * kVT);
    const int nb = a.nb;
    double jx = 0, jy = 0, jz = 0, m = 0;
    const int64_t qb = (int64_t)b * nb - (int64_t)b * (b - 1) / 2;  // item (b, b)
    for (int c = b; c < nb; ++c) {
        const int64_t q = qb + (c - b);
        const int64_t g0 = ((q * kSymChunks + 1) * (int64_t)a.grid - 1) / a.units;
        const int64_t g1 = ((q * kSymChunks + kSymChunks) * (int64_t)a.grid - 1) / a.units;
        for (int64_t g = g0; g <= g1; ++g) {
            const double *slot = a.rowpart + (size_t)(g + q) * 4 * kVT;
            jx += slot[t];
            jy += slot[kVT + t];
            jz += slot[2 * kVT + t];
            m += slot[3 * kVT + t];
        }
    }
    const int chunk = t >> 5, lane = t & 31;
    for (int r = 0; r < b; ++r) {
        const int64_t q = (int64_t)r * nb - (int64_t)r * (r - 1) / 2 + (b - r);
        const double *cp = a.colpart + (size_t)(q * kSymChunks + chunk) * 4 * 32;
        jx += cp[lane];
        jy += cp[32 + lane];
        jz += cp[64 + lane];
        m += cp[96 + lane];
    }
    double4 x = lx[i];
    x.x = fma(G, jx, x.x);
    x.y = fma(G, jy, x.y);
    x.z = fma(G, jz, x.z);
    lx[i] = x;
    mu[i] = fma(G, m, mu[i]);
    if (drift) {
        double4 v = lv[i];
        v.x = fma(h, x.x, v.x);
        v.y = fma(h, x.y, v.y);
        v.z = fma(h, x.z, v.z);
        lv[i] = v;
    }
}

// lx += G J^T w ; mu += G (..) ; then (if drift) lv += h lx ; and w for the next VJP
__global__ void vjp_combine_kernel(int64_t n, int64_t tiles, int64_t total, int grid, int bi, const double *part,
                                   double G, double4 *lx, double4 *lv, double *mu, double h, int drift) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t r = i / bi;
    const int l = (int)(i - r * bi);
    const int64_t g0 = ((r * tiles + 1) * (int64_t)grid - 1) / total;
    const int64_t g1 = (((r + 1) * tiles) * (int64_t)grid - 1) / total;
    double jx = 0, jy = 0, jz = 0, m = 0;
    for (int64_t g = g0; g <= g1; ++g) {
        const double *slot = part + (size_t)(g + r) * 4 * bi;
        jx += slot[l];
        jy += slot[bi + l];
        jz += slot[2 * bi + l];
        m += slot[3 * bi + l];
    }
    double4 x = lx[i];
    x.x = fma(G, jx, x.x);
    x.y = fma(G, jy, x.y);
    x.z = fma(G, jz, x.z);
    lx[i] = x;
    mu[i] = fma(G, m, mu[i]);
    if (drift) {
        double4 v = lv[i];
        v.x = fma(h, x.x, v.x);
        v.y = fma(h, x.y, v.y);
        v.z = fma(h, x.z, v.z);
        lv[i] = v;
    }
}

__global__ void scale_kernel(int64_t n, const double4 *lv, double c, double4 *w) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 v = lv[i];
    w[i] = make_double4(c * v.x, c * v.y, c * v.z, 0.0);
}

// v += c a ; x += h v   (a kick followed by a drift)
__global__ void kick_then_drift_kernel(int64_t n, double4 *x, double4 *v, const double4 *a, double c, double h) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 vv = v[i];
    const double4 aa = a[i];
    vv.x = fma(c, aa.x, vv.x); vv.y = fma(c, aa.y, vv.y); vv.z = fma(c, aa.z, vv.z);
    v[i] = vv;
    double4 xx = x[i];
    xx.x = fma(h, vv.x, xx.x); xx.y = fma(h, vv.y, xx.y); xx.z = fma(h, vv.z, xx.z);
    x[i] = xx;
}

__global__ void kick_kernel(int64_t n, double4 *v, const double4 *a, double c) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 vv = v[i];
    const double4 aa = a[i];
    vv.x = fma(c, aa.x, vv.x); vv.y = fma(c, aa.y, vv.y); vv.z = fma(c, aa.z, vv.z);
    v[i] = vv;
}

__global__ void pack_kernel(int64_t n, const double *x3, const double *m, const double *v3, double4 *x, double4 *v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = make_double4(x3[3 * i], x3[3 * i + 1], x3[3 * i + 2], m[i]);
    if (v) v[i] = make_double4(v3[3 * i], v3[3 * i + 1], v3[3 * i + 2], 0.0);
}

__global__ void unpack_kernel(int64_t n, const double4 *a, double *a3) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 q = a[i];
    a3[3 * i] = q.x;
    a3[3 * i + 1] = q.y;
    a3[3 * i + 2] = q.z;
}

__global__ void copy_triples_kernel(int64_t n, const double *in3, double4 *out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = in3 ? make_double4(in3[3 * i], in3[3 * i + 1], in3[3 * i + 2], 0.0) : make_double4(0, 0, 0, 0);
}

}  // namespace gtd

using namespace gtd;

struct gtd_adjoint {
    int device = 0;
    int64_t n = 0;
    uint64_t steps = 0, every = 1;
    double G = 0, h = 0;
    ForcePlan fplan, vplan;
    double *fpart = nullptr, *vpart = nullptr;
    double4 *x = nullptr, *v = nullptr, *a = nullptr;     // working state
    double4 *ck = nullptr;                                 // checkpoints: (x, v_{k-1/2}, a) * ncheck
    int64_t ncheck = 0;
    double4 *seg = nullptr;                                // positions of one segment [(every+1) * n]
    double4 *lx = nullptr, *lv = nullptr, *w = nullptr;
    double *mu = nullptr;
    // symmetric VJP (vjp_sym_kernel) when its partial sums fit kSymMaxBytes, else vjp_kernel
    bool sym = false;
    SymArgs sa{};
    int2 *item_rc = nullptr;
    double *rowpart = nullptr, *colpart = nullptr;
    bool have_forward = false;
    uint64_t launches = 0;
};

static unsigned g1(int64_t n) { return (unsigned)((n + 255) / 256); }

static int adj_force(gtd_adjoint *A, const double4 *x, cudaStream_t st) {
    int rc = launch_force(GTD_PREC_F64, A->fplan, x, A->G, A->fpart, st);
    if (rc) return rc;
    StepArgs sa{};
    sa.n = A->n;
    sa.src = x;
    sa.cur = x;
    sa.vel = A->v;
    sa.acc = A->a;
    rc = launch_integrate(A->fplan, A->fpart, EPI_ACC, sa, st);
    A->launches += 2;
    return rc;
}

// The symmetric VJP keeps 8 KB of row sums per slot (one slot per item and one per CTA) and 8 KB of
// column sums per item: 37 MB at N = 16384; above this size (N ~ 90000) the ordered-pair kernel
// runs instead.
constexpr size_t kSymMaxBytes = (size_t)1 << 30;

static int adj_vjp(gtd_adjoint *A, const double4 *x, bool drift, cudaStream_t st) {
    if (A->sym) {
        SymArgs a = A->sa;
        a.x = x;
        a.w = A->w;
        vjp_sym_kernel<<<a.grid, kSymThreads, 0, st>>>(a);
        GTD_CHECK_LAUNCH();
        vjp_sym_combine_kernel<<<g1(A->n), 256, 0, st>>>(a, A->G, A->lx, A->lv, A->mu, A->h, drift ? 1 : 0);
        GTD_CHECK_LAUNCH();
        A->launches += 2;
        return GTD_OK;
    }
    const ForcePlan &p = A->vplan;
    VjpArgs va{p.n, p.rows, p.tiles, p.total, p.grid, p.bi, x, A->w, A->G, A->vpart};
    vjp_kernel<<<p.grid, kVT, 0, st>>>(va);
    GTD_CHECK_LAUNCH();
    vjp_combine_kernel<<<g1(A->n), 256, 0, st>>>(A->n, p.tiles, p.total, p.grid, p.bi, A->vpart, A->G, A->lx, A->lv,
                                                 A->mu, A->h, drift ? 1 : 0);
    GTD_CHECK_LAUNCH();
    A->launches += 2;
    return GTD_OK;
}

extern "C" {

int gtd_adjoint_create(gtd_adjoint **out, int device, int64_t n, uint64_t steps, uint64_t checkpoint_every,
                       double G, double dt) {
    if (!out) return fail(GTD_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (n < 2 || steps < 1 || !(dt > 0)) return fail(GTD_ERR_INVALID_ARGUMENT, "need n >= 2, steps >= 1, dt > 0");
    if (checkpoint_every < 1) checkpoint_every = 1;
    GTD_CUDA(cudaSetDevice(device));
    gtd_adjoint *A = new (std::nothrow) gtd_adjoint();
    if (!A) return fail(GTD_ERR_OUT_OF_MEMORY, "host allocation failed");
    A->device = device;
    A->n = n;
    A->steps = steps;
    A->every = std::min<uint64_t>(checkpoint_every, steps);
    A->G = G;
    A->h = dt;
    A->fplan = make_plan(n, GTD_PREC_F64, device, tuned_variant(device, GTD_PREC_F64, n));
    // the VJP kernel runs one i-body per thread against 256-body j-tiles: a plan with 256-body rows
    // and tiles
    A->vplan = A->fplan;
    A->vplan.bi = kVT;
    A->vplan.rows = (n + kVT - 1) / kVT;
    A->vplan.tiles = (n + kVT - 1) / kVT;
    A->vplan.total = A->vplan.rows * A->vplan.tiles;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vjp_kernel, kVT, 0);
    A->vplan.grid = (int)std::min<int64_t>((int64_t)sms * std::max(per_sm, 1), A->vplan.total);
    A->vplan.slots = A->vplan.grid + A->vplan.rows;
    A->ncheck = (int64_t)((steps + A->every - 1) / A->every) + 1;
    {
        const int nb = (int)((n + kVT - 1) / kVT);
        const int64_t items = (int64_t)nb * (nb + 1) / 2;
        const int64_t units = items * kSymChunks;
        int sym_per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sym_per_sm, vjp_sym_kernel, kSymThreads, 0);
        const int64_t grid = std::min<int64_t>((int64_t)sms * std::max(sym_per_sm, 1), units);
        const size_t bytes = ((size_t)(grid + items) + (size_t)units / kSymChunks) * 4 * kVT * sizeof(double);
        if (bytes <= kSymMaxBytes) {
            A->sym = true;
            A->sa.n = n;
            A->sa.nb = nb;
            A->sa.items = items;
            A->sa.units = units;
            A->sa.grid = (int)grid;
        }
    }
    const size_t b4 = sizeof(double4) * (size_t)n;
    cudaError_t e = cudaSuccess;
    auto M = [&](void **p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes); };
    if (A->sym) {
        M((void **)&A->item_rc, sizeof(int2) * (size_t)A->sa.items);
        M((void **)&A->rowpart, (size_t)(A->sa.grid + A->sa.items) * 4 * kVT * sizeof(double));
        M((void **)&A->colpart, (size_t)A->sa.units * 4 * 32 * sizeof(double));
        if (e == cudaSuccess) {
            std::vector<int2> rc;
            rc.reserve((size_t)A->sa.items);
            for (int r = 0; r < A->sa.nb; ++r)
                for (int c = r; c < A->sa.nb; ++c) rc.push_back(make_int2(r, c));
            e = cudaMemcpy(A->item_rc, rc.data(), sizeof(int2) * rc.size(), cudaMemcpyHostToDevice);
        }
        A->sa.item_rc = A->item_rc;
        A->sa.rowpart = A->rowpart;
        A->sa.colpart = A->colpart;
    }
    M((void **)&A->fpart, partial_bytes(A->fplan));
    M((void **)&A->vpart, (size_t)A->vplan.slots * 4 * A->vplan.bi * sizeof(double));
    M((void **)&A->x, b4);
    M((void **)&A->v, b4);
    M((void **)&A->a, b4);
    M((void **)&A->ck, 3 * b4 * (size_t)A->ncheck);
    M((void **)&A->seg, b4 * (size_t)(A->every + 1));
    M((void **)&A->lx, b4);
    M((void **)&A->lv, b4);
    M((void **)&A->w, b4);
    M((void **)&A->mu, sizeof(double) * (size_t)n);
    if (e != cudaSuccess) {
        int rc = cuda_fail(e, "adjoint buffers", __FILE__, __LINE__);
        gtd_adjoint_destroy(A);
        return rc;
    }
    *out = A;
    return GTD_OK;
}

int gtd_adjoint_destroy(gtd_adjoint *A) {
    if (!A) return GTD_OK;
    cudaSetDevice(A->device);
    cudaFree(A->fpart); cudaFree(A->vpart); cudaFree(A->x); cudaFree(A->v); cudaFree(A->a); cudaFree(A->ck);
    cudaFree(A->seg); cudaFree(A->lx); cudaFree(A->lv); cudaFree(A->w); cudaFree(A->mu);
    cudaFree(A->item_rc); cudaFree(A->rowpart); cudaFree(A->colpart);
    delete A;
    return GTD_OK;
}

// Forward KDK over all steps from device arrays x0/v0 (n x 3) and m (n); writes xT/vT (device, may
// be NULL) and keeps the checkpoints for gtd_adjoint_backward.  stream: a cudaStream_t or NULL.
int gtd_adjoint_forward(gtd_adjoint *A, const double *x0, const double *v0, const double *m, double *xT,
                        double *vT, void *stream) {
    if (!A || !x0 || !v0 || !m) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaSetDevice(A->device);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = A->n;
    const size_t b4 = sizeof(double4) * (size_t)n;
    pack_kernel<<<g1(n), 256, 0, st>>>(n, x0, m, v0, A->x, A->v);
    GTD_CHECK_LAUNCH();
    int rc = adj_force(A, A->x, st);
    if (rc) return rc;
    const double h = A->h;
    for (uint64_t k = 0; k < A->steps; ++k) {
        if (k % A->every == 0) {
            double4 *c = A->ck + 3 * (size_t)n * (k / A->every);
            GTD_CUDA(cudaMemcpyAsync(c, A->x, b4, cudaMemcpyDeviceToDevice, st));
            GTD_CUDA(cudaMemcpyAsync(c + n, A->v, b4, cudaMemcpyDeviceToDevice, st));
            GTD_CUDA(cudaMemcpyAsync(c + 2 * n, A->a, b4, cudaMemcpyDeviceToDevice, st));
        }
        kick_then_drift_kernel<<<g1(n), 256, 0, st>>>(n, A->x, A->v, A->a, k == 0 ? 0.5 * h : h, h);
        GTD_CHECK_LAUNCH();
        A->launches += 1;
        rc = adj_force(A, A->x, st);
        if (rc) return rc;
    }
    kick_kernel<<<g1(n), 256, 0, st>>>(n, A->v, A->a, 0.5 * h);
    GTD_CHECK_LAUNCH();
    A->launches += 1;
    if (xT) unpack_kernel<<<g1(n), 256, 0, st>>>(n, A->x, xT);
    if (vT) unpack_kernel<<<g1(n), 256, 0, st>>>(n, A->v, vT);
    GTD_CHECK_LAUNCH();
    A->have_forward = true;
    return GTD_OK;
}

// Reverse sweep: gxT, gvT (device, n x 3, gvT may be NULL) -> gx0, gv0 (n x 3), gm (n).
int gtd_adjoint_backward(gtd_adjoint *A, const double *gxT, const double *gvT, double *gx0, double *gv0, double *gm,
                         void *stream) {
    if (!A || !gxT) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!A->have_forward) return fail(GTD_ERR_INVALID_ARGUMENT, "gtd_adjoint_forward must run first");
    cudaSetDevice(A->device);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = A->n;
    const size_t b4 = sizeof(double4) * (size_t)n;
    const double h = A->h;
    const uint64_t T = A->steps, C = A->every;
    copy_triples_kernel<<<g1(n), 256, 0, st>>>(n, gxT, A->lx);
    copy_triples_kernel<<<g1(n), 256, 0, st>>>(n, gvT, A->lv);
    GTD_CHECK_LAUNCH();
    GTD_CUDA(cudaMemsetAsync(A->mu, 0, sizeof(double) * (size_t)n, st));
    const int64_t nseg = (int64_t)((T + C - 1) / C);
    for (int64_t sgi = nseg - 1; sgi >= 0; --sgi) {
        const uint64_t k0 = (uint64_t)sgi * C, k1 = std::min<uint64_t>(k0 + C, T);
        // recompute positions x_{k0..k1} of this segment from its checkpoint
        const double4 *c = A->ck + 3 * (size_t)n * (size_t)sgi;
        GTD_CUDA(cudaMemcpyAsync(A->x, c, b4, cudaMemcpyDeviceToDevice, st));
        GTD_CUDA(cudaMemcpyAsync(A->v, c + n, b4, cudaMemcpyDeviceToDevice, st));
        GTD_CUDA(cudaMemcpyAsync(A->a, c + 2 * n, b4, cudaMemcpyDeviceToDevice, st));
        GTD_CUDA(cudaMemcpyAsync(A->seg, A->x, b4, cudaMemcpyDeviceToDevice, st));
        for (uint64_t k = k0; k < k1; ++k) {
            kick_then_drift_kernel<<<g1(n), 256, 0, st>>>(n, A->x, A->v, A->a, k == 0 ? 0.5 * h : h, h);
            GTD_CHECK_LAUNCH();
            A->launches += 1;
            GTD_CUDA(cudaMemcpyAsync(A->seg + (size_t)(k + 1 - k0) * n, A->x, b4, cudaMemcpyDeviceToDevice, st));
            if (k + 1 < k1) {
                int rc = adj_force(A, A->x, st);
                if (rc) return rc;
            }
        }
        // VJPs at x_k, k = k1 .. k0 (k0 only for the first segment's x0 handled when sgi == 0)
        const uint64_t kstop = sgi == 0 ? k0 : k0 + 1;
        for (uint64_t k = k1 + 1; k-- > kstop;) {
            const double ck = (k == 0 || k == T) ? 0.5 * h : h;
            scale_kernel<<<g1(n), 256, 0, st>>>(n, A->lv, ck, A->w);
            GTD_CHECK_LAUNCH();
            A->launches += 1;
            int rc = adj_vjp(A, A->seg + (size_t)(k - k0) * n, k > 0, st);
            if (rc) return rc;
        }
    }
    if (gx0) unpack_kernel<<<g1(n), 256, 0, st>>>(n, A->lx, gx0);
    if (gv0) unpack_kernel<<<g1(n), 256, 0, st>>>(n, A->lv, gv0);
    if (gm) GTD_CUDA(cudaMemcpyAsync(gm, A->mu, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    GTD_CHECK_LAUNCH();
    return GTD_OK;
}

int gtd_adjoint_launch_count(const gtd_adjoint *A, uint64_t *count) {
    if (!A || !count) return fail(GTD_ERR_INVALID_ARGUMENT, "NULL argument");
    *count = A->launches;
    return GTD_OK;
}

}  // extern "C"
