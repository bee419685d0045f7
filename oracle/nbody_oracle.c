/* CPU restatement of the gtd:: force-and-step path.  TEST INFRASTRUCTURE ONLY (see
 * nbody_oracle.h): the oracle the CUDA kernels are checked against, never linked by the product.
 *
 * Types follow the reference exactly: positions, velocities, accelerations, masses and radii are
 * double (T = M = R = double), G / dt / half_dt / restitution are long double (gregsys.hpp:171-213,
 * gregbod.hpp:916), and every expression promotes where the reference's operator overloads
 * promote (gregvec.hpp:2069-2073, 2487-2497, 3742-3744, 3792-3796, 3834-3836).  Build with
 * -ffp-contract=off so no multiply-add is fused where the reference rounds twice.
 */
#include "nbody_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef long double ld;

long double orc_G_units(uint64_t m_first, uint64_t m_second, uint64_t d_first, uint64_t d_second, uint64_t t_first,
                        uint64_t t_second) {
    /* gregsys.hpp:258-274: "Ma:b" gives m_denom=a, m_num=b; "Dc:d" gives d_num=c, d_denom=d;
     * "Tx:y" gives t_denom=x, t_num=y.  G starts at 66743 (units of 1e-15 SI). */
    uint64_t m_denom = m_first, m_num = m_second, d_num = d_first, d_denom = d_second, t_denom = t_first,
             t_num = t_second;
    ld G = 66743;
    G *= m_num * d_num * d_num * d_num * t_num * t_num;
    G /= m_denom * d_denom * d_denom * d_denom * t_denom * t_denom;
    G /= 1000000000000000ULL;
    return G;
}

/* vector3D<double>::magnitude, gregvec.hpp:2069-2073 */
static ld mag_ld(double x, double y, double z) {
    return sqrtl((ld)x * (ld)x + (ld)y * (ld)y + (ld)z * (ld)z);
}

/* cumulative_acc, gregsys.hpp:352-357: r12 = x_j - x_i; |((r12.r12) r12)| in long double;
 * a_i += (G m_j / r^3) r12 ; a_j -= (G m_i / r^3) r12, each component rounded into double. */
static void pair_acc(const double *xi, const double *xj, double mi, double mj, ld G, double *ai, double *aj) {
    double rx = xj[0] - xi[0], ry = xj[1] - xi[1], rz = xj[2] - xi[2];
    double r2 = rx * rx + ry * ry + rz * rz;
    ld r3 = mag_ld(r2 * rx, r2 * ry, r2 * rz);
    ld si = (G * (ld)mj) / r3;
    ld sj = (G * (ld)mi) / r3;
    ai[0] = (double)((ld)ai[0] + si * (ld)rx);
    ai[1] = (double)((ld)ai[1] + si * (ld)ry);
    ai[2] = (double)((ld)ai[2] + si * (ld)rz);
    aj[0] = (double)((ld)aj[0] - sj * (ld)rx);
    aj[1] = (double)((ld)aj[1] - sj * (ld)ry);
    aj[2] = (double)((ld)aj[2] - sj * (ld)rz);
}

/* calc_acc_and_e with memFreq == 0, gregsys.hpp:439-447 */
void orc_direct_acc(int n, const double *m, const double *x3, const long double *Gp, double *a3) {
    ld G = *Gp;
    memset(a3, 0, sizeof(double) * 3 * (size_t)n);
    for (int o = 0; o < n; ++o)
        for (int i = o + 1; i < n; ++i) pair_acc(x3 + 3 * o, x3 + 3 * i, m[o], m[i], G, a3 + 3 * o, a3 + 3 * i);
}

/* orc_direct_acc restricted to the bodies rows[0..nrows): each row's acceleration is summed over
 * the other bodies in ascending index order, with pair_acc's arithmetic for that body's side of
 * each pair (a_i -= s r for the pairs (o < i) where the reference updates i as the second body,
 * a_i += s r for o > i), so the rows agree bit for bit with orc_direct_acc.  gross (optional)
 * receives sum_j |G m_j / r^2| per row, the scale of FP rounding in a summed force.  Rows are
 * split over `threads` pthreads. */
typedef struct {
    int n, lo, hi;
    const double *m, *x3;
    ld G;
    const int32_t *rows;
    double *a3, *gross;
} rows_job;

static void *rows_worker(void *arg) {
    const rows_job *J = (const rows_job *)arg;
    for (int q = J->lo; q < J->hi; ++q) {
        const int i = J->rows[q];
        const double *xi = J->x3 + 3 * i;
        double a[3] = {0.0, 0.0, 0.0};
        ld g = 0.0L;
        for (int o = 0; o < J->n; ++o) {
            if (o == i) continue;
            const double *xo = J->x3 + 3 * o;
            if (o < i) { /* pair (o, i): r12 = x_i - x_o, body i is the second body */
                double rx = xi[0] - xo[0], ry = xi[1] - xo[1], rz = xi[2] - xo[2];
                double r2 = rx * rx + ry * ry + rz * rz;
                ld r3 = mag_ld(r2 * rx, r2 * ry, r2 * rz);
                ld sj = (J->G * (ld)J->m[o]) / r3;
                a[0] = (double)((ld)a[0] - sj * (ld)rx);
                a[1] = (double)((ld)a[1] - sj * (ld)ry);
                a[2] = (double)((ld)a[2] - sj * (ld)rz);
                g += (J->G * (ld)J->m[o]) / (ld)r2;
            } else { /* pair (i, o): r12 = x_o - x_i, body i is the first body */
                double rx = xo[0] - xi[0], ry = xo[1] - xi[1], rz = xo[2] - xi[2];
                double r2 = rx * rx + ry * ry + rz * rz;
                ld r3 = mag_ld(r2 * rx, r2 * ry, r2 * rz);
                ld si = (J->G * (ld)J->m[o]) / r3;
                a[0] = (double)((ld)a[0] + si * (ld)rx);
                a[1] = (double)((ld)a[1] + si * (ld)ry);
                a[2] = (double)((ld)a[2] + si * (ld)rz);
                g += (J->G * (ld)J->m[o]) / (ld)r2;
            }
        }
        J->a3[3 * q] = a[0];
        J->a3[3 * q + 1] = a[1];
        J->a3[3 * q + 2] = a[2];
        if (J->gross) J->gross[q] = (double)g;
    }
    return NULL;
}

void orc_direct_acc_rows(int n, const double *m, const double *x3, const long double *Gp, const int32_t *rows,
                         int nrows, double *a3, double *gross, int threads) {
    enum { kMaxThreads = 256 };
    if (threads > nrows) threads = nrows;
    if (threads > kMaxThreads) threads = kMaxThreads;
    if (threads < 1) threads = 1;
    pthread_t tid[kMaxThreads];
    rows_job job[kMaxThreads];
    int started[kMaxThreads];
    for (int k = 0; k < threads; ++k) {
        job[k] = (rows_job){n, (int)((long)nrows * k / threads), (int)((long)nrows * (k + 1) / threads), m, x3, *Gp,
                            rows, a3, gross};
        started[k] = k > 0 && pthread_create(&tid[k], NULL, rows_worker, &job[k]) == 0;
    }
    rows_worker(&job[0]);
    for (int k = 1; k < threads; ++k) {
        if (started[k]) pthread_join(tid[k], NULL);
        else rows_worker(&job[k]); /* a thread that could not start: its rows run here */
    }
}

/* x += s * y with s long double and the sum rounded into double (vector3D += vector3D<long double>) */
static void axpy_ld(double *x, ld s, const double *y) {
    for (int k = 0; k < 3; ++k) x[k] = (double)((ld)x[k] + s * (ld)y[k]);
}

typedef struct {
    int inner; /* position in the iteration order that generated the candidate (ties) */
    int body;  /* body index */
    ld dist;
    double mom_o, mom_i;
    double ux, uy, uz;
} coll_cand;

static int cand_cmp(const void *a, const void *b) {
    const coll_cand *p = (const coll_cand *)a, *q = (const coll_cand *)b;
    if (p->dist < q->dist) return -1;
    if (p->dist > q->dist) return 1;
    return (p->inner > q->inner) - (p->inner < q->inner);
}

static void resolve_group(int o, coll_cand *c, int nc, const double *m, const double *rest, double *v3);

/* s_coll without GREGSYS_MERGERS, gregsys.hpp:690-914.  For each outer body, the overlapping
 * later bodies are keyed by their long-double distance in a std::map (first insertion wins on an
 * equal key) with the momenta along r12 snapshotted at scan time, then resolved in ascending
 * distance with the restitution impulse of gregsys.hpp:810-838. */
void orc_s_coll(int n, const double *m, const double *r, const double *rest, const double *x3, double *v3) {
    coll_cand *c = (coll_cand *)malloc(sizeof(coll_cand) * (size_t)(n > 1 ? n : 1));
    for (int o = 0; o < n; ++o) {
        int nc = 0;
        for (int i = o + 1; i < n; ++i) {
            double rad_dist = r[o] + r[i];
            double ux = x3[3 * i] - x3[3 * o], uy = x3[3 * i + 1] - x3[3 * o + 1], uz = x3[3 * i + 2] - x3[3 * o + 2];
            ld dist = mag_ld(ux, uy, uz);
            ux = (double)((ld)ux / dist);
            uy = (double)((ld)uy / dist);
            uz = (double)((ld)uz / dist);
            if ((ld)rad_dist > dist) {
                /* momentum() = mass * vel (gregbod.hpp:595-597), then the dot product with the unit
                 * r12 in double (gregvec.hpp:3742-3744) */
                double mox = m[o] * v3[3 * o], moy = m[o] * v3[3 * o + 1], moz = m[o] * v3[3 * o + 2];
                double mix = m[i] * v3[3 * i], miy = m[i] * v3[3 * i + 1], miz = m[i] * v3[3 * i + 2];
                double po = mox * ux + moy * uy + moz * uz;
                double pi = mix * ux + miy * uy + miz * uz;
                c[nc].inner = i;
                c[nc].body = i;
                c[nc].dist = dist;
                c[nc].mom_o = po;
                c[nc].mom_i = pi;
                c[nc].ux = ux;
                c[nc].uy = uy;
                c[nc].uz = uz;
                ++nc;
            }
        }
        if (!nc) continue;
        resolve_group(o, c, nc, m, rest, v3);
    }
    free(c);
}

/* The response of s_coll / bh_s_coll to one outer body's candidates (gregsys.hpp:810-838 and
 * 657-681): ascending distance, first of equal keys only, impulse for approaching pairs. */
static void resolve_group(int o, coll_cand *c, int nc, const double *m, const double *rest, double *v3) {
    qsort(c, (size_t)nc, sizeof(coll_cand), cand_cmp);
    for (int k = 0; k < nc; ++k) {
        if (k > 0 && c[k].dist == c[k - 1].dist) continue; /* std::map::emplace keeps the first key */
        int i = c[k].body;
        double o_vel = c[k].mom_o / m[o];
        double i_vel = c[k].mom_i / m[i];
        double o_minus_i = o_vel - i_vel;
        ld avg_rest = ((ld)rest[o] + (ld)rest[i]) / 2;
        if (o_vel > 0 || i_vel < 0) {
            if (o_vel <= 0 && i_vel < 0)
                if (o_vel < i_vel) continue;
            if (o_vel > 0 && i_vel >= 0)
                if (o_vel < i_vel) continue;
            double psum = c[k].mom_o + c[k].mom_i;
            double msum = m[o] + m[i];
            double new_o_vel = (double)(((ld)psum - (ld)m[i] * avg_rest * (ld)o_minus_i) / (ld)msum);
            double new_i_vel = (double)(((ld)psum + (ld)m[o] * avg_rest * (ld)o_minus_i) / (ld)msum);
            double d_o = new_o_vel - o_vel, d_i = new_i_vel - i_vel;
            v3[3 * o] += d_o * c[k].ux;
            v3[3 * o + 1] += d_o * c[k].uy;
            v3[3 * o + 2] += d_o * c[k].uz;
            v3[3 * i] += d_i * c[k].ux;
            v3[3 * i + 1] += d_i * c[k].uy;
            v3[3 * i + 2] += d_i * c[k].uz;
        }
    }
}

int orc_evolve(int method, int coll, int n, const double *m, const double *r, const double *rest, double *x3,
               double *v3, double *a3, long double dt, uint64_t steps, const long double *Gp) {
    ld G = *Gp;
    if (n <= 0) return 0; /* gregsys.hpp:2611-2612: empty system returns immediately */
    ld half_dt = dt / 2;
    size_t sz = sizeof(double) * 3 * (size_t)n;
    if (method == ORC_LEAPFROG_KDK) {
        /* gregsys.hpp:2946-2990 with loop_kdk :477-513 */
        orc_direct_acc(n, m, x3, Gp, a3);
        for (uint64_t s = 0; s < steps; ++s) {
            for (int i = 0; i < n; ++i) {
                axpy_ld(v3 + 3 * i, half_dt, a3 + 3 * i);
                axpy_ld(x3 + 3 * i, dt, v3 + 3 * i);
            }
            orc_direct_acc(n, m, x3, Gp, a3);
            for (int i = 0; i < n; ++i) axpy_ld(v3 + 3 * i, half_dt, a3 + 3 * i);
            if (coll == 3) orc_s_coll(n, m, r, rest, x3, v3);
        }
        return 0;
    }
    if (method == ORC_LEAPFROG_DKD) {
        /* gregsys.hpp:2993-3039 with loop_dkd :540-560 */
        for (uint64_t s = 0; s < steps; ++s) {
            for (int i = 0; i < n; ++i) axpy_ld(x3 + 3 * i, half_dt, v3 + 3 * i);
            orc_direct_acc(n, m, x3, Gp, a3);
            for (int i = 0; i < n; ++i) {
                axpy_ld(v3 + 3 * i, dt, a3 + 3 * i);
                axpy_ld(x3 + 3 * i, half_dt, v3 + 3 * i);
            }
            if (coll == 3) orc_s_coll(n, m, r, rest, x3, v3);
        }
        return 0;
    }
    if (method == ORC_EULER) {
        /* gregsys.hpp:2666-2712 with take_euler_step :380-391 */
        for (uint64_t s = 0; s < steps; ++s) {
            orc_direct_acc(n, m, x3, Gp, a3);
            for (int i = 0; i < n; ++i) {
                axpy_ld(x3 + 3 * i, dt, v3 + 3 * i);
                axpy_ld(v3 + 3 * i, dt, a3 + 3 * i);
            }
            if (coll == 3) orc_s_coll(n, m, r, rest, x3, v3);
        }
        return 0;
    }
    if (method == ORC_MODIFIED_EULER || method == ORC_MIDPOINT) {
        /* modified Euler gregsys.hpp:2722-2760 + take_modified_euler_step :392-405;
         * midpoint gregsys.hpp:2808-2846 + take_midpoint_step :406-419 */
        int mid = method == ORC_MIDPOINT;
        ld h = mid ? half_dt : dt;
        double *px = (double *)malloc(sz), *pv = (double *)malloc(sz), *pa = (double *)malloc(sz);
        if (!px || !pv || !pa) { free(px); free(pv); free(pa); return -3; }
        for (uint64_t s = 0; s < steps; ++s) {
            orc_direct_acc(n, m, x3, Gp, a3);
            for (int i = 0; i < 3 * n; ++i) {
                px[i] = (double)((ld)x3[i] + h * (ld)v3[i]);
                pv[i] = (double)((ld)v3[i] + h * (ld)a3[i]);
            }
            /* the predicted accelerations start from zero (default-constructed / make_zero) */
            memset(pa, 0, sz);
            for (int o = 0; o < n; ++o)
                for (int i = o + 1; i < n; ++i) pair_acc(px + 3 * o, px + 3 * i, m[o], m[i], G, pa + 3 * o, pa + 3 * i);
            for (int i = 0; i < 3 * n; ++i) {
                if (mid) {
                    x3[i] = (double)((ld)x3[i] + dt * (ld)pv[i]);
                    v3[i] = (double)((ld)v3[i] + dt * (ld)pa[i]);
                } else {
                    x3[i] = (double)((ld)x3[i] + half_dt * (ld)(v3[i] + pv[i]));
                    v3[i] = (double)((ld)v3[i] + half_dt * (ld)(a3[i] + pa[i]));
                }
            }
            if (coll == 3) orc_s_coll(n, m, r, rest, x3, v3);
        }
        free(px);
        free(pv);
        free(pa);
        return 0;
    }
    return -1;
}

void orc_energy(int n, const double *m, const double *x3, const double *v3, const long double *Gp, double *ke,
                double *pe) {
    ld G = *Gp;
    /* calc_energy, gregsys.hpp:608-630; KE per body from set_ke, gregbod.hpp:917-920 */
    double *bpe = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    double total_pe = 0, total_ke = 0;
    for (int o = 0; o < n; ++o) {
        for (int i = o + 1; i < n; ++i) {
            double rx = x3[3 * i] - x3[3 * o], ry = x3[3 * i + 1] - x3[3 * o + 1], rz = x3[3 * i + 2] - x3[3 * o + 2];
            ld pot = -(G * (ld)m[o] * (ld)m[i]) / mag_ld(rx, ry, rz);
            bpe[o] = (double)((ld)bpe[o] + pot);
            bpe[i] = (double)((ld)bpe[i] + pot);
        }
        bpe[o] /= 2.0;
        ld mag = mag_ld(v3[3 * o], v3[3 * o + 1], v3[3 * o + 2]);
        ld k = (ld)(0.5 * m[o]) * mag * mag;
        total_pe += bpe[o];
        total_ke = (double)((ld)total_ke + k);
    }
    free(bpe);
    *ke = total_ke;
    *pe = total_pe;
}

void orc_merge_pair(double *a, const double *b) {
    /* gregbod.hpp:1066-1082 with com/vel_com/acc_com gregbod.hpp:1096-1145; rows are
     * {m, r, rest, x, y, z, vx, vy, vz, ax, ay, az} */
    double ma = a[0], mb = b[0], msum = ma + mb;
    double nx[3], nv[3], na[3];
    for (int k = 0; k < 3; ++k) {
        nx[k] = (ma * a[3 + k] + mb * b[3 + k]) / msum;
        nv[k] = (ma * a[6 + k] + mb * b[6 + k]) / msum;
        na[k] = (ma * a[9 + k] + mb * b[9 + k]) / msum;
    }
    for (int k = 0; k < 3; ++k) {
        a[3 + k] = nx[k];
        a[6 + k] = nv[k];
        a[9 + k] = na[k];
    }
    a[2] = (double)(((ld)a[2] + (ld)b[2]) / 2);
    a[0] = ma + mb;
    a[1] = (double)cbrtl((ld)(a[1] * a[1] * a[1] + b[1] * b[1] * b[1]));
}

int orc_merge_overlapping(int n, double *b) {
    int num = n;
    for (int o = 0; o < num; ++o) {
        int i = o + 1;
        while (i < num) {
            if (i == o) { ++i; continue; }
            double *bo = b + 12 * o, *bi = b + 12 * i;
            double dx = bi[3] - bo[3], dy = bi[4] - bo[4], dz = bi[5] - bo[5];
            ld dist = sqrtl((ld)(dx * dx + dy * dy + dz * dz)); /* vec_ops::distance gregvec.hpp:4701-4706 */
            if (dist < (ld)(bo[1] + bi[1])) {
                orc_merge_pair(bo, bi);
                memmove(b + 12 * i, b + 12 * (i + 1), sizeof(double) * 12 * (size_t)(num - i - 1));
                if (i < o) --o;
                --num;
                i = 0;
                continue;
            }
            ++i;
        }
    }
    return num;
}

/* ---------------------------------------------------------------------------------------------- */
/* Barnes-Hut host rebuild                                                                         */

static double roundT(double v, int is_float) { return is_float ? (double)(float)v : v; }
static double addT(double a, double b, int is_float) { return is_float ? (double)((float)a + (float)b) : a + b; }
static double subT(double a, double b, int is_float) { return is_float ? (double)((float)a - (float)b) : a - b; }

void orc_bh_root_box(int n, const double *x3, int is_float, double *box6) {
    /* greg8tree.hpp:1012-1047 */
    double mn[3], mx[3];
    for (int k = 0; k < 3; ++k) mn[k] = mx[k] = roundT(x3[k], is_float);
    for (int i = 1; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            double v = roundT(x3[3 * i + k], is_float);
            if (v < mn[k]) mn[k] = v;
            if (v > mx[k]) mx[k] = v;
        }
    double xr = subT(mx[0], mn[0], is_float), yr = subT(mx[1], mn[1], is_float), zr = subT(mx[2], mn[2], is_float);
    double edge = xr > yr ? (xr > zr ? xr : zr) : (yr > zr ? yr : zr);
    double pad = roundT((double)((ld)edge / 20.0L), is_float);
    for (int k = 0; k < 3; ++k) box6[k] = subT(mn[k], pad, is_float);
    edge = addT(edge, roundT(2 * pad, is_float), is_float);
    for (int k = 0; k < 3; ++k) box6[3 + k] = addT(box6[k], edge, is_float);
}

/* midpoint of set_corners, greg8tree.hpp:83-85: (btm + top) in T, then /2 (exact) */
static double midT(double lo, double hi, int is_float) { return addT(lo, hi, is_float) * 0.5; }

int orc_morton(const double *pos3, const double *box6, int is_float, uint64_t *code) {
    double p[3], lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        p[k] = roundT(pos3[k], is_float);
        lo[k] = box6[k];
        hi[k] = box6[3 + k];
        if (!(lo[k] <= p[k] && p[k] < hi[k])) return -1; /* between(), gregvec.hpp:2115-2120 */
    }
    uint64_t c = 0;
    for (int l = 0; l < 21; ++l) {
        unsigned oct = 0;
        for (int k = 0; k < 3; ++k) {
            double mid = midT(lo[k], hi[k], is_float);
            if (p[k] >= mid) {
                oct |= 1u << k;
                lo[k] = mid;
            } else {
                hi[k] = mid;
            }
        }
        c = (c << 3) | oct;
    }
    *code = c;
    return 0;
}

typedef struct {
    uint64_t code;
    int32_t idx;
} keyidx;

static int keyidx_cmp(const void *a, const void *b) {
    const keyidx *p = (const keyidx *)a, *q = (const keyidx *)b;
    if (p->code != q->code) return p->code < q->code ? -1 : 1;
    return (p->idx > q->idx) - (p->idx < q->idx);
}

static int lcp_digits(uint64_t a, uint64_t b) {
    uint64_t x = a ^ b;
    if (!x) return 21;
    return (__builtin_clzll(x) - 1) / 3;
}

/* last sorted slot whose code shares the first d octal digits with code[a] */
static int range_end(const uint64_t *code, int n, int a, int d) {
    int shift = 63 - 3 * d;
    uint64_t pre = shift >= 64 ? 0 : (code[a] >> shift);
    int lo = a, hi = n - 1;
    while (lo < hi) {
        int midp = lo + (hi - lo + 1) / 2;
        uint64_t pm = shift >= 64 ? 0 : (code[midp] >> shift);
        if (pm == pre) lo = midp;
        else hi = midp - 1;
    }
    return lo;
}

void orc_bh_free(orc_tree *t) {
    free(t->code); free(t->perm); free(t->depth); free(t->is_leaf); free(t->first); free(t->count);
    free(t->skip); free(t->mass); free(t->com3); free(t->width);
    memset(t, 0, sizeof *t);
}

int orc_bh_build(int n, const double *x3, const double *m, int is_float, orc_tree *t) {
    memset(t, 0, sizeof *t);
    t->n = n;
    if (n <= 0) return 0;
    orc_bh_root_box(n, x3, is_float, t->box6);
    keyidx *ki = (keyidx *)malloc(sizeof(keyidx) * (size_t)n);
    int *lcp = (int *)malloc(sizeof(int) * (size_t)n);
    int *start = (int *)malloc(sizeof(int) * (size_t)(n + 1));
    if (!ki || !lcp || !start) { free(ki); free(lcp); free(start); return -3; }
    for (int i = 0; i < n; ++i) {
        ki[i].idx = i;
        if (orc_morton(x3 + 3 * i, t->box6, is_float, &ki[i].code)) { free(ki); free(lcp); free(start); return -1; }
    }
    qsort(ki, (size_t)n, sizeof(keyidx), keyidx_cmp);
    t->code = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    t->perm = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    for (int i = 0; i < n; ++i) { t->code[i] = ki[i].code; t->perm[i] = ki[i].idx; }
    free(ki);
    for (int a = 0; a + 1 < n; ++a) {
        lcp[a] = lcp_digits(t->code[a], t->code[a + 1]);
        if (lcp[a] == 21) {
            const double *p = x3 + 3 * t->perm[a], *q = x3 + 3 * t->perm[a + 1];
            if (roundT(p[0], is_float) == roundT(q[0], is_float) && roundT(p[1], is_float) == roundT(q[1], is_float) &&
                roundT(p[2], is_float) == roundT(q[2], is_float)) {
                free(lcp); free(start); orc_bh_free(t); return -2;
            }
        }
    }
    /* node counts per sorted slot: internal depths (lcp[a-1], min(lcp[a],20)], then one leaf */
    int total = 0;
    for (int a = 0; a < n; ++a) {
        int lm = a > 0 ? lcp[a - 1] : -1, la = a + 1 < n ? lcp[a] : -1;
        int lim = la < 20 ? la : 20;
        int ni = lim - lm > 0 ? lim - lm : 0;
        int leaf = lm < 21;
        start[a] = total;
        total += ni + leaf;
    }
    start[n] = total;
    t->n_nodes = total;
    t->depth = (int8_t *)malloc((size_t)total);
    t->is_leaf = (int8_t *)malloc((size_t)total);
    t->first = (int32_t *)malloc(sizeof(int32_t) * (size_t)total);
    t->count = (int32_t *)malloc(sizeof(int32_t) * (size_t)total);
    t->skip = (int32_t *)malloc(sizeof(int32_t) * (size_t)total);
    t->mass = (double *)malloc(sizeof(double) * (size_t)total);
    t->com3 = (double *)malloc(sizeof(double) * 3 * (size_t)total);
    t->width = (double *)malloc(sizeof(double) * (size_t)total);
    int leaves = 0;
    for (int a = 0; a < n; ++a) {
        int lm = a > 0 ? lcp[a - 1] : -1, la = a + 1 < n ? lcp[a] : -1;
        int lim = la < 20 ? la : 20;
        int node = start[a];
        for (int d = lm + 1; d <= lim; ++d, ++node) {
            int last = range_end(t->code, n, a, d);
            t->depth[node] = (int8_t)d;
            t->is_leaf[node] = 0;
            t->first[node] = a;
            t->count[node] = last - a + 1;
            t->skip[node] = start[last + 1];
        }
        if (lm < 21) {
            int last = la == 21 ? range_end(t->code, n, a, 21) : a;
            int lb = last + 1 < n ? lcp[last] : -1;
            int dl = last > a ? 21 : (lm > lb ? lm : lb) + 1;
            t->depth[node] = (int8_t)dl;
            t->is_leaf[node] = 1;
            t->first[node] = a;
            t->count[node] = last - a + 1;
            t->skip[node] = start[last + 1];
            ++leaves;
        }
    }
    t->n_leaves = leaves;
    /* cell width top.x - btm.x along the node's prefix (set_corners splits, in T) */
    for (int nd = 0; nd < total; ++nd) {
        double lo = t->box6[0], hi = t->box6[3];
        uint64_t c = t->code[t->first[nd]];
        for (int l = 0; l < t->depth[nd]; ++l) {
            double mid = midT(lo, hi, is_float);
            if ((c >> (3 * (20 - l))) & 1u) lo = mid;
            else hi = mid;
        }
        t->width[nd] = subT(hi, lo, is_float);
    }
    /* FP64 mass moments: leaves from their bodies, internal nodes from their children in octant
     * order, deepest first (children are always after their parent in pre-order) */
    for (int nd = total - 1; nd >= 0; --nd) {
        double msum = 0, mx = 0, my = 0, mz = 0;
        if (t->is_leaf[nd]) {
            if (t->count[nd] == 1) {
                int b = t->perm[t->first[nd]];
                t->mass[nd] = roundT(m[b], is_float);
                for (int k = 0; k < 3; ++k) t->com3[3 * nd + k] = roundT(x3[3 * b + k], is_float);
                continue;
            }
            for (int s = t->first[nd]; s < t->first[nd] + t->count[nd]; ++s) {
                int b = t->perm[s];
                double mb = roundT(m[b], is_float);
                msum += mb;
                mx += mb * roundT(x3[3 * b], is_float);
                my += mb * roundT(x3[3 * b + 1], is_float);
                mz += mb * roundT(x3[3 * b + 2], is_float);
            }
        } else {
            for (int c = nd + 1; c < t->skip[nd]; c = t->skip[c]) {
                msum += t->mass[c];
                mx += t->mass[c] * t->com3[3 * c];
                my += t->mass[c] * t->com3[3 * c + 1];
                mz += t->mass[c] * t->com3[3 * c + 2];
            }
        }
        t->mass[nd] = msum;
        t->com3[3 * nd] = mx / msum;
        t->com3[3 * nd + 1] = my / msum;
        t->com3[3 * nd + 2] = mz / msum;
    }
    free(lcp);
    free(start);
    return 0;
}

void orc_bh_acc(const orc_tree *t, const double *x3, const double *m, int is_float, double theta, double eps, double G,
                double *a3, uint32_t *n_inter) {
    int n = t->n;
    /* own leaf of each sorted slot */
    int *own = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int nd = 0; nd < t->n_nodes; ++nd)
        if (t->is_leaf[nd])
            for (int s = t->first[nd]; s < t->first[nd] + t->count[nd]; ++s) own[s] = nd;
    double th2 = theta * theta;
    float th2f = (float)th2;
    ld eps2 = (ld)eps * (ld)eps;
    for (int s = 0; s < n; ++s) {
        int b = t->perm[s];
        double p[3] = {roundT(x3[3 * b], is_float), roundT(x3[3 * b + 1], is_float), roundT(x3[3 * b + 2], is_float)};
        ld ax = 0, ay = 0, az = 0;
        uint32_t cnt = 0;
        int nd = t->n_nodes > 1 ? 1 : t->n_nodes; /* the walk starts at the root's first child */
        while (nd < t->n_nodes) {
            int accept = 0;
            if (t->is_leaf[nd]) {
                if (nd == own[s] && t->count[nd] == 1) { nd = t->skip[nd]; continue; }
                /* a leaf is always a source; a bucket leaf acts body by body */
                for (int q = t->first[nd]; q < t->first[nd] + t->count[nd]; ++q) {
                    int bq = t->perm[q];
                    if (bq == b) continue;
                    ld rx = (ld)roundT(x3[3 * bq], is_float) - (ld)p[0];
                    ld ry = (ld)roundT(x3[3 * bq + 1], is_float) - (ld)p[1];
                    ld rz = (ld)roundT(x3[3 * bq + 2], is_float) - (ld)p[2];
                    ld r2 = rx * rx + ry * ry + rz * rz + eps2;
                    ld f = (ld)G * (ld)roundT(m[bq], is_float) / (r2 * sqrtl(r2));
                    ax += f * rx;
                    ay += f * ry;
                    az += f * rz;
                    ++cnt;
                }
                nd = t->skip[nd];
                continue;
            }
            if (is_float) {
                float cx = (float)t->com3[3 * nd], cy = (float)t->com3[3 * nd + 1], cz = (float)t->com3[3 * nd + 2];
                float dx = cx - (float)p[0], dy = cy - (float)p[1], dz = cz - (float)p[2];
                float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                float w = (float)t->width[nd];
                accept = w * w < th2f * r2;
            } else {
                double dx = t->com3[3 * nd] - p[0], dy = t->com3[3 * nd + 1] - p[1], dz = t->com3[3 * nd + 2] - p[2];
                double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
                double w = t->width[nd];
                accept = w * w < th2 * r2;
            }
            if (accept) {
                ld rx = (ld)t->com3[3 * nd] - (ld)p[0], ry = (ld)t->com3[3 * nd + 1] - (ld)p[1],
                   rz = (ld)t->com3[3 * nd + 2] - (ld)p[2];
                ld r2 = rx * rx + ry * ry + rz * rz + eps2;
                ld f = (ld)G * (ld)t->mass[nd] / (r2 * sqrtl(r2));
                ax += f * rx;
                ay += f * ry;
                az += f * rz;
                ++cnt;
                nd = t->skip[nd];
            } else {
                nd = nd + 1;
            }
        }
        a3[3 * b] = (double)ax;
        a3[3 * b + 1] = (double)ay;
        a3[3 * b + 2] = (double)az;
        if (n_inter) n_inter[b] = cnt;
    }
    free(own);
}

void orc_G_units_into(uint64_t m_first, uint64_t m_second, uint64_t d_first, uint64_t d_second, uint64_t t_first,
                      uint64_t t_second, long double *out) {
    *out = orc_G_units(m_first, m_second, d_first, d_second, t_first, t_second);
}

#include <pthread.h>
#include <time.h>

typedef struct {
    int n;
    const double *m;
    double *x3, *v3, *a3;
    long double dt, G;
    uint64_t steps;
} bench_job;

static void *bench_run(void *p) {
    bench_job *j = (bench_job *)p;
    orc_evolve(ORC_LEAPFROG_KDK, 0, j->n, j->m, NULL, NULL, j->x3, j->v3, j->a3, j->dt, j->steps, &j->G);
    return NULL;
}

int orc_bench_kdk(int n, const double *m, const double *x3, const double *v3, long double dt, uint64_t steps,
                  const long double *G, int threads, long long *wall_ns) {
    if (threads < 1) threads = 1;
    size_t sz = sizeof(double) * 3 * (size_t)n;
    bench_job *jobs = (bench_job *)calloc((size_t)threads, sizeof(bench_job));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; ++t) {
        jobs[t].n = n; jobs[t].m = m; jobs[t].dt = dt; jobs[t].G = *G; jobs[t].steps = steps;
        jobs[t].x3 = (double *)malloc(sz); jobs[t].v3 = (double *)malloc(sz); jobs[t].a3 = (double *)malloc(sz);
        memcpy(jobs[t].x3, x3, sz);
        memcpy(jobs[t].v3, v3, sz);
    }
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (int t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, bench_run, &jobs[t]);
    for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    *wall_ns = (long long)(t1.tv_sec - t0.tv_sec) * 1000000000LL + (t1.tv_nsec - t0.tv_nsec);
    for (int t = 0; t < threads; ++t) { free(jobs[t].x3); free(jobs[t].v3); free(jobs[t].a3); }
    free(jobs);
    free(tid);
    return 0;
}

/* Cell bounds of node nd (set_corners splits of the root box, greg8tree.hpp:81-131, in T). */
static void node_box(const orc_tree *t, int nd, int is_float, double lo[3], double hi[3]) {
    uint64_t c = t->code[t->first[nd]];
    for (int k = 0; k < 3; ++k) {
        lo[k] = t->box6[k];
        hi[k] = t->box6[3 + k];
    }
    for (int l = 0; l < t->depth[nd]; ++l) {
        for (int k = 0; k < 3; ++k) {
            double mid = midT(lo[k], hi[k], is_float);
            if ((c >> (3 * (20 - l) + k)) & 1u) lo[k] = mid;
            else hi[k] = mid;
        }
    }
}

/* bh_s_coll (gregsys.hpp:631-688): for every leaf in DFS order (bh_cube::iterator), the bodies of
 * the leaves whose cells touch its cell (nn_iterator, greg8tree.hpp:615-701: depth-first from the
 * root's children in octant order, descending only into touching cells, closed-interval test of
 * :624-628) that overlap it by radius, resolved exactly as in s_coll.  Leaves shared by bodies with
 * equal 63-bit codes (depth-21 buckets) count their other bodies as touching neighbours. */
int orc_bh_s_coll(const orc_tree *t, const double *m, const double *r, const double *rest, const double *x3,
                  double *v3, int is_float) {
    int n = t->n;
    if (n < 2) return 0;
    int nn = t->n_nodes;
    double *bx = (double *)malloc(sizeof(double) * 6 * (size_t)nn);
    int *own = (int *)malloc(sizeof(int) * (size_t)n);
    coll_cand *c = (coll_cand *)malloc(sizeof(coll_cand) * (size_t)n);
    if (!bx || !own || !c) { free(bx); free(own); free(c); return -3; }
    for (int nd = 0; nd < nn; ++nd) {
        node_box(t, nd, is_float, bx + 6 * nd, bx + 6 * nd + 3);
        if (t->is_leaf[nd])
            for (int q = t->first[nd]; q < t->first[nd] + t->count[nd]; ++q) own[q] = nd;
    }
    for (int a = 0; a < n; ++a) {
        int L = own[a], o = t->perm[a], nc = 0;
        const double *B = bx + 6 * L;
        for (int k = 1; k < nn;) {
            int take = 0;
            if (k == L) {
                take = t->count[k] > 1;
            } else {
                const double *C = bx + 6 * k;
                int touch = !(B[3] < C[0] || B[0] > C[3] || B[4] < C[1] || B[1] > C[4] || B[5] < C[2] || B[2] > C[5]);
                if (!touch) { k = t->skip[k]; continue; }
                if (!t->is_leaf[k]) { ++k; continue; }
                take = 1;
            }
            if (take) {
                for (int q = t->first[k]; q < t->first[k] + t->count[k]; ++q) {
                    if (q == a) continue;
                    int i = t->perm[q];
                    double rad_dist = r[o] + r[i];
                    double ux = x3[3 * i] - x3[3 * o], uy = x3[3 * i + 1] - x3[3 * o + 1],
                           uz = x3[3 * i + 2] - x3[3 * o + 2];
                    ld dist = mag_ld(ux, uy, uz);
                    ux = (double)((ld)ux / dist);
                    uy = (double)((ld)uy / dist);
                    uz = (double)((ld)uz / dist);
                    if ((ld)rad_dist > dist) {
                        double mox = m[o] * v3[3 * o], moy = m[o] * v3[3 * o + 1], moz = m[o] * v3[3 * o + 2];
                        double mix = m[i] * v3[3 * i], miy = m[i] * v3[3 * i + 1], miz = m[i] * v3[3 * i + 2];
                        c[nc].inner = q;
                        c[nc].body = i;
                        c[nc].dist = dist;
                        c[nc].mom_o = mox * ux + moy * uy + moz * uz;
                        c[nc].mom_i = mix * ux + miy * uy + miz * uz;
                        c[nc].ux = ux;
                        c[nc].uy = uy;
                        c[nc].uz = uz;
                        ++nc;
                    }
                }
            }
            k = t->skip[k];
        }
        if (nc) resolve_group(o, c, nc, m, rest, v3);
    }
    free(bx);
    free(own);
    free(c);
    return 0;
}
