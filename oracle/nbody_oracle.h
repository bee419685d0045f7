/* CPU restatement of the gtd:: N-body force-and-step path (GregW10/GregPackagesCPP), in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle the CUDA path is checked against.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the product never does.
 *
 * Every function restates the reference's arithmetic step for step, in the same types
 * (double storage, long double intermediates where the reference promotes to long double) and
 * the same loop order, so that with FMA contraction off it agrees with the reference headers bit
 * for bit (pinned by tests/test_oracle_pins.py against oracle/_ref/libgtdref.so and the fixtures
 * in tests/golden/).  Arrays are SoA-of-triples: x3[3*i+k].
 */
#ifndef GTD_NBODY_ORACLE_H
#define GTD_NBODY_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Integration-method flags, gregsys.hpp:156-165. */
enum { ORC_EULER = 2, ORC_MODIFIED_EULER = 4, ORC_MIDPOINT = 8, ORC_LEAPFROG_KDK = 16, ORC_LEAPFROG_DKD = 32 };

/* G from a units format "Ma:b,Dc:d,Tx:y" already split into its six integers (gregsys.hpp:245-282). */
long double orc_G_units(uint64_t m_first, uint64_t m_second, uint64_t d_first, uint64_t d_second, uint64_t t_first,
                        uint64_t t_second);

/* Same, written through a pointer so callers without a long double type (ctypes) keep all bits. */
void orc_G_units_into(uint64_t m_first, uint64_t m_second, uint64_t d_first, uint64_t d_second, uint64_t t_first,
                      uint64_t t_second, long double *out);

/* Direct-summation accelerations at the given positions, gregsys.hpp:439-476 / 352-357.
 * a3 is zeroed first (MEM_LOOP, gregsys.hpp:107-122). */
void orc_direct_acc(int n, const double *m, const double *x3, const long double *G, double *a3);

/* orc_direct_acc for the bodies rows[0..nrows) only (bit for bit the same values), with
 * gross[q] = sum_j G m_j / r^2 for each row when gross is not NULL; rows are split over
 * `threads` pthreads.  a3 and gross are indexed by position in rows. */
void orc_direct_acc_rows(int n, const double *m, const double *x3, const long double *G, const int32_t *rows,
                         int nrows, double *a3, double *gross, int threads);

/* gtd::system::evolve for the direct-summation methods (gregsys.hpp:2593-3071).  State is updated
 * in place; a3 holds the final accelerations as the reference leaves them.  coll is 0 or 3
 * (s_coll restitution, gregsys.hpp:690-914).  Returns 0, or -1 for an unsupported method. */
int orc_evolve(int method, int coll, int n, const double *m, const double *r, const double *rest, double *x3,
               double *v3, double *a3, long double dt, uint64_t steps, const long double *G);

/* CPU throughput sample: `threads` independent copies of the system, each running
 * orc_evolve(leapfrog_kdk) on its own pthread; *wall_ns covers the evolve calls only. */
int orc_bench_kdk(int n, const double *m, const double *x3, const double *v3, long double dt, uint64_t steps,
                  const long double *G, int threads, long long *wall_ns);

/* One pass of s_coll (non-merging branch), gregsys.hpp:690-914, on the current state. */
void orc_s_coll(int n, const double *m, const double *r, const double *rest, const double *x3, double *v3);

/* Total KE and PE as calc_energy computes them (gregsys.hpp:608-630, gregbod.hpp:917-920). */
void orc_energy(int n, const double *m, const double *x3, const double *v3, const long double *G, double *ke,
                double *pe);

/* body::operator+= (gregbod.hpp:1066-1082): merge body b into body a.  Each body is
 * {m, r, rest, x, y, z, vx, vy, vz, ax, ay, az}; the result is written over a. */
void orc_merge_pair(double *a, const double *b);

/* Add-time overlap merge with the scan order of check_overlap (gregsys.hpp:307-342), as that
 * routine intends it: after a merge the merged body is re-checked against every body from index
 * 0.  Bodies are rows of 12 doubles as in orc_merge_pair; returns the surviving count (rows are
 * compacted in place, order preserved). */
int orc_merge_overlapping(int n, double *bodies12);

/* ---- Barnes-Hut: host rebuild of the linear octree ------------------------------------------ */

/* Root box exactly as bh_tree::find_min_max computes it (greg8tree.hpp:1012-1047), in T=double
 * (is_float=0) or T=float (is_float=1, positions rounded to float first).  box6 = btm xyz, top xyz. */
void orc_bh_root_box(int n, const double *x3, int is_float, double *box6);

/* 63-bit Morton code of one position: 21 levels of the reference's octant descent
 * (set_corners greg8tree.hpp:81-131, dispatch :146-210): split at (btm+top)/2 computed in T,
 * bit set when coordinate >= split, octant bit0=x bit1=y bit2=z.  Returns 0, or -1 when the
 * position is outside [btm, top) (the reference throws invalid_body_placement). */
int orc_morton(const double *pos3, const double *box6, int is_float, uint64_t *code);

typedef struct {
    int n, n_nodes, n_leaves;
    uint64_t *code;    /* [n] sorted codes */
    int32_t *perm;     /* [n] sorted slot -> original body index */
    int8_t *depth;     /* [n_nodes] pre-order */
    int8_t *is_leaf;   /* [n_nodes] */
    int32_t *first;    /* [n_nodes] first sorted slot */
    int32_t *count;    /* [n_nodes] bodies in the node */
    int32_t *skip;     /* [n_nodes] pre-order index after the node's subtree */
    double *mass;      /* [n_nodes] */
    double *com3;      /* [3*n_nodes] */
    double *width;     /* [n_nodes] top.x - btm.x of the cell, in T */
    double box6[6];
} orc_tree;

/* Builds the octree over n bodies: root box, Morton codes, a stable sort by code, node emission
 * in DFS pre-order (children in octant order = ascending code), skip links, FP64 mass moments
 * summed child by child in octant order.  Returns 0, -1 (body outside box), -2 (two bodies at
 * exactly the same position: indistinguishable_bodies, greg8tree.hpp:171-172) or -3 (no memory). */
int orc_bh_build(int n, const double *x3, const double *m, int is_float, orc_tree *t);
void orc_bh_free(orc_tree *t);

/* Barnes-Hut accelerations with the reference walk order and opening rule (cell_iterator,
 * greg8tree.hpp:702-833): start at the root's children, accept leaves (except the body's own)
 * and cells with width/|x - com| < theta, else descend; force G*M/(r^2+eps^2)^{3/2} * r
 * (bh_acc gregsys.hpp:371-375, accumulated).  is_float selects the FP32 arithmetic the GPU uses
 * for T=float (criterion w^2 < theta^2 r^2 and the force in float, sums in float); otherwise FP64
 * with the same criterion.  a3/n_inter are indexed by original body index. */
void orc_bh_acc(const orc_tree *t, const double *x3, const double *m, int is_float, double theta, double eps, double G,
                double *a3, uint32_t *n_inter);

/* bh_s_coll (gregsys.hpp:631-688) over tree t built at x3: restitution impulses between each leaf's
 * body and the overlapping bodies of the leaves whose cells touch its cell (nn_iterator,
 * greg8tree.hpp:615-701), leaves in DFS order; v3 is updated in place.  Returns 0 or -3. */
int orc_bh_s_coll(const orc_tree *t, const double *m, const double *r, const double *rest, const double *x3,
                  double *v3, int is_float);

#ifdef __cplusplus
}
#endif
#endif
