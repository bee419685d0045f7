/* gtd_b200.h - C ABI of the B200 force-and-step engine behind the gtd:: N-body API.
 *
 * This is the boundary the drop-in C++ headers (include/gtd/*.hpp) call.  It takes plain pointers
 * and sizes only (no CUDA, torch or C++ types), returns an int status (0 = GTD_OK) and keeps a
 * thread-local message for gtd_last_error().  Every call is re-entrant per handle: a handle owns
 * its device buffers and one CUDA stream, and no call touches global mutable state.
 *
 * Each entry point names the reference interface it replaces (file:line in
 * GregW10/GregPackagesCPP).  Host arrays of vectors are triples: x3[3*i+k].  long double in the
 * reference API is carried as double across this ABI (there is no long double on the device).
 */
#ifndef GTD_B200_H
#define GTD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GTD_ABI_VERSION 1

#if defined(__GNUC__)
#define GTD_API __attribute__((visibility("default")))
#else
#define GTD_API
#endif

/* ---- status codes; the C++ wrapper maps them onto the reference's exception types ---------- */
#define GTD_OK 0
#define GTD_ERR_INVALID_ARGUMENT 1        /* std::invalid_argument (gregsys.hpp:1403, 1649, ...) */
#define GTD_ERR_CUDA 2                    /* a CUDA runtime call failed */
#define GTD_ERR_OUT_OF_MEMORY 3
#define GTD_ERR_OVERLAPPING_BODIES 4      /* gtd::overlapping_bodies_error (gregbod.hpp:24, gregsys.hpp:322) */
#define GTD_ERR_INVALID_BODY_PLACEMENT 5  /* gtd::invalid_body_placement (greg8tree.hpp:17, 140, 206) */
#define GTD_ERR_INDISTINGUISHABLE 6       /* gtd::indistinguishable_bodies (greg8tree.hpp:32, 171-172) */
#define GTD_ERR_NONFINITE 7               /* a NaN/Inf appeared in the device state */
#define GTD_ERR_TIMEOUT 8                 /* a bounded device-side wait expired */
#define GTD_ERR_TWO_BODY 9                /* gtd::two_body_error (gregbod.hpp:62, gregsys.hpp:2627-2629) */
#define GTD_ERR_NO_DEVICE 10
#define GTD_ERR_CAPACITY 11               /* a size beyond what the entry point supports */
#define GTD_ERR_UNSUPPORTED 12            /* a method the reference leaves empty (rk4, rk3_8, ...) */
#define GTD_ERR_NSYS_LOAD 13              /* gtd::nsys_load_error (gregsys.hpp:125-129) */
#define GTD_ERR_NSYS_FORMAT 14            /* gtd::nsys_format_error (gregsys.hpp:130-134) */
#define GTD_ERR_CALLBACK 15               /* an evolve callback (host step hook or device hook) failed */

/* ---- integration-method flags, identical to gtd::system's (gregsys.hpp:156-165) ------------- */
#define GTD_TWO_BODY 1
#define GTD_EULER 2
#define GTD_MODIFIED_EULER 4
#define GTD_MIDPOINT 8
#define GTD_LEAPFROG_KDK 16
#define GTD_LEAPFROG_DKD 32
#define GTD_RK4 64
#define GTD_RK3_8 128
#define GTD_BARNES_HUT 65536

/* ---- collision modes (gtd::system template parameter `collisions`, gregsys.hpp:166-168) ----- */
#define GTD_NO_COLL 0
#define GTD_OVERLAP_COLL 3  /* s_coll restitution impulses, gregsys.hpp:690-914 */
#define GTD_MERGE_COLL 4    /* overlap merges with momentum conservation (body::operator+=) */

/* ---- arithmetic of the pairwise force ---------------------------------------------------- */
#define GTD_PREC_F64 0   /* FP64 everywhere */
#define GTD_PREC_MIXED 1 /* FP32 pair forces and per-tile sums, FP64 Kahan sums across tiles, FP64 state */

typedef struct gtd_system gtd_system;

GTD_API const char *gtd_last_error(void);
/* *accepted = whether evolve() accepts the method value, by gtd::system::check_option
 * (gregsys.hpp:1406-1411; its word tests let nearly every value through).  Host-only. */
GTD_API int gtd_check_option(int option, int *accepted);
GTD_API int gtd_abi_version(void);
GTD_API int gtd_device_count(int *count);

/* A device-resident N-body system.  Replaces the storage of gtd::system (std::vector<body>,
 * gregsys.hpp:179) for the duration of evolve(): the host vector stays authoritative between
 * calls, the handle holds its SoA copy on the device. */
GTD_API int gtd_system_create(gtd_system **out, int device, int precision);
GTD_API int gtd_system_destroy(gtd_system *sys);

/* Scalars of gtd::system: G (gregsys.hpp:171, 245-282), dt/half_dt (:202-203, set_timestep
 * :1642-1651), iterations (:205, set_iterations :1636-1641), softening (:200-201, set_softening
 * :1660-1666; used by Barnes-Hut only, as in the reference), bh_theta (:212, :1667-1672). */
GTD_API int gtd_system_set_params(gtd_system *sys, double G, double dt, uint64_t iterations, double softening,
                          double bh_theta);
/* Collision handling (the `collisions` / `mergeOverlappingBodies` template parameters,
 * gregsys.hpp:135-137): GTD_NO_COLL, GTD_OVERLAP_COLL or GTD_MERGE_COLL. */
GTD_API int gtd_system_set_collisions(gtd_system *sys, int mode);

/* The add-time overlap check of the system constructors (check_overlap, gregsys.hpp:307-342),
 * scanning in upload order.  merge == 0: returns GTD_ERR_OVERLAPPING_BODIES naming the first
 * overlapping pair found (pair[0..1] = their upload indices, pair may be NULL), as the reference
 * throws overlapping_bodies_error.  merge != 0: merges overlapping bodies with body::operator+=
 * (gregbod.hpp:1066-1082), re-checking a merged body against every body from index 0 (the
 * routine's stated intent: after its first merge the reference loop's counter and pointer fall
 * out of step, gregsys.hpp:329-335, and it then deletes bodies it never merged). */
GTD_API int gtd_system_check_overlap(gtd_system *sys, int merge, int32_t *pair);

/* Gather: the AoS gtd::body fields (gregbod.hpp:906-916) as SoA.  r, rest, v3 may be NULL
 * (zero radius, restitution 1, zero velocity).  n == 0 is an empty system. */
GTD_API int gtd_system_upload(gtd_system *sys, int64_t n, const double *m, const double *r, const double *rest,
                      const double *x3, const double *v3);
/* Scatter back.  *n receives the body count (it shrinks after merges); any output may be NULL.
 * Bodies keep their upload order; merged-away bodies are removed, survivors keep their order. */
GTD_API int gtd_system_download(gtd_system *sys, int64_t *n, double *m, double *r, double *rest, double *x3, double *v3,
                        double *a3);
GTD_API int gtd_system_num_bodies(const gtd_system *sys, int64_t *n);
/* Upload indices of the current bodies in download order (ascending): after merges, which of the
 * uploaded bodies survived (their state holds the merged result). */
GTD_API int gtd_system_survivors(gtd_system *sys, int64_t *upload_index);

/* ---- trajectory frames (memFreq) -------------------------------------------------------------
 * Replaces the recording of gtd::system<..., memFreq, ...> (body trajectories gregbod.hpp:304-320,
 * per-body and total energies gregsys.hpp:219-227, 343-363, 439-476, 608-630).  With every != 0,
 * each direct-summation evolve (gtd_system_evolve, gtd_system_evolve_begin/_steps with host
 * callbacks, gtd_system_evolve_callbacks with device callbacks) records a frame at its start and
 * after every every-th step (after that step's for_all_bods and collision pass, before
 * for_each_bod: FUNC_TEMPL_SELECT, gregsys.hpp:16-106); a frame holds, per body in download order, x, y, z, vx, vy, vz,
 * ke = 0.5 m |v| |v| and pe = 0.5 sum_{j != i} -G m_i m_j / r_ij, computed on the device in FP64.
 * Each evolve starts a new recording; Barnes-Hut evolves record nothing (as the reference).  Which
 * of these values the reference keeps depends on the method and collision mode; the C++ and Python
 * front ends apply its rules.  Merging collisions with recording return GTD_ERR_UNSUPPORTED.
 * gtd_system_recording: frame count, bodies per frame, the step index of each frame (states,
 * [frames]) and the frames (frame8, [frames][n][8]); pass NULL arrays to query the counts. */
GTD_API int gtd_system_set_recording(gtd_system *sys, uint64_t every);
GTD_API int gtd_system_recording(gtd_system *sys, int64_t *frames, int64_t *n, int64_t *states, double *frame8);

/* ---- .nsys snapshots -------------------------------------------------------------------------
 * The reference's on-disk format (header gregsys.hpp:1444-1466, chunk :1467-1477): a 96-byte
 * header, then per body { char r_coeff[16]; M mass; R radius; T x, y, z, vx, vy, vz; } with natural
 * alignment, then zero padding to a multiple of 4 bytes.  m_size/r_size/t_size are sizeof(M),
 * sizeof(R), sizeof(T) of the caller's floating-point types: 4 (float), 8 (double) or 16 (x86-64
 * long double, 80-bit extended); integral M/R/T return GTD_ERR_UNSUPPORTED.  The chunks are packed
 * and unpacked on the device; the file holds the bodies in download order.
 * gtd_nsys_chunk_size: sizeof(nsys_chunk) for those sizes. */
GTD_API int gtd_nsys_chunk_size(int m_size, int r_size, int t_size, int *chunk_bytes);
/* Replaces system::to_nsys (gregsys.hpp:3214-3258).  time_elapsed and dt are stored as long
 * double, g_vals are the six unsigned numbers of the units format (m_num, m_denom, d_num, d_denom,
 * t_num, t_denom).  *bytes_written receives the file size, or 0 (with GTD_OK) when path is NULL or
 * the file cannot be opened, as the reference returns 0. */
GTD_API int gtd_system_to_nsys(gtd_system *sys, const char *path, double time_elapsed, double dt,
                               const uint64_t *g_vals, int m_size, int r_size, int t_size, int64_t *bytes_written);
/* The same, returning once the packing and its device-to-host copy are enqueued on the handle's
 * stream: a host thread writes the file when the copy is done, so the next evolve can run meanwhile
 * (the snapshot is of the state at the call).  Two writes can be in flight per handle; a third
 * call waits for the oldest.  gtd_system_nsys_wait waits for every pending write and returns the
 * first failure, or GTD_OK and the size of the most recent file. */
GTD_API int gtd_system_to_nsys_async(gtd_system *sys, const char *path, double time_elapsed, double dt,
                                     const uint64_t *g_vals, int m_size, int r_size, int t_size);
GTD_API int gtd_system_nsys_wait(gtd_system *sys, int64_t *bytes_written);
/* Replaces the system(const char *nsys_path, ...) constructor's load_from_nsys (gregsys.hpp:947-1400):
 * the same checks in the same order with the same messages (GTD_ERR_NSYS_LOAD / GTD_ERR_NSYS_FORMAT
 * for nsys_load_error / nsys_format_error; GTD_ERR_INVALID_ARGUMENT for a non-positive time-step),
 * then the bodies replace the handle's (upload order = file order).  check_nan_inf scans every field
 * (on the device) and names the first offending chunk and field.  Long doubles are rounded to
 * double.  Outputs (any may be NULL): the stored time and time-step, the six units numbers, and G
 * computed from them as the reference does (gregsys.hpp:1281-1284). */
GTD_API int gtd_system_load_nsys(gtd_system *sys, const char *path, int check_nan_inf, int m_size, int r_size,
                                 int t_size, double *time_elapsed, double *dt, uint64_t *g_vals, double *G);

/* gtd::system::evolve(method) with no callbacks (gregsys.hpp:2593-3071): `iterations` steps of
 * the method on the device, one upload/download around it done by the caller.  *elapsed_ns is
 * the device time of the call (CUDA events), like the reference's returned duration.  Returns
 * GTD_ERR_UNSUPPORTED for the methods the reference leaves empty. */
GTD_API int gtd_system_evolve(gtd_system *sys, int method, int64_t *elapsed_ns);

/* The same loop split for evolve() with callbacks: begin computes what the method needs before
 * its first step (the initial acceleration of leapfrog KDK, gregsys.hpp:2947), steps advances k
 * steps and leaves the state synchronised (positions and velocities at the same time). */
GTD_API int gtd_system_evolve_begin(gtd_system *sys, int method);
GTD_API int gtd_system_evolve_steps(gtd_system *sys, uint64_t k);

/* Accelerations at the current positions: direct summation (calc_acc_and_e, gregsys.hpp:439-476)
 * or, with GTD_BARNES_HUT in `method`, the Barnes-Hut walk.  a3 may be NULL (kept on device). */
GTD_API int gtd_system_accelerations(gtd_system *sys, int method, double *a3);

/* FP64 diagnostics: kinetic and potential energy (calc_energy gregsys.hpp:608-630), total
 * momentum (sum of body::momentum, gregbod.hpp:595-597) and centre of mass (gregbod.hpp:1096-1106).
 * Any output may be NULL. */
GTD_API int gtd_system_energy(gtd_system *sys, double *ke, double *pe, double *p3, double *com3);

/* ---- evolve callbacks -------------------------------------------------------------------------
 * gtd::system::evolve(method, continue_ev_if, for_each_bod, for_all_bods) (gregsys.hpp:2593-3071)
 * calls continue_ev_if() before every step (without it: `iterations` steps), for_all_bods(bodies)
 * after the step's update and before the collision pass (FUNC_TEMPL_SELECT, gregsys.hpp:16-106;
 * leapfrog_kdk_acc_e_and_step, :528-539), and for_each_bod(body) on every body after that.  The
 * Barnes-Hut branch calls none of them (gregsys.hpp:2893-2945).  Two ways to run them here. */

/* Host callbacks.  `hook` runs on the host inside every step of gtd_system_evolve_steps, at
 * for_all_bods' place (the state is synchronised then); it may read and write the bodies with
 * gtd_system_download / gtd_system_update_bodies.  A nonzero return ends the evolve with that
 * status.  NULL removes the hook. */
typedef int (*gtd_step_hook)(void *user);
GTD_API int gtd_system_set_step_hook(gtd_system *sys, gtd_step_hook hook, void *user);
/* Overwrites the given arrays (any may be NULL) of the live bodies, in download order, without
 * touching the accelerations or the evolve in progress (what a callback's writes to the reference's
 * body vector do).  The body count cannot change here. */
GTD_API int gtd_system_update_bodies(gtd_system *sys, const double *m, const double *r, const double *rest,
                                     const double *x3, const double *v3);

/* Device callbacks: GPU work that replaces a host callback, so the bodies never leave the device.
 * A hook ENQUEUES work on `stream` and returns; it must not synchronise, allocate or read the
 * bodies on the host.  gtd_system_evolve_callbacks records each hook's work once per step shape
 * into a CUDA graph and replays it every step, so the work must be the same every step (state
 * that changes belongs in device memory).  The arrays are in device order (upload order whenever
 * collisions are on). */
typedef struct gtd_device_bodies {
    int64_t n;
    double *pos_mass;              /* [n][4]: x, y, z, m */
    double *vel;                   /* [n][4]: vx, vy, vz, unused */
    double *acc;                   /* [n][4]: ax, ay, az, unused */
    double *radius;                /* [n] */
    double *rest;                  /* [n] coefficient of restitution (body::rest_c) */
    const int32_t *upload_index;   /* [n] upload index of the body in each slot */
    unsigned int *cont;            /* a continue_ev_if hook writes its verdict here: nonzero = step */
    void *stream;                  /* cudaStream_t of the handle */
} gtd_device_bodies;
typedef int (*gtd_device_hook)(void *user, const gtd_device_bodies *bodies);
/* Sets all three callbacks to user hooks (NULL: none), replacing the built-ins below. */
GTD_API int gtd_system_set_device_callbacks(gtd_system *sys, gtd_device_hook continue_ev_if, void *cont_user,
                                            gtd_device_hook for_each_bod, void *each_user,
                                            gtd_device_hook for_all_bods, void *all_user);
/* Built-in for_all_bods: random_comet's (gregsys.hpp:1965-1984).  Every step the carried centre
 * becomes (centre + sum of positions) / N -- or (centre + sum of m x) / M with mass_weighted, the
 * GREGSYS_MERGERS form -- with N and M the body count and total mass at this call, then every body
 * takes rest = max_cor - (max_cor - min_cor) d^n_exp / (d^n_exp + scale_factor), d its distance
 * to the centre.  com is the starting centre. */
GTD_API int gtd_system_set_rest_from_com(gtd_system *sys, double min_cor, double max_cor, double scale_factor,
                                         double n_exp, const double com[3], int mass_weighted);
/* The carried centre of the built-in for_all_bods (random_comet reads it after evolve). */
GTD_API int gtd_system_rest_from_com_centre(gtd_system *sys, double com[3]);
/* Built-in continue_ev_if: random_comet's (gregsys.hpp:1936-1963): true while some body has
 * rest < min_max_cor (resetting a counter), then true for probing_iters more evaluations. */
GTD_API int gtd_system_set_continue_while_rest_below(gtd_system *sys, double min_max_cor, uint64_t probing_iters);
/* evolve(method, callbacks) with the device callbacks set above; the predicate is evaluated on the
 * device and the loop runs as CUDA-graph chunks whose conditional nodes stop at the first false
 * verdict, so the host waits once per chunk, not per step.  max_steps > 0 stops after that many
 * steps without evaluating the predicate again (a guard for predicates that never turn false).
 * *steps_taken: steps run; *elapsed_ns: device time. */
GTD_API int gtd_system_evolve_callbacks(gtd_system *sys, int method, uint64_t max_steps, uint64_t *steps_taken,
                                        int64_t *elapsed_ns);
/* How the last gtd_system_evolve_callbacks ran: host waits for the device (one per graph chunk, or
 * one per step in the eager form used with merging collisions, the mixed path's periodic reorder or
 * force timing) and whether the graph form ran. */
GTD_API int gtd_system_callback_stats(const gtd_system *sys, uint64_t *host_waits, int *graph_loop);

/* ---- instrumentation (no counterpart in the reference, which only returns evolve()'s wall time,
 * gregsys.hpp:2608-2625, 3061-3070) ------------------------------------------------------------ */

/* Number of kernels this handle has launched since creation. */
GTD_API int gtd_system_launch_count(const gtd_system *sys, uint64_t *count);
/* The cudaStream_t the handle launches on, so a caller can record its own events on it. */
GTD_API int gtd_system_stream(const gtd_system *sys, void **stream);
/* enable != 0: bracket every force-kernel launch with CUDA events on the handle's stream and
 * accumulate their durations; gtd_system_force_timing reads (and with reset != 0 clears) the total
 * milliseconds and launch count. */
GTD_API int gtd_system_time_force_kernels(gtd_system *sys, int enable);
GTD_API int gtd_system_force_timing(gtd_system *sys, double *total_ms, uint64_t *launches, int reset);
/* Force-kernel variants (i-bodies per thread; for GTD_PREC_MIXED also the j-bodies summed in FP32
 * between FP64 folds).  gtd_system_autotune_direct times every variant on the handle's current
 * bodies (a warm-up and `reps` timed force launches each, median), keeps the fastest for the handle
 * and remembers it for the process: every handle without a pinned variant on the same device, with
 * the same precision and an N of the same bit length, then uses it (untuned: a fixed choice by
 * precision and N).  It leaves the bodies untouched apart from their order on the device.
 * gtd_system_set_direct_variant pins a variant for the handle; variant < 0 unpins it. */
GTD_API int gtd_direct_variant_count(int precision, int *count);
GTD_API int gtd_direct_variant_info(int precision, int variant, int *i_per_thread, int *fold);
GTD_API int gtd_system_set_direct_variant(gtd_system *sys, int variant);
GTD_API int gtd_system_autotune_direct(gtd_system *sys, int reps, int *best, double *best_ms);
/* Accuracy control of the mixed-precision direct sum (no counterpart in the reference, whose
 * evolve is FP64 throughout; it bounds the error of the FP32 form of cumulative_acc,
 * gregsys.hpp:352-357).  The FP32 pair terms use coordinates relative to a per-row centre; a
 * pair closer than 2|X_i|/(k - 1) to body i (X_i its offset from that centre) would lose more
 * than k 2^-24 of its relative accuracy to their rounding, so the j-range holding it is summed
 * again from hi/lo coordinate splits.  Default k = 8; k <= 1 turns the check off. */
GTD_API int gtd_system_set_mixed_near_factor(gtd_system *sys, double k);
/* The split of the handle's direct-sum force (no counterpart in the reference): the work units of
 * one force evaluation (mixed: (row, segment) units taken from a work queue; FP64: (row, tile)
 * pairs) and the bytes of partial sums they write. */
GTD_API int gtd_system_direct_plan_info(gtd_system *sys, int64_t *units, int64_t *partial_bytes);
/* Measured throughput of a dependent-FMA microkernel on `device` (all SMs): precision
 * GTD_PREC_MIXED gives FP32 FFMA FLOP/s, GTD_PREC_F64 gives FP64 DFMA FLOP/s (2 flops per FMA). */
GTD_API int gtd_measure_fma_peak(int device, int precision, double *flops_per_s);

/* ---- Barnes-Hut octree (greg8tree.hpp) ----------------------------------------------------- */

/* Rebuilds the octree from the current positions: root box as bh_tree::find_min_max
 * (greg8tree.hpp:1012-1047), 63-bit Morton codes along the reference's octant splits
 * (set_corners :81-131, dispatch :146-210; depth 21), radix sort, linear octree in DFS pre-order
 * with skip links, FP64 centres of mass (calc_com :213-281).  tree_float = 1 builds in T=float
 * (positions rounded to float), 0 in T=double.  Replaces bh_tree::add_bodies + calc_com. */
GTD_API int gtd_bh_build(gtd_system *sys, int tree_float);
/* Tree geometry for evolve(leapfrog_kdk | barnes_hut): 1 = T=float (the default), 0 = T=double. */
GTD_API int gtd_bh_set_tree_float(gtd_system *sys, int tree_float);
/* Float-tree walk that replaces the cell_iterator loop (greg8tree.hpp:702-833): -1 = default (2),
 * 0 = per-lane walk with position/mass and links in separate arrays, 1 = per-lane walk with both
 * halves of a node in one 32-byte sector (0 and 1 give the same interaction lists and bits), 2 =
 * list walk: the same interaction list per body, classified for a warp's 32 bodies at once and
 * summed in another order.  The next gtd_bh_build applies it. */
GTD_API int gtd_bh_set_walk_variant(gtd_system *sys, int variant);
GTD_API int gtd_bh_tree_size(gtd_system *sys, int64_t *n_nodes, int64_t *n_leaves, double *box6);
/* Copies the tree out (any pointer may be NULL): sorted codes and slot->body permutation [n],
 * then per node in pre-order: depth, leaf flag, first slot, body count, skip, mass, com, width.
 * Replaces walking bh_tree with its iterators (greg8tree.hpp:502-614, 1080-1085). */
GTD_API int gtd_bh_tree_download(gtd_system *sys, uint64_t *codes, int32_t *perm, int8_t *depth, int8_t *is_leaf,
                         int32_t *first, int32_t *count, int32_t *skip, double *mass, double *com3, double *width);
/* Barnes-Hut accelerations of every body with the reference walk (cell_iterator,
 * greg8tree.hpp:702-833) and bh_acc's force (gregsys.hpp:371-375, accumulated), on the tree of the
 * last gtd_bh_build.  n_inter (per body, optional) counts accepted cells and leaves. */
GTD_API int gtd_bh_accelerations(gtd_system *sys, double *a3, uint32_t *n_inter);

/* ---- direct-sum accelerations that allocate nothing ------------------------------------------
 * No counterpart in the reference.  For callers that cannot let a library call cudaMalloc: a
 * process whose device memory is already owned by a pool (a PyTorch caching allocator, a code that
 * reserves everything at start-up) may have none to give, and cudaMalloc/cudaFree synchronise the
 * device, stalling other streams inside a running loop.  The caller passes device buffers: pm4 =
 * n x 4 doubles (x, y, z, m), 16-byte aligned; acc3 = n x 3 doubles, written with the accelerations
 * sum_j G m_j (x_j - x_i) / |x_j - x_i|^3 (as gtd_system_accelerations).  The only scratch, the
 * force kernel's partial sums, lives in a fixed 8 MiB device array compiled into the library (every
 * GPU that loads the library holds it until the process exits); n is limited to 65536 and larger n
 * is rejected with GTD_ERR_CAPACITY.  The first call on a device looks up that array's address
 * (cudaGetSymbolAddress), so make the first call on each device before any stream capture.  All
 * calls share the array: calls whose work overlaps on the GPU (different streams, or different
 * host threads) race on it and must be serialised by the caller.  Nothing in it needs clearing
 * between calls (every partial sum read is written first by the same call).  The array's address
 * is kept per device after the first call; cudaDeviceReset discards the array, so the entry point
 * must not be used after a device reset.  pm4 and acc3 that are not device (or managed) memory of
 * the current device are rejected with GTD_ERR_INVALID_ARGUMENT before anything is launched.
 * GTD_PREC_MIXED sums the bodies in the order given (gtd_system reorders them spatially first);
 * its test bar against the FP64 result is 1e-6 RMS relative.  stream: a cudaStream_t or NULL; the
 * call returns after enqueueing. */
GTD_API int gtd_direct_accelerations_noalloc(int64_t n, const double *pm4, double G, int precision, double *acc3,
                                             void *stream);

/* ---- batched ensemble of independent systems ------------------------------------------------
 * Replaces the drivers' pattern of one gtd::system per std::thread (bdsim.cpp:82-113): every
 * system advances by leapfrog KDK (gregsys.hpp:2946-2990) with FP64 state and FP32 pair forces,
 * one persistent launch per step for all systems, the step loop replayed as a CUDA graph, and
 * overlap merges with body::operator+= in check_overlap's scan order (gregsys.hpp:307-342). */
typedef struct gtd_ensemble gtd_ensemble;

GTD_API int gtd_ensemble_create(gtd_ensemble **out, int device);
GTD_API int gtd_ensemble_destroy(gtd_ensemble *ens);
/* G, dt (as gtd_system_set_params) and merge != 0 to merge overlapping bodies after each step. */
GTD_API int gtd_ensemble_set_params(gtd_ensemble *ens, double G, double dt, int merge);
/* System s owns bodies [offsets[s], offsets[s+1]) (at most 8192 per system); r, rest, v3 may be
 * NULL.  The first evolve computes the initial accelerations (and add-time merges). */
GTD_API int gtd_ensemble_upload(gtd_ensemble *ens, int64_t n_systems, const int64_t *offsets, const double *m,
                                const double *r, const double *rest, const double *x3, const double *v3);
/* Advances every system `steps` KDK steps; *elapsed_ns is the device time (CUDA events). */
GTD_API int gtd_ensemble_evolve(gtd_ensemble *ens, uint64_t steps, int64_t *elapsed_ns);
/* Live bodies per system (counts[n_systems]), merges so far, kernel launches so far. */
GTD_API int gtd_ensemble_counts(gtd_ensemble *ens, int64_t *counts, uint64_t *merges, uint64_t *launches);
/* State at the upload offsets: system s's survivors occupy the first counts[s] rows of its range,
 * in upload order. */
GTD_API int gtd_ensemble_download(gtd_ensemble *ens, double *m, double *r, double *rest, double *x3, double *v3,
                                  double *a3);
/* CTA size of the step kernel (64, 128, 256 or 512) and bodies per thread in its force loop (1, or
 * 2 or 4 with at most 256 threads), or let the autotuner time (128|256|512, 1), (128|256, 2) and
 * (128|256, 4) on the current state (restored afterwards) and keep the fastest; gtd_ensemble_config
 * reads the choice. */
GTD_API int gtd_ensemble_set_threads(gtd_ensemble *ens, int threads);
GTD_API int gtd_ensemble_set_bodies_per_thread(gtd_ensemble *ens, int bodies);
GTD_API int gtd_ensemble_config(const gtd_ensemble *ens, int *threads, int *bodies_per_thread);
GTD_API int gtd_ensemble_autotune(gtd_ensemble *ens, int *best_threads, double *best_ms);

/* ---- adjoint of the FP64 leapfrog KDK evolve (no counterpart in the reference) ---------------
 * Gradients of a loss on the final state of evolve(leapfrog_kdk) (gregsys.hpp:2946-2990) with
 * respect to the initial positions, velocities and masses, by a hand-written reverse sweep with
 * checkpoints every `checkpoint_every` steps and recomputation in between.  All arrays are DEVICE
 * pointers (n x 3 or n doubles, row-major); `stream` is a cudaStream_t or NULL. */
typedef struct gtd_adjoint gtd_adjoint;

GTD_API int gtd_adjoint_create(gtd_adjoint **out, int device, int64_t n, uint64_t steps, uint64_t checkpoint_every,
                               double G, double dt);
GTD_API int gtd_adjoint_destroy(gtd_adjoint *adj);
GTD_API int gtd_adjoint_forward(gtd_adjoint *adj, const double *x0, const double *v0, const double *m, double *xT,
                                double *vT, void *stream);
/* gxT = dL/dx_T (required), gvT = dL/dv_T (may be NULL) -> gx0, gv0, gm (any may be NULL). */
GTD_API int gtd_adjoint_backward(gtd_adjoint *adj, const double *gxT, const double *gvT, double *gx0, double *gv0,
                                 double *gm, void *stream);
GTD_API int gtd_adjoint_launch_count(const gtd_adjoint *adj, uint64_t *count);

#ifdef __cplusplus
}
#endif
#endif /* GTD_B200_H */
