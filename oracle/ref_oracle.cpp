/* Reference-backed oracle: a thin extern "C" driver over the UNMODIFIED gtd:: headers of
 * GregW10/GregPackagesCPP (gregsys.hpp, greg8tree.hpp, gregbod.hpp), compiled from the reference
 * tree by oracle/Makefile into oracle/_ref/libgtdref.so.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (gregpackagescpp_b200/, include/) links or
 * loads this library; only tests/, the fixture generator under tests/golden/ and the CPU-baseline
 * leg of bench.py do, as a checker or as the timed reference CPU arm.
 *
 * Private state of gtd::system / gtd::body / gtd::bh_cube is reached through one explicit
 * specialisation of gtd::system (named `ref_access` below).  Every gtd::system specialisation is
 * a friend of body (gregbod.hpp:869-886), of bh_cube/bh_tree (greg8tree.hpp:954-956, 1107-1108)
 * and of every other system specialisation (gregsys.hpp:3444-3445), so this reads private
 * members without touching the reference sources.
 */
#include "gregsys.hpp"

#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

namespace gtd {
/* Explicit specialisation used purely as a key to the friendship declared by the reference. */
template <>
class system<double, double, double, true, true, 0, 4242, 4242, false> {
public:
    using bod_d = body<double, double, double, 0>;
    using bod_f = body<float, float, float, 0>;

    template <typename S>
    static auto &bodies(S &s) { return s.bods; }

    template <typename B>
    static void set_acc(B &b, double ax, double ay, double az) { b.acc.x = ax; b.acc.y = ay; b.acc.z = az; }

    /* Energy of a system with memFreq != 0, using the reference's own private calc_energy
     * (gregsys.hpp:608-630) after refreshing every body's kinetic energy (gregbod.hpp:325-328). */
    template <typename S>
    static void energy(S &s, long double *ke, long double *pe) {
        for (auto &b : s.bods) b.set_ke();
        s.create_energy_vectors();
        s.calc_energy();
        *ke = s.tot_ke.back();
        *pe = s.tot_pe.back();
    }

    template <typename S>
    static long double G(const S &s) { return s.G; }

    /* gtd::system's private static check_option (gregsys.hpp:1406-1411). */
    static bool check_option(int option) {
        return gtd::system<double, double, double, false, false, 0, 0, 0, false>::check_option(option);
    }
    template <typename S>
    static long double time_elapsed(const S &s) { return s.time_elapsed; }
    template <typename S>
    static long double dt(const S &s) { return s.dt; }
    template <typename B>
    static long double rest(const B &b) { return b.rest_c; }

    /* The recordings of a system with memFreq != 0 (gregsys.hpp:219-227; gregbod.hpp:304-306):
     * every body's positions/velocities/kinetic energies, the per-body pe and energy maps (keyed by
     * body id) and the system totals.  Capacities in frames; returns the frame counts. */
    template <typename S>
    static void recordings(S &s, int max_frames, int *pos_frames, int *pe_frames, double *pos3, double *vel3,
                           double *ke, double *pe, double *energy, double *tot3) {
        const int n = (int)s.bods.size();
        *pos_frames = n ? (int)s.bods[0].get_positions().size() : 0;
        *pe_frames = (int)s.tot_pe.size();
        for (int i = 0; i < n; ++i) {
            const auto &b = s.bods[i];
            const auto &P = b.get_positions();
            const auto &V = b.get_velocities();
            const auto &K = b.get_kinetic_energies();
            for (int f = 0; f < (int)P.size() && f < max_frames; ++f) {
                const size_t o = ((size_t)f * n + i);
                pos3[3 * o] = (double)P[f].x; pos3[3 * o + 1] = (double)P[f].y; pos3[3 * o + 2] = (double)P[f].z;
                vel3[3 * o] = (double)V[f].x; vel3[3 * o + 1] = (double)V[f].y; vel3[3 * o + 2] = (double)V[f].z;
                ke[o] = (double)K[f];
            }
            const auto &PE = s.pe[b.id];
            const auto &E = s.energy[b.id];
            for (int f = 0; f < (int)PE.size() && f < max_frames; ++f) {
                pe[(size_t)f * n + i] = (double)PE[f];
                energy[(size_t)f * n + i] = (double)E[f];
            }
        }
        for (int f = 0; f < *pe_frames && f < max_frames; ++f) {
            tot3[3 * f] = (double)s.tot_pe[f];
            tot3[3 * f + 1] = (double)s.tot_ke[f];
            tot3[3 * f + 2] = (double)s.tot_e[f];
        }
    }

    /* DFS pre-order dump of a bh_tree, children in octant order 0..7 (greg8tree.hpp:74-76). */
    template <typename Tree, typename Bod>
    static long dump_tree(Tree &tree, const Bod *base, long max_nodes, int *depth, int *leaf_body,
                          double *mass, double *com3, double *btm3, double *top3, double *root_box6) {
        auto *root = tree._root;
        if (root_box6) {
            root_box6[0] = tree._btm.x; root_box6[1] = tree._btm.y; root_box6[2] = tree._btm.z;
            root_box6[3] = tree._top.x; root_box6[4] = tree._top.y; root_box6[5] = tree._top.z;
        }
        if (!root) return 0;
        using cube_t = std::remove_pointer_t<decltype(root)>;
        std::vector<std::pair<cube_t *, int>> stack;
        stack.emplace_back(root, 0);
        long count = 0;
        while (!stack.empty()) {
            auto [c, d] = stack.back();
            stack.pop_back();
            if (count < max_nodes) {
                depth[count] = d;
                leaf_body[count] = c->_bod ? int(c->_bod - base) : -1;
                mass[count] = double(c->_mass);
                com3[3 * count + 0] = double(c->_com.x);
                com3[3 * count + 1] = double(c->_com.y);
                com3[3 * count + 2] = double(c->_com.z);
                btm3[3 * count + 0] = double(c->_btm.x);
                btm3[3 * count + 1] = double(c->_btm.y);
                btm3[3 * count + 2] = double(c->_btm.z);
                top3[3 * count + 0] = double(c->_top.x);
                top3[3 * count + 1] = double(c->_top.y);
                top3[3 * count + 2] = double(c->_top.z);
            }
            ++count;
            for (int i = 7; i >= 0; --i)
                if (c->_sub[i]) stack.emplace_back(c->_sub[i], d + 1);
        }
        return count;
    }

    /* Barnes-Hut acceleration of every body: reference tree (greg8tree.hpp:1066-1078), reference
     * calc_com (greg8tree.hpp:1062), reference cell_iterator walk (greg8tree.hpp:702-833) and the
     * reference bh_acc arithmetic (gregsys.hpp:371-375) with the assignment corrected to `+=`. */
    template <typename Tree, typename Bod>
    static void bh_walk(Tree &tree, std::vector<Bod> &bods, long double theta, long double eps_sq,
                        long double Gc, uint64_t *n_inter) {
        using cube_t = std::remove_pointer_t<decltype(tree._root)>;
        for (auto &b : bods) { b.acc.x = 0; b.acc.y = 0; b.acc.z = 0; }
        uint64_t count = 0;
        typename cube_t::iterator it = tree.begin();
        while (it) {
            typename cube_t::cell_iterator cit{tree._root, it, theta};
            Bod *bod = const_cast<Bod *>(it._cptr->_bod);
            while (cit) {
                const cube_t *src = cit++._cptr;
                auto &&r12 = src->_com - bod->curr_pos;
                auto &&r12_sq = r12 * r12 + eps_sq;
                bod->acc += Gc * (src->_mass / (r12_sq)) * (r12 / (sqrtl(r12_sq)));
                ++count;
            }
            ++it;
        }
        if (n_inter) *n_inter = count;
    }

    /* The reference's Barnes-Hut leapfrog schedule (gregsys.hpp:2893-2945) around bh_walk. */
    static void bh_kdk(std::vector<bod_d> &v, long double dt, uint64_t steps, long double theta, long double eps_sq,
                       long double Gc, long long *tb, long long *tw) {
        long double half_dt = dt / 2;
        auto walk = [&]() {
            gtd::bh_tree<double, double, double, 0> tree;
            auto t0 = std::chrono::steady_clock::now();
            tree.add_bodies(v);
            tree.calc_com();
            auto t1 = std::chrono::steady_clock::now();
            bh_walk(tree, v, theta, eps_sq, Gc, nullptr);
            auto t2 = std::chrono::steady_clock::now();
            *tb += std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
            *tw += std::chrono::duration_cast<std::chrono::nanoseconds>(t2 - t1).count();
        };
        walk();
        for (auto &b : v) b.curr_vel += half_dt * b.acc;
        for (uint64_t s = 0; s < steps; ++s) {
            for (auto &b : v) b.curr_pos += dt * b.curr_vel;
            walk();
            for (auto &b : v) b.curr_vel += dt * b.acc;
        }
    }

    /* The same schedule on a system with collisions != 0, so that the reference's own bh_s_coll
     * (gregsys.hpp:631-688) runs after every full kick on the system's own btree, as in
     * gregsys.hpp:2936-2938. */
    template <typename S>
    static void bh_kdk_coll(S &s, long double dt, uint64_t steps, long double theta, long double eps_sq) {
        auto &v = s.bods;
        const long double Gc = s.G;
        const long double half_dt = dt / 2;
        auto walk = [&]() {
            s.btree.delete_tree();
            s.btree.add_bodies(v);
            s.btree.calc_com();
            bh_walk(s.btree, v, theta, eps_sq, Gc, nullptr);
        };
        walk();
        for (auto &b : v) b.curr_vel += half_dt * b.acc;
        for (uint64_t k = 0; k < steps; ++k) {
            for (auto &b : v) b.curr_pos += dt * b.curr_vel;
            walk();
            for (auto &b : v) b.curr_vel += dt * b.acc;
            s.bh_s_coll();
        }
    }

    /* One bh_s_coll on a tree built at the given state (no gravity, no drift). */
    template <typename S>
    static void bh_s_coll_once(S &s) {
        s.btree.delete_tree();
        s.btree.add_bodies(s.bods);
        s.bh_s_coll();
    }

    template <typename A, typename B>
    static void merge_into(A &a, const B &b) { a += b; }

    /* evolve(method, continue_ev_if, for_each_bod, for_all_bods) on the reference's own loop with the
     * callbacks random_comet passes (gregsys.hpp:1935-1984), restated here as lambdas: continue
     * while some body has rest_c < min_max_cor (resetting a counter), then probing_iters more
     * steps; for_all_bods carries the centre (com += positions, then /= N, or m-weighted /= M) and
     * sets rest_c from the distance to it.  for_each_bod (each_mode 1) scales every velocity by
     * each_factor.  max_steps > 0 makes the predicate false once that many steps ran. */
    struct cb_args {
        int cont_mode, all_mode, each_mode, mass_weighted;
        long double min_max_cor, min_cor, max_cor, scale_factor, n_exp;
        uint64_t probing_iters, max_steps;
        double each_factor;
    };
    template <typename S, typename C, typename E, typename A>
    static void call_evolve(S &s, int method, const C &c, const E &e, const A &a) {
        s.evolve(method, c, e, a);
    }
    template <typename S>
    static uint64_t evolve_callbacks(S &s, int method, const cb_args &p, double *com_io) {
        auto &bods = s.bods;
        gtd::vector3D<double> com{com_io[0], com_io[1], com_io[2]};
        const uint64_t n_ = bods.size();
        double tot_mass = 0;
        for (const auto &b : bods) tot_mass += b.mass_;
        uint64_t count = 0, taken = 0;
        auto cont = [&]() -> bool {
            if (p.max_steps && taken >= p.max_steps) return false;
            bool go = false, below = false;
            for (const auto &b : bods)
                if (b.rest_c < p.min_max_cor) {
                    below = true;
                    break;
                }
            if (below) {
                count = 0;
                go = true;
            } else {
                go = count++ < p.probing_iters;
            }
            if (go) ++taken;
            return go;
        };
        auto all = [&](auto &bodies) {
            if (p.mass_weighted) {
                for (const auto &b : bodies) com += b.mass_ * b.curr_pos;
                com /= tot_mass;
            } else {
                for (const auto &b : bodies) com += b.curr_pos;
                com /= n_;
            }
            long double dist_exp;
            for (auto &b : bodies) {
                dist_exp = powl((b.curr_pos - com).magnitude(), p.n_exp);
                b.rest_c = p.max_cor - (p.max_cor - p.min_cor) * (dist_exp / (dist_exp + p.scale_factor));
            }
        };
        auto each = [&](auto &b) { b.curr_vel *= p.each_factor; };
        const bool c = p.cont_mode != 0, a = p.all_mode != 0, e = p.each_mode != 0;
        if (c && e && a) call_evolve(s, method, cont, each, all);
        else if (c && e) call_evolve(s, method, cont, each, nullptr);
        else if (c && a) call_evolve(s, method, cont, nullptr, all);
        else if (c) call_evolve(s, method, cont, nullptr, nullptr);
        else if (e && a) call_evolve(s, method, nullptr, each, all);
        else if (e) call_evolve(s, method, nullptr, each, nullptr);
        else if (a) call_evolve(s, method, nullptr, nullptr, all);
        else call_evolve(s, method, nullptr, nullptr, nullptr);
        com_io[0] = com.get_x();
        com_io[1] = com.get_y();
        com_io[2] = com.get_z();
        return c ? taken : s.iterations;
    }
};
}  // namespace gtd

using ref_access = gtd::system<double, double, double, true, true, 0, 4242, 4242, false>;
using bod_d = ref_access::bod_d;
using bod_f = ref_access::bod_f;

static thread_local char g_err[512];

extern "C" const char *ref_last_error(void) { return g_err; }

#define REF_TRY try {
#define REF_CATCH                                              \
    }                                                          \
    catch (const std::exception &e) {                          \
        std::snprintf(g_err, sizeof g_err, "%s", e.what());    \
        return -1;                                             \
    }                                                          \
    catch (...) {                                              \
        std::snprintf(g_err, sizeof g_err, "unknown exception"); \
        return -1;                                             \
    }

static std::vector<bod_d> make_bodies(int n, const double *m, const double *r, const double *rest,
                                      const double *x3, const double *v3) {
    std::vector<bod_d> v;
    v.reserve(n);
    for (int i = 0; i < n; ++i)
        v.emplace_back(m[i], r ? r[i] : 0.0, gtd::vector3D<double>{x3[3 * i], x3[3 * i + 1], x3[3 * i + 2]},
                       gtd::vector3D<double>{v3 ? v3[3 * i] : 0.0, v3 ? v3[3 * i + 1] : 0.0, v3 ? v3[3 * i + 2] : 0.0},
                       rest ? (long double)rest[i] : 1.0L);
    return v;
}

template <typename S>
static void read_back(S &s, double *x3, double *v3, double *a3, double *m, double *r) {
    auto &b = ref_access::bodies(s);
    for (size_t i = 0; i < b.size(); ++i) {
        if (x3) { x3[3 * i] = b[i].pos().get_x(); x3[3 * i + 1] = b[i].pos().get_y(); x3[3 * i + 2] = b[i].pos().get_z(); }
        if (v3) { v3[3 * i] = b[i].vel().get_x(); v3[3 * i + 1] = b[i].vel().get_y(); v3[3 * i + 2] = b[i].vel().get_z(); }
        if (a3) {
            a3[3 * i] = b[i].acceleration().get_x();
            a3[3 * i + 1] = b[i].acceleration().get_y();
            a3[3 * i + 2] = b[i].acceleration().get_z();
        }
        if (m) m[i] = b[i].mass();
        if (r) r[i] = b[i].rad();
    }
}

template <int coll>
static int evolve_impl(int method, int n, const double *m, const double *r, const double *rest, const double *x3,
                       const double *v3, double dt, uint64_t steps, const char *units, double *x3o, double *v3o,
                       double *a3o, long long *ns) {
    using sys_t = gtd::system<double, double, double, false, false, coll, 0, 0, false>;
    sys_t s{make_bodies(n, m, r, rest, x3, v3), (long double)dt, steps, units, true};
    auto t = s.evolve(method);
    if (ns) *ns = t.count();
    read_back(s, x3o, v3o, a3o, nullptr, nullptr);
    return 0;
}

extern "C" {

/* gtd::system<double,double,double,false,false,coll,0,0,false>::evolve(method) (gregsys.hpp:2593-3071)
 * on n bodies; coll is 0 (none) or 3 (overlap restitution, s_coll gregsys.hpp:690-914). */
int ref_evolve(int method, int coll, int n, const double *m, const double *r, const double *rest, const double *x3,
               const double *v3, double dt, uint64_t steps, const char *units, double *x3o, double *v3o, double *a3o,
               long long *elapsed_ns) {
    REF_TRY
    if (coll == 0) return evolve_impl<0>(method, n, m, r, rest, x3, v3, dt, steps, units, x3o, v3o, a3o, elapsed_ns);
    if (coll == 3) return evolve_impl<3>(method, n, m, r, rest, x3, v3, dt, steps, units, x3o, v3o, a3o, elapsed_ns);
    std::snprintf(g_err, sizeof g_err, "unsupported collision mode %d", coll);
    return -1;
    REF_CATCH
}

/* G as the reference derives it from a units string (gregsys.hpp:245-282), as long double. */
int ref_G(const char *units, long double *G) {
    REF_TRY
    gtd::system<double, double, double, false, false, 0, 0, 0, false> s{1.0L, 1, units};
    *G = ref_access::G(s);
    return 0;
    REF_CATCH
}

/* The reference's setters (gregsys.hpp:1636-1672) on a default system: out4 = the results of
 * set_timestep(dt), set_iterations(iterations), set_softening(eps), set_bh_opening_angle(theta).
 * dt, eps and theta arrive as long double so that values between two doubles can be tried. */
int ref_setters(long double dt, uint64_t iterations, long double eps, long double theta, int *out4) {
    REF_TRY
    gtd::system<double, double, double, false, false, 0, 0, 0, false> s{1.0L, 1, "M1:1,D1:1,T1:1"};
    out4[0] = s.set_timestep(dt) ? 1 : 0;
    out4[1] = s.set_iterations(iterations) ? 1 : 0;
    out4[2] = s.set_softening(eps) ? 1 : 0;
    out4[3] = s.set_bh_opening_angle(theta) ? 1 : 0;
    return 0;
    REF_CATCH
}

/* check_option (gregsys.hpp:1406-1411): 1 when evolve() accepts the method value, else 0. */
int ref_check_option(int option) { return ref_access::check_option(option) ? 1 : 0; }

/* Constructs a system with time step dt (the constructor's check_dt, gregsys.hpp:1401-1405):
 * 0, or -1 with the exception's message in ref_last_error(). */
int ref_construct_dt(long double dt) {
    REF_TRY
    gtd::system<double, double, double, false, false, 0, 0, 0, false> s{dt, 1, "M1:1,D1:1,T1:1"};
    return 0;
    REF_CATCH
}

/* Total kinetic and potential energy with the reference's calc_energy (gregsys.hpp:608-630). */
int ref_energy(int n, const double *m, const double *x3, const double *v3, const char *units, long double *ke,
               long double *pe) {
    REF_TRY
    using sys_t = gtd::system<double, double, double, false, false, 0, 1, 0, false>;
    std::vector<gtd::body<double, double, double, 1>> v;
    v.reserve(n);
    for (int i = 0; i < n; ++i)
        v.emplace_back(m[i], 0.0, gtd::vector3D<double>{x3[3 * i], x3[3 * i + 1], x3[3 * i + 2]},
                       gtd::vector3D<double>{v3[3 * i], v3[3 * i + 1], v3[3 * i + 2]});
    sys_t s{std::move(v), 1.0L, 1, units, true};
    ref_access::energy(s, ke, pe);
    return 0;
    REF_CATCH
}

/* Add-time overlap merge: the system constructor with allow_overlapping_bodies=false runs
 * check_overlap (gregsys.hpp:307-342) with mergeOverlappingBodies=true.  Returns the surviving
 * count in *n_out and their state. */
int ref_check_overlap_merge(int n, const double *m, const double *r, const double *rest, const double *x3,
                            const double *v3, int *n_out, double *m_o, double *r_o, double *x3o, double *v3o) {
    REF_TRY
    using sys_t = gtd::system<double, double, double, false, true, 0, 0, 0, false>;
    sys_t s{make_bodies(n, m, r, rest, x3, v3), 1.0L, 1, "M1:1,D1:1,T1:1", false};
    *n_out = (int)s.num_bodies();
    read_back(s, x3o, v3o, nullptr, m_o, r_o);
    return 0;
    REF_CATCH
}

/* body::operator+= (gregbod.hpp:1066-1082): merges body b into body a; the result's state. */
int ref_merge_pair(const double *ma, const double *mb, double *out_m, double *out_r, double *out_x3, double *out_v3,
                   double *out_a3, double *out_rest) {
    /* ma/mb: {m, r, rest, x, y, z, vx, vy, vz, ax, ay, az} */
    REF_TRY
    bod_d a{ma[0], ma[1], gtd::vector3D<double>{ma[3], ma[4], ma[5]}, gtd::vector3D<double>{ma[6], ma[7], ma[8]},
            (long double)ma[2]};
    bod_d b{mb[0], mb[1], gtd::vector3D<double>{mb[3], mb[4], mb[5]}, gtd::vector3D<double>{mb[6], mb[7], mb[8]},
            (long double)mb[2]};
    ref_access::set_acc(a, ma[9], ma[10], ma[11]);
    ref_access::set_acc(b, mb[9], mb[10], mb[11]);
    ref_access::merge_into(a, b);
    *out_m = a.mass();
    *out_r = a.rad();
    out_x3[0] = a.pos().get_x(); out_x3[1] = a.pos().get_y(); out_x3[2] = a.pos().get_z();
    out_v3[0] = a.vel().get_x(); out_v3[1] = a.vel().get_y(); out_v3[2] = a.vel().get_z();
    out_a3[0] = a.acceleration().get_x(); out_a3[1] = a.acceleration().get_y(); out_a3[2] = a.acceleration().get_z();
    *out_rest = (double)a.restitution();
    return 0;
    REF_CATCH
}

/* Reference octree (bh_tree::add_bodies greg8tree.hpp:1066-1078 + calc_com :1062) dumped in DFS
 * pre-order.  prec 0: T=M=R=double; prec 1: T=M=R=float on the given values rounded to float.
 * Returns the node count (arrays are filled up to max_nodes) or -1 on a reference exception. */
long ref_bh_tree_dump(int prec, int n, const double *x3, const double *m, long max_nodes, int *depth, int *leaf_body,
                      double *mass, double *com3, double *btm3, double *top3, double *root_box6) {
    REF_TRY
    if (prec == 0) {
        std::vector<bod_d> v = make_bodies(n, m, nullptr, nullptr, x3, nullptr);
        gtd::bh_tree<double, double, double, 0> tree;
        tree.add_bodies(v);
        tree.calc_com();
        return ref_access::dump_tree(tree, v.data(), max_nodes, depth, leaf_body, mass, com3, btm3, top3, root_box6);
    } else {
        std::vector<bod_f> v;
        v.reserve(n);
        for (int i = 0; i < n; ++i)
            v.emplace_back((float)m[i], 0.0f,
                           gtd::vector3D<float>{(float)x3[3 * i], (float)x3[3 * i + 1], (float)x3[3 * i + 2]},
                           gtd::vector3D<float>{0.0f, 0.0f, 0.0f});
        gtd::bh_tree<float, float, float, 0> tree;
        tree.add_bodies(v);
        /* no calc_com: the float moments overflow in SI units; topology only */
        return ref_access::dump_tree(tree, v.data(), max_nodes, depth, leaf_body, mass, com3, btm3, top3, root_box6);
    }
    REF_CATCH
}

/* Barnes-Hut accelerations (T=double) with the corrected accumulation; see ref_access::bh_walk. */
int ref_bh_acc(int n, const double *x3, const double *m, double theta, double eps, const char *units, double *a3,
               uint64_t *n_inter) {
    REF_TRY
    long double Gc;
    if (ref_G(units, &Gc)) return -1;
    std::vector<bod_d> v = make_bodies(n, m, nullptr, nullptr, x3, nullptr);
    gtd::bh_tree<double, double, double, 0> tree;
    tree.add_bodies(v);
    tree.calc_com();
    ref_access::bh_walk(tree, v, (long double)theta, (long double)eps * (long double)eps, Gc, n_inter);
    for (int i = 0; i < n; ++i) {
        a3[3 * i] = v[i].acceleration().get_x();
        a3[3 * i + 1] = v[i].acceleration().get_y();
        a3[3 * i + 2] = v[i].acceleration().get_z();
    }
    return 0;
    REF_CATCH
}

/* The reference's Barnes-Hut leapfrog schedule (gregsys.hpp:2893-2945): initial walk and half
 * kick, then per step a full drift, a rebuild, a walk and a full kick (velocities end half a step
 * ahead), with the corrected accumulation and calc_com after every build. */
int ref_bh_kdk(int n, const double *m, const double *x3, const double *v3, double dt, uint64_t steps, double theta,
               double eps, const char *units, double *x3o, double *v3o, double *a3o, long long *build_ns,
               long long *walk_ns) {
    REF_TRY
    long double Gc;
    if (ref_G(units, &Gc)) return -1;
    std::vector<bod_d> v = make_bodies(n, m, nullptr, nullptr, x3, v3);
    long long tb = 0, tw = 0;
    ref_access::bh_kdk(v, (long double)dt, steps, (long double)theta, (long double)eps * (long double)eps, Gc, &tb,
                       &tw);
    if (build_ns) *build_ns = tb;
    if (walk_ns) *walk_ns = tw;
    for (int i = 0; i < n; ++i) {
        if (x3o) { x3o[3 * i] = v[i].pos().get_x(); x3o[3 * i + 1] = v[i].pos().get_y(); x3o[3 * i + 2] = v[i].pos().get_z(); }
        if (v3o) { v3o[3 * i] = v[i].vel().get_x(); v3o[3 * i + 1] = v[i].vel().get_y(); v3o[3 * i + 2] = v[i].vel().get_z(); }
        if (a3o) {
            a3o[3 * i] = v[i].acceleration().get_x();
            a3o[3 * i + 1] = v[i].acceleration().get_y();
            a3o[3 * i + 2] = v[i].acceleration().get_z();
        }
    }
    return 0;
    REF_CATCH
}

}  // extern "C"

/* .nsys snapshots through the reference's own system::to_nsys (gregsys.hpp:3214-3258) and
 * load_from_nsys constructor (gregsys.hpp:1478-1480, 947-1400), for M, R, T in {float, double,
 * long double}: kind 0 = double x3, 1 = float x3, 2 = long double x3, 3 = <float, float, double>. */
template <typename M, typename R, typename T>
static int to_nsys_impl(int n, const double *m, const double *r, const double *rest, const double *x3,
                        const double *v3, double dt, uint64_t steps, const char *units, const char *path,
                        long long *bytes) {
    using sys_t = gtd::system<M, R, T, false, false, 0, 0, 0, false>;
    using bod_t = gtd::body<M, R, T, 0>;
    std::vector<bod_t> v;
    v.reserve(n);
    for (int i = 0; i < n; ++i)
        v.emplace_back((M)m[i], (R)r[i], gtd::vector3D<T>{(T)x3[3 * i], (T)x3[3 * i + 1], (T)x3[3 * i + 2]},
                       gtd::vector3D<T>{(T)v3[3 * i], (T)v3[3 * i + 1], (T)v3[3 * i + 2]}, (long double)rest[i]);
    sys_t s{std::move(v), (long double)dt, steps, units, true};
    if (steps) s.evolve(16);  // leapfrog_kdk
    *bytes = (long long)s.to_nsys(path);
    return 0;
}

template <typename M, typename R, typename T>
static int load_nsys_impl(const char *path, int alloc, int check, int max_n, int *n_out, double *m, double *r,
                          double *rest, double *x3, double *v3, double *t_el, double *dt, double *G) {
    using sys_t = gtd::system<M, R, T, false, false, 0, 0, 0, false>;
    sys_t s{path, alloc != 0, check != 0, true};
    auto &b = ref_access::bodies(s);
    *n_out = (int)b.size();
    for (int i = 0; i < (int)b.size() && i < max_n; ++i) {
        m[i] = (double)b[i].mass();
        r[i] = (double)b[i].rad();
        rest[i] = (double)ref_access::rest(b[i]);
        x3[3 * i] = (double)b[i].pos().get_x(); x3[3 * i + 1] = (double)b[i].pos().get_y();
        x3[3 * i + 2] = (double)b[i].pos().get_z();
        v3[3 * i] = (double)b[i].vel().get_x(); v3[3 * i + 1] = (double)b[i].vel().get_y();
        v3[3 * i + 2] = (double)b[i].vel().get_z();
    }
    *t_el = (double)ref_access::time_elapsed(s);
    *dt = (double)ref_access::dt(s);
    *G = (double)ref_access::G(s);
    return 0;
}

extern "C" {

int ref_to_nsys(int kind, int n, const double *m, const double *r, const double *rest, const double *x3,
                const double *v3, double dt, uint64_t steps, const char *units, const char *path, long long *bytes) {
    REF_TRY
    switch (kind) {
        case 0: return to_nsys_impl<double, double, double>(n, m, r, rest, x3, v3, dt, steps, units, path, bytes);
        case 1: return to_nsys_impl<float, float, float>(n, m, r, rest, x3, v3, dt, steps, units, path, bytes);
        case 2:
            return to_nsys_impl<long double, long double, long double>(n, m, r, rest, x3, v3, dt, steps, units, path,
                                                                       bytes);
        case 3: return to_nsys_impl<float, float, double>(n, m, r, rest, x3, v3, dt, steps, units, path, bytes);
    }
    std::snprintf(g_err, sizeof g_err, "unknown kind %d", kind);
    return -1;
    REF_CATCH
}

/* Returns 0, or -1 (nsys_load_error), -2 (nsys_format_error), -3 (other exception) with the
 * exception's what() in ref_last_error.  alloc = the constructor's alloc_chunks; with alloc != 0 a
 * NaN/Inf chunk makes the reference delete its input stream a second time (gregsys.hpp:1306-1308,
 * then final_handler :950-952) and crash, so NaN/Inf cases are read with alloc = 0. */
int ref_load_nsys(int kind, const char *path, int alloc, int check, int max_n, int *n_out, double *m, double *r,
                  double *rest, double *x3, double *v3, double *t_el, double *dt, double *G) {
    try {
        switch (kind) {
            case 0:
                return load_nsys_impl<double, double, double>(path, alloc, check, max_n, n_out, m, r, rest, x3, v3,
                                                              t_el, dt, G);
            case 1:
                return load_nsys_impl<float, float, float>(path, alloc, check, max_n, n_out, m, r, rest, x3, v3, t_el,
                                                           dt, G);
            case 2:
                return load_nsys_impl<long double, long double, long double>(path, alloc, check, max_n, n_out, m, r,
                                                                             rest, x3, v3, t_el, dt, G);
            case 3:
                return load_nsys_impl<float, float, double>(path, alloc, check, max_n, n_out, m, r, rest, x3, v3, t_el,
                                                            dt, G);
        }
        std::snprintf(g_err, sizeof g_err, "unknown kind %d", kind);
        return -3;
    } catch (const gtd::nsys_format_error &e) {
        std::snprintf(g_err, sizeof g_err, "%s", e.what());
        return -2;
    } catch (const gtd::nsys_load_error &e) {
        std::snprintf(g_err, sizeof g_err, "%s", e.what());
        return -1;
    } catch (const std::exception &e) {
        std::snprintf(g_err, sizeof g_err, "%s", e.what());
        return -3;
    }
}

}  // extern "C"

/* evolve with trajectory recording: gtd::system<double,double,double,false,false,coll,MF,FF,false>,
 * evolve(method) called `calls` times (a second call clears the first one's recordings,
 * gregsys.hpp:2615-2619, 2569-2586); the recordings of the last call and the final state. */
template <uint64_t MF>
static std::vector<gtd::body<double, double, double, MF>> rec_bodies(int n, const double *m, const double *r,
                                                                     const double *rest, const double *x3,
                                                                     const double *v3) {
    std::vector<gtd::body<double, double, double, MF>> v;
    v.reserve(n);
    for (int i = 0; i < n; ++i)
        v.emplace_back(m[i], r ? r[i] : 0.0, gtd::vector3D<double>{x3[3 * i], x3[3 * i + 1], x3[3 * i + 2]},
                       gtd::vector3D<double>{v3[3 * i], v3[3 * i + 1], v3[3 * i + 2]},
                       rest ? (long double)rest[i] : 1.0L);
    return v;
}

template <int coll, uint64_t MF, uint64_t FF>
static int evolve_rec_impl(int method, int n, const double *m, const double *r, const double *rest, const double *x3,
                           const double *v3, double dt, uint64_t steps, const char *units, int calls, int max_frames,
                           int *pos_frames, int *pe_frames, double *pos3, double *vel3, double *ke, double *pe,
                           double *energy, double *tot3, double *x3o, double *v3o) {
    using sys_t = gtd::system<double, double, double, false, false, coll, MF, FF, false>;
    sys_t s{rec_bodies<MF>(n, m, r, rest, x3, v3), (long double)dt, steps, units, true};
    for (int c = 0; c < calls; ++c) s.evolve(method);
    ref_access::recordings(s, max_frames, pos_frames, pe_frames, pos3, vel3, ke, pe, energy, tot3);
    read_back(s, x3o, v3o, nullptr, nullptr, nullptr);
    return 0;
}

/* evolve(method, continue_ev_if, for_each_bod, for_all_bods) of a system with memFreq = MF (fileFreq
 * 0), the callbacks of ref_access::evolve_callbacks: the recordings (FUNC_TEMPL_SELECT,
 * gregsys.hpp:16-106, inside the callback loops), the final state, every rest_c and the steps. */
template <int coll, uint64_t MF>
static int evolve_rec_cb_impl(int method, int n, const double *m, const double *r, const double *rest,
                              const double *x3, const double *v3, double dt, uint64_t iterations, const char *units,
                              const ref_access::cb_args &p, double *com_io, int max_frames, int *pos_frames,
                              int *pe_frames, double *pos3, double *vel3, double *ke, double *pe, double *energy,
                              double *tot3, double *x3o, double *v3o, double *rest_o, uint64_t *steps) {
    using sys_t = gtd::system<double, double, double, false, false, coll, MF, 0, false>;
    sys_t s{rec_bodies<MF>(n, m, r, rest, x3, v3), (long double)dt, iterations, units, true};
    *steps = ref_access::evolve_callbacks(s, method, p, com_io);
    ref_access::recordings(s, max_frames, pos_frames, pe_frames, pos3, vel3, ke, pe, energy, tot3);
    read_back(s, x3o, v3o, nullptr, nullptr, nullptr);
    auto &b = ref_access::bodies(s);
    for (size_t i = 0; i < b.size(); ++i) rest_o[i] = (double)ref_access::rest(b[i]);
    return 0;
}

extern "C" {

/* mem_freq 1, 2 or 3; coll 0 or 3; file_freq must be 0.  With memFreq and fileFreq both non-zero,
 * evolve() does not compile (its Barnes-Hut Euler branch, gregsys.hpp:2640-2646, names members that
 * do not exist); with fileFreq == 0, FUNC_TEMPL_SELECT (gregsys.hpp:15-16) always takes its
 * non-recording branch, so only the energies of calc_acc_and_e / calc_energy are recorded. */
int ref_evolve_record(int method, int coll, uint64_t mem_freq, uint64_t file_freq, int n, const double *m, const double *r,
                      const double *rest, const double *x3, const double *v3, double dt, uint64_t steps,
                      const char *units, int calls, int max_frames, int *pos_frames, int *pe_frames, double *pos3,
                      double *vel3, double *ke, double *pe, double *energy, double *tot3, double *x3o, double *v3o) {
    REF_TRY
#define REC_CASE(C, F, FF)                                                                                      \
    if (coll == C && mem_freq == F && file_freq == FF)                                                         \
        return evolve_rec_impl<C, F, FF>(method, n, m, r, rest, x3, v3, dt, steps, units, calls, max_frames,   \
                                         pos_frames, pe_frames, pos3, vel3, ke, pe, energy, tot3, x3o, v3o);
    REC_CASE(0, 1, 0) REC_CASE(0, 2, 0) REC_CASE(0, 3, 0) REC_CASE(3, 1, 0) REC_CASE(3, 2, 0) REC_CASE(3, 3, 0)
#undef REC_CASE
    std::snprintf(g_err, sizeof g_err, "unsupported coll %d / mem_freq %llu / file_freq %llu", coll,
                  (unsigned long long)mem_freq, (unsigned long long)file_freq);
    return -1;
    REF_CATCH
}

/* mem_freq 1, 2 or 3; coll 0 or 3; the callback arguments as ref_evolve_callbacks. */
int ref_evolve_record_callbacks(int method, int coll, uint64_t mem_freq, int n, const double *m, const double *r,
                                const double *rest, const double *x3, const double *v3, double dt,
                                uint64_t iterations, const char *units, int cont_mode, double min_max_cor,
                                uint64_t probing_iters, int all_mode, double min_cor, double max_cor,
                                double scale_factor, double n_exp, int mass_weighted, int each_mode,
                                double each_factor, uint64_t max_steps, double *com_io, int max_frames,
                                int *pos_frames, int *pe_frames, double *pos3, double *vel3, double *ke, double *pe,
                                double *energy, double *tot3, double *x3o, double *v3o, double *rest_o,
                                uint64_t *steps) {
    REF_TRY
    const ref_access::cb_args p{cont_mode, all_mode, each_mode, mass_weighted, (long double)min_max_cor,
                                (long double)min_cor, (long double)max_cor, (long double)scale_factor,
                                (long double)n_exp, probing_iters, max_steps, each_factor};
#define REC_CB_CASE(C, F)                                                                                      \
    if (coll == C && mem_freq == F)                                                                            \
        return evolve_rec_cb_impl<C, F>(method, n, m, r, rest, x3, v3, dt, iterations, units, p, com_io,       \
                                        max_frames, pos_frames, pe_frames, pos3, vel3, ke, pe, energy, tot3, x3o, \
                                        v3o, rest_o, steps);
    REC_CB_CASE(0, 1) REC_CB_CASE(0, 2) REC_CB_CASE(0, 3) REC_CB_CASE(3, 1) REC_CB_CASE(3, 2) REC_CB_CASE(3, 3)
#undef REC_CB_CASE
    std::snprintf(g_err, sizeof g_err, "unsupported coll %d / mem_freq %llu", coll, (unsigned long long)mem_freq);
    return -1;
    REF_CATCH
}

/* ref_bh_kdk with the reference's bh_s_coll after every full kick: a
 * gtd::system<double,double,double,false,false,3,0,0,false> (overlapping bodies allowed). */
int ref_bh_kdk_coll(int n, const double *m, const double *r, const double *rest, const double *x3, const double *v3,
                    double dt, uint64_t steps, double theta, const char *units, double *x3o, double *v3o) {
    REF_TRY
    using sys_t = gtd::system<double, double, double, false, false, 3, 0, 0, false>;
    sys_t s{make_bodies(n, m, r, rest, x3, v3), (long double)dt, steps, units, true};
    ref_access::bh_kdk_coll(s, (long double)dt, steps, (long double)theta, 0.0L);
    read_back(s, x3o, v3o, nullptr, nullptr, nullptr);
    return 0;
    REF_CATCH
}

/* One reference bh_s_coll on the given state (tree built at x3); v3o receives the velocities. */
int ref_bh_s_coll(int n, const double *m, const double *r, const double *rest, const double *x3, const double *v3,
                  double *v3o) {
    REF_TRY
    using sys_t = gtd::system<double, double, double, false, false, 3, 0, 0, false>;
    sys_t s{make_bodies(n, m, r, rest, x3, v3), 1.0L, 1, "M1:1,D1:1,T1:1", true};
    ref_access::bh_s_coll_once(s);
    read_back(s, nullptr, v3o, nullptr, nullptr, nullptr);
    return 0;
    REF_CATCH
}

}  // extern "C"

#include <thread>

extern "C" {
/* CPU throughput of the reference's evolve(leapfrog_kdk) (gregsys.hpp:2946-2990): `threads`
 * independent copies of the same system evolved concurrently, one std::thread each (the ensemble
 * pattern of bdsim.cpp:82-113; evolve itself is single-threaded).  *wall_ns is the wall time from
 * the first evolve() call to the last one returning (system construction excluded). */
int ref_bench_kdk(int n, const double *m, const double *x3, const double *v3, double dt, uint64_t steps,
                  const char *units, int threads, long long *wall_ns) {
    REF_TRY
    using sys_t = gtd::system<double, double, double, false, false, 0, 0, 0, false>;
    if (threads < 1) threads = 1;
    std::vector<sys_t *> systems;
    for (int t = 0; t < threads; ++t)
        systems.push_back(new sys_t{make_bodies(n, m, nullptr, nullptr, x3, v3), (long double)dt, steps, units, true});
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back([s = systems[t]]() { s->evolve(sys_t::leapfrog_kdk); });
    for (auto &th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    for (auto *s : systems) delete s;
    *wall_ns = std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
    return 0;
    REF_CATCH
}
}

/* evolve(method, continue_ev_if, for_each_bod, for_all_bods) of
 * gtd::system<double,double,double,false,false,coll,0,0,false> (coll 0 or 3) with random_comet's
 * callbacks (ref_access::evolve_callbacks).  cont_mode / all_mode / each_mode 0 pass nullptr.
 * com_io: the starting centre in, the carried centre out; rest_o: every body's rest_c after. */
extern "C" int ref_evolve_callbacks(int method, int coll, int n, const double *m, const double *r, const double *rest,
                                    const double *x3, const double *v3, double dt, uint64_t iterations,
                                    const char *units, int cont_mode, double min_max_cor, uint64_t probing_iters,
                                    int all_mode, double min_cor, double max_cor, double scale_factor, double n_exp,
                                    int mass_weighted, int each_mode, double each_factor, uint64_t max_steps,
                                    double *com_io, double *x3o, double *v3o, double *rest_o, uint64_t *steps) {
    REF_TRY
    ref_access::cb_args p{cont_mode, all_mode, each_mode, mass_weighted, (long double)min_max_cor,
                          (long double)min_cor, (long double)max_cor, (long double)scale_factor, (long double)n_exp,
                          probing_iters, max_steps, each_factor};
    auto finish = [&](auto &s, uint64_t k) {
        read_back(s, x3o, v3o, nullptr, nullptr, nullptr);
        auto &b = ref_access::bodies(s);
        for (size_t i = 0; i < b.size(); ++i) rest_o[i] = (double)ref_access::rest(b[i]);
        *steps = k;
    };
    if (coll == 0) {
        gtd::system<double, double, double, false, false, 0, 0, 0, false> s{make_bodies(n, m, r, rest, x3, v3),
                                                                         (long double)dt, iterations, units, true};
        finish(s, ref_access::evolve_callbacks(s, method, p, com_io));
        return 0;
    }
    if (coll == 3) {
        gtd::system<double, double, double, false, false, 3, 0, 0, false> s{make_bodies(n, m, r, rest, x3, v3),
                                                                         (long double)dt, iterations, units, true};
        finish(s, ref_access::evolve_callbacks(s, method, p, com_io));
        return 0;
    }
    std::snprintf(g_err, sizeof g_err, "unsupported collision mode %d", coll);
    return -1;
    REF_CATCH
}
