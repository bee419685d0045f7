// Drop-in gtd::system (GregW10/GregPackagesCPP gregsys.hpp:135-3612) whose evolve() runs on the
// B200 through the C ABI (gtd_b200.h).  Same template parameters, method flags, constructors,
// setters and evolve() contract; the std::vector<body> stays authoritative on the host between
// calls and is gathered to the device SoA at evolve() entry and scattered back at exit.
//
// Differences, all documented in the engine: no long double arithmetic on the device (FP64 is used
// for every T); per-step file output (fileFreq) and progress printing are not performed (memFreq
// recordings are, from frames computed on the device); evolve-time merges use check_overlap's scan
// as that routine intends.  .nsys files
// (to_nsys and the path constructor) are written and read by the engine, for floating-point M, R
// and T.
#ifndef GTD_B200_GREGSYS_HPP
#define GTD_B200_GREGSYS_HPP

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <functional>
#include <initializer_list>
#include <ios>
#include <iostream>  // the reference's headers provide it to the drivers
#include <type_traits>
#include <regex>
#include <string>
#include <vector>

#include "greg8tree.hpp"
#include "gregbod.hpp"

namespace gtd {

// Device callbacks for evolve(): GPU work in place of the host callables (gtd_b200.h).
namespace device {
// random_comet's for_all_bods (gregsys.hpp:1966-1984): the carried centre *com becomes
// (*com + sum of positions) / N (or (*com + sum m x) / M, the GREGSYS_MERGERS form), then every body
// takes rest_c = max_cor - (max_cor - min_cor) d^n_exp / (d^n_exp + scale_factor), d its distance
// to the centre.  *com is read at evolve() entry and written back at exit, as the reference's lambda
// leaves its captured _com.
template <typename T>
struct rest_from_com {
    long double min_cor, max_cor, scale_factor, n_exp;
    vector3D<T> *com;
    bool mass_weighted = false;
};
// random_comet's continue_ev_if (gregsys.hpp:1936-1963): true while some body has
// rest_c < min_max_cor, then for probing_iters more evaluations.
struct while_rest_below {
    long double min_max_cor;
    uint64_t probing_iters;
};
// The caller's own device callback: fn enqueues GPU work on the handle's stream (gtd_device_hook).
struct hook {
    gtd_device_hook fn;
    void *user;
};
template <typename F>
struct is_rest_from_com : std::false_type {};
template <typename T>
struct is_rest_from_com<rest_from_com<T>> : std::true_type {};
template <typename F>
struct is_callback : std::bool_constant<is_rest_from_com<F>::value || std::is_same_v<F, while_rest_below> ||
                                        std::is_same_v<F, hook>> {};
}  // namespace device

template <isNumWrapper M = long double, isNumWrapper R = long double, isNumWrapper T = long double,
          bool prog = false, bool mergeOverlappingBodies = false, int collisions = 0, uint64_t memFreq = 0,
          uint64_t fileFreq = 1, bool binaryFile = true>
class system {
public:
    static constexpr int two_body = GTD_TWO_BODY;
    static constexpr int euler = GTD_EULER;
    static constexpr int modified_euler = GTD_MODIFIED_EULER;
    static constexpr int midpoint = GTD_MIDPOINT;
    static constexpr int leapfrog_kdk = GTD_LEAPFROG_KDK;
    static constexpr int leapfrog_dkd = GTD_LEAPFROG_DKD;
    static constexpr int rk4 = GTD_RK4;
    static constexpr int rk3_8 = GTD_RK3_8;
    static constexpr int barnes_hut = GTD_BARNES_HUT;
    static constexpr int fast_multipole = 131'072;
    static constexpr int no_coll_check = 0;
    static constexpr int overlap_coll_check = 3;
    static constexpr int pred_coll_check = 7;
    static constexpr long double G_SI = 0.000'000'000'066'743;
    static_assert(collisions <= pred_coll_check && !(collisions & (collisions + 1)),
                  "Invalid collision-checking option.");
    using bod_t = body<M, R, T, memFreq>;

private:
    std::vector<bod_t> bods;
    long double G = 66'743e-15L;
    long double eps = 0, dt = 1, bh_theta = 3.14159265358979323846L / 3;
    uint64_t iterations = 1'000;
    long double time_elapsed{};
    uint64_t G_vals[6] = {1, 1, 1, 1, 1, 1};  // m_num, m_denom, d_num, d_denom, t_num, t_denom
    // memFreq energy records of the last evolve (gregsys.hpp:219-227), per body in body order
    std::vector<std::vector<T>> pe_rec, energy_rec;
    std::vector<T> tot_pe, tot_ke, tot_e;
    bool mixed = false;
    gtd_system *dev = nullptr;
    int device = 0;
    uint64_t callback_step_limit = 0;

    void parse_units_format(const std::string &str) {  // gregsys.hpp:245-282
        static const std::regex re{R"(^\s*(m|M)\s*(?=\d{1,18}\s*:)\d*[1-9]+\d*\s*:\s*(?=\d{1,18}\s*,)\d*[1-9]+\d*\s*,\s*(d|D)\s*(?=\d{1,18}\s*:)\d*[1-9]+\d*\s*:\s*(?=\d{1,18}\s*,)\d*[1-9]+\d*\s*,\s*(t|T)\s*(?=\d{1,18}\s*:)\d*[1-9]+\d*\s*:\s*(?=\d{1,18}\s*$)\d*[1-9]+\d*\s*$)"};
        if (!std::regex_match(str, re))
            throw std::invalid_argument{"The units_format string passed, \"" + str +
                                        "\", does not match the format required:\n\"Ma:b,Dc:x,Ty:z\", where "
                                        "'a', 'b', 'c', 'x', 'y', and 'z' represent any positive integer number of "
                                        "1-18 characters starting with at least one non-zero character.\n"};
        uint64_t v[6];
        int k = 0;
        static const std::regex digits{R"(\d+)"};
        for (std::sregex_iterator it{str.begin(), str.end(), digits}, end; it != end && k < 6; ++it)
            v[k++] = std::stoull(it->str());
        const uint64_t m_den = v[0], m_num = v[1], d_num = v[2], d_den = v[3], t_den = v[4], t_num = v[5];
        const uint64_t gv[6] = {m_num, m_den, d_num, d_den, t_num, t_den};  // gregsys.hpp:275-280
        std::memcpy(G_vals, gv, sizeof gv);
        G = 66'743;
        G *= m_num * d_num * d_num * d_num * t_num * t_num;
        G /= m_den * d_den * d_den * d_den * t_den * t_den;
        G /= 1'000'000'000'000'000;
    }
    void ensure_device() {
        if (!dev) {
            throw_status(gtd_system_create(&dev, device, mixed ? GTD_PREC_MIXED : GTD_PREC_F64));
            throw_status(gtd_system_set_recording(dev, memFreq));
        }
    }
    // The records the reference keeps (fileFreq = 0 is the only setting with which its evolve
    // compiles): FUNC_TEMPL_SELECT (gregsys.hpp:15-105) never takes its recording branch, so the
    // trajectories grow past their first element only through the collision pass (s_coll<true>);
    // energies come from calc_acc_and_e / calc_energy (every frame for Euler, modified Euler and
    // midpoint, the first only for the leapfrogs without collisions) and from the leapfrogs'
    // collision path, with each body's last recorded kinetic energy.  Barnes-Hut records nothing.
    void collect_recordings(int method) {
        pe_rec.clear();
        energy_rec.clear();
        tot_pe.clear();
        tot_ke.clear();
        tot_e.clear();
        int64_t frames = 0, n = 0;
        throw_status(gtd_system_recording(dev, &frames, &n, nullptr, nullptr));
        if (!frames || (method & barnes_hut) == barnes_hut || (size_t)n != bods.size()) return;
        std::vector<int64_t> states((size_t)frames);
        std::vector<double> fr((size_t)frames * (size_t)n * 8);
        throw_status(gtd_system_recording(dev, nullptr, nullptr, states.data(), fr.data()));
        int branch = 0;
        for (int b : {1, 2, 4, 8, 16, 32, 64, 128})
            if ((method & b) == b) { branch = b; break; }
        constexpr bool coll = collisions != 0;
        const int64_t n_e = (!coll && (branch == leapfrog_kdk || branch == leapfrog_dkd)) ? 1 : frames;
        pe_rec.assign((size_t)n, {});
        energy_rec.assign((size_t)n, {});
        for (int64_t k = 0; k < frames; ++k) {
            T tpe{}, tke{};
            for (int64_t i = 0; i < n; ++i) {
                const double *f = &fr[((size_t)k * n + i) * 8];
                bod_t &b = bods[(size_t)i];
                if (coll && k > 0) {
                    b.positions.push_back(vector3D<T>{(T)f[0], (T)f[1], (T)f[2]});
                    b.velocities.push_back(vector3D<T>{(T)f[3], (T)f[4], (T)f[5]});
                    b.curr_ke = f[6];
                    b.energies.push_back(b.curr_ke);
                }
                if (k < n_e) {
                    pe_rec[(size_t)i].push_back((T)f[7]);
                    energy_rec[(size_t)i].push_back((T)(b.curr_ke + f[7]));
                    tpe += (T)f[7];
                    tke += (T)b.curr_ke;
                }
            }
            if (k < n_e) {
                tot_pe.push_back(tpe);
                tot_ke.push_back(tke);
                tot_e.push_back(tpe + tke);
            }
        }
    }
    int coll_mode() const {
        if constexpr (collisions == overlap_coll_check) return mergeOverlappingBodies ? GTD_MERGE_COLL : GTD_OVERLAP_COLL;
        return GTD_NO_COLL;
    }
    void push() {
        ensure_device();
        const int64_t n = (int64_t)bods.size();
        std::vector<double> m(n), r(n), e(n), x(3 * n), v(3 * n);
        for (int64_t i = 0; i < n; ++i) {
            const bod_t &b = bods[i];
            m[i] = (double)b.mass_;
            r[i] = (double)b.radius;
            e[i] = (double)b.rest_c;
            x[3 * i] = (double)b.curr_pos.x; x[3 * i + 1] = (double)b.curr_pos.y; x[3 * i + 2] = (double)b.curr_pos.z;
            v[3 * i] = (double)b.curr_vel.x; v[3 * i + 1] = (double)b.curr_vel.y; v[3 * i + 2] = (double)b.curr_vel.z;
        }
        throw_status(gtd_system_set_params(dev, (double)G, (double)dt, iterations, (double)eps, (double)bh_theta));
        throw_status(gtd_system_set_collisions(dev, coll_mode()));
        throw_status(gtd_bh_set_tree_float(dev, std::is_same_v<T, float> ? 1 : 0));
        throw_status(gtd_system_upload(dev, n, m.data(), r.data(), e.data(), x.data(), v.data()));
    }
    void pull() {
        int64_t n = 0;
        throw_status(gtd_system_num_bodies(dev, &n));
        std::vector<double> m(n), r(n), e(n), x(3 * n), v(3 * n), a(3 * n);
        throw_status(gtd_system_download(dev, &n, m.data(), r.data(), e.data(), x.data(), v.data(), a.data()));
        if ((size_t)n < bods.size()) {
            // merges: the survivors (by upload index) keep their body objects and relative order
            std::vector<int64_t> idx(n);
            throw_status(gtd_system_survivors(dev, idx.data()));
            std::vector<bod_t> kept;
            kept.reserve(n);
            for (int64_t i = 0; i < n; ++i) kept.emplace_back(std::move(bods[(size_t)idx[i]]));
            bods.swap(kept);
        }
        for (int64_t i = 0; i < n; ++i) {
            bod_t &b = bods[i];
            b.mass_ = (M)m[i];
            b.radius = (R)r[i];
            b.rest_c = e[i];
            b.curr_pos = vector3D<T>{(T)x[3 * i], (T)x[3 * i + 1], (T)x[3 * i + 2]};
            b.curr_vel = vector3D<T>{(T)v[3 * i], (T)v[3 * i + 1], (T)v[3 * i + 2]};
            b.acc = vector3D<T>{(T)a[3 * i], (T)a[3 * i + 1], (T)a[3 * i + 2]};
        }
    }
    // A callback's writes to the body vector, sent back without restarting the evolve in progress.
    void update() {
        const int64_t n = (int64_t)bods.size();
        int64_t dn = 0;
        throw_status(gtd_system_num_bodies(dev, &dn));
        if (n != dn) throw std::logic_error{"an evolve callback changed the number of bodies"};
        std::vector<double> m(n), r(n), e(n), x(3 * n), v(3 * n);
        for (int64_t i = 0; i < n; ++i) {
            const bod_t &b = bods[i];
            m[i] = (double)b.mass_;
            r[i] = (double)b.radius;
            e[i] = (double)b.rest_c;
            x[3 * i] = (double)b.curr_pos.x; x[3 * i + 1] = (double)b.curr_pos.y; x[3 * i + 2] = (double)b.curr_pos.z;
            v[3 * i] = (double)b.curr_vel.x; v[3 * i + 1] = (double)b.curr_vel.y; v[3 * i + 2] = (double)b.curr_vel.z;
        }
        throw_status(gtd_system_update_bodies(dev, m.data(), r.data(), e.data(), x.data(), v.data()));
    }
    void check_dt() {
        if (dt <= 0) throw std::invalid_argument{"Time-step cannot be zero or negative.\n"};
    }

public:
    system() : G{G_SI} {}
    explicit system(long double timestep, uint64_t num_iterations, const char *units_format)
        : dt{timestep}, iterations{num_iterations} {
        check_dt();
        parse_units_format(units_format);
    }
    system(std::vector<bod_t> bodies, long double timestep = 1, uint64_t num_iterations = 1'000,
           const char *units_format = "M1:1,D1:1,T1:1", bool allow_overlapping_bodies = false)
        : bods{std::move(bodies)}, dt{timestep}, iterations{num_iterations} {
        check_dt();
        if (!allow_overlapping_bodies) check_overlap();
        parse_units_format(units_format);
    }
    system(const std::initializer_list<bod_t> &list) : bods{list}, G{G_SI} { check_overlap(); }
    // gregsys.hpp:1479-1490: the bodies, time, time-step and units of a .nsys file.  alloc_chunks
    // chose between two host read strategies in the reference; the engine always reads the chunks in
    // one piece and unpacks them on the device.
    explicit system(const char *nsys_path, bool alloc_chunks = true, bool check_nan_inf = true,
                    bool allow_overlapping_bodies = true) {
        static_assert(std::is_floating_point_v<M> && std::is_floating_point_v<R> && std::is_floating_point_v<T>,
                      "the engine reads .nsys files with floating-point M, R and T");
        (void)alloc_chunks;
        if (nsys_path == nullptr) throw std::invalid_argument{"nullptr passed as .nsys file path.\n"};
        ensure_device();
        double t_el = 0, step = 0, g = 0;
        throw_status(gtd_system_load_nsys(dev, nsys_path, check_nan_inf ? 1 : 0, (int)sizeof(M), (int)sizeof(R),
                                          (int)sizeof(T), &t_el, &step, G_vals, &g));
        (void)g;
        time_elapsed = t_el;
        dt = step;
        // G from the stored units in long double, as load_from_nsys does (gregsys.hpp:1281-1284)
        G = 66'743;
        G *= G_vals[0] * G_vals[2] * G_vals[2] * G_vals[2] * G_vals[4] * G_vals[4];
        G /= G_vals[1] * G_vals[3] * G_vals[3] * G_vals[3] * G_vals[5] * G_vals[5];
        G /= 1'000'000'000'000'000;
        int64_t n = 0;
        throw_status(gtd_system_num_bodies(dev, &n));
        std::vector<double> m(n), r(n), e(n), x(3 * n), v(3 * n);
        throw_status(gtd_system_download(dev, &n, m.data(), r.data(), e.data(), x.data(), v.data(), nullptr));
        bods.reserve((size_t)n);
        for (int64_t i = 0; i < n; ++i)
            bods.emplace_back((M)m[i], (R)r[i], (T)x[3 * i], (T)x[3 * i + 1], (T)x[3 * i + 2], (T)v[3 * i],
                              (T)v[3 * i + 1], (T)v[3 * i + 2], (long double)e[i]);
        if (!allow_overlapping_bodies) check_overlap();
    }
    system(const system &other) : bods{other.bods}, G{other.G}, eps{other.eps}, dt{other.dt},
                                  bh_theta{other.bh_theta}, iterations{other.iterations},
                                  time_elapsed{other.time_elapsed}, mixed{other.mixed} {
        std::memcpy(G_vals, other.G_vals, sizeof G_vals);
    }
    system &operator=(const system &) = delete;
    ~system() { gtd_system_destroy(dev); }

    // ---- check_overlap (gregsys.hpp:307-342) on the device --------------------------------------
    void check_overlap() {
        if (bods.size() < 2) return;
        push();
        int32_t pair[2] = {0, 0};
        throw_status(gtd_system_check_overlap(dev, mergeOverlappingBodies ? 1 : 0, pair));
        if constexpr (mergeOverlappingBodies) pull();
    }

    // ---- memFreq energy records of the last evolve (private in the reference; read here for
    // checks): per body (body order) potential and total energies, and the system totals -------------
    const std::vector<std::vector<T>> &recorded_pe() const noexcept { return pe_rec; }
    const std::vector<std::vector<T>> &recorded_energy() const noexcept { return energy_rec; }
    const std::vector<T> &recorded_total_pe() const noexcept { return tot_pe; }
    const std::vector<T> &recorded_total_ke() const noexcept { return tot_ke; }
    const std::vector<T> &recorded_total_e() const noexcept { return tot_e; }

    // ---- .nsys output (gregsys.hpp:3214-3258): returns the bytes written, 0 for a NULL path or a
    // file that cannot be opened ----------------------------------------------------------------------
    std::streamoff to_nsys(const char *path) const {
        static_assert(std::is_floating_point_v<M> && std::is_floating_point_v<R> && std::is_floating_point_v<T>,
                      "the engine writes .nsys files with floating-point M, R and T");
        if (path == nullptr) return 0;
        auto *self = const_cast<system *>(this);
        self->push();
        int64_t bytes = 0;
        throw_status(gtd_system_to_nsys(dev, path, (double)time_elapsed, (double)dt, G_vals, (int)sizeof(M),
                                        (int)sizeof(R), (int)sizeof(T), &bytes));
        return (std::streamoff)bytes;
    }
    // Extension: the snapshot is taken on the device now and written to the file by a host thread,
    // so the next evolve() overlaps the write; nsys_wait() returns the last file's size.
    void to_nsys_async(const char *path) const {
        static_assert(std::is_floating_point_v<M> && std::is_floating_point_v<R> && std::is_floating_point_v<T>,
                      "the engine writes .nsys files with floating-point M, R and T");
        if (path == nullptr) return;
        auto *self = const_cast<system *>(this);
        self->push();
        throw_status(gtd_system_to_nsys_async(dev, path, (double)time_elapsed, (double)dt, G_vals, (int)sizeof(M),
                                              (int)sizeof(R), (int)sizeof(T)));
    }
    std::streamoff nsys_wait() const {
        int64_t bytes = 0;
        if (dev) throw_status(gtd_system_nsys_wait(dev, &bytes));
        return (std::streamoff)bytes;
    }

    // ---- accessors and setters (gregsys.hpp:1627-1672) ------------------------------------------
    typename std::vector<bod_t>::size_type num_bodies() const noexcept { return bods.size(); }
    long double elapsed_time() const noexcept { return time_elapsed; }
    long double G_val() const noexcept { return G; }
    bool set_iterations(uint64_t number) noexcept {
        if (!number) return false;
        iterations = number;
        return true;
    }
    bool set_timestep(const long double &delta_t) noexcept {
        if (delta_t <= 0) return false;
        dt = delta_t;
        return true;
    }
    void set_G_units(const char *units_format) { parse_units_format(units_format); }
    bool set_softening(long double e) noexcept {
        if (e < sqrtl(std::numeric_limits<long double>::min())) return false;
        eps = e;
        return true;
    }
    bool set_bh_opening_angle(long double theta) {
        if (theta < 0 || theta >= 3.14159265358979323846L) return false;
        bh_theta = theta;
        return true;
    }
    // Engine extension: FP32 pair forces with FP64 Kahan sums (true) or FP64 throughout (false).
    void use_mixed_precision(bool on) {
        if (on != mixed) {
            gtd_system_destroy(dev);
            dev = nullptr;
            mixed = on;
        }
    }
    void set_device(int d) {
        gtd_system_destroy(dev);
        dev = nullptr;
        device = d;
    }

    system &add_body(const bod_t &b, bool chk_overlap = true) {
        bods.emplace_back(b);
        if (chk_overlap) check_overlap();
        return *this;
    }
    template <typename... Args>
    system &emplace_body(bool chk_overlap, Args &&...args) {
        bods.emplace_back(std::forward<Args>(args)...);
        if (chk_overlap) check_overlap();
        return *this;
    }
    system &add_bodies(const std::vector<bod_t> &bodies, bool chk_overlap = true) {
        bods.insert(bods.end(), bodies.begin(), bodies.end());
        if (chk_overlap) check_overlap();
        return *this;
    }
    bool remove_body(uint64_t id) {
        for (auto it = bods.begin(); it != bods.end(); ++it)
            if (it->get_id() == id) {
                bods.erase(it);
                return true;
            }
        return false;
    }
    const bod_t &get_body(uint64_t id) const {
        for (const auto &b : bods)
            if (b.get_id() == id) return b;
        throw std::invalid_argument("The id passed does not correspond to any body present in this system object.\n");
    }
    const bod_t &front() const {
        if (bods.empty()) throw std::logic_error{"gtd::system<>::front cannot be called on an empty gtd::system object.\n"};
        return bods.front();
    }
    const bod_t &back() const {
        if (bods.empty()) throw std::logic_error{"gtd::system<>::back cannot be called on an empty gtd::system object.\n"};
        return bods.back();
    }
    const bod_t &operator[](typename std::vector<bod_t>::size_type i) const { return bods[i]; }
    auto begin() { return bods.begin(); }
    auto end() { return bods.end(); }
    auto begin() const { return bods.cbegin(); }
    auto end() const { return bods.cend(); }

    // ---- evolve (gregsys.hpp:2593-3071) -----------------------------------------------------------
    // Callbacks are either host callables (the reference's contract: they see the body vector; the
    // state makes a host round trip per step) or device callbacks (gtd::device::*: GPU work, the
    // bodies stay on the device and the predicate is evaluated there).  The two kinds cannot mix.
    template <typename evFuncT = std::nullptr_t, typename bodFuncT = std::nullptr_t,
              typename bodsFuncT = std::nullptr_t>
        requires(std::same_as<evFuncT, std::nullptr_t> || device::is_callback<evFuncT>::value ||
                 requires(evFuncT f) { { f() } -> std::same_as<bool>; }) &&
                (std::same_as<bodFuncT, std::nullptr_t> || device::is_callback<bodFuncT>::value ||
                 requires(bodFuncT f, bod_t &b) { { f(b) } -> std::same_as<void>; }) &&
                (std::same_as<bodsFuncT, std::nullptr_t> || device::is_callback<bodsFuncT>::value ||
                 requires(bodsFuncT f, std::vector<bod_t> &v) { { f(v) } -> std::same_as<void>; })
    const std::chrono::nanoseconds evolve(int integration_method = leapfrog_kdk,
                                          const evFuncT &continue_ev_if = nullptr,
                                          const bodFuncT &for_each_bod = nullptr,
                                          const bodsFuncT &for_all_bods = nullptr) {
        if (bods.empty()) return std::chrono::nanoseconds::zero();
        constexpr bool no_cb = std::same_as<evFuncT, std::nullptr_t> && std::same_as<bodFuncT, std::nullptr_t> &&
                               std::same_as<bodsFuncT, std::nullptr_t>;
        constexpr bool dev_cb = device::is_callback<evFuncT>::value || device::is_callback<bodFuncT>::value ||
                                device::is_callback<bodsFuncT>::value;
        if constexpr (memFreq != 0)
            for (bod_t &b : bods) b.clear_trajectory();  // clear_evolution (gregsys.hpp:2569-2586)
        push();
        if constexpr (no_cb) {
            int64_t ns = 0;
            throw_status(gtd_system_evolve(dev, integration_method, &ns));
            pull();
            if constexpr (memFreq != 0) collect_recordings(integration_method);
            time_elapsed = iterations * dt;
            return std::chrono::nanoseconds{ns};
        } else if constexpr (dev_cb) {
            static_assert((std::same_as<evFuncT, std::nullptr_t> || device::is_callback<evFuncT>::value) &&
                              (std::same_as<bodFuncT, std::nullptr_t> || device::is_callback<bodFuncT>::value) &&
                              (std::same_as<bodsFuncT, std::nullptr_t> || device::is_callback<bodsFuncT>::value),
                          "device callbacks and host callables cannot be mixed in one evolve");
            gtd_device_hook cf = nullptr, ef = nullptr, af = nullptr;
            void *cu = nullptr, *eu = nullptr, *au = nullptr;
            if constexpr (std::same_as<evFuncT, device::hook>) { cf = continue_ev_if.fn; cu = continue_ev_if.user; }
            if constexpr (std::same_as<bodFuncT, device::hook>) { ef = for_each_bod.fn; eu = for_each_bod.user; }
            if constexpr (std::same_as<bodsFuncT, device::hook>) { af = for_all_bods.fn; au = for_all_bods.user; }
            throw_status(gtd_system_set_device_callbacks(dev, cf, cu, ef, eu, af, au));
            if constexpr (std::same_as<evFuncT, device::while_rest_below>)
                throw_status(gtd_system_set_continue_while_rest_below(dev, (double)continue_ev_if.min_max_cor,
                                                                      continue_ev_if.probing_iters));
            if constexpr (device::is_rest_from_com<bodsFuncT>::value) {
                const double c[3] = {(double)for_all_bods.com->x, (double)for_all_bods.com->y,
                                     (double)for_all_bods.com->z};
                throw_status(gtd_system_set_rest_from_com(dev, (double)for_all_bods.min_cor, (double)for_all_bods.max_cor,
                                                          (double)for_all_bods.scale_factor, (double)for_all_bods.n_exp,
                                                          c, for_all_bods.mass_weighted ? 1 : 0));
            }
            uint64_t steps = 0;
            int64_t ns = 0;
            throw_status(gtd_system_evolve_callbacks(dev, integration_method, callback_step_limit, &steps, &ns));
            pull();
            if constexpr (memFreq != 0) collect_recordings(integration_method);
            if constexpr (device::is_rest_from_com<bodsFuncT>::value) {
                double c[3];
                throw_status(gtd_system_rest_from_com_centre(dev, c));
                for_all_bods.com->x = c[0];
                for_all_bods.com->y = c[1];
                for_all_bods.com->z = c[2];
            }
            throw_status(gtd_system_set_device_callbacks(dev, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr));
            time_elapsed = iterations * dt;  // gregsys.hpp:3069, whatever the steps taken
            return std::chrono::nanoseconds{ns};
        } else {
            // host callables see the bodies every step: the state makes a host round trip for them.
            // Order per step (gregsys.hpp:16-106, 2970-2987): continue_ev_if, the update, for_all_bods
            // (inside the step, before the collision pass), the collision pass, for_each_bod.
            const auto start = std::chrono::steady_clock::now();
            if ((integration_method & barnes_hut) == barnes_hut) {  // this branch calls no callback
                int64_t ns = 0;
                throw_status(gtd_system_evolve(dev, integration_method, &ns));
                pull();
                if constexpr (memFreq != 0) collect_recordings(integration_method);
                time_elapsed = iterations * dt;
                return std::chrono::nanoseconds{ns};
            }
            struct hook_ctx {
                system *self;
                const bodsFuncT *all;
                std::exception_ptr err;
            } ctx{this, &for_all_bods, nullptr};
            struct unhook {
                gtd_system *d;
                ~unhook() { gtd_system_set_step_hook(d, nullptr, nullptr); }
            } guard{dev};
            if constexpr (!std::same_as<bodsFuncT, std::nullptr_t>) {
                throw_status(gtd_system_set_step_hook(dev, +[](void *u) -> int {
                    auto *c = static_cast<hook_ctx *>(u);
                    try {
                        c->self->pull();
                        (*c->all)(c->self->bods);
                        c->self->update();
                        return 0;
                    } catch (...) {
                        c->err = std::current_exception();
                        return GTD_ERR_CALLBACK;
                    }
                }, &ctx));
            }
            throw_status(gtd_system_evolve_begin(dev, integration_method));
            uint64_t steps = 0;
            while (true) {
                if constexpr (std::same_as<evFuncT, std::nullptr_t>) {
                    if (steps >= iterations) break;
                } else {
                    if (!continue_ev_if()) break;
                }
                const int rc = gtd_system_evolve_steps(dev, 1);
                if (ctx.err) std::rethrow_exception(ctx.err);
                throw_status(rc);
                ++steps;
                if constexpr (!std::same_as<bodFuncT, std::nullptr_t>) {
                    pull();
                    for (bod_t &b : bods) for_each_bod(b);
                    update();
                }
            }
            pull();
            if constexpr (memFreq != 0) collect_recordings(integration_method);
            time_elapsed = iterations * dt;  // gregsys.hpp:3069, whatever the steps taken
            return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - start);
        }
    }
    // Guard for device-callback evolves whose predicate might never turn false (0: none).
    void set_callback_step_limit(uint64_t max_steps) noexcept { callback_step_limit = max_steps; }
};

typedef system<long double, long double, long double> sys;
typedef system<long double, long double, long double, false, false, 3> sys_c;
typedef system<long double, long double, long double, false, true> sys_m;
typedef system<long double, long double, long double, false, true, 3> sys_mc;
typedef system<long double, long double, long double, false, false, 0, 0, 0, false> sys_n;
typedef system<long double, long double, long double, false, false, 3, 0, 0, false> sys_c_n;
typedef system<long double, long double, long double, false, true, 0, 0, 0, false> sys_m_n;

}  // namespace gtd
#endif
