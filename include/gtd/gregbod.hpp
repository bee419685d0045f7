// Drop-in gtd::vector3D / gtd::body for code written against GregW10/GregPackagesCPP's gtd::
// N-body API (gregvec.hpp, gregbod.hpp), backed by the B200 engine (gtd_b200.h).  Only the parts
// of those headers the force-and-step path and its callers use are provided; names, template
// parameters, accessors and exception types match the reference.
#ifndef GTD_B200_GREGBOD_HPP
#define GTD_B200_GREGBOD_HPP

#include <atomic>
#include <cmath>
#include <cstdint>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../gtd_b200.h"

namespace gtd {

template <typename T>
concept isNumWrapper = std::is_arithmetic_v<T>;

// ---- exceptions (gregbod.hpp:19-90, greg8tree.hpp:11-46) ------------------------------------------
class nbody_error : public std::logic_error {
public:
    nbody_error() : std::logic_error{"Error with N-body simulation.\n"} {}
    explicit nbody_error(const char *msg) : std::logic_error{msg} {}
};
class overlapping_bodies_error : public nbody_error {
public:
    overlapping_bodies_error() : nbody_error{"Bodies added to the system overlap.\n"} {}
    explicit overlapping_bodies_error(const char *msg) : nbody_error{msg} {}
};
class negative_mass_error : public nbody_error {
public:
    negative_mass_error() : nbody_error{"A body cannot have a negative mass.\n"} {}
    explicit negative_mass_error(const char *msg) : nbody_error{msg} {}
};
class negative_radius_error : public nbody_error {
public:
    negative_radius_error() : nbody_error{"A body cannot have a negative radius.\n"} {}
    explicit negative_radius_error(const char *msg) : nbody_error{msg} {}
};
class two_body_error : public nbody_error {
public:
    two_body_error() : nbody_error{"Two-body integration requires exactly two bodies.\n"} {}
    explicit two_body_error(const char *msg) : nbody_error{msg} {}
};
class empty_system_error : public nbody_error {
public:
    using nbody_error::nbody_error;
};
class no_evolution_error : public nbody_error {
public:
    using nbody_error::nbody_error;
};
class barnes_hut_error : public nbody_error {
public:
    using nbody_error::nbody_error;
    barnes_hut_error() : nbody_error{"An error occurred with the creation and/or usage of a gtd::bh_cube<> object.\n"} {}
};
class invalid_body_placement : public barnes_hut_error {
public:
    using barnes_hut_error::barnes_hut_error;
};
class indistinguishable_bodies : public barnes_hut_error {
public:
    using barnes_hut_error::barnes_hut_error;
};
class nsys_load_error : public nbody_error {  // gregsys.hpp:125-129
public:
    nsys_load_error() : nbody_error{"Error loading N-body data from .nsys file.\n"} {}
    explicit nsys_load_error(const char *msg) : nbody_error{msg} {}
};
class nsys_format_error : public nsys_load_error {  // gregsys.hpp:130-134
public:
    nsys_format_error() : nsys_load_error{"Error loading N-body data from .nsys file.\n"} {}
    explicit nsys_format_error(const char *msg) : nsys_load_error{msg} {}
};

// a CUDA / resource failure of the engine itself (no counterpart: the reference runs on the host)
class device_error : public std::runtime_error {
public:
    explicit device_error(const char *msg) : std::runtime_error{msg} {}
};

// Maps a C ABI status onto the reference's exception types.
inline void throw_status(int rc) {
    if (rc == GTD_OK) return;
    const char *m = gtd_last_error();
    switch (rc) {
        case GTD_ERR_INVALID_ARGUMENT: throw std::invalid_argument{m};
        case GTD_ERR_OVERLAPPING_BODIES: throw overlapping_bodies_error{m};
        case GTD_ERR_INVALID_BODY_PLACEMENT: throw invalid_body_placement{m};
        case GTD_ERR_INDISTINGUISHABLE: throw indistinguishable_bodies{m};
        case GTD_ERR_TWO_BODY: throw two_body_error{m};
        case GTD_ERR_NSYS_LOAD: throw nsys_load_error{m};
        case GTD_ERR_NSYS_FORMAT: throw nsys_format_error{m};
        default: throw device_error{m};
    }
}

// ---- vector3D (the subset of gregvec.hpp the path uses) -----------------------------------------
template <isNumWrapper T>
class vector3D {
public:
    T x{}, y{}, z{};
    vector3D() = default;
    vector3D(T x_, T y_, T z_) : x{x_}, y{y_}, z{z_} {}
    template <isNumWrapper U>
    vector3D(const vector3D<U> &o) : x(o.x), y(o.y), z(o.z) {}
    const T &get_x() const noexcept { return x; }
    const T &get_y() const noexcept { return y; }
    const T &get_z() const noexcept { return z; }
    long double magnitude() const noexcept {  // gregvec.hpp:2069-2073
        return sqrtl((long double)x * x + (long double)y * y + (long double)z * z);
    }
    template <isNumWrapper U, isNumWrapper V>
    bool between(const vector3D<U> &lo, const vector3D<V> &hi) const noexcept {  // gregvec.hpp:2115-2120
        return lo.x <= x && x < hi.x && lo.y <= y && y < hi.y && lo.z <= z && z < hi.z;
    }
    void make_zero() noexcept { x = y = z = T{}; }
    template <isNumWrapper U>
    vector3D &operator+=(const vector3D<U> &o) noexcept { x += o.x; y += o.y; z += o.z; return *this; }
    template <isNumWrapper U>
    vector3D &operator-=(const vector3D<U> &o) noexcept { x -= o.x; y -= o.y; z -= o.z; return *this; }
    T &operator[](unsigned char i) { return i == 0 ? x : (i == 1 ? y : z); }
    const T &operator[](unsigned char i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <isNumWrapper U, isNumWrapper V>
auto operator+(const vector3D<U> &a, const vector3D<V> &b) -> vector3D<decltype(a.x + b.x)> {
    return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <isNumWrapper U, isNumWrapper V>
auto operator-(const vector3D<U> &a, const vector3D<V> &b) -> vector3D<decltype(a.x - b.x)> {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <isNumWrapper U, isNumWrapper V>
auto operator*(const vector3D<U> &a, const vector3D<V> &b) -> decltype(a.x * b.x) {  // dot, gregvec.hpp:3742-3744
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <isNumWrapper U, isNumWrapper V>
auto operator*(const V &s, const vector3D<U> &a) -> vector3D<decltype(s * a.x)> {
    return {s * a.x, s * a.y, s * a.z};
}
template <isNumWrapper U, isNumWrapper V>
auto operator*(const vector3D<U> &a, const V &s) -> vector3D<decltype(a.x * s)> {
    return {a.x * s, a.y * s, a.z * s};
}
template <isNumWrapper U, isNumWrapper V>
auto operator/(const vector3D<U> &a, const V &s) -> vector3D<decltype(a.x / s)> {
    return {a.x / s, a.y / s, a.z / s};
}
template <isNumWrapper U>
std::ostream &operator<<(std::ostream &os, const vector3D<U> &v) {
    return os << +v.x << "i + " << +v.y << "j + " << +v.z << "k";
}
namespace vec_ops {
template <isNumWrapper U, isNumWrapper V>
auto distance(const vector3D<U> &a, const vector3D<V> &b) {  // gregvec.hpp:4701-4706
    auto dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
    return sqrtl(dx * dx + dy * dy + dz * dz);
}
}  // namespace vec_ops

// ---- body (gregbod.hpp:269-1084, history recording omitted: recFreq is accepted and ignored) ------
class body_counter {
    static inline std::atomic<uint64_t> next_id{0};

protected:
    uint64_t id;

public:
    body_counter() : id{next_id++} {}
    body_counter(const body_counter &) : id{next_id++} {}
    body_counter &operator=(const body_counter &) { return *this; }
    uint64_t get_id() const noexcept { return id; }
    virtual ~body_counter() = default;
};

template <isNumWrapper M, isNumWrapper R, isNumWrapper T, bool prog, bool merge, int coll, uint64_t mF,
          uint64_t fF, bool bin>
class system;
template <isNumWrapper, isNumWrapper, isNumWrapper, uint64_t>
class bh_tree;

template <isNumWrapper M = long double, isNumWrapper R = long double, isNumWrapper T = long double,
          uint64_t recFreq = 0>
class body : public body_counter {
public:
    using K = decltype(M{} * T{} * T{});  // kinetic energy type

private:
    M mass_{1};
    R radius{1};
    vector3D<T> curr_pos{}, curr_vel{}, acc{};
    long double rest_c{1};
    K curr_ke{};  // kinetic energy as last recorded (gregbod.hpp:299, 325-328)
    // trajectory (recFreq != 0; gregbod.hpp:304-306): the first element is the state at construction
    std::vector<vector3D<T>> positions, velocities;
    std::vector<K> energies;
    void check() const {
        if (mass_ < M{0}) throw negative_mass_error{};
        if (radius < R{0}) throw negative_radius_error{};
    }
    void set_ke() {
        const auto mag = curr_vel.magnitude();
        curr_ke = 0.5 * mass_ * mag * mag;
    }
    void add_pos_vel_ke() {
        if constexpr (recFreq != 0) {
            set_ke();
            positions.push_back(curr_pos);
            velocities.push_back(curr_vel);
            energies.push_back(curr_ke);
        }
    }
    void clear_trajectory() {  // body::clear (gregbod.hpp:621-628): the current state, ke not recomputed
        positions.assign(1, curr_pos);
        velocities.assign(1, curr_vel);
        energies.assign(1, curr_ke);
    }

public:
    body() { add_pos_vel_ke(); }
    body(const M &m, const R &r) : mass_{m}, radius{r} {
        check();
        add_pos_vel_ke();
    }
    body(const M &m, const R &r, const vector3D<T> &pos, const vector3D<T> &vel, long double restitution = 1)
        : mass_{m}, radius{r}, curr_pos{pos}, curr_vel{vel}, rest_c{restitution} {
        check();
        add_pos_vel_ke();
    }
    body(const M &m, const R &r, const T &x, const T &y, const T &z, const T &vx, const T &vy, const T &vz,
         long double restitution = 1)
        : mass_{m}, radius{r}, curr_pos{x, y, z}, curr_vel{vx, vy, vz}, rest_c{restitution} {
        check();
        add_pos_vel_ke();
    }
    const std::vector<vector3D<T>> &get_positions() const { return positions; }
    const std::vector<vector3D<T>> &get_velocities() const { return velocities; }
    const std::vector<K> &get_kinetic_energies() const { return energies; }
    const M &mass() const noexcept { return mass_; }
    const R &rad() const noexcept { return radius; }
    const vector3D<T> &pos() const noexcept { return curr_pos; }
    const vector3D<T> &vel() const noexcept { return curr_vel; }
    vector3D<T> &acceleration() noexcept { return acc; }
    const vector3D<T> &acceleration() const noexcept { return acc; }
    long double restitution() const noexcept { return rest_c; }
    auto momentum() const { return mass_ * curr_vel; }  // gregbod.hpp:595-597
    long double ke() const { auto mg = curr_vel.magnitude(); return 0.5L * mass_ * mg * mg; }
    bool set_mass(const M &m) { if (m < 0) return false; mass_ = m; return true; }
    bool set_radius(const R &r) { if (r < 0) return false; radius = r; return true; }
    void set_acc(const vector3D<T> &a) { acc = a; }
    bool set_restitution(long double e) noexcept { if (e < 0 || e > 1) return false; rest_c = e; return true; }
    void update(const vector3D<T> &p, const vector3D<T> &v) noexcept { curr_pos = p; curr_vel = v; }
    void shift(const vector3D<T> &dp, const vector3D<T> &dv) noexcept { curr_pos += dp; curr_vel += dv; }
    void reset_acc() { acc.make_zero(); }
    template <isNumWrapper m, isNumWrapper r, isNumWrapper t, bool p, bool mg, int c, uint64_t a, uint64_t b, bool d>
    friend class system;
    template <isNumWrapper, isNumWrapper, isNumWrapper, uint64_t>
    friend class bh_tree;
};

template <isNumWrapper M, isNumWrapper R, isNumWrapper T, uint64_t rF>
std::ostream &operator<<(std::ostream &os, const body<M, R, T, rF> &b) {
    return os << "[gtd::body:id=" << b.get_id() << ",m=" << +b.mass() << ",r=" << +b.rad() << ",current_pos=("
              << b.pos() << "),current_vel=(" << b.vel() << ")]";
}

typedef body<long double, long double, long double, 0> bod_0f;

}  // namespace gtd
#endif
