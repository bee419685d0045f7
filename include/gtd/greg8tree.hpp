// Drop-in gtd::bh_tree and gtd::bh_cube (GregW10/GregPackagesCPP greg8tree.hpp:48-968, 984-1118)
// over the B200 linear octree (gtd_b200.h).  add_bodies builds the tree on the device with the
// reference's root box, octant splits and (for T = float) float geometry; the tree is read back as
// its pre-order node list and rebuilt on the host as linked bh_cube cells, so that code written
// against the reference walks it with the reference's iterators (begin/end over leaves,
// cell_iterator, nn_iterator) and accessors (cube_mass, cube_com, find_leaf, operator[]).
// bh_tree::accelerations runs the reference walk (cell_iterator, greg8tree.hpp:702-833) for every
// body on the device.
#ifndef GTD_B200_GREG8TREE_HPP
#define GTD_B200_GREG8TREE_HPP

#include <cstdint>
#include <stdexcept>
#include <vector>

#include "gregbod.hpp"

namespace gtd {

template <isNumWrapper M, isNumWrapper R, isNumWrapper T, uint64_t rF>
class bh_tree;

// The reference's pi (gregalg.hpp:122), which bounds the opening angle.
inline constexpr long double kBhPi = 3.14159265358979323846264338327950288419716939937510582097494459230L;

// One cell of the octree (greg8tree.hpp:48-968).  The cells of a tree live in one array in DFS
// pre-order (children in octant order 0..7: bit 0 = x, bit 1 = y, bit 2 = z above the split),
// each knowing its position in that order and the position after its subtree, which is what the
// iterators step by; _sub and parent keep the reference's links.
template <isNumWrapper M = long double, isNumWrapper R = long double, isNumWrapper T = long double,
          uint64_t rF = 0>
class bh_cube {
public:
    using bod_t = body<M, R, T, rF>;
    using vec = vector3D<T>;
    using cube_t = bh_cube<M, R, T, rF>;

private:
    vec _btm{}, _top{}, _com{};
    M _mass{};
    const bod_t *_bod = nullptr;  // the body of a leaf, else nullptr
    cube_t *parent = nullptr;
    cube_t *_sub[8]{};
    const std::vector<cube_t> *_all = nullptr;  // every cell of the tree, in pre-order
    int64_t _index = 0, _skip = 0;              // position in _all, and the position after the subtree

    // set_corners (greg8tree.hpp:81-131): the bounds of child octant `oct`, split at (btm + top) / 2
    // computed in T.
    void child_box(unsigned oct, vec &btm, vec &top) const {
        const T half_x = (_btm.x + _top.x) / 2.0l, half_y = (_btm.y + _top.y) / 2.0l, half_z = (_btm.z + _top.z) / 2.0l;
        btm = vec{(oct & 1) ? half_x : _btm.x, (oct & 2) ? half_y : _btm.y, (oct & 4) ? half_z : _btm.z};
        top = vec{(oct & 1) ? _top.x : half_x, (oct & 2) ? _top.y : half_y, (oct & 4) ? _top.z : half_z};
    }
    const cube_t *at(int64_t k) const { return k < (int64_t)_all->size() ? &(*_all)[(size_t)k] : nullptr; }

public:
    const bod_t *get_body() const noexcept { return _bod; }
    cube_t *root() noexcept {
        cube_t *c = this;
        while (c->parent) c = c->parent;
        return c;
    }
    // bh_cube::find_leaf (greg8tree.hpp:859-877): the leaf below this cell whose cell holds pos
    // (between: btm <= pos < top), or nullptr.
    cube_t *find_leaf(const vec &pos) {
        cube_t *c = this;
        for (unsigned i = 0; i < 8;) {
            cube_t *s = c->_sub[i];
            if (s && pos.between(s->_btm, s->_top)) {
                if (s->_bod) return s;
                c = s;
                i = 0;
                continue;
            }
            ++i;
        }
        return nullptr;
    }
    M cube_mass() const { return _mass; }          // greg8tree.hpp:910-912
    vec cube_com() const noexcept { return _com; }  // greg8tree.hpp:913-916 (FP64 moments, rounded to T)
    vec bottom() const noexcept { return _btm; }
    vec top() const noexcept { return _top; }
    const cube_t &operator[](unsigned char index) const {  // greg8tree.hpp:961-968
        if (index > 7)
            throw std::invalid_argument{"gtd::bh_cube<M, R, T, rF>::operator[] error: index cannot be greater than "
                                        "7.\n"};
        if (_sub[index] == nullptr) throw std::invalid_argument{"Error: no gtd::bh_cube<> at index specified.\n"};
        return *_sub[index];
    }

    // greg8tree.hpp:472-501: points at a leaf; dereferences to its body.
    class body_iterator {
    protected:
        const cube_t *_cptr = nullptr;

    public:
        body_iterator() = default;
        explicit body_iterator(const cube_t *c) : _cptr{c} {}
        const bod_t &operator*() const { return *_cptr->_bod; }
        const bod_t *operator->() const { return _cptr->_bod; }
        bool operator==(const body_iterator &o) const noexcept { return _cptr == o._cptr; }
        bool operator!=(const body_iterator &o) const noexcept { return _cptr != o._cptr; }
        const cube_t *cube() const noexcept { return _cptr; }  // the leaf pointed at
    };

    // bh_cube::iterator (greg8tree.hpp:502-614): the leaves below a cell in DFS octant order; the
    // end iterator points at no cell.
    class iterator : public body_iterator {
        using body_iterator::_cptr;
        const cube_t *_root = nullptr;
        void first_leaf_from(int64_t k) {
            const int64_t stop = _root->_skip;
            while (k < stop && !_root->at(k)->_bod) ++k;
            _cptr = k < stop ? _root->at(k) : nullptr;
        }

    public:
        iterator() = default;
        iterator(const cube_t *root, bool is_end = false) : _root{root} {
            if (root == nullptr) throw std::invalid_argument{"Error: nullptr passed as root cube.\n"};
            if (is_end) {
                _cptr = nullptr;
                return;
            }
            first_leaf_from(root->_index);
        }
        iterator &operator++() {
            if (_cptr) first_leaf_from(_cptr->_index + 1);
            return *this;
        }
        iterator operator++(int) {
            iterator c = *this;
            ++*this;
            return c;
        }
        explicit operator bool() const noexcept { return _cptr != nullptr && _cptr->_bod != nullptr; }
    };

    // bh_cube::nn_iterator (greg8tree.hpp:615-701): the leaves whose cells touch the cell of the
    // given body's leaf (closed bounds), the leaf itself excluded, in DFS order from the root's
    // children; converts to false at the end.
    class nn_iterator : public body_iterator {
        using body_iterator::_cptr;
        const cube_t *_bc = nullptr;
        int64_t _next = 0;
        bool touches(const cube_t *c) const noexcept {
            return !(_bc->_top.x < c->_btm.x || _bc->_btm.x > c->_top.x || _bc->_top.y < c->_btm.y ||
                     _bc->_btm.y > c->_top.y || _bc->_top.z < c->_btm.z || _bc->_btm.z > c->_top.z);
        }
        void find_from(int64_t k) {
            const int64_t n = (int64_t)_bc->_all->size();
            while (k < n) {
                const cube_t *c = _bc->at(k);
                if (c != _bc && touches(c)) {
                    if (c->_bod) {
                        _cptr = c;
                        _next = c->_skip;
                        return;
                    }
                    ++k;  // a touching cell: descend
                    continue;
                }
                k = c->_skip;
            }
            _cptr = _bc;
        }

    public:
        nn_iterator(const body_iterator &body_it, bool is_end = false) : body_iterator{body_it.cube()}, _bc{body_it.cube()} {
            if (_bc == nullptr || _bc->_bod == nullptr)
                throw std::invalid_argument{"Error: body iterator does not contain a pointer to a valid "
                                            "body-containing gtd::bh_cube<> object.\n"};
            if (_bc->parent == nullptr || is_end) return;  // a one-body tree has no neighbours
            find_from(1);
        }
        bool has_body() const noexcept { return _cptr != _bc; }
        explicit operator bool() const noexcept { return _cptr != _bc; }
        nn_iterator &operator++() {
            if (_cptr != _bc) find_from(_next);
            return *this;
        }
        nn_iterator operator++(int) {
            nn_iterator c = *this;
            ++*this;
            return c;
        }
    };

    // bh_cube::cell_iterator (greg8tree.hpp:702-833): the cells one body's force is summed over -
    // from the root's children in DFS order, every leaf but the body's own and every cell with
    // (top.x - btm.x) / |x - com| < theta, whose subtree is then skipped; others are opened.
    // Converts to false at the end.
    class cell_iterator {
        const cube_t *_bc = nullptr, *_root = nullptr, *_cptr = nullptr;
        int64_t _next = 0;
        vec _bpos{};
        long double _theta;
        bool is_source_cell(const cube_t *c) const {
            return (c->_top.x - c->_btm.x) / vec_ops::distance(_bpos, c->_com) < _theta;
        }
        void check() const {
            if (_root == nullptr) throw std::invalid_argument{"Error: root cube passed is nullptr.\n"};
            if (_root->parent != nullptr)
                throw std::invalid_argument{"Error: root cube supplied is not root, as parent is not nullptr.\n"};
            if (_theta >= kBhPi || _theta < 0)
                throw std::invalid_argument{"Error: opening angle cannot be negative or equal to or larger than PI "
                                            "radians.\n"};
        }
        void find_from(int64_t k) {
            const int64_t n = (int64_t)_root->_all->size();
            while (k < n) {
                const cube_t *c = _root->at(k);
                if (c == _bc) {
                    k = c->_skip;
                    continue;
                }
                if (c->_bod || is_source_cell(c)) {
                    _cptr = c;
                    _next = c->_skip;
                    return;
                }
                ++k;  // opened: its children come next in pre-order
            }
            _cptr = _bc;
        }

    public:
        explicit cell_iterator(long double opening_angle) : _theta{opening_angle} {
            if (_theta >= kBhPi || _theta < 0)
                throw std::invalid_argument{"Error: opening angle cannot be negative or equal to or larger than PI "
                                            "radians.\n"};
        }
        cell_iterator(const cube_t *root, const body_iterator &body_it, long double opening_angle)
            : _bc{body_it.cube()}, _root{root}, _cptr{body_it.cube()}, _theta{opening_angle} {
            check();
            if (_bc == nullptr || _bc->_bod == nullptr)
                throw std::invalid_argument{"Error: iterator passed does not point to a body-containing cell.\n"};
            _bpos = _bc->_bod->pos();
            if (!_bpos.between(_root->_btm, _root->_top))
                throw invalid_body_placement{"Error: particle does not lie within root cell.\n"};
            find_from(1);
        }
        cell_iterator(const cube_t *root, const vec &particle_pos, long double opening_angle)
            : _root{root}, _bpos{particle_pos}, _theta{opening_angle} {
            check();
            if ((_bc = const_cast<cube_t *>(root)->find_leaf(particle_pos)) == nullptr)
                throw invalid_body_placement{"Error: particle does not lie within root cell.\n"};
            _cptr = _bc;
            find_from(1);
        }
        cell_iterator(const body_iterator &body_it, long double opening_angle)
            : cell_iterator{const_cast<cube_t *>(body_it.cube())->root(), body_it, opening_angle} {}
        cell_iterator &operator++() {
            if (_cptr != _bc) find_from(_next);
            return *this;
        }
        cell_iterator operator++(int) {
            cell_iterator c = *this;
            ++*this;
            return c;
        }
        const cube_t &operator*() const noexcept { return *_cptr; }
        const cube_t *operator->() const noexcept { return _cptr; }
        explicit operator bool() const noexcept { return _cptr != _bc; }
    };

    friend class bh_tree<M, R, T, rF>;
};

template <isNumWrapper M = long double, isNumWrapper R = long double, isNumWrapper T = long double, uint64_t rF = 0>
class bh_tree {
public:
    using bod_t = body<M, R, T, rF>;
    using vec = vector3D<T>;
    using cube_t = bh_cube<M, R, T, rF>;
    struct node {  // one cell of the octree, in DFS pre-order (children in octant order)
        int depth;
        bool leaf;
        int32_t first, count, skip;  // sorted-slot range of its bodies; next node after its subtree
        double mass, width;          // FP64 mass, top.x - btm.x of the cell in T
        vector3D<double> com;
    };

private:
    gtd_system *dev = nullptr;
    const std::vector<bod_t> *src = nullptr;
    std::vector<node> nodes;
    std::vector<int32_t> slot_body;  // sorted slot -> index into the body vector
    std::vector<cube_t> cubes;       // the host cells, pre-order (cubes[0] is the root)
    vec _btm{}, _top{};

    // Links the downloaded pre-order node list into bh_cube cells.  A node at depth d is child
    // octant (code >> 3 (21 - d)) & 7 of the last node seen at depth d - 1, with the bounds
    // set_corners gives it.  The device tree stops at depth 21: the bodies of a leaf there that
    // holds several (positions closer than the depth-21 cell width) become leaves of equal cells
    // under it, in slot order, where the reference would go on splitting.
    void link_cells(const std::vector<uint64_t> &codes) {
        const int64_t nn = (int64_t)nodes.size();
        size_t total = (size_t)nn;
        for (const node &c : nodes)
            if (c.leaf && c.count > 1) total += (size_t)c.count;
        cubes.clear();
        cubes.resize(total);  // never resized again: the links below stay valid
        std::vector<cube_t *> last(64, nullptr);
        size_t w = 0;
        for (int64_t k = 0; k < nn; ++k) {
            const node &nd = nodes[(size_t)k];
            cube_t &c = cubes[w++];
            c._all = &cubes;
            c._mass = (M)nd.mass;
            c._com = vec{(T)nd.com.x, (T)nd.com.y, (T)nd.com.z};
            if (k == 0) {
                c._btm = _btm;
                c._top = _top;
            } else {
                cube_t *p = last[(size_t)nd.depth - 1];
                const unsigned oct = (unsigned)((codes[(size_t)nd.first] >> (3 * (21 - nd.depth))) & 7u);
                p->child_box(oct, c._btm, c._top);
                c.parent = p;
                p->_sub[oct] = &c;
            }
            last[(size_t)nd.depth] = &c;
            if (nd.leaf) {
                if (nd.count == 1) {
                    c._bod = &(*src)[(size_t)slot_body[(size_t)nd.first]];
                } else {
                    if (nd.count > 8) throw barnes_hut_error{"Error: more than 8 bodies share a depth-21 cell.\n"};
                    for (int32_t q = 0; q < nd.count; ++q) {
                        cube_t &l = cubes[w++];
                        l._all = &cubes;
                        l._bod = &(*src)[(size_t)slot_body[(size_t)(nd.first + q)]];
                        l._mass = l._bod->mass();
                        l._com = l._bod->pos();
                        l._btm = c._btm;
                        l._top = c._top;
                        l.parent = &c;
                        c._sub[q] = &l;
                    }
                }
            }
        }
        // pre-order positions and subtree ends (children follow their parent in the array)
        std::vector<int64_t> size(total, 1);
        for (int64_t i = (int64_t)total - 1; i >= 0; --i) {
            cube_t &c = cubes[(size_t)i];
            c._index = i;
            if (c.parent) size[(size_t)(c.parent - cubes.data())] += size[(size_t)i];
        }
        for (size_t i = 0; i < total; ++i) cubes[i]._skip = (int64_t)i + size[i];
    }

public:
    bh_tree() = default;
    bh_tree(const bh_tree &) = delete;
    bh_tree &operator=(const bh_tree &) = delete;
    ~bh_tree() { gtd_system_destroy(dev); }

    // bh_tree::add_bodies (greg8tree.hpp:1066-1078) + calc_com (:1062): the tree is rebuilt from the
    // given bodies (the reference appends to an existing root; a rebuild gives the same octree).
    void add_bodies(const std::vector<bod_t> &bods) {
        if (bods.empty()) return;
        if (!dev) throw_status(gtd_system_create(&dev, 0, GTD_PREC_F64));
        const int64_t n = (int64_t)bods.size();
        std::vector<double> m(n), x(3 * n);
        for (int64_t i = 0; i < n; ++i) {
            m[i] = (double)bods[i].mass();
            x[3 * i] = (double)bods[i].pos().x;
            x[3 * i + 1] = (double)bods[i].pos().y;
            x[3 * i + 2] = (double)bods[i].pos().z;
        }
        throw_status(gtd_system_upload(dev, n, m.data(), nullptr, nullptr, x.data(), nullptr));
        throw_status(gtd_bh_build(dev, std::is_same_v<T, float> ? 1 : 0));
        int64_t nn = 0, nl = 0;
        double box[6];
        throw_status(gtd_bh_tree_size(dev, &nn, &nl, box));
        std::vector<int8_t> depth(nn), leaf(nn);
        std::vector<int32_t> first(nn), count(nn), skip(nn);
        std::vector<double> mass(nn), com(3 * nn), width(nn);
        std::vector<uint64_t> codes(n);
        slot_body.assign(n, 0);
        throw_status(gtd_bh_tree_download(dev, codes.data(), slot_body.data(), depth.data(), leaf.data(), first.data(),
                                          count.data(), skip.data(), mass.data(), com.data(), width.data()));
        nodes.resize(nn);
        for (int64_t k = 0; k < nn; ++k)
            nodes[k] = node{depth[k], leaf[k] != 0, first[k], count[k], skip[k], mass[k], width[k],
                            vector3D<double>{com[3 * k], com[3 * k + 1], com[3 * k + 2]}};
        _btm = vec{(T)box[0], (T)box[1], (T)box[2]};
        _top = vec{(T)box[3], (T)box[4], (T)box[5]};
        src = &bods;
        link_cells(codes);
    }
    void assign_bodies(const std::vector<bod_t> &bods) {
        delete_tree();
        add_bodies(bods);
    }
    void calc_com() {}  // centres of mass are computed (in FP64) when the tree is built
    void delete_tree() noexcept {
        nodes.clear();
        slot_body.clear();
        cubes.clear();
        src = nullptr;
        _btm = _top = vec{};
    }
    vec bottom() { return _btm; }
    vec top() { return _top; }
    const std::vector<node> &cells() const noexcept { return nodes; }

    // bh_tree::begin / end (greg8tree.hpp:1084-1089): the leaves in DFS octant order.
    typename cube_t::iterator begin() {
        if (cubes.empty()) throw std::invalid_argument{"Error: nullptr passed as root cube.\n"};
        return {&cubes[0]};
    }
    typename cube_t::iterator end() {
        if (cubes.empty()) throw std::invalid_argument{"Error: nullptr passed as root cube.\n"};
        return {&cubes[0], true};
    }
    // bh_tree::cell_begin / nn_begin (greg8tree.hpp:1090-1096).
    typename cube_t::cell_iterator cell_begin(const typename cube_t::body_iterator &body_it, long double opening_angle) {
        return {&cubes[0], body_it, opening_angle};
    }
    typename cube_t::nn_iterator nn_begin(const typename cube_t::body_iterator &body_it) { return {body_it}; }
    // The root cell (the reference keeps it private; cell_iterator's (root, position) form needs it).
    cube_t *root() noexcept { return cubes.empty() ? nullptr : &cubes[0]; }

    // Leaf bodies in the reference's iteration order (bh_cube::iterator, greg8tree.hpp:502-614).
    std::vector<const bod_t *> leaf_order() const {
        std::vector<const bod_t *> out;
        for (const cube_t &c : cubes)
            if (c.get_body()) out.push_back(c.get_body());
        return out;
    }

    // Barnes-Hut accelerations of the bodies given to add_bodies, with opening angle theta, the
    // reference's bh_acc force (gregsys.hpp:371-375, accumulated) and softening eps.
    std::vector<vector3D<T>> accelerations(long double theta, long double G, long double eps = 0) {
        if (!src || nodes.empty()) throw std::invalid_argument{"Error: the tree holds no bodies.\n"};
        const int64_t n = (int64_t)src->size();
        throw_status(gtd_system_set_params(dev, (double)G, 1.0, 1, (double)eps, (double)theta));
        throw_status(gtd_bh_build(dev, std::is_same_v<T, float> ? 1 : 0));  // walk records carry G M
        std::vector<double> a(3 * n);
        throw_status(gtd_bh_accelerations(dev, a.data(), nullptr));
        std::vector<vector3D<T>> out(n);
        for (int64_t i = 0; i < n; ++i) out[i] = vector3D<T>{(T)a[3 * i], (T)a[3 * i + 1], (T)a[3 * i + 2]};
        return out;
    }
};

template <uint64_t recFreq>
using octree = bh_tree<long double, long double, long double, recFreq>;
typedef bh_tree<long double, long double, long double, 0> octree_0f;

}  // namespace gtd
#endif
