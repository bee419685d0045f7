// Drop-in gtd::bh_tree (GregW10/GregPackagesCPP greg8tree.hpp:984-1118) over the B200 linear
// octree (gtd_b200.h).  add_bodies builds the tree on the device with the reference's root box,
// octant splits and (for T = float) float geometry; the tree is read back as a pre-order node list
// so callers can walk leaves in the reference's DFS octant order, and bh_accelerations runs the
// reference walk (cell_iterator, greg8tree.hpp:702-833) on the device.
#ifndef GTD_B200_GREG8TREE_HPP
#define GTD_B200_GREG8TREE_HPP

#include <cstdint>
#include <vector>

#include "gregbod.hpp"

namespace gtd {

template <isNumWrapper M = long double, isNumWrapper R = long double, isNumWrapper T = long double, uint64_t rF = 0>
class bh_tree {
public:
    using bod_t = body<M, R, T, rF>;
    using vec = vector3D<T>;
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
    vec _btm{}, _top{};

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
        slot_body.assign(n, 0);
        throw_status(gtd_bh_tree_download(dev, nullptr, slot_body.data(), depth.data(), leaf.data(), first.data(),
                                          count.data(), skip.data(), mass.data(), com.data(), width.data()));
        nodes.resize(nn);
        for (int64_t k = 0; k < nn; ++k)
            nodes[k] = node{depth[k], leaf[k] != 0, first[k], count[k], skip[k], mass[k], width[k],
                            vector3D<double>{com[3 * k], com[3 * k + 1], com[3 * k + 2]}};
        _btm = vec{(T)box[0], (T)box[1], (T)box[2]};
        _top = vec{(T)box[3], (T)box[4], (T)box[5]};
        src = &bods;
    }
    void assign_bodies(const std::vector<bod_t> &bods) {
        delete_tree();
        add_bodies(bods);
    }
    void calc_com() {}  // centres of mass are computed (in FP64) when the tree is built
    void delete_tree() noexcept {
        nodes.clear();
        slot_body.clear();
        src = nullptr;
        _btm = _top = vec{};
    }
    vec bottom() { return _btm; }
    vec top() { return _top; }
    const std::vector<node> &cells() const noexcept { return nodes; }

    // Leaf bodies in the reference's iteration order (bh_cube::iterator, greg8tree.hpp:502-614).
    std::vector<const bod_t *> leaf_order() const {
        std::vector<const bod_t *> out;
        if (!src) return out;
        for (const node &c : nodes)
            if (c.leaf)
                for (int32_t s = c.first; s < c.first + c.count; ++s) out.push_back(&(*src)[slot_body[s]]);
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
