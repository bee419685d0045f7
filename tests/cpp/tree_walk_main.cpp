// Code written against the reference's gtd::bh_tree API (greg8tree.hpp): build a tree over a
// seeded two-cloud body set, iterate its leaves (begin / end), and for every leaf body sum the
// force of the cells its cell_iterator yields (theta = 0.5) and count its nn_iterator neighbours;
// for the first leaf also list the children of each yielded internal cell through operator[].
// The same source compiles against the reference headers and against the drop-in headers
// (include/gtd); their outputs are compared line by line.
//   one line per leaf, in iteration order: index count neighbours ax ay az
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "greg8tree.hpp"

using bod_t = gtd::body<double, double, double, 0>;
using tree_t = gtd::bh_tree<double, double, double, 0>;

int main(int argc, char **argv) {
    const int n = argc > 1 ? std::atoi(argv[1]) : 3000;
    unsigned long long s = 0x9E3779B97F4A7C15ULL;
    auto u = [&]() {
        s ^= s << 13; s ^= s >> 7; s ^= s << 17;
        return ((s >> 11) + 0.5) / 9007199254740992.0;
    };
    std::vector<bod_t> bods;
    bods.reserve(n);
    for (int i = 0; i < n; ++i) {
        // two clumps of different sizes, so that the tree has both deep and shallow branches
        const double scale = i % 3 ? 1.5e11 : 4e10, cx = i % 3 ? 0.0 : 6e11;
        const double r = scale * std::pow(u(), 1.0 / 3.0), ct = 2 * u() - 1, ph = 6.283185307179586 * u();
        const double st = std::sqrt(1 - ct * ct);
        bods.emplace_back(1e30 / n * (0.5 + u()), 0.0,
                          gtd::vector3D<double>{cx + r * st * std::cos(ph), r * st * std::sin(ph), r * ct},
                          gtd::vector3D<double>{0.0, 0.0, 0.0});
    }
    tree_t tree;
    tree.add_bodies(bods);
    tree.calc_com();
    const long double G = 6.674e-11L;
    bool first = true;
    for (auto it = tree.begin(); it != tree.end(); ++it) {
        const bod_t &b = *it;
        long double ax = 0, ay = 0, az = 0;
        unsigned cnt = 0;
        for (auto cit = tree.cell_begin(it, 0.5L); cit; ++cit) {
            const auto com = cit->cube_com();
            const long double dx = (long double)com.get_x() - b.pos().get_x();
            const long double dy = (long double)com.get_y() - b.pos().get_y();
            const long double dz = (long double)com.get_z() - b.pos().get_z();
            const long double d = sqrtl(dx * dx + dy * dy + dz * dz);
            const long double f = G * cit->cube_mass() / (d * d * d);
            ax += f * dx;
            ay += f * dy;
            az += f * dz;
            ++cnt;
            if (first && cit->get_body() == nullptr) {
                std::printf("children");
                for (unsigned char k = 0; k < 8; ++k) {
                    try {
                        std::printf(" %u:%.6e", (unsigned)k, (double)(*cit)[k].cube_mass());
                    } catch (const std::invalid_argument &) {
                        std::printf(" %u:-", (unsigned)k);
                    }
                }
                std::printf("\n");
            }
        }
        first = false;
        unsigned nn = 0;
        for (auto nit = tree.nn_begin(it); nit; ++nit) ++nn;
        std::printf("%ld %u %u %.17Le %.17Le %.17Le\n", (long)(&b - bods.data()), cnt, nn, ax, ay, az);
    }
    try {
        (void)tree.cell_begin(tree.begin(), 3.2L);
        std::printf("theta 3.2 accepted\n");
    } catch (const std::invalid_argument &e) {
        std::printf("theta 3.2 rejected: %s", e.what());
    }
    return 0;
}
