// The guards of gtd::system as code written against the reference's API meets them, through the
// drop-in headers (include/gtd/gregsys.hpp): one command per input line, one result per output line.
//   units <format>                    -> "ok <G as %La>" or "err <message with \n escaped>"
//   set <dt> <iterations> <eps> <theta> -> the four setter results, each 0 or 1
//   dt <value>                        -> "ok" when a system with that time step constructs, else "err <msg>"
// Numbers are read as long double hexfloats (%La) so that no value is rounded on the way in.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>

#include "gtd/gregsys.hpp"

using sys_t = gtd::system<double, double, double, false, false, 0, 0, 0, false>;

static std::string escape(const std::string &s) {
    std::string o;
    for (char c : s) o += c == '\n' ? std::string("\\n") : std::string(1, c);
    return o;
}

int main() {
    std::string line;
    while (std::getline(std::cin, line)) {
        const auto sp = line.find(' ');
        const std::string cmd = line.substr(0, sp), arg = sp == std::string::npos ? "" : line.substr(sp + 1);
        if (cmd == "units") {
            try {
                sys_t s{1.0L, 1, arg.c_str()};
                std::printf("ok %La\n", s.G_val());
            } catch (const std::invalid_argument &e) {
                std::printf("err %s\n", escape(e.what()).c_str());
            }
        } else if (cmd == "set") {
            long double dt, eps, theta;
            unsigned long long it;
            if (std::sscanf(arg.c_str(), "%La %llu %La %La", &dt, &it, &eps, &theta) != 4) return 2;
            sys_t s{1.0L, 1, "M1:1,D1:1,T1:1"};
            std::printf("%d %d %d %d\n", (int)s.set_timestep(dt), (int)s.set_iterations(it), (int)s.set_softening(eps),
                        (int)s.set_bh_opening_angle(theta));
        } else if (cmd == "dt") {
            long double dt;
            if (std::sscanf(arg.c_str(), "%La", &dt) != 1) return 2;
            try {
                sys_t s{dt, 1, "M1:1,D1:1,T1:1"};
                std::printf("ok\n");
            } catch (const std::invalid_argument &e) {
                std::printf("err %s\n", escape(e.what()).c_str());
            }
        } else {
            return 2;
        }
        std::fflush(stdout);
    }
    return 0;
}
