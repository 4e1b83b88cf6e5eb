// shim_driver.cpp -- drives libgg_refshim.so the way the reference CLIs drive
// the reference calculators (cppcode/main.cpp, aspl_cuda.cpp, piece2aspl.cpp,
// box2aspl.cpp, beamer.cpp): read an instance with the reference's own
// load() (cppcode/{graph,part,piece,box}.hpp), construct the calculator by value,
// call its members.  Compiled against the reference headers, so it checks that
// code written for the reference compiles and links unchanged against the shim.
//
//   shim_driver graph|part|piece|box|beamer < instance.txt
// prints one line of key=value results (doubles with 17 significant digits).
#include <cstdio>
#include <iostream>
#include <string>
#include <tuple>

#include "box.hpp"
#include "cudaASPLbeamer.hpp"
#include "cudaASPLbox.hpp"
#include "cudaASPLconv.hpp"
#include "cudaASPLgraph.hpp"
#include "cudaASPLpiece.hpp"
#include "graph.hpp"
#include "part.hpp"
#include "piece.hpp"

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s graph|part|piece|box|beamer < instance\n", argv[0]);
        return 2;
    }
    const std::string kind = argv[1];
    try {
        if (kind == "graph") {
            graphgolf::graph g;
            g.load(std::cin);
            graphgolf::cudaASPLgraph cu(g.N, g.degree_max, 0);
            int diameter;
            int64_t total;
            std::tie(diameter, total) = cu.calc(g);
            std::printf("diameter=%d total=%lld\n", diameter, (long long)total);
        } else if (kind == "part") {
            graphgolf::part p;
            p.load(std::cin);
            graphgolf::cudaASPLconv cu(p.N, p.M, p.degree, 0);
            auto da = cu.diameterASPL(p);
            double c = cu.calc(p);
            auto w = cu.WVCdiameterASPL(p);
            std::printf("diameter=%d aspl=%.17g calc=%.17g wvc=%d wvc_diameter=%d wvc_aspl=%.17g\n",
                        da.first, da.second, c, std::get<0>(w), std::get<1>(w), std::get<2>(w));
        } else if (kind == "piece") {
            graphgolf::piece p;
            p.load(std::cin);
            graphgolf::cudaASPLpiece cu(p.Nx, p.Ny, p.Mx, p.My, p.degree, 0);
            auto da = cu.diameterASPL(p);
            std::printf("diameter=%d aspl=%.17g\n", da.first, da.second);
        } else if (kind == "box") {
            graphgolf::box p;
            p.load(std::cin);
            graphgolf::cudaASPLbox cu(p.Nx, p.Ny, p.Nz, p.Mx, p.My, p.Mz, p.degree, 0);
            auto da = cu.diameterASPL(p);
            std::printf("diameter=%d aspl=%.17g\n", da.first, da.second);
        } else if (kind == "beamer") {
            graphgolf::part p;
            p.load(std::cin);
            graphgolf::cudaASPLbeamer cu(p.N, p.M, p.degree, 0);
            std::printf("aspl=%.17g\n", cu.calc(p));
        } else {
            std::fprintf(stderr, "unknown kind %s\n", kind.c_str());
            return 2;
        }
    } catch (const std::exception &ex) {
        std::fprintf(stderr, "error: %s\n", ex.what());
        return 1;
    }
    return 0;
}
