// refshim.cpp -- the reference calculator classes, defined on the B200 engine.
//
// Built into libgg_refshim.so against the reference's own headers
// (cudacode/cudaASPL*.hpp, cppcode/{graph,part,piece,box}.hpp) found on the
// include path, so that code written for the reference -- the annealers and CLIs
// in cppcode/ that construct a calculator by value and call its members
// (cppcode/annealing.cpp:296,302,403; cppcode/aspl_cuda.cpp:90,94; ...) -- links
// against this library unchanged: the object layout the caller allocates is the
// reference's, and every member function below has the reference's signature.
//
// Each object keeps its engine handle in the first device-pointer member of the
// reference layout (the engine owns all device memory) and its packed edge table
// in the host-table member, exactly the array the reference fills before its
// cudaMemcpy.  Return values and sentinels are those of the C ABI calls, which
// reproduce the reference bit for bit (include/gg.h).  Engine errors, which the
// reference never reports, are raised as std::runtime_error.
#include "gg.h"

#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>

#include "cudaASPLbeamer.hpp"
#include "cudaASPLbox.hpp"
#include "cudaASPLconv.hpp"
#include "cudaASPLgraph.hpp"
#include "cudaASPLpiece.hpp"

namespace {

void check(gg_status s, const char *what) {
    if (s != GG_OK)
        throw std::runtime_error(std::string(what) + ": " + gg_status_str(s) + " (" + gg_last_error() + ")");
}

template <typename P>
gg_engine *engine_of(P *slot) { return reinterpret_cast<gg_engine *>(slot); }

template <typename P>
P *slot_of(gg_engine *e) { return reinterpret_cast<P *>(e); }

}  // namespace

namespace graphgolf {

// ---- cudaASPLgraph (cudacode/cudaASPLgraph.hpp:14-18) ----------------------

cudaASPLgraph::cudaASPLgraph(int N, int degree_max, int device)
    : d_bits(nullptr), h_bits(nullptr), d_diff_bits(nullptr), d_sum(nullptr), d_edges(nullptr),
      h_edges(nullptr), h_ret(nullptr), d_ret(nullptr), h_ret_bits(nullptr), d_ret_bits(nullptr),
      N(N), degree_max(degree_max), device(device), nBlock(0) {
    gg_engine *e = nullptr;
    check(gg_graph_create(N, degree_max, device, &e), "cudaASPLgraph");
    d_bits = slot_of<uint>(e);
    h_edges = new int[(size_t)N * degree_max + 1];
}

cudaASPLgraph::~cudaASPLgraph() {
    gg_destroy(engine_of(d_bits));
    delete[] h_edges;
}

std::pair<int, int64_t> cudaASPLgraph::calc(graph &g) {
    // repack, padding missing slots with self loops (cudaASPLgraph.cu:144-153)
    for (int i = 0; i < N; i++)
        for (int j = 0; j < degree_max; j++)
            h_edges[(size_t)i * degree_max + j] = j < (int)g.edges[i].size() ? g.edges[i][j] : i;
    int diameter = 0;
    int64_t total = 0;
    check(gg_graph_calc(engine_of(d_bits), h_edges, &diameter, &total), "cudaASPLgraph::calc");
    return std::make_pair(diameter, total);
}

// ---- cudaASPLconv (cudacode/cudaASPLconv.hpp:16-22) ------------------------

cudaASPLconv::cudaASPLconv(int N, int M, int degree, int device)
    : d_bits(nullptr), h_bits(nullptr), d_diff_bits(nullptr), d_sum(nullptr), d_edges(nullptr),
      h_edges(nullptr), h_ret(nullptr), d_ret(nullptr), h_ret_bits(nullptr), d_ret_bits(nullptr),
      device(device), width(0), nBlock(0), N(N), M(M), degree(degree) {
    gg_engine *e = nullptr;
    check(gg_conv_create(N, M, degree, device, &e), "cudaASPLconv");
    d_bits = slot_of<uint>(e);
    h_edges = new int[(size_t)M * degree + 1];
}

cudaASPLconv::~cudaASPLconv() {
    gg_destroy(engine_of(d_bits));
    delete[] h_edges;
}

namespace {
// cudaASPLconv.cu:199-201: M x degree diffs, padding 0
void pack_part(const part &p, int M, int degree, int *h) {
    for (int i = 0; i < M; i++)
        for (int j = 0; j < degree; j++)
            h[(size_t)i * degree + j] = j < (int)p.edges[i].size() ? p.edges[i][j] : 0;
}
}  // namespace

double cudaASPLconv::calc(part &p) {
    pack_part(p, M, degree, h_edges);
    double aspl = 0;
    check(gg_conv_calc(engine_of(d_bits), h_edges, &aspl), "cudaASPLconv::calc");
    return aspl;
}

std::pair<int, double> cudaASPLconv::diameterASPL(part &p) {
    pack_part(p, M, degree, h_edges);
    int diameter = 0;
    double aspl = 0;
    check(gg_conv_diameter_aspl(engine_of(d_bits), h_edges, &diameter, &aspl),
          "cudaASPLconv::diameterASPL");
    return std::make_pair(diameter, aspl);
}

std::tuple<int, int, double> cudaASPLconv::WVCdiameterASPL(part &p) {
    pack_part(p, M, degree, h_edges);
    int wvc = 0, diameter = 0;
    double aspl = 0;
    check(gg_conv_wvc_diameter_aspl(engine_of(d_bits), h_edges, &wvc, &diameter, &aspl),
          "cudaASPLconv::WVCdiameterASPL");
    return std::make_tuple(wvc, diameter, aspl);
}

// ---- cudaASPLpiece (cudacode/cudaASPLpiece.hpp:16-20) ----------------------

cudaASPLpiece::cudaASPLpiece(int Nx, int Ny, int Mx, int My, int degree, int device)
    : d_bits(nullptr), h_bits(nullptr), d_diff_bits(nullptr), d_sum(nullptr), d_edges(nullptr),
      h_edges(nullptr), h_ret(nullptr), d_ret(nullptr), h_ret_bits(nullptr), d_ret_bits(nullptr),
      device(device), width(0), nBlock(0), Nx(Nx), Ny(Ny), Mx(Mx), My(My), degree(degree) {
    gg_engine *e = nullptr;
    check(gg_piece_create(Nx, Ny, Mx, My, degree, device, &e), "cudaASPLpiece");
    d_bits = slot_of<uint>(e);
    h_edges = new int[(size_t)Mx * My * degree * 2 + 1];
}

cudaASPLpiece::~cudaASPLpiece() {
    gg_destroy(engine_of(d_bits));
    delete[] h_edges;
}

std::pair<int, double> cudaASPLpiece::diameterASPL(piece &p) {
    // cudaASPLpiece.cu:166-176: (dx, dy) per slot, padding (0, 0)
    for (int x = 0; x < Mx; x++)
        for (int y = 0; y < My; y++)
            for (int e = 0; e < degree; e++) {
                int dx = 0, dy = 0;
                if (e < (int)p.edges[x][y].size()) std::tie(dx, dy) = p.edges[x][y][e];
                h_edges[((size_t)(x * My + y) * degree + e) * 2] = dx;
                h_edges[((size_t)(x * My + y) * degree + e) * 2 + 1] = dy;
            }
    int diameter = 0;
    double aspl = 0;
    check(gg_piece_diameter_aspl(engine_of(d_bits), h_edges, &diameter, &aspl),
          "cudaASPLpiece::diameterASPL");
    return std::make_pair(diameter, aspl);
}

// ---- cudaASPLbox (cudacode/cudaASPLbox.hpp:16-20) --------------------------

cudaASPLbox::cudaASPLbox(int Nx, int Ny, int Nz, int Mx, int My, int Mz, int degree, int device)
    : d_bits(nullptr), h_bits(nullptr), d_diff_bits(nullptr), d_sum(nullptr), d_edges(nullptr),
      h_edges(nullptr), h_ret(nullptr), d_ret(nullptr), h_ret_bits(nullptr), d_ret_bits(nullptr),
      device(device), width(0), nBlock(0), Nx(Nx), Ny(Ny), Nz(Nz), Mx(Mx), My(My), Mz(Mz),
      degree(degree) {
    gg_engine *e = nullptr;
    check(gg_box_create(Nx, Ny, Nz, Mx, My, Mz, degree, device, &e), "cudaASPLbox");
    d_bits = slot_of<uint>(e);
    h_edges = new int[(size_t)Mx * My * Mz * degree * 3 + 1];
}

cudaASPLbox::~cudaASPLbox() {
    gg_destroy(engine_of(d_bits));
    delete[] h_edges;
}

std::pair<int, double> cudaASPLbox::diameterASPL(box &p) {
    // cudaASPLbox.cu:170-184: (dx, dy, dz) per slot, padding (0, 0, 0)
    for (int x = 0; x < Mx; x++)
        for (int y = 0; y < My; y++)
            for (int z = 0; z < Mz; z++)
                for (int e = 0; e < degree; e++) {
                    int dx = 0, dy = 0, dz = 0;
                    if (e < (int)p.edges[x][y][z].size()) std::tie(dx, dy, dz) = p.edges[x][y][z][e];
                    const size_t o = ((size_t)((x * My + y) * Mz + z) * degree + e) * 3;
                    h_edges[o] = dx;
                    h_edges[o + 1] = dy;
                    h_edges[o + 2] = dz;
                }
    int diameter = 0;
    double aspl = 0;
    check(gg_box_diameter_aspl(engine_of(d_bits), h_edges, &diameter, &aspl),
          "cudaASPLbox::diameterASPL");
    return std::make_pair(diameter, aspl);
}

// ---- cudaASPLbeamer (cudacode/cudaASPLbeamer.hpp:12-16) --------------------

cudaASPLbeamer::cudaASPLbeamer(int N, int M, int degree, int device)
    : device(device), d_visited_bits(nullptr), d_updated_bits(nullptr), d_edges(nullptr),
      h_edges(nullptr), d_ret(nullptr), h_ret(nullptr), N(N), M(M), degree(degree) {
    gg_engine *e = nullptr;
    check(gg_beamer_create(N, M, degree, device, &e), "cudaASPLbeamer");
    d_visited_bits = slot_of<uint>(e);
    h_edges = new int[(size_t)M * degree + 1];
}

cudaASPLbeamer::~cudaASPLbeamer() {
    gg_destroy(engine_of(d_visited_bits));
    delete[] h_edges;
}

double cudaASPLbeamer::calc(part &p) {
    if (!p.regular) return 100000000;  // cudaASPLbeamer.cu:72
    pack_part(p, M, degree, h_edges);
    double aspl = 0;
    check(gg_beamer_calc(engine_of(d_visited_bits), h_edges, 1, &aspl), "cudaASPLbeamer::calc");
    return aspl;
}

}  // namespace graphgolf
