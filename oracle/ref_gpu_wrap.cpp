// ref_gpu_wrap.cpp -- C entry points around the REFERENCE's own GPU calculators
// (TEST AND BASELINE INFRASTRUCTURE ONLY; built into oracle/_ref/ by oracle/Makefile).
//
// Each reference calculator (cudacode/cudaASPL*.cu) is compiled for sm_100a from
// the read-only reference tree into its own shared library, because the
// reference .cu files define kernels with identical signatures
// (kernel_aspl_reduce_plus etc.) that cannot share one link unit.  This file is
// compiled once per library with exactly one of REF_GRAPH / REF_CONV /
// REF_PIECE / REF_BOX / REF_BEAMER defined.  It builds the reference data
// structures from flat arrays and calls the reference member functions; the
// reference's progress prints go to a null stream buffer during the call.
//
// The calculator object is created per handle (ggrg_*_create) so that timing
// loops measure calc()/diameterASPL() alone, as the reference annealers call it
// (cppcode/annealing.cpp:296,403; cppcode/aspl_cuda.cpp:90,94).
#include <cstdint>
#include <iostream>
#include <streambuf>
#include <vector>
#include <tuple>

namespace {
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};
struct Quiet {  // silence std::cout for the scope of one reference call
    NullBuf nb;
    std::streambuf *old;
    Quiet() : old(std::cout.rdbuf(&nb)) {}
    ~Quiet() { std::cout.rdbuf(old); }
};
}  // namespace

#if defined(REF_GRAPH)
#include "cudaASPLgraph.hpp"
extern "C" {
// cudaASPLgraph(N, degree_max, device) -- cudacode/cudaASPLgraph.hpp:15
void *ggrg_graph_create(int N, int degree_max, int device) {
    Quiet q;
    return new graphgolf::cudaASPLgraph(N, degree_max, device);
}
void ggrg_graph_destroy(void *h) { delete (graphgolf::cudaASPLgraph *)h; }
// calc(graph&) -- cudacode/cudaASPLgraph.cu:141-199.  adjacency lists as (deg[N], flat).
int ggrg_graph_calc(void *h, int N, const int *deg, const int *nbrs, int *diameter, int64_t *total) {
    graphgolf::graph g;
    g.N = N; g.edges.assign(N, {}); g.degree_max = 0;
    size_t k = 0;
    for (int v = 0; v < N; v++) {
        for (int j = 0; j < deg[v]; j++) g.edges[v].push_back(nbrs[k++]);
        if (deg[v] > g.degree_max) g.degree_max = deg[v];
    }
    Quiet q;
    auto r = ((graphgolf::cudaASPLgraph *)h)->calc(g);
    *diameter = r.first; *total = r.second;
    return 0;
}
}
#elif defined(REF_CONV) || defined(REF_BEAMER)
#ifdef REF_CONV
#include "cudaASPLconv.hpp"
#else
#include "cudaASPLbeamer.hpp"
#endif
static graphgolf::part make_part(int N, int M, const int *deg, const int *diffs) {
    graphgolf::part p;
    p.N = N; p.M = M; p.edges.assign(M, {}); p.degree = 0; p.regular = true;
    size_t k = 0;
    for (int i = 0; i < M; i++) {
        if (!p.degree) p.degree = deg[i];
        else if (p.degree != deg[i]) { p.regular = false; p.degree = std::max(p.degree, deg[i]); }
        for (int j = 0; j < deg[i]; j++) p.edges[i].push_back(diffs[k++]);
    }
    return p;
}
extern "C" {
#ifdef REF_CONV
// cudaASPLconv(N, M, degree, device) -- cudacode/cudaASPLconv.hpp:18
void *ggrg_conv_create(int N, int M, int degree, int device) {
    Quiet q;
    return new graphgolf::cudaASPLconv(N, M, degree, device);
}
void ggrg_conv_destroy(void *h) { delete (graphgolf::cudaASPLconv *)h; }
// calc / diameterASPL / WVCdiameterASPL -- cudacode/cudaASPLconv.cu:151,197,244
int ggrg_conv_calc(void *h, int N, int M, const int *deg, const int *diffs, double *aspl) {
    auto p = make_part(N, M, deg, diffs);
    Quiet q;
    *aspl = ((graphgolf::cudaASPLconv *)h)->calc(p);
    return 0;
}
int ggrg_conv_diameter_aspl(void *h, int N, int M, const int *deg, const int *diffs,
                            int *diameter, double *aspl) {
    auto p = make_part(N, M, deg, diffs);
    Quiet q;
    auto r = ((graphgolf::cudaASPLconv *)h)->diameterASPL(p);
    *diameter = r.first; *aspl = r.second;
    return 0;
}
int ggrg_conv_wvc(void *h, int N, int M, const int *deg, const int *diffs,
                  int *wvc, int *diameter, double *aspl) {
    auto p = make_part(N, M, deg, diffs);
    Quiet q;
    auto r = ((graphgolf::cudaASPLconv *)h)->WVCdiameterASPL(p);
    *wvc = std::get<0>(r); *diameter = std::get<1>(r); *aspl = std::get<2>(r);
    return 0;
}
#else
// cudaASPLbeamer(N, M, degree, device) -- cudacode/cudaASPLbeamer.hpp:14
void *ggrg_beamer_create(int N, int M, int degree, int device) {
    return new graphgolf::cudaASPLbeamer(N, M, degree, device);
}
void ggrg_beamer_destroy(void *h) { delete (graphgolf::cudaASPLbeamer *)h; }
int ggrg_beamer_calc(void *h, int N, int M, const int *deg, const int *diffs, double *aspl) {
    auto p = make_part(N, M, deg, diffs);
    *aspl = ((graphgolf::cudaASPLbeamer *)h)->calc(p);
    return 0;
}
#endif
}
#elif defined(REF_PIECE)
#include "cudaASPLpiece.hpp"
extern "C" {
void *ggrg_piece_create(int Nx, int Ny, int Mx, int My, int degree, int device) {
    Quiet q;
    return new graphgolf::cudaASPLpiece(Nx, Ny, Mx, My, degree, device);
}
void ggrg_piece_destroy(void *h) { delete (graphgolf::cudaASPLpiece *)h; }
// diameterASPL(piece&) -- cudacode/cudaASPLpiece.cu:159-216
int ggrg_piece_diameter_aspl(void *h, int Nx, int Ny, int Mx, int My, const int *deg,
                             const int *vals, int *diameter, double *aspl) {
    graphgolf::piece p(Nx, Ny, Mx, My);
    p.degree = 0; p.regular = true;
    size_t k = 0;
    for (int x = 0; x < Mx; x++)
        for (int y = 0; y < My; y++) {
            int E = deg[x * My + y];
            for (int e = 0; e < E; e++, k += 2) p.edges[x][y].emplace_back(vals[k], vals[k + 1]);
        }
    Quiet q;
    auto r = ((graphgolf::cudaASPLpiece *)h)->diameterASPL(p);
    *diameter = r.first; *aspl = r.second;
    return 0;
}
}
#elif defined(REF_BOX)
#include "cudaASPLbox.hpp"
extern "C" {
void *ggrg_box_create(int Nx, int Ny, int Nz, int Mx, int My, int Mz, int degree, int device) {
    Quiet q;
    return new graphgolf::cudaASPLbox(Nx, Ny, Nz, Mx, My, Mz, degree, device);
}
void ggrg_box_destroy(void *h) { delete (graphgolf::cudaASPLbox *)h; }
// diameterASPL(box&) -- cudacode/cudaASPLbox.cu:166-226
int ggrg_box_diameter_aspl(void *h, int Nx, int Ny, int Nz, int Mx, int My, int Mz,
                           const int *deg, const int *vals, int *diameter, double *aspl) {
    graphgolf::box p(Nx, Ny, Nz, Mx, My, Mz);
    p.regular = true;
    size_t k = 0;
    for (int x = 0; x < Mx; x++)
        for (int y = 0; y < My; y++)
            for (int z = 0; z < Mz; z++) {
                int E = deg[(x * My + y) * Mz + z];
                for (int e = 0; e < E; e++, k += 3)
                    p.edges[x][y][z].emplace_back(vals[k], vals[k + 1], vals[k + 2]);
            }
    Quiet q;
    auto r = ((graphgolf::cudaASPLbox *)h)->diameterASPL(p);
    *diameter = r.first; *aspl = r.second;
    return 0;
}
}
#else
#error "define one of REF_GRAPH REF_CONV REF_PIECE REF_BOX REF_BEAMER"
#endif
