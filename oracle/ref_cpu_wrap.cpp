// ref_cpu_wrap.cpp -- C entry points around the REFERENCE's own CPU calculators
// (TEST INFRASTRUCTURE ONLY; built into oracle/_ref/ by oracle/Makefile).
//
// The reference sources are compiled where they lie (include path points at the
// read-only reference tree); nothing of them is copied here.  This file only
// fills the reference data structures (cppcode/part.hpp:6-44,
// cppcode/piece.hpp:7-53, cppcode/box.hpp:6-81) from flat arrays and calls
//   graphgolf::cpuASPLqueue<cap>::calc / diameterASPL   (cppcode/cpuASPLqueue.cpp:11-96)
//   graphgolf::cpuASPLpiece<cap>::diameterASPL          (cppcode/cpuASPLpiece.cpp:12-63)
//   graphgolf::cpuASPLbox<cap>::diameterASPL            (cppcode/cpuASPLbox.cpp:12-66)
// choosing the smallest template capacity >= N (the reference is undefined for
// N > cap, cppcode/cpuASPLqueue.cpp:23,67).
//
// Edge lists are passed as (deg[M], flat values), one row per orbit vertex, in
// the reference's order: part diffs, piece (dx,dy) pairs, box (dx,dy,dz) triples.
#include <cstdint>
#include <vector>
#include <tuple>
#include <utility>
#include "cpuASPLqueue.cpp"
#include "cpuASPLpiece.cpp"
#include "cpuASPLbox.cpp"

namespace {

using graphgolf::part;
using graphgolf::piece;
using graphgolf::box;

part make_part(int N, int M, const int *deg, const int *vals) {
    part p;
    p.N = N; p.M = M; p.edges.assign(M, {});
    p.degree = 0; p.regular = true;
    size_t k = 0;
    for (int i = 0; i < M; i++) {
        if (!p.degree) p.degree = deg[i];
        else if (p.degree != deg[i]) { p.regular = false; p.degree = std::max(p.degree, deg[i]); }
        for (int j = 0; j < deg[i]; j++) p.edges[i].push_back(vals[k++]);
    }
    return p;
}

piece make_piece(int Nx, int Ny, int Mx, int My, const int *deg, const int *vals) {
    piece p(Nx, Ny, Mx, My);
    p.degree = 0; p.regular = true;
    size_t k = 0;
    for (int x = 0; x < Mx; x++)
        for (int y = 0; y < My; y++) {
            int E = deg[x * My + y];
            if (!p.degree) p.degree = E; else if (p.degree != E) p.regular = false;
            for (int e = 0; e < E; e++, k += 2) p.edges[x][y].emplace_back(vals[k], vals[k + 1]);
        }
    return p;
}

box make_box(int Nx, int Ny, int Nz, int Mx, int My, int Mz, const int *deg, const int *vals) {
    box p(Nx, Ny, Nz, Mx, My, Mz);
    p.regular = true;
    size_t k = 0;
    for (int x = 0; x < Mx; x++)
        for (int y = 0; y < My; y++)
            for (int z = 0; z < Mz; z++) {
                int E = deg[(x * My + y) * Mz + z];
                if (!p.degree) p.degree = E; else if (p.degree != E) p.regular = false;
                for (int e = 0; e < E; e++, k += 3)
                    p.edges[x][y][z].emplace_back(vals[k], vals[k + 1], vals[k + 2]);
            }
    return p;
}

// Dispatch on the smallest capacity that holds N vertices.
template <template <int> class Calc, typename F>
int with_cap(int N, F &&f) {
    if (N <= 1024) { Calc<1024> c; f(c); return 0; }
    if (N <= 4096) { Calc<4096> c; f(c); return 0; }
    if (N <= 16384) { Calc<16384> c; f(c); return 0; }
    if (N <= 65536) { Calc<65536> c; f(c); return 0; }
    if (N <= 131072) { Calc<131072> c; f(c); return 0; }
    return -1;
}

}  // namespace

extern "C" {

// cpuASPLqueue<cap>::diameterASPL (cppcode/cpuASPLqueue.cpp:54-96)
int ggr_queue_diameter_aspl(int N, int M, const int *deg, const int *diffs,
                            int *diameter, double *aspl) {
    part p = make_part(N, M, deg, diffs);
    return with_cap<graphgolf::cpuASPLqueue>(N, [&](auto &c) {
        auto r = c.diameterASPL(p);
        *diameter = r.first; *aspl = r.second;
    });
}

// cpuASPLqueue<cap>::calc (cppcode/cpuASPLqueue.cpp:11-53)
int ggr_queue_calc(int N, int M, const int *deg, const int *diffs, double *aspl) {
    part p = make_part(N, M, deg, diffs);
    return with_cap<graphgolf::cpuASPLqueue>(N, [&](auto &c) { *aspl = c.calc(p); });
}

// cpuASPLpiece<cap>::diameterASPL (cppcode/cpuASPLpiece.cpp:12-63)
int ggr_piece_diameter_aspl(int Nx, int Ny, int Mx, int My, const int *deg, const int *vals,
                            int *diameter, double *aspl) {
    piece p = make_piece(Nx, Ny, Mx, My, deg, vals);
    return with_cap<graphgolf::cpuASPLpiece>(Nx * Ny, [&](auto &c) {
        auto r = c.diameterASPL(p);
        *diameter = r.first; *aspl = r.second;
    });
}

// cpuASPLbox<cap>::diameterASPL (cppcode/cpuASPLbox.cpp:12-66)
int ggr_box_diameter_aspl(int Nx, int Ny, int Nz, int Mx, int My, int Mz, const int *deg,
                          const int *vals, int *diameter, double *aspl) {
    box p = make_box(Nx, Ny, Nz, Mx, My, Mz, deg, vals);
    return with_cap<graphgolf::cpuASPLbox>(Nx * Ny * Nz, [&](auto &c) {
        auto r = c.diameterASPL(p);
        *diameter = r.first; *aspl = r.second;
    });
}

}  // extern "C"
