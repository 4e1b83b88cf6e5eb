// gg_gen.cpp -- deterministic instance generators (host only, no GPU).
//
// Random numbers: SplitMix64 seeds xoshiro256** (Blackman & Vigna, "Scrambled
// linear pseudorandom number generators", 2021); bounded integers use Lemire's
// multiply-and-reject method ("Fast random integer generation in an interval",
// ACM TOMACS 2019).  Both are spelled out here so that a seed means the same
// graph on every platform (std::uniform_int_distribution is library-defined).
//
// The reference draws its random instances with std::mt19937 + std::shuffle
// stub pairing and does not reject loops or multi-edges (cppcode/initTemp.cpp:399-405,
// cppcode/RNDpiecegen.cpp).  The generators here are the seeded synthetic
// inputs of the benchmark configurations instead: simple and connected by
// construction.
#include "gg.h"

#include <algorithm>
#include <cstdint>
#include <string>
#include <unordered_set>
#include <vector>

namespace {

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (auto &w : s) {  // SplitMix64
            x += 0x9e3779b97f4a7c15ull;
            uint64_t z = x;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            w = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {  // xoshiro256**
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    uint32_t below(uint32_t n) {  // uniform in [0, n), Lemire
        uint32_t x = (uint32_t)(next() >> 32);
        uint64_t m = (uint64_t)x * n;
        uint32_t l = (uint32_t)m;
        if (l < n) {
            const uint32_t t = (uint32_t)(-n) % n;
            while (l < t) {
                x = (uint32_t)(next() >> 32);
                m = (uint64_t)x * n;
                l = (uint32_t)m;
            }
        }
        return (uint32_t)(m >> 32);
    }
};

inline uint64_t ekey(int a, int b) {
    if (a > b) std::swap(a, b);
    return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
}

bool connected(int n, const std::vector<std::vector<int>> &g) {
    std::vector<char> seen(n, 0);
    std::vector<int> st{0};
    seen[0] = 1;
    int cnt = 1;
    while (!st.empty()) {
        int v = st.back();
        st.pop_back();
        for (int u : g[v])
            if (!seen[u]) { seen[u] = 1; ++cnt; st.push_back(u); }
    }
    return cnt == n;
}

// One attempt: stub pairing, then double-edge switches that move every loop and
// repeated edge onto a uniformly drawn partner edge until the multigraph is simple.
bool regular_attempt(int n, int d, Rng &rng, std::vector<std::pair<int, int>> &E) {
    std::vector<int> stubs((size_t)n * d);
    for (int v = 0; v < n; ++v)
        for (int k = 0; k < d; ++k) stubs[(size_t)v * d + k] = v;
    for (size_t i = stubs.size(); i > 1; --i) std::swap(stubs[i - 1], stubs[rng.below((uint32_t)i)]);
    const size_t m = stubs.size() / 2;
    E.resize(m);
    for (size_t i = 0; i < m; ++i) E[i] = {stubs[2 * i], stubs[2 * i + 1]};
    std::unordered_multiset<uint64_t> ms;
    ms.reserve(m * 2);
    for (auto &e : E) ms.insert(ekey(e.first, e.second));
    auto bad = [&](size_t i) {
        const auto &e = E[i];
        return e.first == e.second || ms.count(ekey(e.first, e.second)) > 1;
    };
    const size_t budget = 200 * m + 100000;
    size_t tries = 0;
    for (size_t i = 0; i < m; ++i) {
        while (bad(i)) {
            if (++tries > budget) return false;
            const size_t j = rng.below((uint32_t)m);
            if (j == i) continue;
            int a = E[i].first, b = E[i].second, c = E[j].first, x = E[j].second;
            if (rng.below(2)) std::swap(c, x);
            // (a,b),(c,x) -> (a,c),(b,x)
            if (a == c || b == x) continue;
            if (ms.count(ekey(a, c)) || ms.count(ekey(b, x))) continue;
            if (ekey(a, c) == ekey(b, x)) continue;
            ms.erase(ms.find(ekey(E[i].first, E[i].second)));
            ms.erase(ms.find(ekey(E[j].first, E[j].second)));
            E[i] = {a, c};
            E[j] = {b, x};
            ms.insert(ekey(a, c));
            ms.insert(ekey(b, x));
            if (j < i && bad(j)) i = j;  // re-examine an earlier edge if it became bad
        }
    }
    return true;
}

}  // namespace

extern "C" {

gg_status gg_gen_random_regular(int n, int d, uint64_t seed, int32_t *adj) {
    if (!adj || n < 2 || d < 1 || d >= n || ((long long)n * d) % 2 != 0 || (long long)n * d > (1ll << 31))
        return GG_BAD_ARG;
    Rng rng(seed);
    std::vector<std::pair<int, int>> E;
    for (int attempt = 0; attempt < 1000; ++attempt) {
        if (!regular_attempt(n, d, rng, E)) continue;
        std::vector<std::vector<int>> g(n);
        for (auto &e : E) { g[e.first].push_back(e.second); g[e.second].push_back(e.first); }
        if (!connected(n, g)) continue;
        for (int v = 0; v < n; ++v) {
            std::sort(g[v].begin(), g[v].end());
            std::copy(g[v].begin(), g[v].end(), adj + (size_t)v * d);
        }
        return GG_OK;
    }
    return GG_BAD_ARG;
}

gg_status gg_gen_swaps(int n, int degree, const int32_t *adj, int base_id, int count, uint64_t seed,
                       gg_swap *out) {
    if (!adj || !out || n < 4 || degree < 1 || count < 0) return GG_BAD_ARG;
    // undirected edge list, each edge once
    std::vector<std::pair<int, int>> E;
    for (int v = 0; v < n; ++v)
        for (int k = 0; k < degree; ++k) {
            const int u = adj[(size_t)v * degree + k];
            if (u < 0 || u >= n) return GG_BAD_ARG;
            if (v < u) E.emplace_back(v, u);
        }
    if (E.size() < 2) return GG_BAD_ARG;
    auto has_edge = [&](int x, int y) {
        for (int k = 0; k < degree; ++k)
            if (adj[(size_t)x * degree + k] == y) return true;
        return false;
    };
    Rng rng(seed);
    const uint32_t m = (uint32_t)E.size();
    for (int i = 0; i < count; ++i) {
        for (int tries = 0;; ++tries) {
            if (tries > 1000000) return GG_BAD_ARG;
            auto e1 = E[rng.below(m)], e2 = E[rng.below(m)];
            if (rng.below(2)) std::swap(e1.first, e1.second);
            if (rng.below(2)) std::swap(e2.first, e2.second);
            const int a = e1.first, b = e1.second, c = e2.first, d = e2.second;
            if (a == c || a == d || b == c || b == d) continue;  // needs two disjoint edges
            const int mode = (int)rng.below(2);
            const int p = mode ? d : c, q = mode ? c : d;       // new edges (a,p), (b,q)
            if (has_edge(a, p) || has_edge(b, q)) continue;    // would repeat an edge
            out[i] = gg_swap{base_id, a, b, c, d, mode};
            break;
        }
    }
    return GG_OK;
}

}  // extern "C"

namespace {

// Moves of a lift of K = 1, 2 or 3 axes (see gg.h).  Axis j has the lifted size
// n[j] and the orbit size m[j]; orbit row r has coordinates r_j (row-major, last
// axis fastest, the calculators' table order).  Slot (r, i) holds the diff vector
// of an orbit edge from orbit r to orbit (r_j + diff_j) mod n_j mod m_j; its reverse
// slot is the first slot of that orbit's row holding -diff (componentwise mod n_j),
// the search of cppcode/annealing.cpp:117-124 and pieceannealing.cpp:126-133.  A
// new shift for an edge from orbit x to orbit y is (y_j - x_j) + m_j k_j, k_j
// uniform in [0, n_j / m_j) (annealing.cpp:131, pieceannealing.cpp:135-136).
gg_status lift_moves(int K, const int n[3], const int m[3], int degree, const int32_t *table, int count,
                     uint64_t seed, gg_lift_edit *out) {
    if (!table || !out || K < 1 || K > 3 || degree < 1 || count < 0) return GG_BAD_ARG;
    int M = 1;
    bool lifted = false;
    for (int j = 0; j < K; ++j) {
        if (m[j] < 1 || n[j] < 1 || m[j] > n[j] || n[j] % m[j] != 0) return GG_BAD_ARG;
        M *= m[j];
        lifted |= n[j] / m[j] > 1;
    }
    struct Vec { int32_t c[3]; };
    auto norm = [&](long long x, int j) { return (int32_t)(((x % n[j]) + n[j]) % n[j]); };
    std::vector<Vec> nd((size_t)M * degree);
    for (size_t q = 0; q < nd.size(); ++q) {
        nd[q] = Vec{{0, 0, 0}};
        for (int j = 0; j < K; ++j) nd[q].c[j] = norm(table[q * K + j], j);
    }
    auto at = [&](int r, int i) -> Vec & { return nd[(size_t)r * degree + i]; };
    auto coords = [&](int r, int c[3]) {
        for (int j = K - 1; j >= 0; --j) { c[j] = r % m[j]; r /= m[j]; }
    };
    auto row_of = [&](const int c[3]) {
        int r = 0;
        for (int j = 0; j < K; ++j) r = r * m[j] + c[j];
        return r;
    };
    auto zero = [&](const Vec &v) { return v.c[0] == 0 && v.c[1] == 0 && v.c[2] == 0; };
    auto same = [&](const Vec &a, const Vec &b) { return a.c[0] == b.c[0] && a.c[1] == b.c[1] && a.c[2] == b.c[2]; };
    auto neg = [&](const Vec &v) {
        Vec w{{0, 0, 0}};
        for (int j = 0; j < K; ++j) w.c[j] = norm(-(long long)v.c[j], j);
        return w;
    };
    auto target = [&](int r, const Vec &v) {
        int c[3] = {0, 0, 0};
        coords(r, c);
        for (int j = 0; j < K; ++j) c[j] = (int)(((long long)c[j] + v.c[j]) % n[j] % m[j]);
        return row_of(c);
    };
    auto reverse = [&](int r, int i, int *rr) {
        const int to = target(r, at(r, i));
        const Vec back = neg(at(r, i));
        for (int q = 0; q < degree; ++q)
            if (same(at(to, q), back) && !(to == r && q == i)) { *rr = to; return q; }
        return -1;
    };
    Rng rng(seed);
    auto shift = [&](int from, int to) {
        int a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
        coords(from, a);
        coords(to, b);
        Vec v{{0, 0, 0}};
        for (int j = 0; j < K; ++j)
            v.c[j] = norm((long long)(b[j] - a[j]) + (long long)m[j] * rng.below((uint32_t)(n[j] / m[j])), j);
        return v;
    };
    // rows touched by an edit stay simple: edited slots nonzero, nonzero diffs pairwise distinct
    auto simple_after = [&](int cnt, const int *er, const int *es, const Vec *ev) {
        for (int j = 0; j < cnt; ++j) {
            std::vector<Vec> row(nd.begin() + (size_t)er[j] * degree, nd.begin() + (size_t)(er[j] + 1) * degree);
            std::vector<char> edited(degree, 0);
            for (int k = 0; k < cnt; ++k)
                if (er[k] == er[j]) { row[es[k]] = ev[k]; edited[es[k]] = 1; }
            for (int k = 0; k < degree; ++k) {
                if (zero(row[k])) {
                    if (edited[k]) return false;
                    continue;
                }
                for (int q = k + 1; q < degree; ++q)
                    if (same(row[q], row[k])) return false;
            }
        }
        return true;
    };
    for (int c = 0; c < count; ++c) {
        for (long long tries = 0;; ++tries) {
            if (tries > 1000000) return GG_BAD_ARG;
            const bool sh = lifted && rng.below(2) == 0;
            const int a = (int)rng.below((uint32_t)M), ia = (int)rng.below((uint32_t)degree);
            if (zero(at(a, ia))) continue;
            int b = -1;
            const int ib = reverse(a, ia, &b);
            if (ib < 0) continue;
            int er[4], es[4], cnt;
            Vec ev[4];
            if (sh) {
                const Vec v = shift(a, b);
                cnt = 2;
                er[0] = a; es[0] = ia; ev[0] = v;
                er[1] = b; es[1] = ib; ev[1] = neg(v);
            } else {
                const int cc = (int)rng.below((uint32_t)M), ic = (int)rng.below((uint32_t)degree);
                if (zero(at(cc, ic))) continue;
                int d = -1;
                const int id = reverse(cc, ic, &d);
                if (id < 0) continue;
                const int rs[4] = {a, b, cc, d}, ss[4] = {ia, ib, ic, id};
                bool distinct = true;
                for (int x = 0; x < 4; ++x)
                    for (int y = x + 1; y < 4; ++y) distinct &= !(rs[x] == rs[y] && ss[x] == ss[y]);
                if (!distinct) continue;  // the same orbit edge twice
                // a-b, c-d -> a-d, b-c
                const Vec vad = shift(a, d), vbc = shift(b, cc);
                cnt = 4;
                er[0] = a;  es[0] = ia; ev[0] = vad;
                er[1] = d;  es[1] = id; ev[1] = neg(vad);
                er[2] = b;  es[2] = ib; ev[2] = vbc;
                er[3] = cc; es[3] = ic; ev[3] = neg(vbc);
            }
            if (!simple_after(cnt, er, es, ev)) continue;
            gg_lift_edit e{};
            e.count = cnt;
            for (int j = 0; j < cnt; ++j) {
                e.row[j] = er[j];
                e.slot[j] = es[j];
                for (int q = 0; q < 3; ++q) e.diff[j][q] = ev[j].c[q];
            }
            out[c] = e;
            break;
        }
    }
    return GG_OK;
}

}  // namespace

extern "C" {

gg_status gg_gen_lift_moves(int N, int M, int degree, const int32_t *diffs, int count, uint64_t seed,
                            gg_lift_edit *out) {
    const int n[3] = {N, 1, 1}, m[3] = {M, 1, 1};
    if (N < 2) return GG_BAD_ARG;
    return lift_moves(1, n, m, degree, diffs, count, seed, out);
}

gg_status gg_gen_piece_moves(int Nx, int Ny, int Mx, int My, int degree, const int32_t *vals, int count,
                             uint64_t seed, gg_lift_edit *out) {
    const int n[3] = {Nx, Ny, 1}, m[3] = {Mx, My, 1};
    if ((long long)Nx * Ny < 2) return GG_BAD_ARG;
    return lift_moves(2, n, m, degree, vals, count, seed, out);
}

gg_status gg_gen_box_moves(int Nx, int Ny, int Nz, int Mx, int My, int Mz, int degree, const int32_t *vals,
                           int count, uint64_t seed, gg_lift_edit *out) {
    const int n[3] = {Nx, Ny, Nz}, m[3] = {Mx, My, Mz};
    if ((long long)Nx * Ny * Nz < 2) return GG_BAD_ARG;
    return lift_moves(3, n, m, degree, vals, count, seed, out);
}

gg_status gg_gen_cyclic_lift(int m, int g, int d, uint64_t seed, int32_t *diffs) {
    if (!diffs || m < 1 || g < 1 || d < 1 || ((long long)m * d) % 2 != 0 ||
        (long long)m * g >= (1ll << 31))
        return GG_BAD_ARG;
    const int N = m * g;
    Rng rng(seed);
    for (int attempt = 0; attempt < 100000; ++attempt) {
        std::vector<int> stubs((size_t)m * d);
        for (int v = 0; v < m; ++v)
            for (int k = 0; k < d; ++k) stubs[(size_t)v * d + k] = v;
        for (size_t i = stubs.size(); i > 1; --i) std::swap(stubs[i - 1], stubs[rng.below((uint32_t)i)]);
        std::vector<std::vector<int>> rows(m);
        for (size_t i = 0; i + 1 < stubs.size(); i += 2) {
            int a = stubs[i], b = stubs[i + 1];
            if (a > b) std::swap(a, b);
            const int s = (int)rng.below((uint32_t)g);
            const int diff = (b - a) + m * s;  // quotient edge (a, b, s)
            rows[a].push_back(diff);
            rows[b].push_back(-diff);
        }
        // Simple lift: the neighbours (u + diff) mod N of each orbit vertex u are
        // distinct and differ from u (then every lifted copy of u is simple too).
        bool ok = true;
        for (int u = 0; u < m && ok; ++u) {
            std::unordered_set<long long> seen;
            for (int df : rows[u]) {
                long long to = (((long long)u + df) % N + N) % N;
                if (to == u || !seen.insert(to).second) { ok = false; break; }
            }
        }
        if (!ok) continue;
        // Connected lift.
        std::vector<std::vector<int>> gl(N);
        for (int v = 0; v < N; ++v)
            for (int df : rows[v % m]) gl[v].push_back((int)((((long long)v + df) % N + N) % N));
        if (!connected(N, gl)) continue;
        for (int u = 0; u < m; ++u) std::copy(rows[u].begin(), rows[u].end(), diffs + (size_t)u * d);
        return GG_OK;
    }
    return GG_BAD_ARG;
}

gg_status gg_gen_piece_lift(int Mx, int My, int kx, int ky, int d, uint64_t seed, int32_t *vals) {
    const long long M = (long long)Mx * My, Nx = (long long)Mx * kx, Ny = (long long)My * ky;
    if (!vals || Mx < 1 || My < 1 || kx < 1 || ky < 1 || d < 1 || (M * d) % 2 != 0 || Nx * Ny >= (1ll << 30))
        return GG_BAD_ARG;
    Rng rng(seed);
    for (int attempt = 0; attempt < 100000; ++attempt) {
        std::vector<int> stubs((size_t)M * d);
        for (int v = 0; v < M; ++v)
            for (int k = 0; k < d; ++k) stubs[(size_t)v * d + k] = v;
        for (size_t i = stubs.size(); i > 1; --i) std::swap(stubs[i - 1], stubs[rng.below((uint32_t)i)]);
        std::vector<std::vector<std::pair<int, int>>> rows(M);
        for (size_t i = 0; i + 1 < stubs.size(); i += 2) {
            const int a = stubs[i], b = stubs[i + 1];
            const int ax = a / My, ay = a % My, bx = b / My, by = b % My;
            const int dx = (bx - ax) + Mx * (int)rng.below((uint32_t)kx);
            const int dy = (by - ay) + My * (int)rng.below((uint32_t)ky);
            rows[a].push_back({dx, dy});
            rows[b].push_back({-dx, -dy});
        }
        // simple lift: the neighbours of each tile vertex are distinct and differ from it
        bool ok = true;
        for (int u = 0; u < M && ok; ++u) {
            std::unordered_set<long long> seen;
            const long long ux = u / My, uy = u % My;
            for (auto &p : rows[u]) {
                const long long tx = ((ux + p.first) % Nx + Nx) % Nx, ty = ((uy + p.second) % Ny + Ny) % Ny;
                const long long to = tx * Ny + ty;
                if (to == ux * Ny + uy || !seen.insert(to).second) { ok = false; break; }
            }
        }
        if (!ok) continue;
        const int N = (int)(Nx * Ny);
        std::vector<std::vector<int>> gl(N);
        for (int v = 0; v < N; ++v) {
            const long long x = v / Ny, y = v % Ny;
            for (auto &p : rows[(x % Mx) * My + (y % My)])
                gl[v].push_back((int)((((x + p.first) % Nx + Nx) % Nx) * Ny + (((y + p.second) % Ny + Ny) % Ny)));
        }
        if (!connected(N, gl)) continue;
        for (int u = 0; u < M; ++u)
            for (int k = 0; k < d; ++k) {
                vals[((size_t)u * d + k) * 2] = rows[u][k].first;
                vals[((size_t)u * d + k) * 2 + 1] = rows[u][k].second;
            }
        return GG_OK;
    }
    return GG_BAD_ARG;
}

}  // extern "C"
