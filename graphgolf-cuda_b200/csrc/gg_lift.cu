// gg_lift.cu -- batched exact evaluation of lifted candidates (gg_lift_* in gg.h):
// cyclic lifts ("part"), 2-D and 3-D torus lifts ("piece", "box").
//
// The part form of cudaASPLconv: M orbit vertices with d diffs each; vertex v of
// the N-vertex lift has the neighbours (v + diffs[v % M][i]) mod N, and the BFS
// runs from the M vertices 0..M-1 (cudaASPLconv.cu:197-243).  Piece and box
// tables hold 2- or 3-component diffs per orbit of a corner tile, the BFS runs
// from that tile (cudaASPLpiece.cu:159-216, cudaASPLbox.cu:166-226).  The
// reference's annealers change 2 or 4 slots of the table per proposal
// (cppcode/annealing.cpp:112-197, pieceannealing.cpp:113-204) and score each with
// one calculator call.
//
// Here one cooperative launch scores a population.  `lift_tables` writes every
// candidate's table (base + edit, diffs reduced to [0, n) per axis); for piece and
// box, `lift_expand` turns each into a pull adjacency and the kernel's EXPL
// variant reads adjacency rows and finds sources through a vertex ->
// representative map.  `lift_kernel`
// runs the candidates in rounds of G side by side: a round's bitsets hold, per
// vertex, W = G * cpc uint4 chunks (cpc = ceil(M/128)), chunk group g being the
// M sources of candidate g of the round, source s at bit s % 128 of chunk s / 128
// of its group.  A level is one pass over all (vertex, chunk) items:
//     new = (OR_i F[(v + diff_g[v % M][i]) mod N][w]) & ~V[v][w];  V |= new;  F' = new
// where g is the item's group, so neighbours always come from the item's own
// candidate.  Each thread owns one chunk column w (so one group, one counter and
// one table) and walks the vertices v = v0, v0 + VS, ...; consecutive lanes own
// consecutive columns, so the gathers of a neighbour row are contiguous 16-byte
// loads, all issued before the first is used.  Level 1 is the round's reset pass
// (a chunk's level-1 pairs are the sources among its own neighbours: no gather).
// Late in a round (past 85 % of its
// pairs reached) a chunk gathers half its neighbours first and the rest only
// while it still misses sources.  New pairs are counted per thread, reduced per
// group at the end of the level (shared atomics, then one global atomic per block
// and group into counts[L][k]); after the grid barrier every block reads the
// round's counts, and the round ends when no candidate found a pair or every
// candidate reached all M*N pairs.
#include "gg.h"
#include "gg_internal.h"
#include "gg_kernels.cuh"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

constexpr int kLiftBlock = 256;
constexpr int kMaxGroup = 32;
constexpr int kFirstLevels = 256;   // count rows a launch starts with (see gg_lift_eval)

struct LiftArgs {
    const int32_t *tab;              // part form: [K][M][d] diffs in [0, N), rows 16-byte aligned when d % 4 == 0
    const int32_t *adj;              // piece / box: [K][N][d] pull adjacency of each candidate
    const int32_t *inv;              // piece / box: [N] representative index of a vertex, or -1
    int N, M, d, K, G, cpc, W;       // W = G * cpc chunks per vertex
    unsigned cols_threads;           // threads that own a column: the largest multiple of W <= grid threads
    unsigned vstep;                  // cols_threads / W: vertices between a thread's items
    int half_ppm;                    // past this share of the round's pairs reached: half gathers
    uint4 *V, *F0, *F1;              // [N][W]
    unsigned long long *counts;      // [max_levels + 1][K]: pairs first reached at level L
    int max_levels;
    unsigned long long *level_ns;    // [max_levels + 1]: device clock at the start ([0]) and
                                     // at the end of each level of the first round
    gg::Ctl *ctl;
    unsigned expected;
    long long wait_ns;
};

// Candidate tables ([K][M][d][comps], comps = axes of the lift): slot (k, r, i)
// is the base slot unless candidate k's edit names slot (r, i).
__global__ void lift_tables(const int32_t *base, const gg_lift_edit *ed, int K, int M, int d, int comps,
                            int32_t *tab) {
    const long long per = (long long)M * d, total = per * K;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total;
         x += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(x / per);
        const int e = (int)(x - (long long)k * per);
        const int r = e / d, i = e - r * d;
        const gg_lift_edit &q = ed[k];
        int hit = -1;
        for (int j = 0; j < q.count; ++j)
            if (q.row[j] == r && q.slot[j] == i) hit = j;
        for (int c = 0; c < comps; ++c)
            tab[x * comps + c] = hit >= 0 ? q.diff[hit][c] : __ldg(base + (size_t)e * comps + c);
    }
}

// Pull adjacency of every candidate of a 2-D or 3-D torus lift (axes sizes n,
// orbit sizes m; vertex (x * ny + y) * nz + z), from its table of diffs already
// reduced to [0, n): the expansion of cudaASPLpiece.cu:41-50 / cudaASPLbox.cu:44-57.
// One thread per (candidate, vertex): the coordinates and the orbit row once, then
// the row's d entries.
__global__ void lift_expand(const int32_t *tab, int K, int M, int d, int comps, int nx, int ny, int nz, int mx,
                            int my, int mz, int32_t *adj) {
    const long long N = (long long)nx * ny * nz, total = N * K;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(q / N);
        const int v = (int)(q - (long long)k * N);
        const int x = v / (ny * nz), rem = v - x * (ny * nz), y = rem / nz, z = rem - y * nz;
        const int r = ((x % mx) * my + (y % my)) * mz + (z % mz);
        const int32_t *t = tab + ((size_t)k * M + r) * d * comps;
        int32_t *out = adj + (size_t)q * d;
        for (int i = 0; i < d; ++i) {
            int tx = x + __ldg(t + i * comps), ty = y + __ldg(t + i * comps + 1);
            int tz = comps > 2 ? z + __ldg(t + i * comps + 2) : z;
            tx -= tx >= nx ? nx : 0;
            ty -= ty >= ny ? ny : 0;
            tz -= tz >= nz ? nz : 0;
            out[i] = (tx * ny + ty) * nz + tz;
        }
    }
}

// OR of F[u][w] over the neighbours u of slots [B, E) of `row` (u = v + diff,
// diff in [0, N)): every load of the span is issued before the first is used.
template <int B, int E, bool EXPL>
__device__ __forceinline__ void gather_span(const int32_t *row, unsigned v, unsigned w, unsigned N, unsigned W,
                                            const uint4 *Fc, uint4 &acc) {
    int32_t df[E - B];
    if constexpr (B % 4 == 0 && (E - B) % 4 == 0) {
#pragma unroll
        for (int i = 0; i < E - B; i += 4) {
            const int4 q = __ldg(reinterpret_cast<const int4 *>(row + B + i));
            df[i] = q.x; df[i + 1] = q.y; df[i + 2] = q.z; df[i + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < E - B; ++i) df[i] = __ldg(row + B + i);
    }
    uint4 x[E - B];
#pragma unroll
    for (int i = 0; i < E - B; ++i) {
        unsigned u = (unsigned)df[i];
        if constexpr (!EXPL) {   // a diff: u = (v + diff) mod N
            u += v;
            u -= u >= N ? N : 0u;
        }
        x[i] = __ldcg(Fc + (size_t)u * W + w);
    }
#pragma unroll
    for (int i = 0; i < E - B; ++i) gg::or_into(acc, x[i]);
}

// The same for a run-time degree: slots [b, e).
template <bool EXPL>
__device__ __forceinline__ void gather_any(const int32_t *row, int b, int e, unsigned v, unsigned w, unsigned N,
                                           unsigned W, const uint4 *Fc, uint4 &acc) {
#pragma unroll 4
    for (int i = b; i < e; ++i) {
        unsigned u = (unsigned)__ldg(row + i);
        if constexpr (!EXPL) {
            u += v;
            u -= u >= N ? N : 0u;
        }
        gg::or_into(acc, __ldcg(Fc + (size_t)u * W + w));
    }
}

// Representative index of vertex u: u itself for a part (sources 0..M-1),
// inv[u] for a piece or box; -1 for a vertex that is no source.
template <bool EXPL>
__device__ __forceinline__ int source_of(unsigned u, unsigned M, const int32_t *inv) {
    if constexpr (EXPL) return __ldg(inv + u);
    else return u < M ? (int)u : -1;
}

// The sources among the pull neighbours of v (row `row`, slots [B, E)) that lie in
// the chunk of sources [lo, lo + 128), as bits.
template <int B, int E, bool EXPL>
__device__ __forceinline__ void sources_span(const int32_t *row, unsigned v, unsigned lo, unsigned N, unsigned M,
                                             const int32_t *inv, unsigned nb[4]) {
    int32_t df[E - B];
    if constexpr (B % 4 == 0 && (E - B) % 4 == 0) {
#pragma unroll
        for (int i = 0; i < E - B; i += 4) {
            const int4 q = __ldg(reinterpret_cast<const int4 *>(row + B + i));
            df[i] = q.x; df[i + 1] = q.y; df[i + 2] = q.z; df[i + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < E - B; ++i) df[i] = __ldg(row + B + i);
    }
#pragma unroll
    for (int i = 0; i < E - B; ++i) {
        unsigned u = (unsigned)df[i];
        if constexpr (!EXPL) {
            u += v;
            u -= u >= N ? N : 0u;
        }
        const int sv = source_of<EXPL>(u, M, inv);
        const unsigned o = (unsigned)sv - lo;
        if (sv >= 0 && o < 128u) nb[o >> 5] |= 1u << (o & 31u);
    }
}

// The reset pass of a round with level 1 folded in: the pairs a chunk (v, w)
// reaches at level 1 are the sources among its pull neighbours that lie in the
// chunk, so the pass writes the padding bits, the diagonal and those pairs into V
// and their frontier into F1 (`Fn`) without a gather.  Columns of candidates past
// the last one (mine == false) start full.  `rows`: the column's candidate's diff
// table (part, row v % M) or pull adjacency (piece / box, row v).  Returns the
// thread's new pairs.
template <int D, bool EXPL>
__device__ __forceinline__ unsigned level1_pass(const LiftArgs &a, const int32_t *rows, unsigned v0,
                                                unsigned vstep, unsigned rstep, unsigned w, unsigned cc,
                                                bool mine, uint4 *Fn) {
    const unsigned N = (unsigned)a.N, M = (unsigned)a.M, W = (unsigned)a.W;
    const uint4 pad = mine ? gg::pad_mask((int)cc, a.M)
                           : make_uint4(0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu);
    const unsigned lo = cc * 128u;     // sources of this chunk: [lo, lo + 128) of the group
    unsigned cnt = 0, r = v0 % M;
    for (unsigned v = v0; v < N; v += vstep) {
        uint4 vis = pad, n1 = gg::u4zero();
        if (mine) {
            const int sv = source_of<EXPL>(v, M, a.inv);
            const unsigned o = (unsigned)sv - lo;
            if (sv >= 0 && o < 128u) {   // the diagonal
                const unsigned bit = 1u << (o & 31u);
                switch (o >> 5) {
                    case 0: vis.x |= bit; break;
                    case 1: vis.y |= bit; break;
                    case 2: vis.z |= bit; break;
                    default: vis.w |= bit; break;
                }
            }
            const int32_t *row = rows + (size_t)(EXPL ? v : r) * a.d;
            unsigned nb[4] = {0u, 0u, 0u, 0u};
            if constexpr (D > 0) {
                sources_span<0, D, EXPL>(row, v, lo, N, M, a.inv, nb);
            } else {
                for (int i = 0; i < a.d; ++i) {
                    unsigned u = (unsigned)__ldg(row + i);
                    if constexpr (!EXPL) {
                        u += v;
                        u -= u >= N ? N : 0u;
                    }
                    const int su = source_of<EXPL>(u, M, a.inv);
                    const unsigned ou = (unsigned)su - lo;
                    if (su >= 0 && ou < 128u) nb[ou >> 5] |= 1u << (ou & 31u);
                }
            }
            n1 = gg::andnot(make_uint4(nb[0], nb[1], nb[2], nb[3]), vis);
            gg::or_into(vis, n1);
            cnt += gg::u4popc(n1);
        }
        a.V[(size_t)v * W + w] = vis;
        Fn[(size_t)v * W + w] = n1;
        r += rstep;
        r -= r >= M ? M : 0u;
    }
    return cnt;
}

// D > 0: the degree at compile time; D == 0: a.d at run time.  EXPL: piece / box
// (per-candidate pull adjacency and representative map); otherwise part (diffs).
template <int D, bool EXPL>
__global__ void __launch_bounds__(kLiftBlock, 4) lift_kernel(const LiftArgs a) {
    __shared__ unsigned s_cnt[kMaxGroup];
    __shared__ unsigned long long s_reached[kMaxGroup];
    __shared__ int s_half;
    if (threadIdx.x < kMaxGroup) s_cnt[threadIdx.x] = 0u;
    unsigned epoch = 0;
    const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x;
    // this thread's column (threads past cols_threads own none)
    const bool owner = tid < a.cols_threads;
    const unsigned w = owner ? tid % (unsigned)a.W : 0u;
    const unsigned g = w / (unsigned)a.cpc, cc = w - g * (unsigned)a.cpc;
    const unsigned v0 = owner ? tid / (unsigned)a.W : (unsigned)a.N;
    const unsigned N = (unsigned)a.N, W = (unsigned)a.W, M = (unsigned)a.M;
    const unsigned vstep = a.vstep, rstep = vstep % M;
    const unsigned long long all_pairs = (unsigned long long)a.M * (unsigned long long)a.N;
    const int dh = a.d / 2;
    const int rounds = (a.K + a.G - 1) / a.G;
    int zeroed = 1;        // rows 0 and 1 of counts are zeroed by the host
    int levels_run = 0;
    for (int rd = 0; rd < rounds; ++rd) {
        const int k0 = rd * a.G;
        const int live = min(a.G, a.K - k0);
        const bool mine = owner && (int)g < live;   // a column of a live candidate
        const int kc = k0 + (mine ? (int)g : 0);
        const int32_t *rows = EXPL ? a.adj + (size_t)kc * a.N * a.d : a.tab + (size_t)kc * a.M * a.d;
        if (threadIdx.x == 0) s_half = 0;   // read after the next barrier
        if (rd == 0 && a.level_ns && blockIdx.x == 0 && threadIdx.x == 0) a.level_ns[0] = gg::gtimer();
        unsigned long long reached = threadIdx.x < (unsigned)live ? (unsigned long long)a.M : 0ull;
        for (int L = 1; L <= a.max_levels; ++L) {
            const uint4 *Fc = (L & 1) ? a.F0 : a.F1;
            uint4 *Fn = (L & 1) ? a.F1 : a.F0;
            // the next level's count row, before any block can add to it
            if (blockIdx.x == 0 && L + 1 > zeroed && L + 1 <= a.max_levels)
                for (int k = threadIdx.x; k < a.K; k += blockDim.x) a.counts[(size_t)(L + 1) * a.K + k] = 0ull;
            zeroed = max(zeroed, L + 1);
            unsigned cnt = 0;
            unsigned r = v0 % M;
            if (L == 1) {
                // level 1 is the round's reset pass
                cnt = level1_pass<D, EXPL>(a, rows, v0, vstep, rstep, w, cc, mine, Fn);
            } else {
                const bool half = s_half != 0;
                for (unsigned v = v0; v < N; v += vstep) {
                    const size_t t = (size_t)v * W + w;
                    const uint4 own = __ldcg(a.V + t);
                    uint4 nw = gg::u4zero();
                    if (!gg::u4full(own)) {
                        // full from the reset pass unless the column is a live candidate's
                        const int32_t *row = rows + (size_t)(EXPL ? v : r) * a.d;
                        uint4 acc = gg::u4zero();
                        if constexpr (D > 0) {
                            if (!half && D <= 12) {
                                gather_span<0, D, EXPL>(row, v, w, N, W, Fc, acc);
                            } else if (!half) {   // two spans keep the loads within the registers
                                gather_span<0, D / 2, EXPL>(row, v, w, N, W, Fc, acc);
                                gather_span<D / 2, D, EXPL>(row, v, w, N, W, Fc, acc);
                            } else {
                                gather_span<0, D / 2, EXPL>(row, v, w, N, W, Fc, acc);
                                if (!gg::u4full(gg::u4or(own, acc))) gather_span<D / 2, D, EXPL>(row, v, w, N, W, Fc, acc);
                            }
                        } else {
                            gather_any<EXPL>(row, 0, half ? dh : a.d, v, w, N, W, Fc, acc);
                            if (half && !gg::u4full(gg::u4or(own, acc))) gather_any<EXPL>(row, dh, a.d, v, w, N, W, Fc, acc);
                        }
                        nw = gg::andnot(acc, own);
                        if (gg::u4any(nw)) {
                            a.V[t] = gg::u4or(own, nw);
                            cnt += gg::u4popc(nw);
                        }
                    }
                    Fn[t] = nw;
                    r += rstep;   // (v + vstep) % M
                    r -= r >= M ? M : 0u;
                }
            }
            // per group: lanes of one group share a key
            const int key = cnt ? (int)g : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            const unsigned sum = __reduce_add_sync(peers, cnt);
            if (key >= 0 && (int)(threadIdx.x & 31u) == __ffs((int)peers) - 1) atomicAdd(&s_cnt[key], sum);
            __syncthreads();
            if (threadIdx.x < (unsigned)live && s_cnt[threadIdx.x]) {
                atomicAdd(a.counts + (size_t)L * a.K + k0 + threadIdx.x, (unsigned long long)s_cnt[threadIdx.x]);
                s_cnt[threadIdx.x] = 0u;
            }
            if (!gg::grid_sync(a.ctl, a.expected, a.wait_ns, L, epoch)) return;
            if (rd == 0 && a.level_ns && blockIdx.x == 0 && threadIdx.x == 0) a.level_ns[L] = gg::gtimer();
            levels_run = max(levels_run, L);
            int more = 0;
            if (threadIdx.x < (unsigned)live) {
                const unsigned long long n = gg::ld_relaxed_u64(a.counts + (size_t)L * a.K + k0 + threadIdx.x);
                reached += n;
                more = n != 0ull && reached < all_pairs;
                s_reached[threadIdx.x] = reached;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned long long sum_r = 0;
                for (int q = 0; q < live; ++q) sum_r += s_reached[q];
                s_half = (double)sum_r > (double)a.half_ppm * 1e-6 * (double)live * (double)all_pairs;
            }
            if (!__syncthreads_or(more)) break;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl->levels_run = levels_run;
}

template <bool EXPL>
void *lift_kernel_for_t(int d) {
    switch (d) {
        case 3: return (void *)lift_kernel<3, EXPL>;
        case 4: return (void *)lift_kernel<4, EXPL>;
        case 5: return (void *)lift_kernel<5, EXPL>;
        case 6: return (void *)lift_kernel<6, EXPL>;
        case 8: return (void *)lift_kernel<8, EXPL>;
        case 10: return (void *)lift_kernel<10, EXPL>;
        case 12: return (void *)lift_kernel<12, EXPL>;
        case 16: return (void *)lift_kernel<16, EXPL>;
        default: return (void *)lift_kernel<0, EXPL>;
    }
}
void *lift_kernel_for(int d, bool expl) { return expl ? lift_kernel_for_t<true>(d) : lift_kernel_for_t<false>(d); }

gg_status lfail(gg_status s, const std::string &m) {
    (void)cudaGetLastError();
    gg::set_last_error(m.c_str());
    return s;
}

#define GL_CK(call)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return lfail(e_ == cudaErrorMemoryAllocation ? GG_OUT_OF_MEMORY : GG_CUDA_ERROR, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                \
    } while (0)

}  // namespace

struct gg_lift {
    int N = 0, M = 0, d = 0, device = 0;
    int axes = 1;                                    // 1 part, 2 piece, 3 box
    int n[3] = {1, 1, 1}, m[3] = {1, 1, 1};          // lifted and orbit size of each axis
    int32_t *d_inv = nullptr;                        // piece / box: [N] representative index or -1
    int32_t *d_adj = nullptr;                        // piece / box: [cap][N][d] candidate adjacency
    int cpc = 0, g_auto = 1, g_max = 0, group = 0;   // group 0: automatic
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int32_t *d_base = nullptr, *d_tab = nullptr;
    gg_lift_edit *d_ed = nullptr, *h_ed = nullptr;
    int cap = 0;                                     // candidates the buffers hold
    uint4 *V = nullptr, *F0 = nullptr, *F1 = nullptr;
    unsigned long long *d_counts = nullptr, *h_counts = nullptr;
    size_t counts_cap = 0;                           // entries
    gg::Ctl *d_ctl = nullptr, *h_ctl = nullptr;
    unsigned long long *d_level_ns = nullptr, *h_level_ns = nullptr;
    int level_ns_n = 0;                              // entries the buffers hold
    int grid = 0;                                    // blocks of the cooperative launch
    int half_ppm = 850000;
    long long wait_ns = 10ll * 1000 * 1000 * 1000;
    bool base_set = false;
    float last_ms = 0.f;
};

namespace {

void lift_free(gg_lift *h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->d_base); cudaFree(h->d_tab); cudaFree(h->d_ed); cudaFreeHost(h->h_ed);
    cudaFree(h->d_inv); cudaFree(h->d_adj);
    cudaFree(h->V); cudaFree(h->F0); cudaFree(h->F1);
    cudaFree(h->d_counts); cudaFreeHost(h->h_counts);
    cudaFree(h->d_level_ns); cudaFreeHost(h->h_level_ns);
    cudaFree(h->d_ctl); cudaFreeHost(h->h_ctl);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

gg_status ensure_cand(gg_lift *h, int n) {
    if (n <= h->cap) return GG_OK;
    int cap = std::max(n, 2 * h->cap);
    cudaFree(h->d_tab); cudaFree(h->d_ed); cudaFreeHost(h->h_ed); cudaFree(h->d_adj);
    h->d_tab = nullptr; h->d_ed = nullptr; h->h_ed = nullptr; h->d_adj = nullptr; h->cap = 0;
    GL_CK(cudaMalloc(&h->d_tab, (size_t)cap * h->M * h->d * h->axes * sizeof(int32_t)));
    if (h->axes > 1) GL_CK(cudaMalloc(&h->d_adj, (size_t)cap * h->N * h->d * sizeof(int32_t)));
    GL_CK(cudaMalloc(&h->d_ed, (size_t)cap * sizeof(gg_lift_edit)));
    GL_CK(cudaMallocHost(&h->h_ed, (size_t)cap * sizeof(gg_lift_edit)));
    h->cap = cap;
    return GG_OK;
}

gg_status ensure_counts(gg_lift *h, size_t entries) {
    if (entries <= h->counts_cap) return GG_OK;
    const size_t cap = std::max(entries, 2 * h->counts_cap);
    cudaFree(h->d_counts); cudaFreeHost(h->h_counts);
    h->d_counts = nullptr; h->h_counts = nullptr; h->counts_cap = 0;
    GL_CK(cudaMalloc(&h->d_counts, cap * sizeof(unsigned long long)));
    GL_CK(cudaMallocHost(&h->h_counts, cap * sizeof(unsigned long long)));
    h->counts_cap = cap;
    return GG_OK;
}

std::string lift_tune_key(const gg_lift *h) {
    return gg::tune_key(h->device, "lift", {h->axes, h->n[0], h->n[1], h->n[2], h->m[0], h->m[1], h->m[2], h->d});
}

gg_status alloc_group(gg_lift *h, int groups) {
    cudaFree(h->V); cudaFree(h->F0); cudaFree(h->F1);
    h->V = h->F0 = h->F1 = nullptr;
    h->g_max = 0;
    const size_t bits = (size_t)h->N * h->cpc * groups * sizeof(uint4);
    GL_CK(cudaMalloc(&h->V, bits));
    GL_CK(cudaMalloc(&h->F0, bits));
    GL_CK(cudaMalloc(&h->F1, bits));
    h->g_max = groups;
    return GG_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// A handle for a lift of `axes` axes: lifted sizes n, orbit sizes m.
gg_status lift_open(int axes, const int n_in[3], const int m_in[3], int degree, int device, gg_lift **out) {
    if (!out) return lfail(GG_BAD_ARG, "null argument");
    *out = nullptr;
    long long N = 1, M = 1;
    for (int j = 0; j < axes; ++j) {
        if (m_in[j] < 1 || n_in[j] < 1 || m_in[j] > n_in[j] || n_in[j] % m_in[j] != 0)
            return lfail(GG_BAD_ARG, "every lifted size must be a positive multiple of its orbit size");
        N *= n_in[j];
        M *= m_in[j];
    }
    if (N < 2 || N >= (1ll << 30) || degree < 1 || degree > 4096)
        return lfail(GG_BAD_ARG, "need 2 <= N < 2^30 vertices and 1 <= degree <= 4096");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return lfail(GG_NO_DEVICE, "no such CUDA device");
    gg_lift *h = new gg_lift();
    h->axes = axes;
    for (int j = 0; j < axes; ++j) { h->n[j] = n_in[j]; h->m[j] = m_in[j]; }
    h->N = (int)N; h->M = (int)M; h->d = degree; h->device = device;
    h->cpc = (h->M + 127) / 128;
    auto fail = [&](gg_status s) { lift_free(h); return s; };
    if (cudaSetDevice(device) != cudaSuccess) return fail(lfail(GG_NO_DEVICE, "cudaSetDevice failed"));
    int l2 = 0, coop = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lift_kernel_for(degree, axes > 1), kLiftBlock, 0) !=
            cudaSuccess)
        return fail(lfail(GG_CUDA_ERROR, "device query failed"));
    if (!coop || per_sm < 1) return fail(lfail(GG_CUDA_ERROR, "cooperative launch unavailable"));
    h->grid = per_sm * h->sms;
    // one candidate's round share: three bitsets of N * cpc uint4
    // (half the L2: lines gathered from both dies' SMs are held in both halves;
    // at m=1024, g=32, d=12 a sweep of 2-8 candidates per round put the optimum at 5)
    const double per_cand = 3.0 * h->N * h->cpc * 16.0;
    const int fit = (int)std::max(1.0, 0.5 * l2 / per_cand);
    // items N * W must stay below 2^31
    const long long by_items = std::max(1ll, (1ll << 31) / ((long long)h->N * h->cpc));
    h->g_auto = (int)std::min<long long>({(long long)fit, (long long)kMaxGroup, by_items});
    {
        // a group recorded by gg_lift_autotune for this lift shape on this kind of GPU
        std::vector<int> tuned;
        if (gg::tune_get(lift_tune_key(h), &tuned) && !tuned.empty() && tuned[0] >= 1 &&
            tuned[0] <= kMaxGroup && tuned[0] <= by_items)
            h->g_auto = tuned[0];
    }
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_base, (size_t)h->M * degree * axes * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_ctl, sizeof(gg::Ctl));
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_ctl, sizeof(gg::Ctl));
    if (e == cudaSuccess && axes > 1) {
        // representatives: the corner tile, numbered like the table's rows
        // (cpuASPLpiece.cpp:199-200, cpuASPLbox.cpp:133-134)
        std::vector<int32_t> inv((size_t)h->N, -1);
        const int nz = h->n[2], ny = h->n[1];
        for (int x = 0; x < h->m[0]; ++x)
            for (int y = 0; y < h->m[1]; ++y)
                for (int z = 0; z < h->m[2]; ++z)
                    inv[((size_t)x * ny + y) * nz + z] = (x * h->m[1] + y) * h->m[2] + z;
        e = cudaMalloc(&h->d_inv, inv.size() * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMemcpy(h->d_inv, inv.data(), inv.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess)
        return fail(lfail(e == cudaErrorMemoryAllocation ? GG_OUT_OF_MEMORY : GG_CUDA_ERROR,
                          cudaGetErrorString(e)));
    // bitsets for the automatic group (a larger group set later reallocates)
    const gg_status s = alloc_group(h, h->g_auto);
    if (s != GG_OK) return fail(s);
    *out = h;
    return GG_OK;
}

}  // namespace

extern "C" {

gg_status gg_lift_create(int N, int M, int degree, int device, gg_lift **out) {
    const int n[3] = {N, 1, 1}, m[3] = {M, 1, 1};
    return lift_open(1, n, m, degree, device, out);
}

gg_status gg_lift_create_piece(int Nx, int Ny, int Mx, int My, int degree, int device, gg_lift **out) {
    const int n[3] = {Nx, Ny, 1}, m[3] = {Mx, My, 1};
    return lift_open(2, n, m, degree, device, out);
}

gg_status gg_lift_create_box(int Nx, int Ny, int Nz, int Mx, int My, int Mz, int degree, int device,
                             gg_lift **out) {
    const int n[3] = {Nx, Ny, Nz}, m[3] = {Mx, My, Mz};
    return lift_open(3, n, m, degree, device, out);
}

gg_status gg_lift_set_base(gg_lift *h, const int32_t *table) {
    if (!h || !table) return lfail(GG_BAD_ARG, "null argument");
    std::vector<int32_t> nd((size_t)h->M * h->d * h->axes);
    for (size_t k = 0; k < nd.size(); ++k) {
        const long long n = h->n[k % h->axes];
        nd[k] = (int32_t)((((long long)table[k] % n) + n) % n);
    }
    GL_CK(cudaSetDevice(h->device));
    GL_CK(cudaMemcpyAsync(h->d_base, nd.data(), nd.size() * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
    GL_CK(cudaStreamSynchronize(h->stream));
    h->base_set = true;
    return GG_OK;
}

gg_status gg_lift_set_group(gg_lift *h, int group) {
    if (!h || group < 0 || group > kMaxGroup) return lfail(GG_BAD_ARG, "group must be in [0, 32]");
    if (group > 0 && (long long)h->N * h->cpc * group >= (1ll << 31))
        return lfail(GG_BAD_ARG, "group too large for this lift");
    const int need = group ? group : h->g_auto;
    if (need > h->g_max) {
        GL_CK(cudaSetDevice(h->device));
        GL_CK(cudaStreamSynchronize(h->stream));
        const gg_status s = alloc_group(h, need);
        if (s != GG_OK) return s;
    }
    h->group = group;
    return GG_OK;
}

gg_status gg_lift_autotune(gg_lift *h, int n_cand, const gg_lift_edit *edits, int max_levels, int trials,
                           int *best_group, double *best_ms) {
    if (!h || n_cand < 1 || !edits || trials < 1 || max_levels < 0) return lfail(GG_BAD_ARG, "bad arguments");
    if (!h->base_set) return lfail(GG_BAD_ARG, "no base table set");
    std::vector<gg_cand_result> out((size_t)n_cand);
    const int keep = h->group;
    int best = 0;
    double best_t = 1e300;
    const long long by_items = std::max(1ll, (1ll << 31) / ((long long)h->N * h->cpc));
    for (int G = 1; G <= std::min<long long>({(long long)kMaxGroup, by_items, (long long)n_cand}); ++G) {
        if (G > 12 && G != 16 && G != 24 && G != 32) continue;
        gg_status s = gg_lift_set_group(h, G);
        if (s == GG_OUT_OF_MEMORY) { (void)cudaGetLastError(); break; }
        if (s != GG_OK) return s;
        s = gg_lift_eval(h, n_cand, edits, max_levels, out.data());  // warm
        if (s == GG_BAD_ARG) break;  // more chunk columns than threads: larger groups fail too
        if (s != GG_OK) return s;
        double t = 1e300;
        for (int k = 0; k < trials; ++k) {
            s = gg_lift_eval(h, n_cand, edits, max_levels, out.data());
            if (s != GG_OK) return s;
            t = std::min(t, (double)h->last_ms);
        }
        if (t < best_t) { best_t = t; best = G; }
    }
    if (!best) {
        gg_lift_set_group(h, keep);
        return lfail(GG_OUT_OF_MEMORY, "no group fits");
    }
    gg::tune_put(lift_tune_key(h), {best});
    h->g_auto = best;
    gg_status s = gg_lift_set_group(h, 0);
    if (s != GG_OK) return s;
    if (best_group) *best_group = best;
    if (best_ms) *best_ms = best_t;
    return GG_OK;
}

gg_status gg_lift_group(gg_lift *h, int *group) {
    if (!h || !group) return lfail(GG_BAD_ARG, "null argument");
    *group = h->group ? h->group : h->g_auto;
    return GG_OK;
}

gg_status gg_lift_eval(gg_lift *h, int n_cand, const gg_lift_edit *edits, int max_levels,
                       gg_cand_result *out) {
    if (!h || n_cand < 0 || (n_cand && (!edits || !out)) || max_levels < 0)
        return lfail(GG_BAD_ARG, "bad arguments");
    if (!h->base_set) return lfail(GG_BAD_ARG, "no base table set");
    if (n_cand == 0) return GG_OK;
    if (h->g_max < 1) return lfail(GG_OUT_OF_MEMORY, "bitsets were not allocated");
    GL_CK(cudaSetDevice(h->device));
    gg_status s = ensure_cand(h, n_cand);
    if (s != GG_OK) return s;
    for (int k = 0; k < n_cand; ++k) {
        const gg_lift_edit &q = edits[k];
        if (q.count < 0 || q.count > 4) return lfail(GG_BAD_ARG, "edit count must be in [0, 4]");
        gg_lift_edit &o = h->h_ed[k];
        o = gg_lift_edit{};
        o.count = q.count;
        for (int j = 0; j < q.count; ++j) {
            if (q.row[j] < 0 || q.row[j] >= h->M || q.slot[j] < 0 || q.slot[j] >= h->d)
                return lfail(GG_BAD_ARG, "edit slot outside the table");
            o.row[j] = q.row[j];
            o.slot[j] = q.slot[j];
            for (int c = 0; c < h->axes; ++c) {
                const long long n = h->n[c];
                o.diff[j][c] = (int32_t)((((long long)q.diff[j][c] % n) + n) % n);
            }
        }
    }
    // Count rows for the first kFirstLevels levels; a population where some candidate
    // still finds pairs there (a lift of very large diameter) runs again with rows
    // for the full cap, so the buffers stay small for the usual diameters.
    const int ml_full = max_levels > 0 ? std::min(max_levels, h->N) : h->N;
    for (int ml = std::min(ml_full, kFirstLevels);; ml = ml_full) {
        s = ensure_counts(h, (size_t)(ml + 1) * n_cand);
        if (s != GG_OK) return s;
        if (ml + 1 > h->level_ns_n) {
            cudaFree(h->d_level_ns); cudaFreeHost(h->h_level_ns);
            h->d_level_ns = nullptr; h->h_level_ns = nullptr; h->level_ns_n = 0;
            GL_CK(cudaMalloc(&h->d_level_ns, (size_t)(ml + 1) * sizeof(unsigned long long)));
            GL_CK(cudaMallocHost(&h->h_level_ns, (size_t)(ml + 1) * sizeof(unsigned long long)));
            h->level_ns_n = ml + 1;
        }
        const int G = std::min(h->group ? h->group : h->g_auto, n_cand);
        const cudaStream_t st = h->stream;
        GL_CK(cudaMemcpyAsync(h->d_ed, h->h_ed, (size_t)n_cand * sizeof(gg_lift_edit), cudaMemcpyHostToDevice, st));
        GL_CK(cudaMemsetAsync(h->d_ctl, 0, sizeof(gg::Ctl), st));
        GL_CK(cudaMemsetAsync(h->d_counts, 0, (size_t)std::min(ml + 1, 2) * n_cand * sizeof(unsigned long long), st));
        GL_CK(cudaEventRecord(h->ev0, st));
        const long long tab_n = (long long)n_cand * h->M * h->d;
        lift_tables<<<(int)std::min<long long>((tab_n + 255) / 256, (long long)h->sms * 16), 256, 0, st>>>(
            h->d_base, h->d_ed, n_cand, h->M, h->d, h->axes, h->d_tab);
        GL_CK(cudaGetLastError());
        if (h->axes > 1) {
            const long long rows_n = (long long)n_cand * h->N;
            lift_expand<<<(int)std::min<long long>((rows_n + 255) / 256, (long long)h->sms * 16), 256, 0, st>>>(
                h->d_tab, n_cand, h->M, h->d, h->axes, h->n[0], h->n[1], h->n[2], h->m[0], h->m[1], h->m[2], h->d_adj);
            GL_CK(cudaGetLastError());
        }
        LiftArgs a{};
        a.tab = h->d_tab;
        a.adj = h->d_adj;
        a.inv = h->d_inv;
        a.N = h->N; a.M = h->M; a.d = h->d; a.K = n_cand; a.G = G; a.cpc = h->cpc; a.W = G * h->cpc;
        a.V = h->V; a.F0 = h->F0; a.F1 = h->F1;
        a.counts = h->d_counts;
        a.max_levels = ml;
        const unsigned threads = (unsigned)h->grid * kLiftBlock;
        if ((unsigned)a.W > threads) return lfail(GG_BAD_ARG, "more chunk columns than threads: lower the group");
        a.cols_threads = threads / (unsigned)a.W * (unsigned)a.W;
        a.vstep = a.cols_threads / (unsigned)a.W;
        a.half_ppm = h->half_ppm;
        a.level_ns = h->d_level_ns;
        a.ctl = h->d_ctl;
        a.wait_ns = h->wait_ns;
        a.expected = (unsigned)h->grid;
        GL_CK(cudaMemsetAsync(h->d_level_ns, 0, (size_t)(ml + 1) * sizeof(unsigned long long), st));
        void *args[] = {&a};
        GL_CK(cudaLaunchCooperativeKernel(lift_kernel_for(h->d, h->axes > 1), dim3(h->grid), dim3(kLiftBlock), args, 0,
                                          st));
        GL_CK(cudaEventRecord(h->ev1, st));
        GL_CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(gg::Ctl), cudaMemcpyDeviceToHost, st));
        GL_CK(cudaStreamSynchronize(st));
        if (h->h_ctl->err) return lfail(GG_TIMEOUT, "grid barrier wait exceeded the limit");
        const int lr = std::min(h->h_ctl->levels_run, ml);
        GL_CK(cudaMemcpyAsync(h->h_counts, h->d_counts, (size_t)(lr + 1) * n_cand * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, st));
        GL_CK(cudaMemcpyAsync(h->h_level_ns, h->d_level_ns, (size_t)(lr + 1) * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, st));
        GL_CK(cudaStreamSynchronize(st));
        GL_CK(cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
        const unsigned long long all = (unsigned long long)h->M * (unsigned long long)h->N;
        for (int k = 0; k < n_cand; ++k) {
            unsigned long long tot = 0, reach = (unsigned long long)h->M;
            int lev = 0;
            for (int L = 1; L <= lr; ++L) {
                const unsigned long long c = h->h_counts[(size_t)L * n_cand + k];
                if (!c) continue;
                tot += (unsigned long long)L * c;
                reach += c;
                lev = L;
            }
            const bool capped = lev == ml && reach < all;
            out[k] = gg_cand_result{tot, reach, lev, (!capped && reach == all) ? 1 : 0};
        }
        bool again = false;
        for (int k = 0; k < n_cand && ml < ml_full; ++k)
            again |= out[k].levels == ml && out[k].reached < all;
        if (!again) break;
    }
    return GG_OK;
}

gg_status gg_lift_set_half_ppm(gg_lift *h, int half_ppm) {
    if (!h || half_ppm < 0 || half_ppm > 1000000) return lfail(GG_BAD_ARG, "half_ppm must be in [0, 1e6]");
    h->half_ppm = half_ppm;
    return GG_OK;
}

gg_status gg_lift_last_level_ns(gg_lift *h, uint64_t *ns, int n) {
    if (!h || !ns || n < 0) return lfail(GG_BAD_ARG, "bad arguments");
    const int lr = h->h_ctl ? h->h_ctl->levels_run : 0;
    for (int i = 0; i < n; ++i) ns[i] = (i <= lr && i < h->level_ns_n && h->h_level_ns) ? h->h_level_ns[i] : 0;
    return GG_OK;
}

gg_status gg_lift_last_ms(gg_lift *h, double *ms) {
    if (!h || !ms) return lfail(GG_BAD_ARG, "null argument");
    *ms = h->last_ms;
    return GG_OK;
}

gg_status gg_lift_destroy(gg_lift *h) {
    lift_free(h);
    return GG_OK;
}

}  // extern "C"
