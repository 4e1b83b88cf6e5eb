// gg_kernels.cuh -- device code of the bit-parallel all-pairs BFS (sm_100a).
//
// Data layout in HBM, per source batch of `ns` sources (ns <= 128 * nC):
//   V   [rows][nC] uint4   visited bits: bit i of row v = "source i has reached v"
//   F0/F1 [rows][nC] uint4 frontier bits (pairs first reached at the previous level),
//                          ping-ponged between levels
//   fl0/fl1 [ceil(rows*nC/32)] u32  one bit per uint4 of F: set iff that uint4 holds
//                          new bits; a reader touches F only where the bit is set
//   counts[L]              pairs first reached at level L (u64, atomics)
//   masks[L]               AND of every visited u32 after level L (WVC only)
// Source i lives at bit (i % 32) of u32 component ((i / 32) % 4) of chunk i / 128,
// which is the reference's word/bit mapping (cudaASPLconv.cu:12-13,28-30) seen
// through 128-bit loads, so the lane-aggregated AND masks agree bit for bit.
//
// One BFS level (cudaASPLconv.cu:35-56 fused with :80-99):
//   new[v] = OR_{u in adj[v], flag(u)} F[u]  &  ~V[v];   V[v] |= new;  F'[v] = new
// The whole level loop runs inside one cooperative launch; levels are separated
// by a grid barrier whose waits are bounded (globaltimer) and report GG_TIMEOUT.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gg {

constexpr int kBlock = 256;

// Division by a run-time invariant divisor via multiply-high (Granlund &
// Montgomery, "Division by invariant integers using multiplication", PLDI 1994,
// round-up variant): q = (umulhi(n, m) + n) >> s with s = ceil(log2 d),
// m = floor(2^32 (2^s - d) / d) + 1.  Exact for all 32-bit n when the sum is
// formed in 64 bits.
struct FastDiv {
    uint32_t d, m, s;
    __host__ __device__ FastDiv() : d(1), m(1), s(0) {}
    __host__ explicit FastDiv(uint32_t dv) : d(dv) {
        s = 0;
        while ((1ull << s) < dv) ++s;
        m = (uint32_t)((((1ull << 32) * ((1ull << s) - dv)) / dv) + 1);
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
        uint32_t hi = __umulhi(n, m);
#else
        uint32_t hi = (uint32_t)(((uint64_t)n * m) >> 32);
#endif
        return (uint32_t)(((uint64_t)hi + n) >> s);
    }
};

// Control block of one cooperative launch (zeroed by the host before launch).
// The barrier's arrival counter and the word the blocks wait on sit on
// separate 128-byte lines, so the waiting loads do not contend with arrivals.
struct Ctl {
    unsigned int arrive;      // grid-barrier arrivals, counted over the whole launch
    int err;                  // 0, or 1 = a barrier wait exceeded the limit
    int err_level;            // level at which the first wait gave up
    int levels_run;           // last level executed (single-batch callers)
    int pad0[28];
    unsigned int passed;      // grid barriers completed so far
    unsigned int pad_p;
    // (epoch << 40) | value published by the last arrival of a grid_sync_value
    unsigned long long result;
    int pad1[28];
};
static_assert(offsetof(Ctl, passed) == 128 && offsetof(Ctl, result) == 136 && sizeof(Ctl) == 256,
              "arrivals and the published words on separate 128-byte lines");

struct BfsArgs {
    const int32_t *adj;       // [rows][d] pull adjacency
    // Sources.  The evaluation's sources are entries [src_begin, src_begin +
    // ns_total) of a source list; batch b holds the next 128 * nC of them.
    // inv[v] = index of vertex v in the list (-1: not a source); inv nullptr:
    // entry i of the list is vertex src_first + i.
    const int32_t *inv;
    int src_first, src_begin, ns_total, nb;
    uint4 *V, *F0, *F1;
    uint32_t *fl0, *fl1;
    unsigned long long *counts;   // [nb][stride]: pairs first reached at level L of batch b
    unsigned int *masks;          // [nb][stride] or nullptr (WVC)
    int stride;
    int *levels_run;              // [nb]: last level executed in batch b
    unsigned long long *level_ns; // [max_levels + 1] or nullptr: globaltimer at each level end (batch 0)
    unsigned long long *batch_ns; // [2 * nb] or nullptr: globaltimer at each batch's start and end
    Ctl *ctl;
    const int *bad;           // nonzero: the table failed its range check; do nothing
    unsigned int expected;    // blocks the barrier waits for (the grid size)
    FastDiv div_nc;           // division by nC
    uint32_t items;           // rows * nC
    int rows, d, nC;
    int max_levels;
    int dense_w_ppm;          // write F whole when the feeding frontier >= ppm of the pairs
    int dense_r_ppm;          // read F without flags when it was written whole and >= ppm
    int full_skip_ppm;        // own-first, skip full chunks once reached >= ppm of the pairs
    int split_ppm;            // dense levels gather half the neighbours first, and the rest
                              // only where the chunk is not yet covered, once reached >= ppm
    int adj_smem_rows;        // >0: each block keeps its vertex range's adjacency rows
                              // (at most this many) in dynamic shared memory
    long long wait_ns;        // barrier wait limit
    // Push (top-down) levels.  P0/P1 [rows][nC] uint4 and pf0/pf1 (one bit per
    // uint4) hold the frontier of push levels; both are all zero between
    // launches (every consumer clears what it read).  nullptr or push_ppm 0:
    // every level pulls.
    uint4 *P0, *P1;
    uint32_t *pf0, *pf1;
    int push_ppm;             // push while the feeding frontier < ppm of the pairs
    // A push level equals the reference's pull level only when the adjacency is
    // symmetric (u in adj[w] <=> w in adj[u]); the launch tests that first and
    // stores 1 into *asym (zeroed by the host) on any one-way entry.  nullptr:
    // no push levels.
    int *asym;
    // [ceil(rows * nC / 32)] bit per uint4 of V: set iff that chunk is not yet
    // full.  Written by levels that load every visited chunk; a later level in
    // the skip-full stage passes over tiles whose word is 0.  nullptr: unused.
    uint32_t *nf;
    // The second not-full array of the visited-set pull (levels alternate between
    // nf and nf2, so that a level reads its neighbours' words of the level before).
    uint32_t *nf2;
    // Distance bit-planes (nullptr: not written).  Plane k holds bit k of the
    // distance of every (vertex, source) pair: planes[k * plane_stride + v *
    // plane_cols + s / 128] bit s % 128, for the sources of the whole evaluation
    // (batch b writes columns b * nC ...).  nplanes planes hold distances up to
    // 2^nplanes - 1; pairs never reached keep 0.
    uint4 *planes;
    int nplanes;
    unsigned plane_cols;
    unsigned long long plane_stride;
    // Walk pass (see walk_rows): levels 1..walk_K of every batch computed from the
    // walk index of each row (walk_index_kernel, launched before) instead of phase 0
    // and pull/push levels.  0: off.  Needs the batch's counts zeroed by the host
    // (blocks add into them before any grid barrier) and walk buffers in dynamic
    // shared memory at byte offset walk_smem_off.
    int walk_K;
    int walk_rpg;             // rows per group: lcm(nC, 32) / nC
    unsigned walk_smem_off;
    const uint16_t *walk_ent, *walk_off;
    int walk_cap, walk_off_stride;
    // Nonzero (with a walk pass): the levels after the walk pull visited sets from
    // two alternating copies (V and F0) instead of frontiers (see vpull_level), and
    // the walk writes no frontier rows.
    int walk_vpull;
    // One-way flag of the table from walk_index_kernel (0: every row's entries list
    // it back), or nullptr.  With 0, dense visited-set pull levels skip their own
    // chunks: for L >= 2, V_{L-1}[v] lies within the union of the neighbours'
    // V_{L-1}[u] (the source v through any neighbour, every other source through the
    // neighbour on a shortest path).  Such a level adds its rows' popcounts into
    // vtot[3b + L % 3] (3 slots a batch: zeroed two levels ahead), and its count is
    // that total less the padding bits and the pairs reached before it.
    const int *walk_asym;
    unsigned long long *vtot;   // [nb][3], zeroed by the host
    // walk_all_kernel's output (nullptr: a walk pass per batch): the level-K visited
    // rows of batch b at vall + b * items and the level-K frontier flag words at
    // vall_fl + b * tiles.  Level K+1 reads the slice and writes V; the levels after
    // it alternate between V and `third` (when set), which level K+2 writes whole,
    // so the slice is only read and every batch writes the same two buffers.
    // Without `third`, or when level K+2 is a skip-full level (not written whole),
    // they alternate between the slice and V.
    uint4 *vall;
    const uint32_t *vall_fl;
    uint4 *third;
};

// Where a level's new pairs go in the distance planes.
struct PlaneOut {
    uint4 *planes;
    unsigned long long stride;
    unsigned cols, col0;         // columns of the evaluation, first column of the batch
    int nplanes, L;
};

// The block's current PlaneOut, kept in shared memory (the plane-writing
// kernel's thread 0 sets it between barriers), so that the functions below take
// no extra arguments and the kernel without planes carries none of this.
__device__ __forceinline__ PlaneOut &plane_slot() {
    __shared__ PlaneOut s;
    return s;
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_acquire_i(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned *p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_relaxed(const unsigned *p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier with a bounded wait.  Requires co-resident blocks
// (cooperative launch).  `epoch` counts the barriers this block has passed in
// the launch (the same number in every block).  Each block adds 1 to `arrive`;
// the block whose add makes it (epoch + 1) * expected is the last one and
// publishes `passed` = epoch + 1; every block waits until it reads that value.
// One acquire-release atomic per block (no separate fences), and the waiting
// acquire loads go to a line no arrival touches.
// `expected` above gridDim.x makes the wait run out (fault-injection tests).
// Returns false on every block once any block's wait ran past `wait_ns`; the
// kernel then returns and the host reports GG_TIMEOUT.
__device__ __forceinline__ bool grid_sync(Ctl *ctl, unsigned expected, long long wait_ns, int level,
                                          unsigned &epoch) {
    __shared__ int s_ok;
    __syncthreads();
    const unsigned next = epoch + 1u;
    if (threadIdx.x == 0) {
        int ok = 1;
        // release: the block's writes (ordered before this thread by the block
        // barrier) are published with the arrival; acquire: the last arrival sees
        // every other block's, and publishes them with its release store
        const unsigned old = atom_add_acq_rel(&ctl->arrive, 1u);
        if (old + 1u == next * expected) st_release(&ctl->passed, next);
        const unsigned long long t0 = gtimer();
        for (unsigned it = 1;; ++it) {
            if (ld_acquire(&ctl->passed) == next) break;
            if ((it & 255u) == 0u) {
                if (ld_acquire_i(&ctl->err)) { ok = 0; break; }
                if ((long long)(gtimer() - t0) > wait_ns) {
                    if (atomicCAS(&ctl->err, 0, 1) == 0) ctl->err_level = level;
                    ok = 0;
                    break;
                }
            }
        }
        s_ok = ok;
    }
    epoch = next;
    __syncthreads();
    return s_ok != 0;
}

// grid_sync that also hands every block one 64-bit value (< 2^40) read after all
// arrivals: the last arrival reads *src (every block's additions into it come
// before their arrivals) and publishes (epoch << 40) | value with a release store
// on the line the waiters poll, so the value costs no round trip after the
// barrier.  The value is valid in thread 0 only.  `passed` is kept up to date for
// the plain grid_sync.
__device__ __forceinline__ bool grid_sync_value(Ctl *ctl, unsigned expected, long long wait_ns, int level,
                                                unsigned &epoch, const unsigned long long *src,
                                                unsigned long long &value) {
    __shared__ int s_ok2;
    __syncthreads();
    const unsigned next = epoch + 1u;
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned long long tag = (unsigned long long)(next & 0xffffffu) << 40;
        const unsigned old = atom_add_acq_rel(&ctl->arrive, 1u);
        if (old + 1u == next * expected) {
            const unsigned long long v = ld_relaxed_u64(src) & ((1ull << 40) - 1ull);
            st_release_u64(&ctl->result, tag | v);
            st_release(&ctl->passed, next);
        }
        const unsigned long long t0 = gtimer();
        for (unsigned it = 1;; ++it) {
            const unsigned long long w = ld_acquire_u64(&ctl->result);
            if ((w & ~((1ull << 40) - 1ull)) == tag) {
                value = w & ((1ull << 40) - 1ull);
                break;
            }
            if ((it & 255u) == 0u) {
                if (ld_acquire_i(&ctl->err)) { ok = 0; break; }
                if ((long long)(gtimer() - t0) > wait_ns) {
                    if (atomicCAS(&ctl->err, 0, 1) == 0) ctl->err_level = level;
                    ok = 0;
                    break;
                }
            }
        }
        s_ok2 = ok;
    }
    epoch = next;
    __syncthreads();
    return s_ok2 != 0;
}

__device__ __forceinline__ uint4 u4zero() { return make_uint4(0u, 0u, 0u, 0u); }
__device__ __forceinline__ void or_into(uint4 &a, const uint4 b) {
    a.x |= b.x; a.y |= b.y; a.z |= b.z; a.w |= b.w;
}
__device__ __forceinline__ uint4 andnot(const uint4 a, const uint4 b) {
    return make_uint4(a.x & ~b.x, a.y & ~b.y, a.z & ~b.z, a.w & ~b.w);
}
__device__ __forceinline__ uint4 u4or(const uint4 a, const uint4 b) {
    return make_uint4(a.x | b.x, a.y | b.y, a.z | b.z, a.w | b.w);
}
__device__ __forceinline__ bool u4any(const uint4 a) { return (a.x | a.y | a.z | a.w) != 0u; }
__device__ __forceinline__ bool u4full(const uint4 a) {
    return (a.x & a.y & a.z & a.w) == 0xffffffffu;
}
__device__ __forceinline__ unsigned u4and(const uint4 a) { return a.x & a.y & a.z & a.w; }
__device__ __forceinline__ unsigned u4popc(const uint4 a) {
    return __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w);
}

// Bits of chunk c that belong to no source (index >= ns): preset as visited,
// like the padding sources of cudaASPLconv.cu:15-21.
__device__ __forceinline__ unsigned pad_word(int lo, int ns) {
    if (ns <= lo) return 0xffffffffu;
    if (ns >= lo + 32) return 0u;
    return ~((1u << (ns - lo)) - 1u);
}
__device__ __forceinline__ uint4 pad_mask(int c, int ns) {
    const int b = c * 128;
    return make_uint4(pad_word(b, ns), pad_word(b + 32, ns), pad_word(b + 64, ns),
                      pad_word(b + 96, ns));
}

#ifndef GG_GRAB
#define GG_GRAB 1
#endif
constexpr int kGrab = GG_GRAB;  // tiles a warp takes (and keeps in flight) at once

// One level's work on tiles [tile0, tile0 + U) of the calling warp (a tile is 32
// consecutive uint4 chunks, one per lane).  Every load of the U tiles is issued
// before any result is used, so each warp keeps U*(d+1) 16-byte loads in flight.
template <int D, int U, bool PL>
__device__ __forceinline__ void level_tiles(const BfsArgs &a, const int d, const int32_t *adj,
                                            const unsigned v_base, const unsigned tile0,
                                            const unsigned t_hi, const uint4 *Fc, uint4 *Fn,
                                            const uint32_t *fc, uint32_t *fn, const bool dense,
                                            const bool write_all, const bool skip_full,
                                            const bool split, const unsigned lane, unsigned &cnt, unsigned &and_pre,
                                            unsigned &and_post) {
    unsigned t[U], c[U];
    bool ok[U], have[U];
    uint4 own[U], acc[U], nw[U];
    const int32_t *arow[U];
    const bool own_early = skip_full || dense || a.masks != nullptr;
#pragma unroll
    for (int u = 0; u < U; ++u) {
        t[u] = (tile0 + u) * 32u + lane;
        ok[u] = (tile0 + u) < t_hi && t[u] < a.items;
        const unsigned v = ok[u] ? a.div_nc.div(t[u]) : v_base;
        c[u] = t[u] - v * (unsigned)a.nC;
        arow[u] = adj + (size_t)(v - v_base) * (size_t)d;
        own[u] = acc[u] = nw[u] = u4zero();
        have[u] = false;
        if (ok[u] && own_early) { own[u] = __ldcg(a.V + t[u]); have[u] = true; }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        if (!ok[u] || (skip_full && u4full(own[u]))) continue;
        if constexpr (D > 0) {
            // Staged so that each step's loads are all in flight together:
            // neighbour ids, then (sparse) their flag words, then the gathers.
            unsigned tu[D];
#pragma unroll
            for (int i = 0; i < D; ++i) tu[i] = (unsigned)arow[u][i] * (unsigned)a.nC + c[u];
            if (dense && split && D >= 8) {
                // Late dense level: few sources still miss this chunk, and half
                // the neighbours usually bring all of them.
                constexpr int H = D / 2;
                uint4 x[H];
#pragma unroll
                for (int i = 0; i < H; ++i) x[i] = __ldcg(Fc + tu[i]);
#pragma unroll
                for (int i = 0; i < H; ++i) or_into(acc[u], x[i]);
                if (!u4full(u4or(own[u], acc[u]))) {
#pragma unroll
                    for (int i = 0; i < D - H; ++i) x[i] = __ldcg(Fc + tu[H + i]);
#pragma unroll
                    for (int i = 0; i < D - H; ++i) or_into(acc[u], x[i]);
                }
            } else if (dense) {
                uint4 x[D];
#pragma unroll
                for (int i = 0; i < D; ++i) x[i] = __ldcg(Fc + tu[i]);
#pragma unroll
                for (int i = 0; i < D; ++i) or_into(acc[u], x[i]);
            } else {
                unsigned fw[D];
#pragma unroll
                for (int i = 0; i < D; ++i) fw[i] = __ldcg(fc + (tu[i] >> 5));
#pragma unroll
                for (int i = 0; i < D; ++i)
                    if ((fw[i] >> (tu[i] & 31u)) & 1u) or_into(acc[u], __ldcg(Fc + tu[i]));
            }
        } else if (dense) {
            for (int i = 0; i < d; ++i)
                or_into(acc[u], __ldcg(Fc + (unsigned)arow[u][i] * (unsigned)a.nC + c[u]));
        } else {
            for (int i = 0; i < d; ++i) {
                const unsigned tu = (unsigned)arow[u][i] * (unsigned)a.nC + c[u];
                if ((__ldcg(fc + (tu >> 5)) >> (tu & 31u)) & 1u) or_into(acc[u], __ldcg(Fc + tu));
            }
        }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        if (ok[u]) {
            if (u4any(acc[u])) {
                if (!have[u]) { own[u] = __ldcg(a.V + t[u]); have[u] = true; }
                nw[u] = andnot(acc[u], own[u]);
                if (u4any(nw[u])) a.V[t[u]] = u4or(own[u], nw[u]);
            }
            if (write_all || u4any(nw[u])) Fn[t[u]] = nw[u];
            if constexpr (PL) {
                // distance L of the new pairs into the planes (one writer per chunk)
                if (u4any(nw[u])) {
                    const PlaneOut &po = plane_slot();
                    const size_t pi = (size_t)a.div_nc.div(t[u]) * po.cols + po.col0 + c[u];
                    for (int p = 0; p < po.nplanes; ++p)
                        if ((po.L >> p) & 1) {
                            uint4 *q = po.planes + (size_t)p * po.stride + pi;
                            *q = u4or(*q, nw[u]);
                        }
                }
            }
            if (a.masks) {
                and_pre &= u4and(own[u]);
                and_post &= u4and(u4or(own[u], nw[u]));
            }
            cnt += u4popc(nw[u]);
        }
        const unsigned b = __ballot_sync(0xffffffffu, u4any(nw[u]));
        if (lane == 0 && (tile0 + u) < t_hi) fn[tile0 + u] = b;
        if (a.nf && own_early) {
            // not-full bits of the tile after this level (own is loaded for every chunk)
            const unsigned nfb = __ballot_sync(0xffffffffu, ok[u] && !u4full(u4or(own[u], nw[u])));
            if (lane == 0 && (tile0 + u) < t_hi) a.nf[tile0 + u] = nfb;
        }
    }
}

// Whether the levels after a walk pass pull visited sets (both not-full arrays given).
__device__ __forceinline__ bool vpull_on(const BfsArgs &a) {
    return a.walk_K > 0 && a.walk_vpull != 0 && a.nf != nullptr && a.nf2 != nullptr;
}

// Visited-set pull (levels after a walk pass).  With V_L[v] the sources within
// distance L of v (chunk by chunk),
//     V_L[v] = V_{L-1}[v] | OR of V_{L-1}[u] over the neighbours u of v
// whose chunk changed at level L-1 (every neighbour, when dense): each V_{L-1}[u]
// lies within V_L[v], and a source first reached at level L reaches v through a
// neighbour that holds it at exactly L - 1, whose chunk therefore changed.  So a
// level needs no frontier rows, only their flag words: X holds V_{L-1}, Y holds
// V_{L-2} and is brought to V_L by writing the chunks that changed at level L-1 or
// L (all chunks while Y holds no level yet: `wr_all`).  A dense level moves 10 row
// transfers per chunk (own, d = 8 gathers, one write) against 11 with frontiers
// (own, gathers, the visited and the frontier writes).  The new pairs are
// V_L & ~V_{L-1}, as in level_tiles; fn gets their flag words, nfn the not-full
// words of V_L.
//
// LAZY (the skip-full stage, nfc = the not-full words of V_{L-1}): a chunk whose
// not-full bit is clear is full whatever X holds there, so full chunks are never
// read or written again -- its own chunk is passed over, and a neighbour chunk that
// is full makes the sum full without a load.  The buffers then hold V_L exactly on
// the chunks that are not full, which is all that later levels read.
template <int D, int U, bool LAZY>
__device__ __forceinline__ void vpull_tiles(const BfsArgs &a, const int d, const int32_t *adj,
                                            const unsigned v_base, const unsigned tile0, const unsigned t_hi,
                                            const uint4 *X, uint4 *Y, const uint32_t *fc, uint32_t *fn,
                                            const uint32_t *nfc, uint32_t *nfn, const unsigned nfo,
                                            const bool dense, const bool wr_all, const bool skip_full,
                                            const bool split, const bool no_own, const unsigned lane,
                                            unsigned &cnt) {
    unsigned t[U], c[U], chg[U];
    bool ok[U];
    uint4 own[U], acc[U];
    const int32_t *arow[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        t[u] = (tile0 + u) * 32u + lane;
        ok[u] = (tile0 + u) < t_hi && t[u] < a.items;
        if (LAZY) ok[u] = ok[u] && ((nfo >> lane) & 1u);   // not full at L-1
        const unsigned v = ok[u] ? a.div_nc.div(t[u]) : v_base;
        c[u] = t[u] - v * (unsigned)a.nC;
        arow[u] = adj + (size_t)(v - v_base) * (size_t)d;
        own[u] = ok[u] && !(!LAZY && no_own) ? __ldcg(X + t[u]) : u4zero();
        acc[u] = u4zero();
        chg[u] = (!wr_all && (tile0 + u) < t_hi) ? __ldcg(fc + tile0 + u) : 0u;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        if (!ok[u] || (skip_full && u4full(own[u]))) continue;
        if constexpr (D > 0) {
            unsigned tu[D];
#pragma unroll
            for (int i = 0; i < D; ++i) tu[i] = (unsigned)arow[u][i] * (unsigned)a.nC + c[u];
            if constexpr (LAZY) {
                // neighbours' not-full words first: a full neighbour fills the sum
                unsigned nw[D], fw[D];
                bool nb_full = false;
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    nw[i] = __ldcg(nfc + (tu[i] >> 5));
                    fw[i] = dense ? ~0u : __ldcg(fc + (tu[i] >> 5));
                }
#pragma unroll
                for (int i = 0; i < D; ++i) nb_full |= !((nw[i] >> (tu[i] & 31u)) & 1u);
                if (nb_full) {
                    acc[u] = make_uint4(~0u, ~0u, ~0u, ~0u);
                } else {
#pragma unroll
                    for (int i = 0; i < D; ++i)
                        if ((fw[i] >> (tu[i] & 31u)) & 1u) or_into(acc[u], __ldcg(X + tu[i]));
                }
            } else if (dense && split && D >= 8) {
                constexpr int H = D / 2;
                uint4 x[H];
#pragma unroll
                for (int i = 0; i < H; ++i) x[i] = __ldcg(X + tu[i]);
#pragma unroll
                for (int i = 0; i < H; ++i) or_into(acc[u], x[i]);
                if (!u4full(u4or(own[u], acc[u]))) {
#pragma unroll
                    for (int i = 0; i < D - H; ++i) x[i] = __ldcg(X + tu[H + i]);
#pragma unroll
                    for (int i = 0; i < D - H; ++i) or_into(acc[u], x[i]);
                }
            } else if (dense) {
                uint4 x[D];
#pragma unroll
                for (int i = 0; i < D; ++i) x[i] = __ldcg(X + tu[i]);
#pragma unroll
                for (int i = 0; i < D; ++i) or_into(acc[u], x[i]);
            } else {
                unsigned fw[D];
#pragma unroll
                for (int i = 0; i < D; ++i) fw[i] = __ldcg(fc + (tu[i] >> 5));
#pragma unroll
                for (int i = 0; i < D; ++i)
                    if ((fw[i] >> (tu[i] & 31u)) & 1u) or_into(acc[u], __ldcg(X + tu[i]));
            }
        } else {
            for (int i = 0; i < d; ++i) {
                const unsigned tu = (unsigned)arow[u][i] * (unsigned)a.nC + c[u];
                if (LAZY && !((__ldcg(nfc + (tu >> 5)) >> (tu & 31u)) & 1u)) {
                    acc[u] = make_uint4(~0u, ~0u, ~0u, ~0u);
                    break;
                }
                if (dense || ((__ldcg(fc + (tu >> 5)) >> (tu & 31u)) & 1u)) or_into(acc[u], __ldcg(X + tu));
            }
        }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        uint4 nw = u4zero();
        bool not_full = false;
        if (ok[u]) {
            nw = andnot(acc[u], own[u]);
            const uint4 vn = u4or(own[u], nw);
            not_full = !u4full(vn);
            const bool need = wr_all || u4any(nw) || ((chg[u] >> lane) & 1u);
            if (need && (!LAZY || not_full)) Y[t[u]] = vn;
            cnt += u4popc(nw);
        }
        const unsigned b = __ballot_sync(0xffffffffu, u4any(nw));
        const unsigned nfb = __ballot_sync(0xffffffffu, not_full);
        if (lane == 0 && (tile0 + u) < t_hi) {
            fn[tile0 + u] = b;
            nfn[tile0 + u] = nfb;
        }
    }
}

// One visited-set pull level over the block's tiles [s_next, t_hi) (s_next set by the
// caller); returns this thread's count of new pairs (no_own: of the pairs in the
// rows it wrote, padding included; every chunk is then written).  nf_use (the skip-full stage,
// with nfc written whole by the level before): a warp takes 32 tiles, passes over
// those whose chunks are all full, and runs the others LAZY.
template <int D>
static __device__ __noinline__ unsigned vpull_level(const BfsArgs &a, const int d, const int32_t *adj,
                                                    const unsigned v_base, const unsigned t_hi, const uint4 *X,
                                                    uint4 *Y, const uint32_t *fc, uint32_t *fn, const uint32_t *nfc,
                                                    uint32_t *nfn, const bool dense, const bool wr_all,
                                                    const bool skip_full, const bool split, const bool nf_use,
                                                    const bool no_own, unsigned *s_next) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned cnt = 0u;
    if (nf_use) {
        for (;;) {
            unsigned tile0 = 0;
            if (lane == 0) tile0 = atomicAdd(s_next, 32u);
            tile0 = __shfl_sync(0xffffffffu, tile0, 0);
            if (tile0 >= t_hi) break;
            const unsigned my = tile0 + lane;
            const unsigned w = my < t_hi ? __ldcg(nfc + my) : 0u;
            if (my < t_hi && w == 0u) {
                fn[my] = 0u;
                nfn[my] = 0u;
            }
            for (unsigned todo = __ballot_sync(0xffffffffu, w != 0u); todo; todo &= todo - 1u) {
                const int k = __ffs((int)todo) - 1;
                const unsigned wk = __shfl_sync(0xffffffffu, w, k);
                vpull_tiles<D, 1, true>(a, d, adj, v_base, tile0 + (unsigned)k, t_hi, X, Y, fc, fn, nfc, nfn, wk,
                                        dense, false, skip_full, split, false, lane, cnt);
            }
        }
    } else {
        for (;;) {
            unsigned tile0 = 0;
            if (lane == 0) tile0 = atomicAdd(s_next, (unsigned)kGrab);
            tile0 = __shfl_sync(0xffffffffu, tile0, 0);
            if (tile0 >= t_hi) break;
            vpull_tiles<D, kGrab, false>(a, d, adj, v_base, tile0, t_hi, X, Y, fc, fn, nfc, nfn, 0u, dense,
                                         wr_all || no_own, skip_full, split, no_own, lane, cnt);
        }
    }
    return cnt;
}

// Dense visited-set pull level without own chunks on 32-chunk rows (a tile is one
// row; tables without one-way entries): Y[v] = OR of the D neighbours' X rows, every
// chunk written, the row's flag and not-full words, and this thread's popcount of what
// it wrote (the level's total, see BfsArgs::walk_asym).  The same result as
// vpull_level with no_own, in a loop with nothing else in it: the generic tile function
// measured 3-4 us slower a level on the 65536-row, 8-regular graph.  With `half`, the
// first D/2 neighbours alone where they already fill the chunk.  Out of line: inlined,
// it raised the level loop's spills.
template <int D>
static __device__ __noinline__ unsigned dense_rows32(const uint4 *X, uint4 *Y, const int32_t *adj,
                                                     const unsigned v_base, const unsigned t_hi, uint32_t *fn,
                                                     uint32_t *nfn, const bool half, unsigned *s_next) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned cnt = 0u;
    for (;;) {
        unsigned v = 0u;
        if (lane == 0) v = atomicAdd(s_next, 1u);
        v = __shfl_sync(0xffffffffu, v, 0);
        if (v >= t_hi) break;
        const int32_t *row = adj + (size_t)(v - v_base) * D;
        unsigned tu[D];
#pragma unroll
        for (int i = 0; i < D; ++i) tu[i] = (unsigned)row[i] * 32u + lane;
        uint4 x[D];
        uint4 q;
        if (D >= 8 && half) {
            // the first half alone where it already fills the chunk
            constexpr int H = D / 2;
#pragma unroll
            for (int i = 0; i < H; ++i) x[i] = __ldcg(X + tu[i]);
            q = x[0];
#pragma unroll
            for (int i = 1; i < H; ++i) or_into(q, x[i]);
            if (!u4full(q)) {
#pragma unroll
                for (int i = H; i < D; ++i) x[i] = __ldcg(X + tu[i]);
#pragma unroll
                for (int i = H; i < D; ++i) or_into(q, x[i]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < D; ++i) x[i] = __ldcg(X + tu[i]);
            q = x[0];
#pragma unroll
            for (int i = 1; i < D; ++i) or_into(q, x[i]);
        }
        Y[(size_t)v * 32 + lane] = q;
        cnt += u4popc(q);
        const unsigned fb = __ballot_sync(0xffffffffu, u4any(q));
        const unsigned nb = __ballot_sync(0xffffffffu, !u4full(q));
        if (lane == 0) {
            fn[v] = fb;
            nfn[v] = nb;
        }
    }
    return cnt;
}

// Component k of a uint4 (k is a compile-time constant after unrolling).
__device__ __forceinline__ unsigned comp_of(const uint4 &f, const int k) {
    return k == 0 ? f.x : (k == 1 ? f.y : (k == 2 ? f.z : f.w));
}

// Push item (u, c) with frontier chunk f to the neighbour chunk tw = (w, c).
// The visited words are ORed first (all four in flight before any returned value
// is used); the bits that were not visited yet -- exact under concurrency,
// atomicOr returns the old word -- are this level's new pairs and go into Pn and
// the flag words with fire-and-forget reductions.
template <bool PL>
__device__ __forceinline__ void push_item(uint4 *V, const uint4 f, const unsigned tw, uint4 *Pn,
                                          uint32_t *pfn, const unsigned w, const unsigned c,
                                          unsigned &cnt) {
    unsigned any = 0u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const unsigned fk = comp_of(f, k);
        if (!fk) continue;
        const unsigned nb = fk & ~atomicOr(reinterpret_cast<unsigned *>(V + tw) + k, fk);
        if (nb) {
            atomicOr(reinterpret_cast<unsigned *>(Pn + tw) + k, nb);
            cnt += __popc(nb);
            any = 1u;
            if constexpr (PL) {
                const PlaneOut &po = plane_slot();
                const size_t pi = (size_t)w * po.cols + po.col0 + c;
                for (int p = 0; p < po.nplanes; ++p)
                    if ((po.L >> p) & 1)
                        atomicOr(reinterpret_cast<unsigned *>(po.planes + (size_t)p * po.stride + pi) + k, nb);
            }
        }
    }
    if (any) atomicOr(pfn + (tw >> 5), 1u << (tw & 31u));
}

// One push level.  The frontier of level L-1 is the set bits of the flag words
// `pfc` (item t = (u, c) of `Pc`).  Thread (k, i) of a group of D lanes takes
// flag word k and neighbour slot i: for each item (u, c) of the word it pushes
// F[u][c] to w = adj[u][i] (the adjacency is symmetric, so the pull rows are also
// the push rows): new = F[u][c] & ~V[w][c] goes into V, into Pn[w][c], and sets
// the flag bit of (w, c) in `pfn`.  Each thread thus waits on one atomic per
// item, and the D pushes of an item run in parallel.  After the group's lanes
// have read them, lane 0 zeroes the items and the flag word, so Pc is all zero
// again when the level ends.  Work is proportional to the frontier, not to
// rows * nC.  Needs D to divide 32 (a group never straddles two warps).  Kept
// out of line: it runs a few times per batch, and inlined it would take
// registers from the pull levels.
template <int D, bool PL>
static __device__ __noinline__ unsigned push_level(const int32_t *adj, uint4 *V, const FastDiv div_nc,
                                            const unsigned nC, uint4 *Pc, uint4 *Pn, uint32_t *pfc,
                                            uint32_t *pfn, const unsigned fwords, const unsigned gtid,
                                            const unsigned nthr) {
    static_assert(D > 0 && 32 % D == 0, "push levels need D | 32");
    unsigned cnt = 0u;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned i = lane % (unsigned)D;
    const unsigned long long total = (unsigned long long)fwords * D;
    // warp-uniform trip count: every lane reaches the __syncwarp below
    for (unsigned long long base = gtid - lane; base < total; base += nthr) {
        const unsigned long long g = base + lane;
        const unsigned k = (unsigned)(g / D);
        const unsigned m0 = g < total ? __ldcg(pfc + k) : 0u;
        for (unsigned m = m0; m;) {
            const unsigned b = (unsigned)(__ffs((int)m) - 1);
            m &= m - 1u;
            const unsigned t = k * 32u + b;
            const unsigned u = div_nc.div(t);
            const unsigned c = t - u * nC;
            const uint4 f = __ldcg(Pc + t);
            const unsigned w = (unsigned)__ldg(adj + (size_t)u * D + i);
            push_item<PL>(V, f, w * nC + c, Pn, pfn, w, c, cnt);
        }
        __syncwarp();
        if (i == 0u && m0) {
            for (unsigned m = m0; m; m &= m - 1u) Pc[k * 32u + (unsigned)(__ffs((int)m) - 1)] = u4zero();
            pfc[k] = 0u;
        }
    }
    return cnt;
}

// Zero the items flagged in `pf` and the flag words themselves (the push buffer
// a pull level read last), restoring the all-zero state the next batch expects.
static __device__ __noinline__ void clear_push_buffer(uint4 *P, uint32_t *pf, const unsigned fwords,
                                               const unsigned gtid, const unsigned nthr) {
    for (unsigned k = gtid; k < fwords; k += nthr) {
        unsigned m = __ldcg(pf + k);
        if (!m) continue;
        do {
            const unsigned b = (unsigned)(__ffs((int)m) - 1);
            m &= m - 1u;
            P[k * 32u + b] = u4zero();
        } while (m);
        pf[k] = 0u;
    }
}

// Phase 0 of batch b: every visited chunk rewritten with its padding bits and
// the diagonal, the diagonal stored as the level-1 frontier (push buffer P_diag
// or F0) with its flag words.  The sources of a batch are distinct vertices, so a
// chunk holds at most one of them.  One warp per tile of 32 chunks.  Out of line
// for the same reason as push_level.
template <bool PL>
static __device__ __noinline__ void phase0_tiles(const int32_t *inv, const int src_first, const int first,
                                          const int ns, uint4 *V, uint4 *F0, uint32_t *fl0,
                                          uint4 *P_diag, uint32_t *pf_diag, const FastDiv div_nc,
                                          const unsigned nC, const unsigned items, const bool push_on,
                                          const unsigned gtid, const unsigned nthr) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned ntiles = (items + 31u) >> 5;
    for (unsigned tile = gtid >> 5; tile < ntiles; tile += nthr >> 5) {
        const unsigned t = tile * 32u + lane;
        const bool ok = t < items;
        const unsigned v = ok ? div_nc.div(t) : 0u;
        const unsigned c = t - v * nC;
        const int g = ok ? (inv ? __ldg(inv + v) : (int)v - src_first) : -1;
        const int j = g - first;
        const bool has = ok && g >= 0 && j >= 0 && j < ns && (unsigned)(j >> 7) == c;
        uint4 one = u4zero();
        if (has) {
            const unsigned bit = 1u << (j & 31), comp = ((unsigned)j >> 5) & 3u;
            if (comp == 0u) one.x = bit; else if (comp == 1u) one.y = bit; else if (comp == 2u) one.z = bit; else one.w = bit;
        }
        if (ok) V[t] = u4or(pad_mask((int)c, ns), one);
        if constexpr (PL) {
            const PlaneOut &po = plane_slot();
            if (ok)
                for (int p = 0; p < po.nplanes; ++p)
                    po.planes[(size_t)p * po.stride + (size_t)v * po.cols + po.col0 + c] = u4zero();
        }
        const unsigned fb = __ballot_sync(0xffffffffu, has);
        if (push_on) {
            if (has) P_diag[t] = one;
            if (lane == 0 && fb) pf_diag[tile] = fb;
        } else {
            if (has) F0[t] = one;
            if (lane == 0) fl0[tile] = fb;
        }
    }
}

// ---------------------------------------------------------------------------
// Walk pass: phase 0 and levels 1..K of a batch in one pass over the rows.
//
// Pull BFS gives V_L[v] = V_{L-1}[v] | OR_{u in adj[v]} V_{L-1}[u], so by
// induction V_L[v] holds exactly the sources whose vertex is the end of some
// walk of length <= L from v along the pull table (adj[v], adj[adj[v]], ...),
// for any table, symmetric or not.  The first levels of a batch touch few pairs
// (about d^L per source), but a pull level still visits every chunk.  Instead:
//
//  * once per evaluation, walk_index_kernel enumerates the walk ends of every row
//    -- level 1 = adj[v] (d), level 2 = H2[v] (d^2; H2 = adj of adj, built by
//    h2_kernel when K >= 3, else read row by row), level 3 = H2 of adj[v] (d^3),
//    level 4 = H2 of H2[v] (d^4) -- keeps those that are sources (consecutive ids,
//    or the inverse list of the lifted forms' representatives) and counting-sorts
//    them per row by (batch, level): ent[v][...] holds each kept end's source index
//    within its batch (16 bits), off[v][b * K + L - 1] where bucket (b, L) starts;
//  * per batch, walk_rows gives each row to one warp, which reads the row's
//    entries of this batch (a few dozen: the ends of the other batches never come
//    back), sets their bits level by level in a shared-memory copy of the row with
//    atomicOr -- its returned old word says whether the pair is new at that level,
//    so the counts are exact, repeated ends included -- and writes the row once:
//    V = V_K with the padding bits, the level-(K+1) frontier F = V_K & ~V_{K-1}
//    (every chunk, zeros included) and its flag words.
//
// K is chosen on the host so that d + ... + d^K stays a few hundred.  Rows go to
// warps in groups of whole rows that also cover whole 32-chunk tiles (lcm(nC, 32)
// chunks), so that each flag word has one writer.
// ---------------------------------------------------------------------------
struct WalkIndexArgs {
    const int32_t *adj;       // [rows][d]
    const int32_t *h2;        // [rows][d*d] or nullptr (K <= 2)
    const int32_t *inv;       // source index of each vertex (-1: none), or nullptr
    int src_first, src_begin, ns_total;   // the evaluation's sources (see BfsArgs)
    FastDiv div_S;            // division by the batch width S = 128 * nC
    int S, nb, K;
    int rows, d;
    int cap;                  // entries per row: d + ... + d^K
    uint16_t *ent;            // [rows][cap]
    uint16_t *off;            // [rows][off_stride]: bucket starts, nb * K + 1 used
    int off_stride;
    const int *bad;           // nonzero: the table failed its range check
    int *asym;                // set to 1 when some row u lacks v for an entry u of row v (nullptr: not checked)
    // walk_all_kernel only: the level-K visited rows of every batch and their flag words
    uint4 *vall;              // [nb][rows * 32]
    uint32_t *vall_fl;        // [nb][rows]
    unsigned long long *counts;   // [nb][counts_stride]: levels 1..K added
    int counts_stride;
    const int *oneway;        // walk_check_kernel's flag (0: counts from the sources' side), or nullptr
};

constexpr int kIndexBlock = 256;

// The row's entries from shared memory to the index, 16 bytes a lane (cap is a
// multiple of 8, so rows start 16-byte aligned; the last word may carry stale
// entries past `total`, which no reader looks at).
__device__ __forceinline__ void copy_row_out(const WalkIndexArgs &a, const int v, const unsigned lane,
                                             const uint16_t *row, const unsigned total) {
    uint4 *dst = reinterpret_cast<uint4 *>(a.ent + (size_t)v * a.cap);
    const uint4 *src = reinterpret_cast<const uint4 *>(row);
    for (unsigned k = lane; k < (total + 7u) / 8u; k += 32) dst[k] = src[k];
    __syncwarp();
}

// One-way check of row v: every entry u of the row must list v in its own row,
// else *a.asym = 1 (the visited-set pull levels then read their own chunks).
__device__ __forceinline__ void row_oneway_check(const WalkIndexArgs &a, const int v, const unsigned lane, const int d) {
    for (int i = (int)lane; i < d; i += 32) {
        const int32_t *ur = a.adj + (size_t)__ldg(a.adj + (size_t)v * d + i) * d;
        bool f = false;
        for (int j = 0; j < d; ++j) f |= __ldg(ur + j) == v;
        if (!f) *a.asym = 1;
    }
}
constexpr int kIndexMaxKeys = 256;   // nb * K buckets per row
constexpr int kIndexMaxCap = 1024;   // entries per row

// Every walk end of row v with its level, in level order within each lane.
template <int D, typename Fn>
__device__ __forceinline__ void for_walk_ends(const WalkIndexArgs &a, const int v, const unsigned lane, Fn &&fn) {
    const int d = D > 0 ? D : a.d;
    const int dd = d * d;
    const int32_t *arow = a.adj + (size_t)v * d;
    for (int i = (int)lane; i < d; i += 32) fn(__ldg(arow + i), 1);
    if (a.K >= 2) {
        if (a.h2) {
            for (int i = (int)lane; i < dd; i += 32) fn(__ldg(a.h2 + (size_t)v * dd + i), 2);
        } else {
            for (int i = (int)lane; i < dd; i += 32) fn(__ldg(a.adj + (size_t)__ldg(arow + i / d) * d + i % d), 2);
        }
    }
    if (a.K >= 3) {
        if constexpr (D > 0 && D <= 8 && (D * D) % 4 == 0) {
            // d H2 rows, 16 bytes at a time, every load in flight before any use
            constexpr int Q = D * D / 4, U = D * Q, SL = (U + 31) / 32;
            uint4 q[SL];
#pragma unroll
            for (int s = 0; s < SL; ++s) {
                const int i = s * 32 + (int)lane;
                q[s] = make_uint4(0u, 0u, 0u, 0u);
                if (i < U)
                    q[s] = __ldg(reinterpret_cast<const uint4 *>(a.h2 + (size_t)__ldg(arow + i / Q) * dd) + i % Q);
            }
#pragma unroll
            for (int s = 0; s < SL; ++s)
                if (s * 32 + (int)lane < U) {
                    fn((int32_t)q[s].x, 3); fn((int32_t)q[s].y, 3); fn((int32_t)q[s].z, 3); fn((int32_t)q[s].w, 3);
                }
        } else {
            for (int i = (int)lane; i < d * dd; i += 32)
                fn(__ldg(a.h2 + (size_t)__ldg(arow + i / dd) * dd + i % dd), 3);
        }
    }
    if (a.K >= 4)
        for (int i = (int)lane; i < dd * dd; i += 32)
            fn(__ldg(a.h2 + (size_t)__ldg(a.h2 + (size_t)v * dd + i / dd) * dd + i % dd), 4);
}

// The walk ends of row v in registers (D <= 8 with D*D % 4 == 0, K <= 3, level-2
// ends from H2 or the adjacency rows), each classified as (key << 16) | payload with
// key = batch * K + level - 1 and payload the source's place in its batch, or -1;
// also the row's one-way check.  NV slots a lane.
template <int D>
struct RowEnds {
    static constexpr int DD = D * D, Q = DD / 4;           // uint4 per level-2 list
    static constexpr int U3 = D * Q, S3 = (U3 + 31) / 32;  // uint4 of the level-3 ends, per lane
    static constexpr int NV = 1 + 4 * ((Q + 31) / 32) + 4 * S3;
};

// The raw walk ends of a row in registers: level 1 (lanes < D), level 2 (lanes < Q,
// 4 a lane), level 3 (S3 uint4 a lane, lanes' slot s3 * 32 + lane < U3).
template <int D>
struct RowEndsRaw {
    int32_t x1;
    uint4 q2[(RowEnds<D>::Q + 31) / 32];
    uint4 q3[RowEnds<D>::S3];
};

// Loads of row v's walk ends (all in flight together), and the row's one-way check.
template <int D>
__device__ __forceinline__ void row_ends_load(const WalkIndexArgs &a, const int v, const unsigned lane,
                                              RowEndsRaw<D> &r) {
    constexpr int DD = RowEnds<D>::DD, Q = RowEnds<D>::Q, U3 = RowEnds<D>::U3, S3 = RowEnds<D>::S3;
    const int32_t *arow = a.adj + (size_t)v * D;
    r.x1 = lane < (unsigned)D ? __ldg(arow + lane) : 0;
#pragma unroll
    for (int s2 = 0; s2 < (Q + 31) / 32; ++s2) {
        const int i = s2 * 32 + (int)lane;
        r.q2[s2] = make_uint4(0u, 0u, 0u, 0u);
        if (a.K >= 2 && i < Q)
            r.q2[s2] = a.h2 ? __ldg(reinterpret_cast<const uint4 *>(a.h2 + (size_t)v * DD) + i)
                            : __ldg(reinterpret_cast<const uint4 *>(a.adj + (size_t)__ldg(arow + i / (D / 4)) * D) +
                                    i % (D / 4));
    }
#pragma unroll
    for (int s3 = 0; s3 < S3; ++s3) {
        const int i = s3 * 32 + (int)lane;
        r.q3[s3] = make_uint4(0u, 0u, 0u, 0u);
        if (a.K >= 3 && i < U3)
            r.q3[s3] = __ldg(reinterpret_cast<const uint4 *>(a.h2 + (size_t)__ldg(arow + i / Q) * DD) + i % Q);
    }
    if (a.asym) {
        if (a.K >= 2) {
            // the level-2 lists are the neighbours' rows, D / 4 lanes per row
            bool f = (int)lane < Q && ((int)r.q2[0].x == v || (int)r.q2[0].y == v || (int)r.q2[0].z == v ||
                                       (int)r.q2[0].w == v);
            if constexpr (D / 4 == 2) f |= __shfl_xor_sync(0xffffffffu, f, 1) != 0;
            if ((int)lane < Q && (int)lane % (D / 4) == 0 && !f) *a.asym = 1;
        } else {
            row_oneway_check(a, v, lane, D);
        }
    }
}

// Each raw end classified: (key << 16) | payload, key = batch * K + level - 1, payload
// the source's place in its batch; -1 for ends that are no source of the evaluation.
template <int D>
__device__ __forceinline__ void row_ends_classify(const WalkIndexArgs &a, const unsigned lane, const RowEndsRaw<D> &r,
                                                  int (&pk)[RowEnds<D>::NV]) {
    constexpr int Q = RowEnds<D>::Q, U3 = RowEnds<D>::U3, S3 = RowEnds<D>::S3;
    auto classify = [&](const int32_t w, const int L) -> int {
        const int g = a.inv ? __ldg(a.inv + w) : w - a.src_first;
        const int j = g - a.src_begin;
        if (!(g >= 0 && (unsigned)j < (unsigned)a.ns_total)) return -1;
        const unsigned b = a.div_S.div((unsigned)j);
        return (int)(((b * (unsigned)a.K + (unsigned)(L - 1)) << 16) | ((unsigned)j - b * (unsigned)a.S));
    };
    int n = 0;
    pk[n++] = lane < (unsigned)D ? classify(r.x1, 1) : -1;
#pragma unroll
    for (int s2 = 0; s2 < (Q + 31) / 32; ++s2) {
        const bool ok = a.K >= 2 && s2 * 32 + (int)lane < Q;
        pk[n++] = ok ? classify((int32_t)r.q2[s2].x, 2) : -1;
        pk[n++] = ok ? classify((int32_t)r.q2[s2].y, 2) : -1;
        pk[n++] = ok ? classify((int32_t)r.q2[s2].z, 2) : -1;
        pk[n++] = ok ? classify((int32_t)r.q2[s2].w, 2) : -1;
    }
#pragma unroll
    for (int s3 = 0; s3 < S3; ++s3) {
        const bool ok = a.K >= 3 && s3 * 32 + (int)lane < U3;
        pk[n++] = ok ? classify((int32_t)r.q3[s3].x, 3) : -1;
        pk[n++] = ok ? classify((int32_t)r.q3[s3].y, 3) : -1;
        pk[n++] = ok ? classify((int32_t)r.q3[s3].z, 3) : -1;
        pk[n++] = ok ? classify((int32_t)r.q3[s3].w, 3) : -1;
    }
}

template <int D>
__device__ __forceinline__ void row_ends_regs(const WalkIndexArgs &a, const int v, const unsigned lane,
                                              int (&pk)[RowEnds<D>::NV]) {
    RowEndsRaw<D> r;
    row_ends_load<D>(a, v, lane, r);
    row_ends_classify<D>(a, lane, r, pk);
}

// One row of the walk index from its ends in registers: counted and placed.
template <int D>
__device__ __forceinline__ void index_row_regs(const WalkIndexArgs &a, const int v, const unsigned lane,
                                               unsigned *cur, uint16_t *row, const int nkeys) {
    constexpr int NV = RowEnds<D>::NV;
    int pk[NV];
    row_ends_regs<D>(a, v, lane, pk);
#pragma unroll
    for (int k = 0; k < NV; ++k)
        if (pk[k] >= 0) atomicAdd(cur + (pk[k] >> 16), 1u);
    __syncwarp();
    // exclusive prefix over the buckets: lane l owns keys [l * per, (l + 1) * per)
    const int per = (nkeys + 31) / 32;
    unsigned mine = 0u;
    for (int k = (int)lane * per; k < min(nkeys, ((int)lane + 1) * per); ++k) mine += cur[k];
    unsigned incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)lane >= o) incl += t;
    }
    unsigned run = incl - mine;
    uint16_t *offrow = a.off + (size_t)v * a.off_stride;
    for (int k = (int)lane * per; k < min(nkeys, ((int)lane + 1) * per); ++k) {
        const unsigned c = cur[k];
        offrow[k] = (uint16_t)run;
        cur[k] = run;
        run += c;
    }
    const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
    if (lane == 0) offrow[nkeys] = (uint16_t)total;
    __syncwarp();
#pragma unroll
    for (int k = 0; k < NV; ++k)
        if (pk[k] >= 0) row[atomicAdd(cur + (pk[k] >> 16), 1u)] = (uint16_t)(pk[k] & 0xffff);
    __syncwarp();
    copy_row_out(a, v, lane, row, total);
}

// Walk pass of every batch at once (4096-source batches, D = 4 or 8, K <= 3): one warp
// per row loads the row's walk ends once (row_ends_load) and writes the row's
// level-K visited row of every batch to vall[b] (padding, the diagonal and every
// end of that batch), a flag word to vall_fl[b] and the level counts into counts[b].
//
// Tables without one-way entries (*a.oneway == 0, from walk_check_kernel): the count
// of level L of batch b is the sum over the batch's sources s of n_L(s), the number
// of vertices at distance exactly L from s (pairs (v, s) at distance L, counted
// from the source's side).  Row s gives n_L(s): its ends inserted level by level
// into a per-warp vertex set (s itself first) -- an end is new at its first level.
// The rows then need no level split (one OR copy a batch, kWalkAllOrGroup batches at
// a time), and the flag word marks the chunks holding any end: every source first
// reached at level K has an end of length K there, so these flags contain the
// level-K frontier's, which is all the visited-set pull levels need of them.
//
// Tables with one-way entries: per batch, exactly walk_rows32's construction (each
// level's ends ORed into their own copy of the row, V_L = V_{L-1} | A_L from the
// padding and the diagonal up, the level's new pairs popc(V_L) - popc(V_{L-1}), the
// flag word from the level-K new bits), kWalkAllGroup batches at a time.
constexpr int kWalkAllGroup = 4;       // batches a warp builds at once with level copies
constexpr int kWalkAllOrGroup = 8;     // ... with one OR copy a batch and the full vertex set
constexpr int kWalkAllWide = 16;       // ... when every vertex is a source (small vertex set)
constexpr int kWalkSetSlots = 1024;    // a warp's vertex set (more than 1 + d + d^2 + d^3 for d <= 8)
constexpr int kWalkSetSmall = 256;     // ... for levels below K only (more than 1 + d + d^2 for d <= 8)
__host__ __device__ constexpr int cmax(int x, int y) { return x > y ? x : y; }
__host__ __device__ constexpr int walk_all_warp_bytes(int K) {
    return cmax(kWalkAllGroup * K * 512,
                cmax(kWalkAllOrGroup * 512 + kWalkSetSlots * 4, kWalkAllWide * 512 + kWalkSetSmall * 4));
}
__host__ __device__ constexpr int walk_all_smem(int K) { return (kIndexBlock / 32) * walk_all_warp_bytes(K); }

// Inserts w into a warp's open-addressing vertex set of 2^bits slots; 1 when new.
__device__ __forceinline__ unsigned set_insert(int *T, const int w, const int bits) {
    const unsigned mask = (1u << bits) - 1u;
    unsigned h = ((unsigned)w * 2654435761u) >> (32 - bits);
    for (unsigned probe = 0; probe <= mask; ++probe) {
        const int old = atomicCAS(T + h, -1, w);
        if (old == -1) return 1u;
        if (old == w) return 0u;
        h = (h + 1u) & mask;
    }
    return 0u;   // not reached: the set holds fewer vertices than slots
}

// One-way check of the whole table (one thread an entry): *oneway = 1 when some
// entry u of row v has no v in row u.
static __global__ void walk_check_kernel(const int32_t *adj, const int rows, const int d, int *oneway,
                                         const int *bad) {
    if (bad && *bad) return;
    const long long n = (long long)rows * d;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(k / d);
        const int32_t *ur = adj + (size_t)__ldg(adj + k) * d;
        bool f = false;
        for (int j = 0; j < d; ++j) f |= __ldg(ur + j) == v;
        if (!f) *oneway = 1;
    }
}

template <int D, int K>
__global__ void __launch_bounds__(kIndexBlock, 3) walk_all_kernel(const WalkIndexArgs a) {
    extern __shared__ __align__(16) unsigned char s_walk[];
    __shared__ unsigned long long s_cnt[kIndexMaxKeys];
    if (a.bad && *a.bad) return;
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const int nb = a.nb, nkeys = nb * K;   // a.K == K
    // mode 0: one-way entries (level copies); 1: counts from the full vertex set;
    // 2: every vertex a source -- the set holds levels below K, and n_K(s) is the
    // popcount of row s's own level-K rows less the padding, s and the lower levels
    const bool sym = a.oneway != nullptr && ld_acquire_i(a.oneway) == 0;
    const bool every = a.inv == nullptr && a.src_first == 0 && a.src_begin == 0 && a.ns_total == a.rows;
    const int mode = !sym ? 0 : (every ? 2 : 1);
    const int GG = mode == 0 ? kWalkAllGroup : (mode == 1 ? kWalkAllOrGroup : kWalkAllWide);
    const int set_bits = mode == 2 ? 8 : 10;
    for (int k = (int)threadIdx.x; k < nkeys; k += (int)blockDim.x) s_cnt[k] = 0ull;
    __syncthreads();
    unsigned char *mine = s_walk + (size_t)wib * walk_all_warp_bytes(K);
    uint4 *buf4 = reinterpret_cast<uint4 *>(mine);
    uint32_t *buf = reinterpret_cast<uint32_t *>(mine);
    int *set = reinterpret_cast<int *>(mine + (mode == 2 ? kWalkAllWide : kWalkAllOrGroup) * 512);
    constexpr int Q = RowEnds<D>::Q, U3 = RowEnds<D>::U3, S3 = RowEnds<D>::S3, NV = RowEnds<D>::NV;
    RowEndsRaw<D> r;
    int pk[NV];
    const size_t items = (size_t)a.rows * 32u;
    const unsigned long long pad_all = (unsigned long long)nb * (unsigned long long)a.S - (unsigned long long)a.ns_total;
    for (int v = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); v < a.rows;
         v += (int)((gridDim.x * blockDim.x) >> 5)) {
        row_ends_load<D>(a, v, lane, r);
        // the row's own source: its batch and place (the diagonal bit)
        const int g = a.inv ? __ldg(a.inv + v) : v - a.src_first;
        const int jd = (g >= 0 && (unsigned)(g - a.src_begin) < (unsigned)a.ns_total) ? g - a.src_begin : -1;
        const int bd = jd >= 0 ? jd / a.S : -1, jj_d = jd - bd * a.S;
        unsigned n1 = 0u, n2 = 0u, n3 = 0u;   // vertices first at levels 1..3 (this lane's share)
        if (mode != 0 && jd >= 0) {
            // level by level into the vertex set (mode 2: levels below K)
            const int slots = 1 << set_bits;
            for (int i = (int)lane; i < slots / 4; i += 32) reinterpret_cast<int4 *>(set)[i] = make_int4(-1, -1, -1, -1);
            __syncwarp();
            if (lane == 0) set_insert(set, v, set_bits);
            __syncwarp();
            const int top = mode == 2 ? K - 1 : K;
            if (top >= 1) {
                n1 = lane < (unsigned)D ? set_insert(set, r.x1, set_bits) : 0u;
                __syncwarp();
            }
            if (top >= 2) {
#pragma unroll
                for (int s2 = 0; s2 < (Q + 31) / 32; ++s2)
                    if (s2 * 32 + (int)lane < Q)
                        n2 += set_insert(set, (int)r.q2[s2].x, set_bits) + set_insert(set, (int)r.q2[s2].y, set_bits) +
                              set_insert(set, (int)r.q2[s2].z, set_bits) + set_insert(set, (int)r.q2[s2].w, set_bits);
                __syncwarp();
            }
            if (top >= 3) {
#pragma unroll
                for (int s3 = 0; s3 < S3; ++s3)
                    if (s3 * 32 + (int)lane < U3)
                        n3 += set_insert(set, (int)r.q3[s3].x, set_bits) + set_insert(set, (int)r.q3[s3].y, set_bits) +
                              set_insert(set, (int)r.q3[s3].z, set_bits) + set_insert(set, (int)r.q3[s3].w, set_bits);
                __syncwarp();
            }
        }
        row_ends_classify<D>(a, lane, r, pk);
        unsigned ball = 0u;   // mode 2: popcount of this lane's chunks of the row's level-K rows
        for (int g0 = 0; g0 < nb; g0 += GG) {
            const int G = min(GG, nb - g0);
            const int copies = mode == 0 ? G * K : G;
            for (int i = 0; i < copies; ++i) buf4[i * 32 + lane] = u4zero();
            __syncwarp();
#pragma unroll
            for (int k = 0; k < NV; ++k)
                if (pk[k] >= 0) {
                    const int key = pk[k] >> 16, b = key / K;
                    if (b >= g0 && b < g0 + G) {
                        const int jj = pk[k] & 0xffff;
                        const int copy = mode == 0 ? (b - g0) * K + (key - b * K) : b - g0;
                        atomicOr(buf + copy * 128 + (jj >> 5), 1u << (jj & 31));
                    }
                }
            __syncwarp();
            uint4 *out = a.vall + (size_t)g0 * items + (size_t)v * 32 + lane;
            for (int bb = 0; bb < G; ++bb, out += items) {
                const int b = g0 + bb;
                const int ns = min(a.S, a.ns_total - b * a.S);
                uint4 vv = ns < a.S ? pad_mask((int)lane, ns) : u4zero();
                if (b == bd && (unsigned)(jj_d >> 7) == lane) {
                    const unsigned bit = 1u << (jj_d & 31), comp = ((unsigned)jj_d >> 5) & 3u;
                    if (comp == 0u) vv.x |= bit; else if (comp == 1u) vv.y |= bit;
                    else if (comp == 2u) vv.z |= bit; else vv.w |= bit;
                }
                bool flag;
                if (mode != 0) {
                    const uint4 al = buf4[bb * 32 + lane];
                    vv = u4or(vv, al);
                    flag = u4any(al);
                    if (mode == 2) ball += u4popc(vv);
                } else {
                    uint4 prev = vv;
                    unsigned pc = u4popc(vv);
#pragma unroll
                    for (int L = 0; L < K; ++L) {
                        const uint4 al = buf4[(bb * K + L) * 32 + lane];
                        prev = vv;
                        vv = u4or(vv, al);
                        const unsigned pn = u4popc(vv);
                        const unsigned t = __reduce_add_sync(0xffffffffu, pn - pc);
                        if (lane == 0 && t) atomicAdd(s_cnt + b * K + L, (unsigned long long)t);
                        pc = pn;
                    }
                    flag = u4any(andnot(vv, prev));
                }
                *out = vv;
                const unsigned m = __ballot_sync(0xffffffffu, flag);
                if (lane == 0) a.vall_fl[(size_t)b * a.rows + v] = m;
            }
            __syncwarp();
        }
        if (mode != 0 && jd >= 0) {
            n1 = __reduce_add_sync(0xffffffffu, n1);
            n2 = __reduce_add_sync(0xffffffffu, n2);
            n3 = __reduce_add_sync(0xffffffffu, n3);
            if (mode == 2) {
                // the vertices within K of s, less s and the levels below K
                const unsigned long long in_ball =
                    (unsigned long long)__reduce_add_sync(0xffffffffu, ball) - pad_all - 1ull;
                const unsigned nK = (unsigned)in_ball - n1 - n2;
                if (K == 1) n1 = nK; else if (K == 2) n2 = nK; else n3 = nK;
            }
            if (lane == 0) {
                atomicAdd(s_cnt + bd * K, (unsigned long long)n1);
                if (K >= 2) atomicAdd(s_cnt + bd * K + 1, (unsigned long long)n2);
                if (K >= 3) atomicAdd(s_cnt + bd * K + 2, (unsigned long long)n3);
            }
        }
    }
    __syncthreads();
    for (int k = (int)threadIdx.x; k < nkeys; k += (int)blockDim.x)
        if (s_cnt[k]) atomicAdd(a.counts + (size_t)(k / K) * a.counts_stride + (k % K) + 1, s_cnt[k]);
}

template <int D>
__global__ void __launch_bounds__(kIndexBlock) walk_index_kernel(const WalkIndexArgs a) {
    __shared__ unsigned s_cur[kIndexBlock / 32][kIndexMaxKeys];
    __shared__ __align__(16) uint16_t s_ent[kIndexBlock / 32][kIndexMaxCap];
    if (a.bad && *a.bad) return;
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    unsigned *cur = s_cur[wib];
    uint16_t *row = s_ent[wib];
    const int nkeys = a.nb * a.K;
    const int per = (nkeys + 31) / 32;   // keys per lane in the scan
    // source index within the evaluation of end w, or -1
    auto src_of = [&](const int32_t w) -> int {
        const int g = a.inv ? __ldg(a.inv + w) : w - a.src_first;
        const int j = g - a.src_begin;
        return (g >= 0 && (unsigned)j < (unsigned)a.ns_total) ? j : -1;
    };
    for (int v = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); v < a.rows;
         v += (int)((gridDim.x * blockDim.x) >> 5)) {
        for (int k = (int)lane; k < nkeys; k += 32) cur[k] = 0u;
        __syncwarp();
        if constexpr (D > 0 && D <= 8 && (D * D) % 4 == 0 && D % 4 == 0) {
            if (a.K <= 3) {
                index_row_regs<D>(a, v, lane, cur, row, nkeys);
                continue;
            }
        }
        if (a.asym) row_oneway_check(a, v, lane, D > 0 ? D : a.d);
        // pass 1: bucket sizes
        for_walk_ends<D>(a, v, lane, [&](const int32_t w, const int L) {
            const int j = src_of(w);
            if (j >= 0) atomicAdd(cur + (int)a.div_S.div((unsigned)j) * a.K + (L - 1), 1u);
        });
        __syncwarp();
        // exclusive prefix over the buckets: lane l owns keys [l * per, (l + 1) * per)
        unsigned mine = 0u;
        for (int k = (int)lane * per; k < min(nkeys, ((int)lane + 1) * per); ++k) mine += cur[k];
        unsigned incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
            if ((int)lane >= o) incl += t;
        }
        unsigned run = incl - mine;
        uint16_t *offrow = a.off + (size_t)v * a.off_stride;
        for (int k = (int)lane * per; k < min(nkeys, ((int)lane + 1) * per); ++k) {
            const unsigned c = cur[k];
            offrow[k] = (uint16_t)run;
            cur[k] = run;
            run += c;
        }
        const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
        if (lane == 0) offrow[nkeys] = (uint16_t)total;
        __syncwarp();
        // pass 2: each kept end at its bucket's next slot (the row's ends again, now from L1)
        for_walk_ends<D>(a, v, lane, [&](const int32_t w, const int L) {
            const int j = src_of(w);
            if (j >= 0) {
                const unsigned b = a.div_S.div((unsigned)j);
                const unsigned pos = atomicAdd(cur + (int)b * a.K + (L - 1), 1u);
                row[pos] = (uint16_t)((unsigned)j - b * (unsigned)a.S);
            }
        });
        __syncwarp();
        copy_row_out(a, v, lane, row, total);
    }
}

struct WalkArgs {
    const uint16_t *ent, *off;  // the walk index (walk_index_kernel)
    int cap, off_stride;
    int b;                    // the batch: buckets b * K .. b * K + K - 1
    const int32_t *inv;       // source index of each vertex (-1: none), or nullptr
    int src_first, first, ns; // source j of the batch is vertex src_first + first + j (inv == nullptr)
    uint4 *V, *F;             // visited bits (V_K), frontier of level K+1
    uint32_t *fl;             // flag words of F
    int rows, nC, K;
    unsigned items;
    int rows_per_group;       // lcm(nC, 32) / nC
};

constexpr int kWalkMaxNC = 64;    // row width (uint4 chunks) the per-warp buffers hold

// Shared-memory bytes of the walk buffers of one warp.
constexpr int kWalkStageRows = 12;    // rows walk_rows32 stages at once
constexpr int kWalkStageWords = 33;   // entry words staged per row (64 entries from an odd start)
__host__ __device__ constexpr int walk_smem_per_warp(int nC) {
    // walk_rows32: 4 level copies of the row and the staged entry words
    return nC == 32 ? 32 * 16 * 4 + kWalkStageRows * kWalkStageWords * 4 : nC * 16 * 2 + kWalkMaxNC * 4;
}
static_assert(walk_smem_per_warp(32) % 16 == 0, "per-warp walk buffers stay 16-byte aligned");
static_assert(kWalkStageRows * 5 <= 64, "bounds of the staged rows fit two registers a lane");

// A row's index entries of this batch: bucket bounds (lanes 0..K hold off[bK + lane])
// and its first 64 entries (lanes hold entries e0 + lane and e0 + 32 + lane, or -1).
struct WalkRowLoad {
    int o;
    int x0, x1;
};

static __device__ __noinline__ void walk_rows(const WalkArgs &w, unsigned char *smem, const unsigned gwarp,
                                              const unsigned nwarps, unsigned long long *s_cnt) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned char *mine = smem + (size_t)(threadIdx.x >> 5) * walk_smem_per_warp(w.nC);
    uint4 *Vb4 = reinterpret_cast<uint4 *>(mine);     // the row, 16 bytes per chunk (conflict-free)
    uint4 *Fb4 = Vb4 + w.nC;
    uint32_t *Vb = reinterpret_cast<uint32_t *>(Vb4);
    uint32_t *Fb = reinterpret_cast<uint32_t *>(Fb4);
    uint32_t *flw = reinterpret_cast<uint32_t *>(Fb4 + w.nC);
    const int K = w.K, rpg = w.rows_per_group;
    unsigned cnt[4] = {0u, 0u, 0u, 0u};
    const int gwords = (rpg * w.nC) >> 5;               // flag words per group
    const unsigned ntiles = (w.items + 31u) >> 5;
    // this warp's rows in order: the rows of groups gwarp, gwarp + nwarps, ...
    auto next_row = [&](const int v) -> int {
        if (v < 0) return -1;
        int n = v + 1;
        if (n % rpg == 0) n = (n / rpg - 1 + (int)nwarps) * rpg;
        return n < w.rows ? n : -1;
    };
    auto load_off = [&](const int v) -> int {
        return (v >= 0 && lane <= (unsigned)K) ? (int)__ldg(w.off + (size_t)v * w.off_stride + w.b * K + lane) : 0;
    };
    auto load_ents = [&](const int v, const int o) -> WalkRowLoad {
        WalkRowLoad r{o, -1, -1};
        const int e0 = __shfl_sync(0xffffffffu, o, 0), eK = __shfl_sync(0xffffffffu, o, K);
        if (v >= 0) {
            const uint16_t *ents = w.ent + (size_t)v * w.cap;
            if (e0 + (int)lane < eK) r.x0 = __ldg(ents + e0 + lane);
            if (e0 + 32 + (int)lane < eK) r.x1 = __ldg(ents + e0 + 32 + lane);
        }
        return r;
    };
    int v = (int)gwarp * rpg;
    if (v >= w.rows) v = -1;
    // two rows ahead: the entries of the next row and the bounds of the one after
    WalkRowLoad cur = load_ents(v, load_off(v));
    int vn = next_row(v);
    int o_n = load_off(vn);
    for (; v >= 0;) {
        const int vnn = next_row(vn);
        const WalkRowLoad nxt = load_ents(vn, o_n);
        const int o_nn = load_off(vnn);
        const int r = v % rpg;
        if (r == 0)
            for (int k = (int)lane; k < gwords; k += 32) flw[k] = 0u;
        // the row starts as its padding bits and the diagonal
        for (int c = (int)lane; c < w.nC; c += 32) {
            Vb4[c] = pad_mask(c, w.ns);
            Fb4[c] = u4zero();
        }
        __syncwarp();
        if (lane == 0) {
            const int g = w.inv ? __ldg(w.inv + v) : v - w.src_first;
            const int j = g - w.first;
            if (g >= 0 && (unsigned)j < (unsigned)w.ns) Vb[j >> 5] |= 1u << (j & 31);
        }
        __syncwarp();
        // the entries level by level (bucket order is level order)
        const int e0 = __shfl_sync(0xffffffffu, cur.o, 0);
        const int e1 = __shfl_sync(0xffffffffu, cur.o, 1);
        const int e2 = __shfl_sync(0xffffffffu, cur.o, K >= 2 ? 2 : 1);
        const int e3 = __shfl_sync(0xffffffffu, cur.o, K >= 3 ? 3 : 1);
        const int eK = __shfl_sync(0xffffffffu, cur.o, K);
        auto level_of = [&](const int i) { return i < e1 ? 1 : (i < e2 ? 2 : (i < e3 ? 3 : 4)); };
        auto put = [&](const int j, const int L) {
            const uint32_t bit = 1u << (j & 31);
            const uint32_t old = atomicOr(Vb + (j >> 5), bit);
            if (!(old & bit)) {
                cnt[L - 1] += 1u;
                if (L == K) atomicOr(Fb + (j >> 5), bit);
            }
        };
        const int L0 = cur.x0 >= 0 ? level_of(e0 + (int)lane) : 0;
        const int L1 = cur.x1 >= 0 ? level_of(e0 + 32 + (int)lane) : 0;
        for (int L = 1; L <= K; ++L) {
            if (L0 == L) put(cur.x0, L);
            if (L1 == L) put(cur.x1, L);
            __syncwarp();
        }
        // rows with more than 64 entries in this batch: the rest, 32 at a time,
        // still in level order (every chunk's levels are at least the last one's)
        for (int base = e0 + 64; base < eK; base += 32) {
            const int i = base + (int)lane;
            const int x = i < eK ? (int)__ldg(w.ent + (size_t)v * w.cap + i) : -1;
            const int Li = x >= 0 ? level_of(i) : 0;
            for (int L = 1; L <= K; ++L) {
                if (Li == L) put(x, L);
                __syncwarp();
            }
        }
        // write the row: V = V_K (padding included), F = new at level K, and the flag
        // bits of F (one ballot per 32 chunks; lane 0 merges it into the group's words)
        const unsigned t0 = (unsigned)v * (unsigned)w.nC;
        const unsigned b0 = (unsigned)r * (unsigned)w.nC;   // chunk index within the group
        for (int cb = 0; cb < w.nC; cb += 32) {
            const int c = cb + (int)lane;
            bool any = false;
            if (c < w.nC) {
                const uint4 vv = Vb4[c], ff = Fb4[c];
                w.V[t0 + c] = vv;
                if (w.F) w.F[t0 + c] = ff;
                any = u4any(ff);
            }
            const unsigned m = __ballot_sync(0xffffffffu, any);
            if (lane == 0 && m) {
                const unsigned first = b0 + (unsigned)cb, off = first & 31u;
                flw[first >> 5] |= m << off;
                if (off && (m >> (32u - off))) flw[(first >> 5) + 1] |= m >> (32u - off);  // stays in the group
            }
        }
        __syncwarp();
        if (r == rpg - 1 || v == w.rows - 1) {
            // the group's flag words (the group starts on a tile boundary)
            const unsigned tile0 = (unsigned)(v / rpg) * (unsigned)gwords;
            for (int k = (int)lane; k < gwords; k += 32)
                if (tile0 + k < ntiles) w.fl[tile0 + k] = flw[k];
            __syncwarp();
        }
        v = vn;
        vn = vnn;
        cur = nxt;
        o_n = o_nn;
    }
#pragma unroll
    for (int L = 0; L < 4; ++L) {
        const unsigned s = __reduce_add_sync(0xffffffffu, cnt[L]);
        if (lane == 0 && s) atomicAdd(s_cnt + L, (unsigned long long)s);
    }
}

// H2[v][i*d + j] = adj[adj[v][i]][j]: the level-2 walk ends of every row, built once
// per evaluation (after the table's range check: a bad table builds nothing).
// When d % 4 == 0 a thread copies 16 bytes (one quarter-row of a neighbour's row).
// With `oneway` (d % 4 == 0, d / 4 a power of two, rows * d * d / 4 a multiple of 32,
// so that every warp iteration is full and a neighbour's row lies within one warp):
// also the table's one-way check, *oneway = 1 when some row u = adj[v][i] lacks v.
static __global__ void h2_kernel(const int32_t *adj, int32_t *h2, int rows, int d, const int *bad,
                                 int *oneway = nullptr) {
    if (bad && *bad) return;
    const long long dd = (long long)d * d;
    if (d % 4 == 0) {
        const int q = d / 4;                           // uint4 per adjacency row
        const long long n = (long long)rows * d * q;   // uint4 of H2
        for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
             k += (long long)gridDim.x * blockDim.x) {
            const long long v = k / ((long long)d * q), r = k % ((long long)d * q);
            const int p = __ldg(adj + v * d + r / q);
            const uint4 w = __ldg(reinterpret_cast<const uint4 *>(adj + (size_t)p * d) + r % q);
            reinterpret_cast<uint4 *>(h2)[k] = w;
            if (oneway) {
                bool hit = (long long)(int)w.x == v || (long long)(int)w.y == v || (long long)(int)w.z == v ||
                           (long long)(int)w.w == v;
                for (int o = 1; o < q; o <<= 1) hit |= __shfl_xor_sync(0xffffffffu, hit, o) != 0;
                if ((threadIdx.x & (unsigned)(q - 1)) == 0u && !hit) *oneway = 1;
            }
        }
        return;
    }
    const long long n = (long long)rows * dd;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const long long v = k / dd, r = k % dd;
        h2[k] = __ldg(adj + (size_t)__ldg(adj + v * d + r / d) * d + r % d);
    }
}

// Resident blocks per SM the register allocation targets: 4 (64 registers).  At 6
// (40 registers) the level loop and its out-of-line level functions spill, and
// the dense levels of a 65536-vertex, 8-regular evaluation ran about 25 % slower
// (38 against 30 us a level); 32 resident warps a SM keep the gathers in flight.
#ifndef GG_MIN_BLOCKS_SMALL_D
#define GG_MIN_BLOCKS_SMALL_D 4
#endif
__host__ __device__ constexpr int min_blocks_for(int D) {
    return (D > 0 && D <= 8) ? GG_MIN_BLOCKS_SMALL_D : 4;
}

// Block-uniform state of the batch and level loops.  It lives in shared memory
// (thread 0 updates it between barriers) so that the level work keeps its
// registers.
struct LoopState {
    unsigned long long reached;  // pairs reached so far in the batch
    unsigned long long c_prev;   // pairs first reached at the previous level
    unsigned long long pairs;    // sources x rows of the batch
    int push_on;                 // push levels allowed in this launch
    int in_p;                    // push buffer holding the previous level's frontier, or -1
    int dirty_p;                 // push buffer still to be cleared, or -1
    int wrote_all_prev;          // the previous level wrote F whole
    int nf_valid;                // a.nf describes V as the previous level left it
    int done;                    // the batch's level loop ends
    int L_next;                  // first level the level loop runs (after a walk pass)
    int sym;                     // the table has no one-way entries (walk_asym read 0)
    uint4 *Pv, *Qv;              // the batch's visited-set pull buffers (Pv holds level walk_K)
    uint4 *Rv;                   // the buffer levels walk_K+2.. alternate with Qv, when r_on
    int r_on;                    // level walk_K + 2 wrote Rv whole (set by that level)
    const uint32_t *fl_walk;     // the flag words level walk_K + 1 reads
    unsigned long long *vt;      // the batch's 3 level totals (a.vtot + 3b), or nullptr
};

// 4-byte asynchronous copy global -> shared (no registers held while in flight).
__device__ __forceinline__ void cp_async4(void *smem_dst, const void *gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// walk_rows for rows of exactly 32 chunks (4096-source batches): a row is one tile
// and one flag word, so lane c owns chunk c of the row.  A warp takes a contiguous
// run of rows and works through it kWalkStageRows at a time in three steps:
//  1. the bucket bounds of every staged row (one load round trip; lane l holds
//     bound l % (K+1) of row l / (K+1), lanes 32.. in a second register);
//  2. the words holding each row's first 64 entries of this batch, copied into
//     shared memory with 4-byte cp.async (second round trip; no registers held);
//  3. per row, from shared memory: each level's entries ORed into their own copy of
//     the row (A_L, non-returning atomics), then every lane builds, for its chunk,
//     V_L = V_{L-1} | A_L from the diagonal up, counts popc(V_L) - popc(V_{L-1})
//     pairs at level L (a source reached at several levels counts at the first),
//     and writes V = V_K, F = V_K & ~V_{K-1} (unless F is null) and the frontier's
//     flag word (one ballot).  Entries past the first 64 of a row are read directly.

template <int K>
static __device__ __noinline__ void walk_rows32(const BfsArgs &a, const int b, const int first, const int ns,
                                                uint4 *F, uint32_t *fl, unsigned char *wsm,
                                                const unsigned gwarp, const unsigned nwarps,
                                                unsigned long long *s_cnt) {
    const unsigned lane = threadIdx.x & 31u;
    uint4 *Ab4 = reinterpret_cast<uint4 *>(wsm);              // A_1 .. A_K (4 copies reserved)
    uint32_t *Ab = reinterpret_cast<uint32_t *>(wsm);
    uint32_t *Es = reinterpret_cast<uint32_t *>(wsm + 4 * 512);   // [kWalkStageRows][kWalkStageWords]
    const int rows = a.rows, off_stride = a.walk_off_stride, cap = a.walk_cap;
    const uint16_t *off_b = a.walk_off + b * K;
    const uint16_t *ent = a.walk_ent;
    const int32_t *inv = a.inv;
    const uint4 pad = pad_mask((int)lane, ns);
    unsigned cnt[K];
#pragma unroll
    for (int L = 0; L < K; ++L) {
        cnt[L] = 0u;
        Ab4[L * 32 + lane] = u4zero();
    }
    __syncwarp();
    const int per = (int)(((unsigned)rows + nwarps - 1u) / nwarps);
    const int v_lo = min(rows, (int)gwarp * per), v_hi = min(rows, v_lo + per);
    for (int r0 = v_lo; r0 < v_hi; r0 += kWalkStageRows) {
        const int R = min(kWalkStageRows, v_hi - r0);
        // 1. bucket bounds (and the lifted forms' source ids of the rows)
        int oA = 0, oB = 0, gd = 0;
        {
            const int rA = (int)lane / (K + 1), rB = ((int)lane + 32) / (K + 1);
            if (rA < R) oA = (int)__ldg(off_b + (size_t)(r0 + rA) * off_stride + ((int)lane - rA * (K + 1)));
            if (rB < R) oB = (int)__ldg(off_b + (size_t)(r0 + rB) * off_stride + ((int)lane + 32 - rB * (K + 1)));
            if (inv && (int)lane < R) gd = __ldg(inv + r0 + (int)lane);
        }
        auto bound = [&](const int i) {   // bound i of the staged rows (i uniform)
            return __shfl_sync(0xffffffffu, i < 32 ? oA : oB, i & 31);
        };
        // 2. entry words of each row (rows start 4-byte aligned: cap is even)
        for (int r = 0; r < R; ++r) {
            const int e0 = bound(r * (K + 1)), eK = bound(r * (K + 1) + K);
            const int w0 = e0 >> 1, w1 = min((eK + 1) >> 1, w0 + kWalkStageWords);
            const uint32_t *src = reinterpret_cast<const uint32_t *>(ent + (size_t)(r0 + r) * cap);
            for (int w = w0 + (int)lane; w < w1; w += 32) cp_async4(Es + r * kWalkStageWords + (w - w0), src + w);
        }
        cp_async_wait_all();
        __syncwarp();
        // 3. the rows
        for (int r = 0; r < R; ++r) {
            const int v = r0 + r;
            int e[K + 1];
#pragma unroll
            for (int k = 0; k <= K; ++k) e[k] = bound(r * (K + 1) + k);
            const int n = e[K] - e[0];
            const uint16_t *Er = reinterpret_cast<const uint16_t *>(Es + r * kWalkStageWords) + (e[0] & 1);
            for (int i = (int)lane; i < n; i += 32) {
                const int x = i < 64 ? (int)Er[i] : (int)__ldg(ent + (size_t)v * cap + e[0] + i);
                int L = 0;
#pragma unroll
                for (int k = 1; k < K; ++k) L += (e[0] + i >= e[k]) ? 1 : 0;
                atomicOr(Ab + L * 128 + (x >> 5), 1u << (x & 31));
            }
            __syncwarp();
            uint4 vv = pad;
            {
                const int g = inv ? __shfl_sync(0xffffffffu, gd, r) : v - a.src_first;
                const int j = g - first;
                if (g >= 0 && (unsigned)j < (unsigned)ns && (unsigned)(j >> 7) == lane) {
                    const unsigned bit = 1u << (j & 31), comp = ((unsigned)j >> 5) & 3u;
                    if (comp == 0u) vv.x |= bit; else if (comp == 1u) vv.y |= bit;
                    else if (comp == 2u) vv.z |= bit; else vv.w |= bit;
                }
            }
            // level by level (a branch-free form: skipping the popcounts and clearing
            // stores of empty lanes measured slower)
            uint4 prev = vv;
            unsigned pc = u4popc(vv);
#pragma unroll
            for (int L = 0; L < K; ++L) {
                const uint4 al = Ab4[L * 32 + lane];
                Ab4[L * 32 + lane] = u4zero();          // clean for the next row
                prev = vv;
                vv = u4or(vv, al);
                const unsigned pn = u4popc(vv);
                cnt[L] += pn - pc;
                pc = pn;
            }
            const uint4 ff = andnot(vv, prev);
            a.V[(size_t)v * 32 + lane] = vv;
            if (F) F[(size_t)v * 32 + lane] = ff;
            const unsigned m = __ballot_sync(0xffffffffu, u4any(ff));
            if (lane == 0) fl[v] = m;
            __syncwarp();
        }
    }
#pragma unroll
    for (int L = 0; L < K; ++L) {
        const unsigned t = __reduce_add_sync(0xffffffffu, cnt[L]);
        if (lane == 0 && t) atomicAdd(s_cnt + L, (unsigned long long)t);
    }
}

// The walk pass of batch b, its counts and the loop state it leaves (levels
// 1..K done; S.L_next = K + 1, or the level at which the batch ended).  Out of
// line so that the level loop keeps its registers.  Returns the barrier count
// after the pass, or kWaitGaveUp when a barrier wait gave up.
constexpr unsigned kWaitGaveUp = 0xffffffffu;
// The loop state after the walk's levels 1..K of batch b (their counts complete):
// S.L_next = K + 1, or the level at which the batch ended, and the batch's buffers.
__device__ __forceinline__ void walk_state(const BfsArgs &a, const int b, const int ns, LoopState &S) {
    unsigned long long *counts = a.counts + (size_t)b * (size_t)a.stride;
    const int K = a.walk_K;
    if (threadIdx.x == 0) {
        S.pairs = (unsigned long long)ns * (unsigned long long)a.rows;
        S.reached = (unsigned long long)ns;
        S.in_p = -1;
        S.wrote_all_prev = 1;
        S.nf_valid = 0;
        S.done = 0;
        int L = 1;
        for (; L <= K; ++L) {
            const unsigned long long cL = ld_relaxed_u64(counts + L);
            S.reached += cL;
            S.c_prev = cL;
            if (cL == 0ull || L >= a.max_levels || S.reached == S.pairs) { S.done = 1; break; }
        }
        S.L_next = S.done ? L : K + 1;
        S.Pv = a.vall ? a.vall + (size_t)b * a.items : a.V;
        S.Qv = a.vall ? a.V : a.F0;
        S.Rv = a.vall && a.third ? a.third : S.Pv;
        S.vt = a.vtot ? a.vtot + 3 * (size_t)b : nullptr;
        S.fl_walk = a.vall ? a.vall_fl + (size_t)b * ((a.items + 31u) >> 5) : (((K + 1) & 1) ? a.fl0 : a.fl1);
        if (b == 0 && a.level_ns && blockIdx.x == 0)
            for (int k = 1; k <= K; ++k) a.level_ns[k] = gtimer();
    }
    __syncthreads();
}

template <int D>
static __device__ __noinline__ unsigned walk_batch(const BfsArgs &a, const int b, const int ns, const int d,
                                                   const unsigned items, const unsigned gtid, const unsigned nthr,
                                                   unsigned epoch, LoopState &S) {
    extern __shared__ int32_t s_adj[];
    // Levels 1..K from the walk ends of every row (walk_rows): the counts
    // were zeroed by the host, so blocks add into them right away.
    __shared__ unsigned long long s_wcnt[4];
    unsigned long long *counts = a.counts + (size_t)b * (size_t)a.stride;
    if (threadIdx.x < 4) s_wcnt[threadIdx.x] = 0ull;
    if (blockIdx.x == 0 && threadIdx.x == 0) counts[0] = (unsigned long long)ns;
    if (b == 0 && a.level_ns && gtid == 0) a.level_ns[0] = gtimer();
    const int K = a.walk_K;
    if (a.vall) {
        // levels 1..K of every batch came from walk_all_kernel (launched before)
        walk_state(a, b, ns, S);
        return epoch;
    }
    // the pass's arguments in shared memory (one copy per block, not a
    // by-value struct on every thread's stack)
    __shared__ WalkArgs w;
    if (threadIdx.x == 0) {
        w.ent = a.walk_ent; w.off = a.walk_off; w.cap = a.walk_cap; w.off_stride = a.walk_off_stride;
        w.b = b;
        w.inv = a.inv;
        w.src_first = a.src_first; w.first = a.src_begin + b * 128 * a.nC; w.ns = ns;
        w.V = a.V;
        w.F = vpull_on(a) ? nullptr : (((K + 1) & 1) ? a.F0 : a.F1);   // what level K + 1 reads
        w.fl = ((K + 1) & 1) ? a.fl0 : a.fl1;
        w.rows = a.rows; w.nC = a.nC; w.K = K; w.items = items;
        w.rows_per_group = a.walk_rpg;
    }
    __syncthreads();
    if (a.nC == 32) {
        unsigned char *wsm = reinterpret_cast<unsigned char *>(s_adj) + a.walk_smem_off +
                             (size_t)(threadIdx.x >> 5) * walk_smem_per_warp(32);
        uint4 *Fw = vpull_on(a) ? nullptr : (((K + 1) & 1) ? a.F0 : a.F1);
        uint32_t *flw = ((K + 1) & 1) ? a.fl0 : a.fl1;
        const int first = a.src_begin + b * 128 * a.nC;
        switch (K) {
            case 1: walk_rows32<1>(a, b, first, ns, Fw, flw, wsm, gtid >> 5, nthr >> 5, s_wcnt); break;
            case 2: walk_rows32<2>(a, b, first, ns, Fw, flw, wsm, gtid >> 5, nthr >> 5, s_wcnt); break;
            case 3: walk_rows32<3>(a, b, first, ns, Fw, flw, wsm, gtid >> 5, nthr >> 5, s_wcnt); break;
            default: walk_rows32<4>(a, b, first, ns, Fw, flw, wsm, gtid >> 5, nthr >> 5, s_wcnt); break;
        }
    } else {
        walk_rows(w, reinterpret_cast<unsigned char *>(s_adj) + a.walk_smem_off, gtid >> 5, nthr >> 5, s_wcnt);
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int L = 1; L <= K; ++L)
            if (s_wcnt[L - 1]) atomicAdd(counts + L, s_wcnt[L - 1]);
    if (!grid_sync(a.ctl, a.expected, a.wait_ns, 0, epoch)) return kWaitGaveUp;
    walk_state(a, b, ns, S);
    return epoch;
}

// One cooperative launch = every source batch of an evaluation, all levels.
//
// Per batch: phase 0 (one pass over the chunks: visited bits reset, padding and
// the diagonal set, level-1 frontier and its flags written) -> grid barrier ->
// levels, each ended by a grid barrier.  One launch instead of one per batch
// saves the launch gap and the shared-memory adjacency reload per batch.
template <int D, bool PL>
__global__ void __launch_bounds__(kBlock, min_blocks_for(D)) bfs_batch_kernel(const __grid_constant__ BfsArgs a) {
    const int d = D > 0 ? D : a.d;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned nthr = gridDim.x * blockDim.x;
    const unsigned items = a.items, ntiles = (items + 31u) >> 5;
    __shared__ unsigned long long s_sum[kBlock / 32];
    __shared__ unsigned s_and[2][kBlock / 32];
    __shared__ unsigned s_next;
    __shared__ LoopState S;
    if (a.bad && *a.bad) return;  // uniform across the grid: no block reaches a barrier
    unsigned epoch = 0u;          // grid barriers passed
    const unsigned t_lo = (unsigned)((unsigned long long)ntiles * blockIdx.x / gridDim.x);
    const unsigned t_hi = (unsigned)((unsigned long long)ntiles * (blockIdx.x + 1) / gridDim.x);

    // The block's tile range covers vertices [v_lo, v_hi]; their adjacency rows
    // stay in shared memory for the whole launch when they fit.
    extern __shared__ int32_t s_adj[];
    const int32_t *adj = a.adj;
    unsigned v_base = 0;
    if (a.adj_smem_rows > 0 && t_hi > t_lo) {
        const unsigned v_lo = a.div_nc.div(t_lo * 32u);
        const unsigned last = min(t_hi * 32u, items) - 1u;
        const unsigned v_hi = a.div_nc.div(last);
        const unsigned nv = v_hi - v_lo + 1u;
        if (nv <= (unsigned)a.adj_smem_rows) {
            const size_t n = (size_t)nv * (size_t)d;
            const int32_t *g = a.adj + (size_t)v_lo * (size_t)d;
            for (size_t k = threadIdx.x; k < n; k += blockDim.x) s_adj[k] = __ldg(g + k);
            adj = s_adj;
            v_base = v_lo;
        }
    }
    // Push levels need the all-zero push buffers, a symmetric adjacency and
    // plain OR rows (the WVC masks are taken over every chunk, which only pull
    // levels visit).
    if (threadIdx.x == 0) {
        S.sym = a.walk_asym != nullptr && a.vtot != nullptr && ld_acquire_i(a.walk_asym) == 0;
        S.push_on = D > 0 && 32 % D == 0 && a.push_ppm > 0 && a.P0 != nullptr && a.asym != nullptr &&
                    a.masks == nullptr && (PL || a.walk_K == 0);
        S.dirty_p = -1;
    }
    __syncthreads();
    if (S.push_on) {
        const unsigned long long n = (unsigned long long)a.rows * (unsigned long long)d;
        for (unsigned long long k = gtid; k < n; k += nthr) {
            const unsigned v = (unsigned)(k / (unsigned)d);
            const int32_t *row = a.adj + (size_t)__ldg(a.adj + k) * (size_t)d;
            bool found = false;
            for (int j = 0; j < d; ++j) found |= (unsigned)__ldg(row + j) == v;
            if (!found) *a.asym = 1;
        }
        if (!grid_sync(a.ctl, a.expected, a.wait_ns, 0, epoch)) return;
        if (threadIdx.x == 0) S.push_on = ld_acquire_i(a.asym) == 0;
        __syncthreads();
    }

    const bool walk = !PL && a.walk_K > 0;
    const bool vp = walk && vpull_on(a);   // visited-set pull after the walk
    for (int b = 0; b < a.nb; ++b) {
        const int ns = min(128 * a.nC, a.ns_total - b * 128 * a.nC);
        if (a.batch_ns && gtid == 0) a.batch_ns[2 * b] = gtimer();
        if (walk) {
            epoch = walk_batch<D>(a, b, ns, d, items, gtid, nthr, epoch, S);
            if (epoch == kWaitGaveUp) return;
        } else {
            if (threadIdx.x == 0) S.L_next = 1;
            // Phase 0 (cudaASPLconv.cu:9-33): counters zeroed, padding bits and
            // the diagonal visited, the diagonal as the level-1 frontier.  The
            // sources of a batch are distinct vertices, so a chunk holds at most
            // one of them.
            unsigned long long *counts = a.counts + (size_t)b * (size_t)a.stride;
            unsigned *masks = a.masks ? a.masks + (size_t)b * (size_t)a.stride : nullptr;
            if (blockIdx.x == 0)
                for (int i = threadIdx.x; i <= a.max_levels; i += blockDim.x) {
                    counts[i] = i == 0 ? (unsigned long long)ns : 0ull;
                    if (masks) masks[i] = 0xffffffffu;
                }
            const int dirty = S.dirty_p, clean = dirty == 0 ? 1 : 0;
            const bool push_on = S.push_on != 0;
            if (dirty >= 0) clear_push_buffer(dirty ? a.P1 : a.P0, dirty ? a.pf1 : a.pf0, ntiles, gtid, nthr);
            if constexpr (PL) {
                if (threadIdx.x == 0)
                    plane_slot() = PlaneOut{a.planes, a.plane_stride, a.plane_cols, (unsigned)(b * a.nC),
                                            a.nplanes, 0};
                __syncthreads();
            }
            phase0_tiles<PL>(a.inv, a.src_first, a.src_begin + b * 128 * a.nC, ns, a.V, a.F0, a.fl0,
                             clean ? a.P1 : a.P0, clean ? a.pf1 : a.pf0, a.div_nc, (unsigned)a.nC, items,
                             push_on, gtid, nthr);
            if (!grid_sync(a.ctl, a.expected, a.wait_ns, 0, epoch)) return;
            if (threadIdx.x == 0) {
                S.reached = S.c_prev = (unsigned long long)ns;
                S.pairs = (unsigned long long)ns * (unsigned long long)a.rows;
                S.in_p = push_on ? clean : -1;
                S.dirty_p = -1;
                S.wrote_all_prev = 0;
                S.nf_valid = 0;
                S.done = 0;
                if constexpr (PL) plane_slot().L = 1;
            }
            __syncthreads();
        }
        if (!walk && b == 0 && a.level_ns && gtid == 0) a.level_ns[0] = gtimer();

        int L = 1;
        for (;; ++L) {
            // levels a walk pass already computed; a batch the walk finished
            // ends at its last level
            if (L < S.L_next) continue;
            if (S.done) break;
            // Per-level access modes.  Every block derives them from the same level
            // counts (read after the barrier), so writer and reader always agree:
            //  * push(L): top-down from the push buffer while the frontier feeding
            //    level L is below push_ppm of the pairs (only from the start);
            //  * write_all(L): F' is stored for every chunk, zeros included, when the
            //    frontier feeding level L already covered >= dense_w_ppm of the pairs;
            //  * dense(L): level L reads F without its flag words (one dependent memory
            //    round trip fewer) when F was written whole and covers >= dense_r_ppm;
            //  * skip_full(L): own visited chunk first and no gathers when it is full,
            //    once >= full_skip_ppm of the pairs are reached (late, bottom-up levels);
            //    with not-full words from the previous level, full tiles are passed
            //    over (and F' is then written only where it is nonzero).
            const unsigned long long c_prev = S.c_prev, pairs = S.pairs;
            const int in_p = S.in_p;
            const bool push = in_p >= 0 && c_prev * 1000000ull < pairs * (unsigned long long)a.push_ppm;
            // (visited-set pull levels always read complete rows: dense by the count alone)
            const bool dense = (vp || S.wrote_all_prev) &&
                               c_prev * 1000000ull >= pairs * (unsigned long long)a.dense_r_ppm;
            const bool skip_full = S.reached * 1000000ull >= pairs * (unsigned long long)a.full_skip_ppm;
            const bool nf_use = !push && skip_full && S.nf_valid;
            const bool split = dense && S.reached * 1000000ull >= pairs * (unsigned long long)a.split_ppm;
            const bool write_all =
                !nf_use && c_prev * 1000000ull >= pairs * (unsigned long long)a.dense_w_ppm;
            // dense visited-set pull on a table without one-way entries: no own chunks
            const bool no_own = vp && S.sym && dense && !nf_use;
            const bool odd = (L & 1) != 0;
            unsigned cnt = 0u, and_pre = 0xffffffffu, and_post = 0xffffffffu;
            if (push) {
                uint4 *Pc = in_p ? a.P1 : a.P0;
                uint4 *Pn = in_p ? a.P0 : a.P1;
                uint32_t *pfc = in_p ? a.pf1 : a.pf0;
                uint32_t *pfn = in_p ? a.pf0 : a.pf1;
                if constexpr (D > 0 && 32 % D == 0) cnt = push_level<D, PL>(a.adj, a.V, a.div_nc, (unsigned)a.nC, Pc, Pn, pfc, pfn, ntiles,
                                           gtid, nthr);
            } else if (vp) {
                // Level walk_K + 1 reads S.Pv (the walk's V, or the batch's
                // walk_all_kernel slice) and the walk's flag words and writes S.Qv;
                // later levels alternate between S.Qv and S.Rv, or S.Pv when level
                // walk_K + 2 cannot write S.Rv whole (a skip-full level)
                const bool first = L == a.walk_K + 1;
                bool r_on = false;
                if (L == a.walk_K + 2) {
                    r_on = S.Rv != S.Pv && !nf_use;
                } else {
                    r_on = S.r_on;   // written by level walk_K + 2 before its barrier
                }
                uint4 *R = r_on ? S.Rv : S.Pv;
                const bool even = ((L - a.walk_K) & 1) == 0;
                const uint4 *X = first ? S.Pv : (even ? S.Qv : R);
                uint4 *Y = first ? S.Qv : (even ? R : S.Qv);
                if (threadIdx.x == 0) {
                    s_next = t_lo;
                    if (L == a.walk_K + 2) S.r_on = r_on;
                }
                __syncthreads();
                if (D > 0 && no_own && !nf_use && a.nC == 32)
                    cnt = dense_rows32<(D > 0 ? D : 1)>(X, Y, adj, v_base, t_hi, odd ? a.fl1 : a.fl0,
                                                        odd ? a.nf2 : a.nf, split, &s_next);
                else
                    cnt = vpull_level<D>(a, d, adj, v_base, t_hi, X, Y,
                                         first ? S.fl_walk : (odd ? a.fl0 : a.fl1), odd ? a.fl1 : a.fl0,
                                         odd ? a.nf : a.nf2, odd ? a.nf2 : a.nf, dense,
                                         first || (L == a.walk_K + 2 && r_on), skip_full, split, nf_use, no_own,
                                         &s_next);
            } else {
                const uint4 *Fc = in_p >= 0 ? (in_p ? a.P1 : a.P0) : (odd ? a.F0 : a.F1);
                const uint32_t *fc = in_p >= 0 ? (in_p ? a.pf1 : a.pf0) : (odd ? a.fl0 : a.fl1);
                uint4 *Fn = odd ? a.F1 : a.F0;
                uint32_t *fn = odd ? a.fl1 : a.fl0;
                // Balanced contiguous tile range per block; the block's warps pull
                // tiles from it through a shared-memory counter.
                if (threadIdx.x == 0) s_next = t_lo;
                __syncthreads();
                if (nf_use) {
                    // Skip-full stage: a warp takes 32 tiles, reads their not-full
                    // words in one load, clears the frontier flags of the full ones
                    // and works only on the others.
                    for (;;) {
                        unsigned tile0 = 0;
                        if (lane == 0) tile0 = atomicAdd(&s_next, 32u);
                        tile0 = __shfl_sync(0xffffffffu, tile0, 0);
                        if (tile0 >= t_hi) break;
                        const unsigned my = tile0 + lane;
                        const unsigned w = my < t_hi ? __ldcg(a.nf + my) : 0u;
                        if (my < t_hi && w == 0u) fn[my] = 0u;
                        for (unsigned todo = __ballot_sync(0xffffffffu, w != 0u); todo; todo &= todo - 1u) {
                            const unsigned tj = tile0 + (unsigned)(__ffs((int)todo) - 1);
                            level_tiles<D, 1, PL>(a, d, adj, v_base, tj, t_hi, Fc, Fn, fc, fn, dense, write_all,
                                              skip_full, split, lane, cnt, and_pre, and_post);
                        }
                    }
                } else {
                    for (;;) {
                        unsigned tile0 = 0;
                        if (lane == 0) tile0 = atomicAdd(&s_next, (unsigned)kGrab);
                        tile0 = __shfl_sync(0xffffffffu, tile0, 0);
                        if (tile0 >= t_hi) break;
                        level_tiles<D, kGrab, PL>(a, d, adj, v_base, tile0, t_hi, Fc, Fn, fc, fn, dense,
                                              write_all, skip_full, split, lane, cnt, and_pre,
                                              and_post);
                    }
                }
            }

            // Level reduction: one 64-bit atomic per block (cudaASPLconv.cu:59-99 fused).
            unsigned long long *counts = a.counts + (size_t)b * (size_t)a.stride;
            unsigned *masks = a.masks ? a.masks + (size_t)b * (size_t)a.stride : nullptr;
            const unsigned wsum = __reduce_add_sync(0xffffffffu, cnt);
            if (lane == 0) s_sum[threadIdx.x >> 5] = wsum;
            if (masks) {
                const unsigned w0 = __reduce_and_sync(0xffffffffu, and_pre);
                const unsigned w1 = __reduce_and_sync(0xffffffffu, and_post);
                if (lane == 0) { s_and[0][threadIdx.x >> 5] = w0; s_and[1][threadIdx.x >> 5] = w1; }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned long long bsum = 0;
                for (int w = 0; w < kBlock / 32; ++w) bsum += s_sum[w];
                if (bsum) atomicAdd(no_own ? S.vt + L % 3 : counts + L, bsum);
                if (vp && S.vt && blockIdx.x == 0) S.vt[(L + 1) % 3] = 0ull;   // read last after level L - 2
                if (masks) {
                    unsigned m0 = 0xffffffffu, m1 = 0xffffffffu;
                    for (int w = 0; w < kBlock / 32; ++w) { m0 &= s_and[0][w]; m1 &= s_and[1][w]; }
                    if (L == 1) atomicAnd(masks, m0);
                    atomicAnd(masks + L, m1);
                }
            }
            // the level's sum comes with the barrier (read by its last arrival)
            unsigned long long lsum = 0;
            if (!grid_sync_value(a.ctl, a.expected, a.wait_ns, L, epoch, no_own ? S.vt + L % 3 : counts + L,
                                 lsum))
                return;
            if (b == 0 && a.level_ns && gtid == 0) a.level_ns[L] = gtimer();
            if (threadIdx.x == 0) {
                unsigned long long cL = lsum;
                if (no_own) {
                    // total bits of V_L less the padding and the pairs reached before
                    const unsigned long long pad = (unsigned long long)a.rows * (unsigned long long)(128 * a.nC - ns);
                    cL = lsum - pad - S.reached;
                    if (blockIdx.x == 0) counts[L] = cL;
                }
                S.reached += cL;
                S.c_prev = cL;
                S.wrote_all_prev = !push && write_all;
                S.nf_valid = a.nf != nullptr && !push && (vp || skip_full || dense || masks != nullptr);
                if (push) {
                    S.in_p = in_p ^ 1;    // the frontier is now in Pn; Pc was cleared by its readers
                } else if (in_p >= 0) {
                    S.dirty_p = in_p;     // read by this pull level; cleared before it is written again
                    S.in_p = -1;
                }
                // Stop on an empty level, at the cap, or as soon as every pair is
                // reached (the next level is then empty by construction).
                S.done = cL == 0ull || L >= a.max_levels || S.reached == S.pairs;
                if constexpr (PL) plane_slot().L = L + 1;
            }
            __syncthreads();
            if (S.done) break;
        }
        if (threadIdx.x == 0) {
            if (blockIdx.x == 0) a.levels_run[b] = L;
            if (S.in_p >= 0) S.dirty_p = S.in_p;
        }
        __syncthreads();
        if (a.batch_ns && gtid == 0) a.batch_ns[2 * b + 1] = gtimer();
    }
    // Nothing reads the push buffers any more: return the one still holding
    // bits to all zero.
    const int dirty = S.dirty_p;
    if (dirty >= 0) clear_push_buffer(dirty ? a.P1 : a.P0, dirty ? a.pf1 : a.pf0, ntiles, gtid, nthr);
}

// Expansion of the calculator tables into the pull adjacency adj[rows][d].
struct ExpandArgs {
    const int32_t *table;
    int32_t *adj;
    int form;                 // 1 part/beamer, 2 piece, 3 box
    int rows, d;
    int N, M;                 // part
    int Nx, Ny, Nz, Mx, My, Mz;
};

__device__ __forceinline__ int pmod64(long long a, int n) {
    long long r = a % n;
    return (int)(r < 0 ? r + n : r);
}

static __global__ void expand_kernel(const ExpandArgs e) {
    const long long total = (long long)e.rows * e.d;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(k / e.d), i = (int)(k % e.d);
        int to;
        if (e.form == 1) {
            // cudaASPLconv.cu:41-44: (N + v + diff) % N
            to = pmod64((long long)v + e.table[(size_t)(v % e.M) * e.d + i], e.N);
        } else if (e.form == 2) {
            // cudaASPLpiece.cu:41-50
            const int x = v / e.Ny, y = v % e.Ny;
            const size_t o = ((size_t)((x % e.Mx) * e.My + (y % e.My)) * e.d + i) * 2;
            const int tx = pmod64((long long)x + e.table[o], e.Nx);
            const int ty = pmod64((long long)y + e.table[o + 1], e.Ny);
            to = tx * e.Ny + ty;
        } else {
            // cudaASPLbox.cu:44-57
            const int x = v / (e.Ny * e.Nz), r = v % (e.Ny * e.Nz), y = r / e.Nz, z = r % e.Nz;
            const size_t o =
                ((size_t)(((x % e.Mx) * e.My + (y % e.My)) * e.Mz + (z % e.Mz)) * e.d + i) * 3;
            const int tx = pmod64((long long)x + e.table[o], e.Nx);
            const int ty = pmod64((long long)y + e.table[o + 1], e.Ny);
            const int tz = pmod64((long long)z + e.table[o + 2], e.Nz);
            to = (tx * e.Ny + ty) * e.Nz + tz;
        }
        e.adj[k] = to;
    }
}

// Range check of a plain-graph table (every entry a vertex id), so that a bad
// table becomes GG_BAD_ARG instead of an out-of-bounds gather.
static __global__ void check_table_kernel(const int32_t *t, long long n, int rows, int *bad) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        if ((unsigned)t[k] >= (unsigned)rows) atomicExch(bad, 1);
}

}  // namespace gg
