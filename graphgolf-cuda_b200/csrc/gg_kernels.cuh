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
struct Ctl {
    unsigned int bar_count;   // arrivals at the current barrier
    unsigned int bar_gen;     // barrier generation
    int err;                  // 0, or 1 = a barrier wait exceeded the limit
    int err_level;            // level at which the first wait gave up
    int levels_run;           // last level executed
    int pad[3];
};

struct BfsArgs {
    const int32_t *adj;       // [rows][d] pull adjacency
    const int32_t *src;       // batch sources: vertex id of source i, i < ns
    uint4 *V, *F0, *F1;
    uint32_t *fl0, *fl1;
    unsigned long long *counts;   // [max_levels + 1]
    unsigned int *masks;          // [max_levels + 1] or nullptr
    Ctl *ctl;
    const int *bad;           // nonzero: the table failed its range check; do nothing
    unsigned int expected;    // blocks the barrier waits for (the grid size)
    FastDiv div_nc;           // division by nC
    uint32_t items;           // rows * nC
    int rows, d, nC, ns;
    int max_levels;
    int bu_permille;          // switch to own-first order once reached > permille/1000 of pairs
    long long wait_ns;        // barrier wait limit
};

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

// Grid-wide barrier with a bounded wait.  Requires co-resident blocks
// (cooperative launch).  Returns false on every block once any block's wait
// ran past the limit; the kernel then returns and the host reports GG_TIMEOUT.
__device__ __forceinline__ bool grid_barrier(Ctl *ctl, unsigned expected, long long wait_ns,
                                             int level) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned gen = ld_acquire(&ctl->bar_gen);
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->bar_count, 1u);
        if (prev + 1 == expected) {
            atomicExch(&ctl->bar_count, 0u);
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            const unsigned long long t0 = gtimer();
            while (ld_acquire(&ctl->bar_gen) == gen) {
                if (ld_acquire_i(&ctl->err)) { ok = 0; break; }
                __nanosleep(64);
                if ((long long)(gtimer() - t0) > wait_ns) {
                    if (atomicCAS(&ctl->err, 0, 1) == 0) ctl->err_level = level;
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (ok && ld_acquire_i(&ctl->err)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
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

// One cooperative launch = one source batch, all levels.
template <int D>
__global__ void __launch_bounds__(kBlock) bfs_batch_kernel(const BfsArgs a) {
    const int d = D > 0 ? D : a.d;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned nthr = gridDim.x * blockDim.x;
    const unsigned wid = gtid >> 5, nwarps = nthr >> 5;
    const unsigned items = a.items, ntiles = (items + 31u) >> 5;
    __shared__ unsigned long long s_sum[kBlock / 32];
    __shared__ unsigned s_and[2][kBlock / 32];
    if (a.bad && *a.bad) return;  // uniform across the grid: no block reaches a barrier

    // Phase 0: per-batch reset (cudaASPLconv.cu:9-33): padding bits visited,
    // frontier and flags cleared, counters zeroed.
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i <= a.max_levels; i += blockDim.x) {
            a.counts[i] = 0ull;
            if (a.masks) a.masks[i] = 0xffffffffu;
        }
    for (unsigned t = gtid; t < items; t += nthr) {
        const unsigned c = t - a.div_nc.div(t) * (unsigned)a.nC;
        a.V[t] = pad_mask((int)c, a.ns);
        a.F0[t] = u4zero();
    }
    for (unsigned w = gtid; w < ntiles; w += nthr) a.fl0[w] = 0u;
    if (!grid_barrier(a.ctl, a.expected, a.wait_ns, 0)) return;

    // Phase 1: the diagonal -- source i has reached its own vertex at level 0.
    for (unsigned i = gtid; i < (unsigned)a.ns; i += nthr) {
        const unsigned t = (unsigned)a.src[i] * (unsigned)a.nC + (i >> 7);
        const unsigned bit = 1u << (i & 31u), comp = (i >> 5) & 3u;
        atomicOr(reinterpret_cast<unsigned *>(a.V + t) + comp, bit);
        atomicOr(reinterpret_cast<unsigned *>(a.F0 + t) + comp, bit);
        atomicOr(a.fl0 + (t >> 5), 1u << (t & 31u));
    }
    if (gtid == 0) a.counts[0] = (unsigned long long)a.ns;
    if (!grid_barrier(a.ctl, a.expected, a.wait_ns, 0)) return;

    const unsigned long long pairs = (unsigned long long)a.ns * (unsigned long long)a.rows;
    const unsigned long long bu_at =
        a.bu_permille >= 1000 ? ~0ull : pairs / 1000ull * (unsigned long long)a.bu_permille;
    unsigned long long reached = (unsigned long long)a.ns;

    for (int L = 1;; ++L) {
        const bool odd = (L & 1) != 0;
        const uint4 *Fc = odd ? a.F0 : a.F1;
        uint4 *Fn = odd ? a.F1 : a.F0;
        const uint32_t *fc = odd ? a.fl0 : a.fl1;
        uint32_t *fn = odd ? a.fl1 : a.fl0;
        // Own-first ("bottom-up") order once most pairs are reached: a chunk
        // whose visited bits are all set skips its gathers entirely.
        const bool own_first = reached > bu_at || a.masks != nullptr;
        unsigned cnt = 0u, and_pre = 0xffffffffu, and_post = 0xffffffffu;

        for (unsigned tile = wid; tile < ntiles; tile += nwarps) {
            const unsigned t = tile * 32u + lane;
            uint4 nw = u4zero();
            if (t < items) {
                const unsigned v = a.div_nc.div(t);
                const unsigned c = t - v * (unsigned)a.nC;
                const int32_t *arow = a.adj + (size_t)v * (size_t)d;
                uint4 own = u4zero();
                bool have = false;
                if (own_first) { own = __ldcg(a.V + t); have = true; }
                if (!(have && u4full(own))) {
                    uint4 acc = u4zero();
#pragma unroll 8
                    for (int i = 0; i < d; ++i) {
                        const unsigned tu = (unsigned)__ldg(arow + i) * (unsigned)a.nC + c;
                        if ((__ldcg(fc + (tu >> 5)) >> (tu & 31u)) & 1u) or_into(acc, __ldcg(Fc + tu));
                    }
                    if (u4any(acc)) {
                        if (!have) { own = __ldcg(a.V + t); have = true; }
                        nw = andnot(acc, own);
                        if (u4any(nw)) {
                            a.V[t] = u4or(own, nw);
                            Fn[t] = nw;
                        }
                    }
                }
                if (a.masks) {
                    and_pre &= u4and(own);
                    and_post &= u4and(u4or(own, nw));
                }
                cnt += u4popc(nw);
            }
            const unsigned b = __ballot_sync(0xffffffffu, u4any(nw));
            if (lane == 0) fn[tile] = b;
        }

        // Level reduction: one 64-bit atomic per block (cudaASPLconv.cu:59-99 fused).
        const unsigned wsum = __reduce_add_sync(0xffffffffu, cnt);
        if (lane == 0) s_sum[threadIdx.x >> 5] = wsum;
        if (a.masks) {
            const unsigned w0 = __reduce_and_sync(0xffffffffu, and_pre);
            const unsigned w1 = __reduce_and_sync(0xffffffffu, and_post);
            if (lane == 0) { s_and[0][threadIdx.x >> 5] = w0; s_and[1][threadIdx.x >> 5] = w1; }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long bsum = 0;
            for (int w = 0; w < kBlock / 32; ++w) bsum += s_sum[w];
            if (bsum) atomicAdd(a.counts + L, bsum);
            if (a.masks) {
                unsigned m0 = 0xffffffffu, m1 = 0xffffffffu;
                for (int w = 0; w < kBlock / 32; ++w) { m0 &= s_and[0][w]; m1 &= s_and[1][w]; }
                if (L == 1) atomicAnd(a.masks, m0);
                atomicAnd(a.masks + L, m1);
            }
        }
        if (!grid_barrier(a.ctl, a.expected, a.wait_ns, L)) return;
        const unsigned long long cL = ld_relaxed_u64(a.counts + L);
        reached += cL;
        if (cL == 0ull || L >= a.max_levels) {
            if (gtid == 0) a.ctl->levels_run = L;
            break;
        }
    }
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
