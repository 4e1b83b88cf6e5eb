// gg_batch.cu -- batched exact evaluation of 2-opt candidates (gg_batch_* in gg.h).
//
// One persistent launch scores every candidate of a batch.  Work unit ("task") =
// one candidate x one chunk of its sources.  A CTA takes a task, builds the
// candidate's adjacency in shared memory (the base rows as uint16, then the four
// rows the 2-opt edit touches), and runs the whole BFS of the chunk's sources
// with both visited bitsets resident in shared memory:
//     next[v][c] = cur[v][c] | (OR_{u in adj[v]} cur[u][c])        (all rows, one level)
// i.e. the level step of cudaASPLconv.cu:35-56 with the reduction of :59-99
// folded into per-thread popcounts and one __syncthreads_or per level.  The grid
// barrier of the single-graph path is not needed: a task never leaves its CTA.
//
// Affected sources (default): per base, one pass of the same kernel also writes
// the base's distance matrix as 4 bit-planes, from which every source's distance
// sum and eccentricity follow.  A candidate then searches only from the sources
// its 2-opt can affect (the test of gg_inc.cu: a removed edge between
// consecutive BFS levels whose deeper end has no other parent, or an added edge
// between vertices whose distances differ by 2 or more); its result is the base's
// total minus those sources' old sums plus their new sums, and the larger of their
// new eccentricities and the others' old ones.  Bases that are not symmetric,
// not connected or of diameter above 15 (and the histogram pass) search every
// source.  GG_BATCH_FULL=1 searches every source for every candidate.
//
// Task order: t -> chunk = maxchunks-1 - t / n_cand, cand = t % n_cand, so the
// extra chunks of the largest bases come first and the common chunks fill the
// tail (largest-first scheduling with no task list on the host).  Both n_cand and
// maxchunks are read from device memory, so one captured CUDA graph serves every
// batch size up to the capacity it was captured for.
#include "gg.h"
#include "gg_internal.h"
#include "gg_planes.cuh"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>


namespace {

constexpr int kBatchBlock = 1024;
constexpr size_t kSmemBudget = 220 * 1024;

constexpr int kPlanes = 4;   // distance bit-planes: distances up to 15

struct BatchBase {
    const int32_t *adj;   // [n][d] in global memory
    const uint16_t *adj16;   // the same rows as uint16, padded to adj16_bytes (a multiple of 16)
    unsigned adj16_bytes;
    int n, d;
    int log_nc;           // chunks (of 128 sources) per task row = 1 << log_nc
    int chunks;           // tasks per candidate = ceil(n / (128 << log_nc))
    // affected-source mode (valid != 0)
    const uint4 *planes;  // [kPlanes][n][cols]: bit k of dist(source, vertex)
    unsigned cols;        // chunks << log_nc
    const unsigned *rowsum;  // [n]: distance sum of each source
    const unsigned *ecc;     // [n]: eccentricity of each source
    unsigned long long total, reached;  // the base's own counts
    int levels;
    int valid;            // symmetric, connected, diameter <= 15
};

// Per candidate, from the affected-source test.
struct IncCand {
    unsigned long long old_sum;   // base distance sums of the affected sources
    unsigned count;               // affected sources (the candidate's search list)
    unsigned max_other;           // largest eccentricity among the other sources
    int full;                     // search every source instead
    int pad;
};

struct BatchCtl {
    unsigned task_ctr;
    int n_cand;
    int max_chunks;
    int bad;              // set by batch_reset when a candidate is outside the domain
    int n_bases;          // registered bases
    int bad_index;        // lowest index of such a candidate (INT_MAX: none)
    int timeout;          // a CTA's wait for its adjacency copy ran past its limit
    int pad;
};

struct BatchArgs {
    const BatchBase *bases;
    const gg_swap *cands;
    gg_cand_result *out;
    BatchCtl *ctl;
    unsigned *hist;       // nullptr, or [n][hist_k]: per-vertex new pairs at levels 1..hist_k
    int hist_k;           // (only meaningful for a launch of one candidate)
    IncCand *inc;         // nullptr: every candidate searches every source
    uint16_t *lists;      // [cand][list_stride]: affected sources
    int list_stride;
};

__device__ __forceinline__ uint4 z4() { return make_uint4(0u, 0u, 0u, 0u); }
__device__ __forceinline__ unsigned padw(int lo, int ns) {
    if (ns <= lo) return 0xffffffffu;
    if (ns >= lo + 32) return 0u;
    return ~((1u << (ns - lo)) - 1u);
}

// Bulk copy (the TMA unit's untiled cp.async.bulk, no multicast, this GPU's
// memory) of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global
// memory into this CTA's shared memory, completing on the mbarrier `bar`.
__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void bulk_to_smem(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(smem_addr(bar)), "r"(phase) : "memory");
    return ok != 0;
}

constexpr long long kCopyWaitNs = 2000000000ll;   // 2 s: a copy of at most 128 KB never takes that

__global__ void __launch_bounds__(kBatchBlock, 1) batch_kernel(const BatchArgs a) {
    extern __shared__ uint4 sm[];
    __shared__ unsigned s_task;
    __shared__ unsigned long long s_tot[kBatchBlock / 32], s_reach[kBatchBlock / 32];
    __shared__ __align__(8) uint64_t s_bar;   // completion of the adjacency copy
    __shared__ int s_late;
    if (a.ctl->bad) return;   // batch_reset rejected a candidate: index nothing
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n_cand = a.ctl->n_cand, max_chunks = a.ctl->max_chunks;
    const unsigned n_tasks = (unsigned)n_cand * (unsigned)max_chunks;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&s_bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned phase = 0;

    for (;;) {
        if (tid == 0) s_task = atomicAdd(&a.ctl->task_ctr, 1u);
        __syncthreads();
        const unsigned task = s_task;
        if (task >= n_tasks) return;
        const int cand = (int)(task % (unsigned)n_cand);
        const int chunk = max_chunks - 1 - (int)(task / (unsigned)n_cand);
        const gg_swap sw = a.cands[cand];
        const BatchBase B = a.bases[sw.base];
        const int n = B.n, d = B.d, lnc = B.log_nc, nC = 1 << lnc;
        const int S = 128 << lnc;
        // sources of this candidate: every vertex, or its affected-source list
        const bool full = a.inc == nullptr || a.inc[cand].full;
        const int count = full ? n : (int)a.inc[cand].count;
        if (chunk * S >= count) {  // this candidate has fewer chunks
            __syncthreads();
            continue;
        }
        const int s0 = chunk * S;
        const int ns = min(S, count - s0);
        const int items = n << lnc;

        // shared memory: adjacency (uint16, padded to 16 bytes), then two bitsets.
        // The base's packed rows arrive by one bulk copy; every thread waits on the
        // mbarrier (bounded: past kCopyWaitNs the CTA flags a timeout and stops).
        uint16_t *adj = reinterpret_cast<uint16_t *>(sm);
        uint4 *cur = sm + (((size_t)n * d * 2 + 15) / 16);
        uint4 *nxt = cur + items;
        if (tid == 0) {
            // the previous task's generic-proxy accesses to this memory come first
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bulk_to_smem(adj, B.adj16, B.adj16_bytes, &s_bar);
            s_late = 0;
        }
        {
            bool done = mbar_try_wait(&s_bar, phase);
            if (!done) {
                unsigned long long t0;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
                for (unsigned it = 1; !done; ++it) {
                    done = mbar_try_wait(&s_bar, phase);
                    if (!done && (it & 63u) == 0u) {
                        unsigned long long t;
                        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                        if ((long long)(t - t0) > kCopyWaitNs) break;
                    }
                }
            }
            if (!done) s_late = 1;
        }
        phase ^= 1u;
        __syncthreads();
        if (s_late) {
            // the copy did not complete: report it and leave (the host sees
            // GG_TIMEOUT); only this CTA's tail of tasks is left unscored
            if (tid == 0) atomicExch(&a.ctl->timeout, 1);
            return;
        }
        if (sw.a >= 0 && tid < 4) {
            // 2-opt: (a,b),(c,d) -> (a,c),(b,d) [mode 0] or (a,d),(b,c) [mode 1]
            const int x[4] = {sw.a, sw.b, sw.c, sw.d};
            const int from[4] = {sw.b, sw.a, sw.d, sw.c};
            const int to0[4] = {sw.c, sw.d, sw.a, sw.b};
            const int to1[4] = {sw.d, sw.c, sw.b, sw.a};
            const int row = x[tid], f = from[tid], t = sw.mode ? to1[tid] : to0[tid];
            for (int j = 0; j < d; ++j)
                if (adj[row * d + j] == (uint16_t)f) { adj[row * d + j] = (uint16_t)t; break; }
        }
        // visited after level 0: the diagonal plus the padding sources
        for (int t = tid; t < items; t += kBatchBlock) {
            const int v = t >> lnc, c = t & (nC - 1);
            const int b = c * 128;
            uint4 w = make_uint4(padw(b, ns), padw(b + 32, ns), padw(b + 64, ns), padw(b + 96, ns));
            const int i = v - s0;
            if (full && i >= b && i < b + 128 && i < ns) {
                const unsigned bit = 1u << (i & 31);
                switch ((i - b) >> 5) {
                    case 0: w.x |= bit; break;
                    case 1: w.y |= bit; break;
                    case 2: w.z |= bit; break;
                    default: w.w |= bit; break;
                }
            }
            cur[t] = w;
        }
        __syncthreads();
        if (!full) {
            // source j of the chunk is vertex lists[s0 + j]
            const uint16_t *lst = a.lists + (size_t)cand * a.list_stride + s0;
            for (int j = tid; j < ns; j += kBatchBlock) {
                const int v = lst[j];
                atomicOr(reinterpret_cast<unsigned *>(cur + ((v << lnc) + (j >> 7))) + ((j >> 5) & 3),
                         1u << (j & 31));
            }
            __syncthreads();
        }

        unsigned long long tot = 0, reach = 0;
        int L = 1;
        for (;; ++L) {
            unsigned cnt = 0;
            for (int t = tid; t < items; t += kBatchBlock) {
                const int v = t >> lnc, c = t & (nC - 1);
                const uint4 own = cur[t];
                uint4 out = own;
                if ((own.x & own.y & own.z & own.w) != 0xffffffffu) {
                    uint4 acc = z4();
                    const uint16_t *ar = adj + v * d;
                    for (int i = 0; i < d; ++i) {
                        const uint4 x = cur[((int)ar[i] << lnc) + c];
                        acc.x |= x.x; acc.y |= x.y; acc.z |= x.z; acc.w |= x.w;
                    }
                    out = make_uint4(own.x | acc.x, own.y | acc.y, own.z | acc.z, own.w | acc.w);
                    const unsigned pc = __popc(acc.x & ~own.x) + __popc(acc.y & ~own.y) +
                                        __popc(acc.z & ~own.z) + __popc(acc.w & ~own.w);
                    cnt += pc;
                    if (a.hist && L <= a.hist_k && pc) atomicAdd(a.hist + (size_t)v * a.hist_k + (L - 1), pc);
                }
                nxt[t] = out;
            }
            tot += (unsigned long long)L * cnt;
            reach += cnt;
            if (!__syncthreads_or(cnt != 0)) break;
            uint4 *sw2 = cur; cur = nxt; nxt = sw2;
        }
        // L is the first level without new pairs
        unsigned long long wt = tot, wr = reach;
        for (int o = 16; o; o >>= 1) {
            wt += __shfl_down_sync(0xffffffffu, wt, o);
            wr += __shfl_down_sync(0xffffffffu, wr, o);
        }
        if (lane == 0) { s_tot[warp] = wt; s_reach[warp] = wr; }
        __syncthreads();
        if (tid == 0) {
            unsigned long long bt = 0, br = (unsigned long long)ns;
            for (int w = 0; w < kBatchBlock / 32; ++w) { bt += s_tot[w]; br += s_reach[w]; }
            atomicAdd(reinterpret_cast<unsigned long long *>(&a.out[cand].total), bt);
            atomicAdd(reinterpret_cast<unsigned long long *>(&a.out[cand].reached), br);
            atomicMax(&a.out[cand].levels, L - 1);
        }
        __syncthreads();  // the next task overwrites shared memory
    }
}

__global__ void batch_finalize(const BatchArgs a) {
    const int n_cand = a.ctl->n_cand;
    if (a.ctl->bad || a.ctl->timeout) {
        // a rejected or timed-out launch scores nothing: every result says so
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cand; i += gridDim.x * blockDim.x)
            a.out[i] = gg_cand_result{0ull, 0ull, -1, 0};
        return;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cand; i += gridDim.x * blockDim.x) {
        const BatchBase B = a.bases[a.cands[i].base];
        gg_cand_result r = a.out[i];
        if (a.inc && !a.inc[i].full) {
            // the other sources keep the base's distances
            const IncCand &ic = a.inc[i];
            r.total = B.total - ic.old_sum + r.total;
            r.reached = B.reached - (unsigned long long)ic.count * B.n + r.reached;
            r.levels = max(r.levels, (int)ic.max_other);
        }
        r.connected = r.reached == (unsigned long long)B.n * (unsigned long long)B.n;
        a.out[i] = r;
    }
}

// Zeroes the results and range-checks every candidate (the device-array entry
// point gets candidates the host never saw): base registered, endpoints inside the
// base, distinct, mode 0 or 1.  One bad candidate sets ctl->bad, and the kernels
// after this one return before reading a base or a row through it.
__global__ void batch_reset(const BatchArgs a) {
    const int n_cand = a.ctl->n_cand;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cand; i += gridDim.x * blockDim.x) {
        a.out[i] = gg_cand_result{0ull, 0ull, 0, 0};
        if (a.inc) a.inc[i] = IncCand{0ull, 0u, 0u, 0, 0};
        const gg_swap sw = a.cands[i];
        bool ok = sw.base >= 0 && sw.base < a.ctl->n_bases;
        if (ok && sw.a >= 0) {
            const unsigned n = (unsigned)a.bases[sw.base].n;
            ok = (unsigned)sw.a < n && (unsigned)sw.b < n && (unsigned)sw.c < n && (unsigned)sw.d < n &&
                 (sw.mode == 0 || sw.mode == 1) && sw.a != sw.b && sw.a != sw.c && sw.a != sw.d &&
                 sw.b != sw.c && sw.b != sw.d && sw.c != sw.d;
        }
        if (!ok) {
            atomicExch(&a.ctl->bad, 1);
            atomicMin(&a.ctl->bad_index, i);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl->task_ctr = 0u;
}

__device__ __forceinline__ unsigned plane_dist(const uint32_t *pw, size_t pstride_w, unsigned cols4,
                                               unsigned x, unsigned s) {
    const size_t base = (size_t)x * cols4 + (s >> 5);
    unsigned dv = 0;
#pragma unroll
    for (int k = 0; k < kPlanes; ++k) dv |= ((__ldg(pw + (size_t)k * pstride_w + base) >> (s & 31u)) & 1u) << k;
    return dv;
}

// One thread per (candidate, source): the affected-source test (see the file
// comment).  Affected sources join the candidate's list with their base
// distance sums; the others give the largest eccentricity that stays.
__global__ void batch_affected(const BatchArgs a, int max_n, int force_full) {
    if (a.ctl->bad) return;   // batch_reset rejected a candidate
    const int n_cand = a.ctl->n_cand;
    const unsigned long long total = (unsigned long long)n_cand * (unsigned long long)max_n;
    const unsigned lane = threadIdx.x & 31u;
    for (unsigned long long g0 = (unsigned long long)blockIdx.x * blockDim.x; g0 < total;
         g0 += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long g = g0 + threadIdx.x;
        const bool in = g < total;
        const int cand = in ? (int)(g / (unsigned)max_n) : 0;
        const int s = in ? (int)(g % (unsigned)max_n) : 0;
        const gg_swap sw = a.cands[cand];
        const BatchBase &B = a.bases[sw.base];
        const bool live = in && s < B.n;
        bool aff = false, other = false;
        if (live && (force_full || !B.valid)) {
            if (s == 0) a.inc[cand].full = 1;
        } else if (live) {
            other = true;
            if (sw.a >= 0) {
                const uint32_t *pw = reinterpret_cast<const uint32_t *>(B.planes);
                const size_t psw = (size_t)B.n * B.cols * 4;
                const unsigned c4 = B.cols * 4;
                const int ends[2][2] = {{sw.a, sw.b}, {sw.c, sw.d}};
                for (int e = 0; e < 2 && !aff; ++e) {
                    const int x = ends[e][0], y = ends[e][1];
                    const unsigned dx = plane_dist(pw, psw, c4, x, s), dy = plane_dist(pw, psw, c4, y, s);
                    if (dx == dy) continue;
                    const int lo = dx < dy ? x : y, hi = dx < dy ? y : x;
                    const unsigned l = min(dx, dy);
                    bool par = false, skipped = false;
                    for (int i = 0; i < B.d && !par; ++i) {
                        const int z = __ldg(B.adj + (size_t)hi * B.d + i);
                        if (z == lo && !skipped) { skipped = true; continue; }
                        par = plane_dist(pw, psw, c4, (unsigned)z, s) == l;
                    }
                    aff = !par;
                }
                if (!aff) {
                    const int p = sw.mode ? sw.d : sw.c, q = sw.mode ? sw.c : sw.d;
                    const unsigned da = plane_dist(pw, psw, c4, sw.a, s), dp = plane_dist(pw, psw, c4, p, s);
                    const unsigned db = plane_dist(pw, psw, c4, sw.b, s), dq = plane_dist(pw, psw, c4, q, s);
                    aff = (da > dp ? da - dp : dp - da) >= 2u || (db > dq ? db - dq : dq - db) >= 2u;
                }
            }
            other = !aff;
        }
        // one set of atomics per candidate present in the warp
        const unsigned peers = __match_any_sync(0xffffffffu, live ? cand : -1);
        const unsigned am = __ballot_sync(0xffffffffu, aff) & peers;
        const int leader = __ffs((int)peers) - 1;
        const unsigned rs = __reduce_add_sync(peers, aff ? __ldg(B.rowsum + s) : 0u);
        const unsigned mx = __reduce_max_sync(peers, other ? __ldg(B.ecc + s) : 0u);
        unsigned first = 0;
        if ((int)lane == leader && live) {
            if (am) {
                first = atomicAdd(&a.inc[cand].count, (unsigned)__popc(am));
                atomicAdd(&a.inc[cand].old_sum, (unsigned long long)rs);
            }
            atomicMax(&a.inc[cand].max_other, mx);
        }
        first = __shfl_sync(0xffffffffu, first, leader);
        if (aff) a.lists[(size_t)cand * a.list_stride + first + __popc(am & ((1u << lane) - 1u))] = (uint16_t)s;
    }
}

gg_status bfail(gg_status s, const std::string &m) {
    (void)cudaGetLastError();
    gg::set_last_error(m.c_str());
    return s;
}

#define GB_CK(call)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return bfail(e_ == cudaErrorMemoryAllocation ? GG_OUT_OF_MEMORY : GG_CUDA_ERROR, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                \
    } while (0)

}  // namespace

struct gg_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<BatchBase> bases;          // host copy (adj = device pointers)
    std::vector<int32_t *> base_adj;       // device adjacency per base
    std::vector<uint16_t *> base_adj16;    // the same, packed as uint16 for the bulk copy
    BatchBase *d_bases = nullptr;
    BatchCtl *d_ctl = nullptr, *h_ctl = nullptr;
    int cap = 0;                           // candidates the buffers hold
    gg_swap *d_cands = nullptr, *h_cands = nullptr;
    gg_cand_result *d_out = nullptr, *h_out = nullptr;
    size_t smem = 0;
    int grid = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const gg_swap *graph_cands = nullptr;  // pointers baked into the graph
    gg_cand_result *graph_out = nullptr;
    cudaStream_t graph_stream = nullptr;
    unsigned *d_hist = nullptr;            // vertex histogram output
    size_t hist_cap = 0;
    double last_ms = 0.0;
    // affected-source mode
    bool full_only = false;                // GG_BATCH_FULL=1: every candidate searches every source
    std::vector<uint4 *> base_planes;      // per base: [kPlanes][n][cols]
    std::vector<unsigned *> base_stats;    // per base: rowsum[n] then ecc[n]
    std::vector<std::pair<std::pair<int, int>, gg_engine *>> engines;  // per (n, degree): base passes
    int *d_flag = nullptr, *h_flag = nullptr;
    IncCand *d_inc = nullptr;              // [cap]
    uint16_t *d_lists = nullptr;           // [cap][list_stride]
    int list_stride = 0;                   // largest base n
};

namespace {

void drop_graph(gg_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

bool log_nc_fits(int n, int d, int l) {
    const size_t adj = ((size_t)n * d * 2 + 15) / 16 * 16;
    return adj + 2 * (size_t)n * (16u << l) <= kSmemBudget;
}

std::string batch_tune_key(int device, int n, int d) { return gg::tune_key(device, "batch", {n, d}); }

// Chunk count per task row (a power of two): the one gg_batch_autotune recorded for
// this base shape on this kind of GPU, else the widest whose bitsets and adjacency
// fit the shared-memory budget.
int auto_log_nc(int device, int n, int d) {
    std::vector<int> tuned;
    if (gg::tune_get(batch_tune_key(device, n, d), &tuned) && !tuned.empty() && tuned[0] >= 0 &&
        tuned[0] <= 4 && log_nc_fits(n, d, tuned[0]))
        return tuned[0];
    int best = -1;
    for (int l = 0; l <= 4; ++l) {
        if (log_nc_fits(n, d, l)) best = l;
        if ((128 << l) >= n) break;
    }
    return best;
}

gg_status refresh_plan(gg_batch *b) {
    size_t smem = 0;
    int max_chunks = 1;
    for (auto &B : b->bases) {
        const size_t need = ((size_t)B.n * B.d * 2 + 15) / 16 * 16 + 2 * (size_t)B.n * (16u << B.log_nc);
        smem = std::max(smem, need);
        max_chunks = std::max(max_chunks, B.chunks);
    }
    b->smem = smem;
    GB_CK(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, sms = 0;
    GB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, kBatchBlock, smem));
    GB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    if (per_sm < 1) return bfail(GG_BAD_ARG, "batch task does not fit in shared memory");
    b->grid = per_sm * sms;
    b->h_ctl->max_chunks = max_chunks;
    GB_CK(cudaMemcpy(b->d_bases, b->bases.data(), b->bases.size() * sizeof(BatchBase),
                     cudaMemcpyHostToDevice));
    drop_graph(b);
    return GG_OK;
}

gg_status ensure_cap(gg_batch *b, int n) {
    int max_n = 0;
    for (auto &B : b->bases) max_n = std::max(max_n, B.n);
    if (n <= b->cap && max_n <= b->list_stride) return GG_OK;
    const int cap = std::max({n, 2 * b->cap, 1});
    cudaFree(b->d_cands); cudaFree(b->d_out); cudaFree(b->d_inc); cudaFree(b->d_lists);
    cudaFreeHost(b->h_cands); cudaFreeHost(b->h_out);
    b->d_cands = nullptr; b->d_out = nullptr; b->h_cands = nullptr; b->h_out = nullptr;
    b->d_inc = nullptr; b->d_lists = nullptr;
    b->cap = 0;
    GB_CK(cudaMalloc(&b->d_cands, (size_t)cap * sizeof(gg_swap)));
    GB_CK(cudaMalloc(&b->d_out, (size_t)cap * sizeof(gg_cand_result)));
    GB_CK(cudaMallocHost(&b->h_cands, (size_t)cap * sizeof(gg_swap)));
    GB_CK(cudaMallocHost(&b->h_out, (size_t)cap * sizeof(gg_cand_result)));
    GB_CK(cudaMalloc(&b->d_inc, (size_t)cap * sizeof(IncCand)));
    b->list_stride = std::max(max_n, 1);
    GB_CK(cudaMalloc(&b->d_lists, (size_t)cap * b->list_stride * sizeof(uint16_t)));
    b->cap = cap;
    drop_graph(b);
    return GG_OK;
}

// Enqueue reset -> batch kernel -> finalize on `st` for candidates `cands`,
// results `out`; the candidate count and task geometry come from d_ctl.
gg_status enqueue(gg_batch *b, const gg_swap *cands, gg_cand_result *out, cudaStream_t st,
                  unsigned *hist = nullptr, int hist_k = 0) {
    // the histogram pass searches every source of its one candidate
    const bool inc = !hist;
    BatchArgs a{b->d_bases, cands, out, b->d_ctl, hist, hist_k, inc ? b->d_inc : nullptr,
                b->d_lists, b->list_stride};
    batch_reset<<<64, 256, 0, st>>>(a);
    if (inc) {
        const unsigned long long pairs = (unsigned long long)b->cap * b->list_stride;
        const int g = (int)std::min<unsigned long long>((pairs + 255) / 256, 148ull * 16);
        batch_affected<<<g, 256, 0, st>>>(a, b->list_stride, b->full_only ? 1 : 0);
    }
    batch_kernel<<<b->grid, kBatchBlock, b->smem, st>>>(a);
    batch_finalize<<<64, 256, 0, st>>>(a);
    GB_CK(cudaGetLastError());
    return GG_OK;
}

constexpr int kIncMaxN = 16384;   // larger bases search every source (planes of 4 n^2/8 bytes)

// The base pass of base `id` (affected-source mode): the single-graph engine
// evaluates the base with its distance planes (at most 16 levels), then every
// source's distance sum and eccentricity follow from the planes.  valid = 0
// (every candidate of the base searches every source) unless the base is
// symmetric, connected and of diameter <= 15.
gg_status base_pass(gg_batch *b, int id) {
    BatchBase &B = b->bases[id];
    const cudaStream_t st = b->stream;
    B.valid = 0;
    if (!b->full_only && B.n <= kIncMaxN) {
        gg_engine *eng = nullptr;
        for (auto &pe : b->engines)
            if (pe.first == std::make_pair(B.n, B.d)) eng = pe.second;
        if (!eng) {
            gg_status s = gg_graph_create(B.n, B.d, b->device, &eng);
            if (s != GG_OK) return s;
            b->engines.push_back({{B.n, B.d}, eng});
            GB_CK(cudaSetDevice(b->device));
        }
        if (!b->base_planes[id]) {
            B.cols = (unsigned)gg::engine_plane_cols(eng);
            GB_CK(cudaMalloc(&b->base_planes[id], (size_t)kPlanes * B.n * B.cols * sizeof(uint4)));
            GB_CK(cudaMalloc(&b->base_stats[id], 2 * (size_t)B.n * sizeof(unsigned)));
        }
        GB_CK(cudaMemsetAsync(b->d_flag, 0, sizeof(int), st));
        const long long ent = (long long)B.n * B.d;
        table_symmetry<<<(int)((ent + 255) / 256), 256, 0, st>>>(b->base_adj[id], B.n, B.d, b->d_flag);
        GB_CK(cudaGetLastError());
        gg_eval_opts o{};
        o.max_levels = 1 << kPlanes;      // a base that needs more levels searches every source
        gg::EvalExtra x;
        x.planes = b->base_planes[id];
        x.nplanes = kPlanes;
        x.no_graph = true;
        gg_result r{};
        gg_status s = gg::engine_eval(eng, b->base_adj[id], &o, &r, st, &x);
        if (s != GG_OK) return s;
        int sms = 0;
        GB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
        // rows of the planes = sources: valid only on a symmetric base, which
        // `valid` below requires
        plane_row_stats<kPlanes><<<plane_row_stats_grid(B.n, sms), 256, 0, st>>>(
            b->base_planes[id], (unsigned long long)B.n * B.cols, B.cols, B.n, b->base_stats[id],
            b->base_stats[id] + B.n);
        GB_CK(cudaGetLastError());
        GB_CK(cudaMemcpyAsync(b->h_flag, b->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        GB_CK(cudaStreamSynchronize(st));
        if (!*b->h_flag && r.connected && !r.capped && r.levels < (1 << kPlanes)) {
            B.valid = 1;
            B.total = r.total;
            B.reached = r.reached;
            B.levels = r.levels;
            B.planes = b->base_planes[id];
            B.rowsum = b->base_stats[id];
            B.ecc = b->base_stats[id] + B.n;
        }
    }
    GB_CK(cudaMemcpyAsync(b->d_bases + id, &B, sizeof(BatchBase), cudaMemcpyHostToDevice, st));
    GB_CK(cudaStreamSynchronize(st));
    return GG_OK;
}

__global__ void set_ctl(BatchCtl *ctl, const BatchCtl v) { *ctl = v; }

// int32 rows -> uint16 rows (vertex ids < 65536), zero padding to `padded` entries.
__global__ void pack16_kernel(const int32_t *adj, uint16_t *out, int n_ent, int padded) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < padded; k += gridDim.x * blockDim.x)
        out[k] = k < n_ent ? (uint16_t)adj[k] : (uint16_t)0;
}

unsigned adj16_bytes(int n, int d) { return (unsigned)((((size_t)n * d * 2) + 15) / 16 * 16); }

// The device-side candidate check starts clean for every launch.
void arm_check(gg_batch *b) {
    b->h_ctl->bad = 0;
    b->h_ctl->timeout = 0;
    b->h_ctl->bad_index = 0x7fffffff;
    b->h_ctl->n_bases = (int)b->bases.size();
}

gg_status validate(const gg_batch *b, int n_cand, const gg_swap *c) {
    for (int i = 0; i < n_cand; ++i) {
        const gg_swap &s = c[i];
        if (s.base < 0 || s.base >= (int)b->bases.size())
            return bfail(GG_BAD_ARG, "candidate " + std::to_string(i) + ": unknown base");
        if (s.a < 0) continue;
        const int n = b->bases[s.base].n;
        if (s.a >= n || s.b < 0 || s.b >= n || s.c < 0 || s.c >= n || s.d < 0 || s.d >= n ||
            (s.mode != 0 && s.mode != 1))
            return bfail(GG_BAD_ARG, "candidate " + std::to_string(i) + ": vertex or mode out of range");
        if (s.a == s.b || s.a == s.c || s.a == s.d || s.b == s.c || s.b == s.d || s.c == s.d)
            return bfail(GG_BAD_ARG, "candidate " + std::to_string(i) + ": endpoints must be distinct");
    }
    return GG_OK;
}

}  // namespace

extern "C" {

gg_status gg_batch_create(int device, gg_batch **out) {
    if (!out) return bfail(GG_BAD_ARG, "null out");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return bfail(GG_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return bfail(GG_NO_DEVICE, "device index out of range");
    gg_batch *b = new gg_batch();
    b->device = device;
    auto fail_and_free = [&](gg_status s) { gg_batch_destroy(b); return s; };
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaMalloc(&b->d_ctl, sizeof(BatchCtl)) != cudaSuccess ||
        cudaMallocHost(&b->h_ctl, sizeof(BatchCtl)) != cudaSuccess ||
        cudaMalloc(&b->d_bases, 256 * sizeof(BatchBase)) != cudaSuccess ||
        cudaMalloc(&b->d_flag, sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&b->h_flag, sizeof(int)) != cudaSuccess)
        return fail_and_free(bfail(GG_CUDA_ERROR, "batch set-up failed"));
    std::memset(b->h_ctl, 0, sizeof(BatchCtl));
    const char *f = std::getenv("GG_BATCH_FULL");
    b->full_only = f && std::atoi(f) != 0;
    *out = b;
    return GG_OK;
}

gg_status gg_batch_add_base(gg_batch *b, int n, int degree, const int32_t *adj, int *base_id) {
    if (!b || !adj || !base_id || n < 1 || n > 65535 || degree < 1 || b->bases.size() >= 256)
        return bfail(GG_BAD_ARG, "need 1 <= n <= 65535, degree >= 1, at most 256 bases");
    for (long long k = 0; k < (long long)n * degree; ++k)
        if (adj[k] < 0 || adj[k] >= n) return bfail(GG_BAD_ARG, "adjacency entry outside [0, n)");
    const int lnc = auto_log_nc(b->device, n, degree);
    if (lnc < 0) return bfail(GG_BAD_ARG, "base graph too large for a shared-memory task");
    GB_CK(cudaSetDevice(b->device));
    int32_t *d = nullptr;
    uint16_t *d16 = nullptr;
    const unsigned b16 = adj16_bytes(n, degree);
    GB_CK(cudaMalloc(&d, (size_t)n * degree * sizeof(int32_t)));
    cudaError_t me = cudaMalloc(&d16, b16);
    if (me != cudaSuccess) { cudaFree(d); GB_CK(me); }
    GB_CK(cudaMemcpy(d, adj, (size_t)n * degree * sizeof(int32_t), cudaMemcpyHostToDevice));
    pack16_kernel<<<64, 256, 0, b->stream>>>(d, d16, n * degree, (int)(b16 / 2));
    GB_CK(cudaGetLastError());
    BatchBase B{};
    B.adj = d; B.adj16 = d16; B.adj16_bytes = b16;
    B.n = n; B.d = degree; B.log_nc = lnc; B.chunks = (n + (128 << lnc) - 1) / (128 << lnc);
    b->bases.push_back(B);
    b->base_adj.push_back(d);
    b->base_adj16.push_back(d16);
    b->base_planes.push_back(nullptr);
    b->base_stats.push_back(nullptr);
    const int id = (int)b->bases.size() - 1;
    gg_status s = refresh_plan(b);
    if (s == GG_OK) s = base_pass(b, id);
    if (s != GG_OK) return s;
    *base_id = id;
    return GG_OK;
}

gg_status gg_batch_set_base(gg_batch *b, int base_id, const int32_t *adj) {
    if (!b || !adj || base_id < 0 || base_id >= (int)b->bases.size())
        return bfail(GG_BAD_ARG, "bad base or adjacency");
    const BatchBase &B = b->bases[base_id];
    for (long long k = 0; k < (long long)B.n * B.d; ++k)
        if (adj[k] < 0 || adj[k] >= B.n) return bfail(GG_BAD_ARG, "adjacency entry outside [0, n)");
    GB_CK(cudaSetDevice(b->device));
    // ordered on the batch stream: launches already enqueued see the old table
    GB_CK(cudaMemcpyAsync(b->base_adj[base_id], adj, (size_t)B.n * B.d * sizeof(int32_t),
                          cudaMemcpyHostToDevice, b->stream));
    pack16_kernel<<<64, 256, 0, b->stream>>>(b->base_adj[base_id], b->base_adj16[base_id], B.n * B.d,
                                            (int)(B.adj16_bytes / 2));
    GB_CK(cudaGetLastError());
    return base_pass(b, base_id);
}

gg_status gg_batch_set_chunk(gg_batch *b, int base_id, int sources) {
    if (!b || base_id < 0 || base_id >= (int)b->bases.size() || sources < 128 || sources % 128)
        return bfail(GG_BAD_ARG, "bad base or chunk width");
    int l = 0;
    while ((128 << l) < sources) ++l;
    if ((128 << l) != sources) return bfail(GG_BAD_ARG, "chunk width must be 128 * 2^k");
    BatchBase &B = b->bases[base_id];
    const size_t need = ((size_t)B.n * B.d * 2 + 15) / 16 * 16 + 2 * (size_t)B.n * (16u << l);
    if (need > kSmemBudget) return bfail(GG_BAD_ARG, "chunk does not fit in shared memory");
    B.log_nc = l;
    B.chunks = (B.n + (128 << l) - 1) / (128 << l);
    GB_CK(cudaSetDevice(b->device));
    return refresh_plan(b);
}

gg_status gg_batch_autotune(gg_batch *b, int n_cand, const gg_swap *cands, int trials, double *best_ms) {
    if (!b || n_cand < 1 || !cands || trials < 1) return bfail(GG_BAD_ARG, "bad arguments");
    gg_status s = validate(b, n_cand, cands);
    if (s != GG_OK) return s;
    std::vector<gg_cand_result> out((size_t)n_cand);
    auto time_it = [&](double *t) -> gg_status {
        gg_status r = gg_batch_eval(b, n_cand, cands, out.data());  // warm (and capture)
        if (r != GG_OK) return r;
        *t = 1e300;
        for (int k = 0; k < trials; ++k) {
            r = gg_batch_eval(b, n_cand, cands, out.data());
            if (r != GG_OK) return r;
            *t = std::min(*t, b->last_ms);
        }
        return GG_OK;
    };
    std::vector<char> used(b->bases.size(), 0);
    for (int i = 0; i < n_cand; ++i) used[cands[i].base] = 1;
    double best_t = 1e300;
    s = time_it(&best_t);
    if (s != GG_OK) return s;
    // coordinate descent over the bases the candidates use: each base's chunk width
    // with the others fixed
    for (size_t id = 0; id < b->bases.size(); ++id) {
        if (!used[id]) continue;
        const int n = b->bases[id].n, d = b->bases[id].d;
        int best_l = b->bases[id].log_nc;
        for (int l = 0; l <= 4; ++l) {
            if (l == best_l || !log_nc_fits(n, d, l)) continue;
            if (l > 0 && (128 << (l - 1)) >= n) break;   // wider than the base's sources
            s = gg_batch_set_chunk(b, (int)id, 128 << l);
            if (s != GG_OK) return s;
            double t = 0;
            s = time_it(&t);
            if (s != GG_OK) return s;
            if (t < best_t) { best_t = t; best_l = l; }
        }
        s = gg_batch_set_chunk(b, (int)id, 128 << best_l);
        if (s != GG_OK) return s;
        gg::tune_put(batch_tune_key(b->device, n, d), {best_l});
    }
    if (best_ms) *best_ms = best_t;
    return GG_OK;
}

gg_status gg_batch_chunk(gg_batch *b, int base_id, int *sources) {
    if (!b || !sources || base_id < 0 || base_id >= (int)b->bases.size()) return bfail(GG_BAD_ARG, "bad base");
    *sources = 128 << b->bases[base_id].log_nc;
    return GG_OK;
}

gg_status gg_batch_eval(gg_batch *b, int n_cand, const gg_swap *cands, gg_cand_result *out) {
    if (!b || n_cand < 0 || (n_cand && (!cands || !out))) return bfail(GG_BAD_ARG, "bad arguments");
    if (n_cand == 0) return GG_OK;
    gg_status s = validate(b, n_cand, cands);
    if (s != GG_OK) return s;
    GB_CK(cudaSetDevice(b->device));
    s = ensure_cap(b, n_cand);
    if (s != GG_OK) return s;
    std::memcpy(b->h_cands, cands, (size_t)n_cand * sizeof(gg_swap));
    b->h_ctl->n_cand = n_cand;
    b->h_ctl->task_ctr = 0;
    arm_check(b);
    GB_CK(cudaMemcpyAsync(b->d_cands, b->h_cands, (size_t)n_cand * sizeof(gg_swap),
                          cudaMemcpyHostToDevice, b->stream));
    GB_CK(cudaMemcpyAsync(b->d_ctl, b->h_ctl, sizeof(BatchCtl), cudaMemcpyHostToDevice, b->stream));
    if (!b->exec) {  // capture reset -> kernel -> finalize once per buffer set
        GB_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        gg_status es = enqueue(b, b->d_cands, b->d_out, b->stream);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (es != GG_OK) { if (g) cudaGraphDestroy(g); return es; }
        GB_CK(ce);
        b->graph = g;
        GB_CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    GB_CK(cudaEventRecord(b->ev0, b->stream));
    GB_CK(cudaGraphLaunch(b->exec, b->stream));
    GB_CK(cudaEventRecord(b->ev1, b->stream));
    GB_CK(cudaMemcpyAsync(b->h_out, b->d_out, (size_t)n_cand * sizeof(gg_cand_result),
                          cudaMemcpyDeviceToHost, b->stream));
    GB_CK(cudaStreamSynchronize(b->stream));
    float ms = 0.f;
    GB_CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->last_ms = ms;
    std::memcpy(out, b->h_out, (size_t)n_cand * sizeof(gg_cand_result));
    if (out[0].levels < 0) return gg_batch_device_status(b, b->stream, nullptr);  // a flagged launch
    return GG_OK;
}

gg_status gg_batch_eval_device(gg_batch *b, int n_cand, const gg_swap *d_cands,
                               gg_cand_result *d_out, void *stream) {
    if (!b || n_cand < 0 || (n_cand && (!d_cands || !d_out))) return bfail(GG_BAD_ARG, "bad arguments");
    if (n_cand == 0) return GG_OK;
    GB_CK(cudaSetDevice(b->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    gg_status cs = ensure_cap(b, n_cand);   // per-candidate lists of the affected-source mode
    if (cs != GG_OK) return cs;
    b->h_ctl->n_cand = n_cand;
    b->h_ctl->task_ctr = 0;
    arm_check(b);
    // the control block goes by value as a kernel argument: this call returns
    // before the GPU runs it, and the next call may change the host copy
    set_ctl<<<1, 1, 0, st>>>(b->d_ctl, *b->h_ctl);
    GB_CK(cudaGetLastError());
    GB_CK(cudaEventRecord(b->ev0, st));
    gg_status s = enqueue(b, d_cands, d_out, st);
    if (s != GG_OK) return s;
    GB_CK(cudaEventRecord(b->ev1, st));
    return GG_OK;
}

gg_status gg_batch_device_status(gg_batch *b, void *stream, int *first_bad) {
    if (!b) return bfail(GG_BAD_ARG, "null batch");
    GB_CK(cudaSetDevice(b->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    GB_CK(cudaStreamSynchronize(st));
    BatchCtl c{};
    GB_CK(cudaMemcpy(&c, b->d_ctl, sizeof(BatchCtl), cudaMemcpyDeviceToHost));
    if (first_bad) *first_bad = c.bad ? c.bad_index : -1;
    if (c.timeout) return bfail(GG_TIMEOUT, "a CTA's wait for its adjacency copy ran past its limit");
    if (c.bad)
        return bfail(GG_BAD_ARG, "device candidate " + std::to_string(c.bad_index) +
                                     ": unknown base, vertex or mode out of range, or repeated endpoint");
    return GG_OK;
}

gg_status gg_batch_vertex_hist(gg_batch *b, int base_id, int K, uint32_t *hist) {
    if (!b || !hist || base_id < 0 || base_id >= (int)b->bases.size() || K < 1 || K > 64)
        return bfail(GG_BAD_ARG, "bad base, K or output");
    GB_CK(cudaSetDevice(b->device));
    gg_status s = ensure_cap(b, 1);
    if (s != GG_OK) return s;
    const int n = b->bases[base_id].n;
    const size_t need = (size_t)n * K;
    if (need > b->hist_cap) {
        cudaFree(b->d_hist);
        b->d_hist = nullptr;
        b->hist_cap = 0;
        GB_CK(cudaMalloc(&b->d_hist, need * sizeof(unsigned)));
        b->hist_cap = need;
    }
    unsigned *d_hist = b->d_hist;
    const gg_swap self{base_id, -1, -1, -1, -1, 0};
    b->h_cands[0] = self;
    b->h_ctl->n_cand = 1;
    b->h_ctl->task_ctr = 0;
    arm_check(b);
    cudaError_t e = cudaMemsetAsync(d_hist, 0, (size_t)n * K * sizeof(unsigned), b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_cands, b->h_cands, sizeof(gg_swap), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_ctl, b->h_ctl, sizeof(BatchCtl), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) s = enqueue(b, b->d_cands, b->d_out, b->stream, d_hist, K);
    if (e == cudaSuccess && s == GG_OK)
        e = cudaMemcpyAsync(hist, d_hist, (size_t)n * K * sizeof(unsigned), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (s != GG_OK) return s;
    GB_CK(e);
    return GG_OK;
}

gg_status gg_batch_last_ms(gg_batch *b, double *ms) {
    if (!b || !ms) return bfail(GG_BAD_ARG, "null argument");
    float f = 0.f;
    if (cudaEventElapsedTime(&f, b->ev0, b->ev1) == cudaSuccess) b->last_ms = f;
    else (void)cudaGetLastError();
    *ms = b->last_ms;
    return GG_OK;
}

gg_status gg_batch_destroy(gg_batch *b) {
    if (!b) return GG_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    for (auto p : b->base_adj) cudaFree(p);
    for (auto p : b->base_adj16) cudaFree(p);
    for (auto p : b->base_planes) cudaFree(p);
    for (auto p : b->base_stats) cudaFree(p);
    for (auto &pe : b->engines) gg_destroy(pe.second);
    cudaFree(b->d_inc); cudaFree(b->d_lists);
    cudaFree(b->d_flag); cudaFreeHost(b->h_flag);
    cudaFree(b->d_bases); cudaFree(b->d_ctl); cudaFreeHost(b->h_ctl);
    cudaFree(b->d_cands); cudaFree(b->d_out); cudaFreeHost(b->h_cands); cudaFreeHost(b->h_out);
    cudaFree(b->d_hist);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return GG_OK;
}

}  // extern "C"
