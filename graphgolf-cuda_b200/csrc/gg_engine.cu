// gg_engine.cu -- host side of the engine and the C ABI declared in include/gg.h.
//
// One gg_engine owns every device and pinned buffer of one calculator, sized at
// construction from its form and dimensions, the way the reference calculators
// size theirs in their constructors (cudaASPLconv.cu:122-137,
// cudaASPLgraph.cu:114-127).  An evaluation is:
//   H2D of the packed table -> expand_kernel (lifted forms) -> one cooperative
//   bfs_batch_kernel launch per source batch -> one D2H of the level counters
//   -> exact host fold into gg_result -> the reference's return convention.
// There is no per-level host round trip: the level loop, its termination test
// and the connectivity test live on the device.
#include "gg.h"
#include "gg_kernels.cuh"
#include "gg_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

using gg::BfsArgs;
using gg::Ctl;
using gg::ExpandArgs;
using gg::FastDiv;

namespace {

thread_local std::string g_err;

gg_status fail(gg_status s, const std::string &msg) {
    g_err = msg;
    return s;
}

#define GG_CK(call)                                                                     \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            (void)cudaGetLastError();                                                   \
            return fail(e_ == cudaErrorMemoryAllocation ? GG_OUT_OF_MEMORY : GG_CUDA_ERROR, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));            \
        }                                                                               \
    } while (0)

enum Form { FORM_GRAPH = 0, FORM_PART = 1, FORM_PIECE = 2, FORM_BOX = 3 };

constexpr int kBeamerRows = 1000000;   // cudaASPLbeamer.cu:10-12
constexpr int kBeamerLevels = 7;       // cudaASPLbeamer.cu:17
constexpr int kSentinel = 100000000;   // cudaASPLconv.cu:207

int env_int(const char *name, int dflt) {
    const char *s = std::getenv(name);
    return (s && *s) ? std::atoi(s) : dflt;
}

// Host-side fault injection for the failure-path tests (GG_FAULT_INJECT):
//   "barrier" -- the grid barrier waits for one block more than is launched, so
//                its bounded wait runs out and the call returns GG_TIMEOUT;
//   "alloc"   -- engine creation reports an allocation failure;
//   "launch"  -- the BFS launch reports a CUDA error before anything is enqueued.
// Nothing here faults, traps or hangs the GPU.
bool fault(const char *what) {
    const char *s = std::getenv("GG_FAULT_INJECT");
    return s && std::strcmp(s, what) == 0;
}

}  // namespace

namespace gg {
// Shared with the other translation units of the library (not exported).
__attribute__((visibility("hidden"))) void set_last_error(const char *msg) { g_err = msg; }
}  // namespace gg

// What a captured evaluation depends on (see run_eval).
struct EvalKey {
    const void *table, *status, *bitsets, *inv, *planes;
    int s0, ns, cap;
    bool wvc, want_ns;
    bool operator==(const EvalKey &o) const {
        return table == o.table && status == o.status && bitsets == o.bitsets && inv == o.inv &&
               planes == o.planes && s0 == o.s0 && ns == o.ns && cap == o.cap && wvc == o.wvc &&
               want_ns == o.want_ns;
    }
};

struct gg_engine {
    int form = FORM_PART;
    int device = 0;
    int N = 0, M = 0, d = 0, rows = 0;
    int dims[6] = {0, 0, 0, 0, 0, 0};    // Nx Ny Nz Mx My Mz
    uint64_t scale = 1;
    size_t table_elems = 0;
    std::vector<int32_t> reps;           // source vertex ids, in source order

    // plan
    int batch_bits = 0;                  // sources per batch (multiple of 128)
    int nC = 0;                          // uint4 chunks per row
    uint32_t items = 0;
    int grid = 0;
    int dense_w_ppm = 100;               // level-mode thresholds (see bfs_batch_kernel)
    int dense_r_ppm = 4000;
    int full_skip_ppm = 995000;
    int split_ppm = 850000;
    int push_ppm = 300;                  // push (top-down) levels below this frontier share
    int push_min_items = 1 << 20;        // ... on bitsets of at least this many chunks
    int adj_smem_rows = 0;               // shared-memory adjacency slice (rows per block)
    size_t smem_bytes = 0;
    int bps_cap = 0;                     // resident blocks per SM (0: as many as fit)
    int walk_pref = -1;                  // walk depth: -1 automatic, 0 off, K > 0 forced
    int walk_K = 0;                      // levels computed by the walk pass (0: off)
    int walk_vpull = 1;                  // levels after the walk pull visited sets (GG_VPULL=0: frontiers)
    int walk_own_skip = 1;               // dense ones skip own chunks on tables without one-way entries (GG_OWN_SKIP)
    int walk_third = 1;                  // after the walk of all batches, levels alternate V and F0 (GG_WALK_THIRD)
    int walk_rpg = 1;                    // rows per walk group
    unsigned walk_smem_off = 0;          // byte offset of the walk buffers in dynamic smem
    int32_t *d_h2 = nullptr;             // [rows][d*d] level-2 walk ends (walk_K >= 3)
    size_t h2_elems = 0;
    // walk index (walk_index_kernel): [rows][walk_cap] entries, [rows][walk_off_stride] bucket starts
    uint16_t *d_went = nullptr, *d_woff = nullptr;
    size_t went_elems = 0, woff_elems = 0;
    int walk_cap = 0, walk_off_stride = 0;
    long long wait_ns = 10ll * 1000 * 1000 * 1000;
    int cap_alloc = 0;                   // levels the counter arrays hold
    int nb_alloc = 0;                    // batches the counter arrays hold

    // device
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int32_t *d_table = nullptr, *d_adj = nullptr;
    // Status block of an evaluation (one device allocation, mirrored in pinned
    // host memory, so that an evaluation needs one memset and one copy back):
    //   [0, 256) Ctl | bad, asym | levels_run[nb_alloc] | batch_ns[2 nb_alloc] |
    //   counts[nb][cap_req + 1]
    unsigned char *d_status = nullptr, *h_status = nullptr;
    size_t off_levels_run = 0, off_batch_ns = 0, off_counts = 0;
    int *d_bad = nullptr;                // the table failed its range check
    int *d_asym = nullptr;               // adjacency not symmetric: no push levels
    uint4 *d_V = nullptr, *d_F0 = nullptr, *d_F1 = nullptr;
    uint32_t *d_fl0 = nullptr, *d_fl1 = nullptr;
    uint4 *d_P0 = nullptr, *d_P1 = nullptr;     // push-level frontier, all zero between launches
    uint32_t *d_pf0 = nullptr, *d_pf1 = nullptr;
    uint32_t *d_nf = nullptr;            // not-full bit per visited chunk
    uint32_t *d_nf2 = nullptr;           // its second copy (visited-set pull levels alternate)
    int *d_wasym = nullptr;              // one-way flag of the table (walk_index_kernel)
    unsigned long long *d_vtot = nullptr;   // [nb][3] level totals (dense visited-set pull without own chunks)
    // walk_all_kernel output: the level-K rows of every batch and their flag words
    uint4 *d_vall = nullptr;
    uint32_t *d_vall_fl = nullptr;
    size_t vall_batches = 0;             // batches d_vall holds
    long long walk_all_mb = 4096;        // budget for d_vall (GG_WALK_ALL_MB; 0: per-batch walk passes)
    bool p_dirty = true;                 // push buffers must be zeroed before the next launch
    unsigned long long *d_counts = nullptr;
    unsigned *d_masks = nullptr;
    unsigned long long *d_level_ns = nullptr, *h_level_ns = nullptr;
    int *d_levels_run = nullptr, *h_levels_run = nullptr;                 // [nb_alloc]
    unsigned long long *d_batch_ns = nullptr, *h_batch_ns = nullptr;     // [2 * nb_alloc]
    int32_t *d_inv = nullptr;            // source index of each vertex, when the sources
    int src_first = 0;                   // are not the consecutive ids src_first, src_first+1, ...
    Ctl *d_ctl = nullptr;
    // pinned host
    int32_t *h_table = nullptr;
    unsigned long long *h_counts = nullptr;
    unsigned *h_masks = nullptr;
    Ctl *h_ctl = nullptr;
    int *h_bad = nullptr;

    bool use_graph = true;               // replay captured evaluations (GG_NO_GRAPH=1: never)
    cudaGraphExec_t graph_exec = nullptr;
    EvalKey graph_key{};

    double last_ms = 0.0;
    int last_launches = 0;
    int last_batches = 0;                // batches of the last evaluation
    uint64_t last_h2d = 0, last_d2h = 0;
};

namespace {

void free_batch_buffers(gg_engine *e) {
    cudaFree(e->d_vall); cudaFree(e->d_vall_fl);
    e->d_vall = nullptr;
    e->d_vall_fl = nullptr;
    e->vall_batches = 0;
    cudaFree(e->d_V); cudaFree(e->d_F0); cudaFree(e->d_F1);
    cudaFree(e->d_fl0); cudaFree(e->d_fl1);
    cudaFree(e->d_P0); cudaFree(e->d_P1); cudaFree(e->d_pf0); cudaFree(e->d_pf1);
    cudaFree(e->d_nf);
    cudaFree(e->d_nf2);
    e->d_nf = e->d_nf2 = nullptr;
    e->d_V = e->d_F0 = e->d_F1 = nullptr;
    e->d_fl0 = e->d_fl1 = nullptr;
    e->d_P0 = e->d_P1 = nullptr;
    e->d_pf0 = e->d_pf1 = nullptr;
}

void free_counters(gg_engine *e) {
    cudaFree(e->d_status); cudaFree(e->d_masks); cudaFree(e->d_level_ns); cudaFree(e->d_vtot);
    cudaFreeHost(e->h_status); cudaFreeHost(e->h_masks);
    cudaFreeHost(e->h_level_ns);
    e->d_status = e->h_status = nullptr;
    e->d_bad = e->d_asym = e->d_wasym = e->h_bad = nullptr;
    e->d_vtot = nullptr;
    e->d_levels_run = e->h_levels_run = nullptr;
    e->d_batch_ns = e->h_batch_ns = nullptr;
    e->d_counts = nullptr; e->d_masks = nullptr; e->d_ctl = nullptr; e->d_level_ns = nullptr;
    e->h_counts = nullptr; e->h_masks = nullptr; e->h_ctl = nullptr; e->h_level_ns = nullptr;
    e->cap_alloc = e->nb_alloc = 0;
}

// A captured evaluation holds buffer addresses, the plan and the wait limit:
// drop it whenever one of them changes.
void invalidate_graph(gg_engine *e) {
    if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
    e->graph_exec = nullptr;
}

void destroy_all(gg_engine *e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    free_batch_buffers(e);
    free_counters(e);
    if (e->d_adj != e->d_table) cudaFree(e->d_adj);  // the graph form aliases the two
    cudaFree(e->d_h2);
    cudaFree(e->d_went);
    cudaFree(e->d_woff);
    cudaFree(e->d_table); cudaFree(e->d_inv);
    cudaFreeHost(e->h_table);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    invalidate_graph(e);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

int kernel_degree_slot(int d) {
    switch (d) {
        case 3: case 4: case 6: case 8: case 12: case 16: return d;
        default: return 0;
    }
}

template <bool PL>
void *kernel_for_t(int d) {
    switch (kernel_degree_slot(d)) {
        case 3: return (void *)gg::bfs_batch_kernel<3, PL>;
        case 4: return (void *)gg::bfs_batch_kernel<4, PL>;
        case 6: return (void *)gg::bfs_batch_kernel<6, PL>;
        case 8: return (void *)gg::bfs_batch_kernel<8, PL>;
        case 12: return (void *)gg::bfs_batch_kernel<12, PL>;
        case 16: return (void *)gg::bfs_batch_kernel<16, PL>;
        default: return (void *)gg::bfs_batch_kernel<0, PL>;
    }
}

// The BFS kernel for degree d; `planes`: the variant that also writes the
// distance planes.
void *kernel_for(int d, bool planes = false) {
    return planes ? kernel_for_t<true>(d) : kernel_for_t<false>(d);
}

// Walk ends per row up to depth K: d + d^2 + ... + d^K.
long long walk_cap_for(int d, int K) {
    long long sum = 0, p = 1;
    for (int k = 1; k <= K; ++k) { p *= d; sum += p; }
    return sum;
}

// Levels the walk pass computes for this plan: the largest K <= 4 whose walk ends
// per row stay within 600 (d = 8: 3 levels, 584 ends; d = 16: 2; d = 4: 4), within
// the index kernel's row buffer and bucket count (kIndexMaxCap ends, kIndexMaxKeys
// = batches * K buckets), with the level-2 table (rows * d^2 int32, K >= 3) within
// 64 MiB and the index (rows * (ends + buckets) uint16) within 1 GiB; off for
// evaluations of a single source batch.  GG_WALK_LEVELS overrides the depth (0 = off;
// still within the size limits).
int walk_levels(const gg_engine *e) {
    const int env = env_int("GG_WALK_LEVELS", e->walk_pref);
    const int d = e->d;
    if (d <= 0 || e->nC > gg::kWalkMaxNC || env == 0) return 0;
    int K = 0;
    for (int k = 1; k <= 4 && walk_cap_for(d, k) <= 600; ++k) K = k;
    const long long nb = ((long long)e->reps.size() + e->batch_bits - 1) / e->batch_bits;
    // The index costs one pass over every row's walk ends per evaluation; with a
    // single source batch the pass it saves is not worth it (n = 4096, d = 16: 0.070
    // against 0.060 ms; a lift with one batch: 0.135 against 0.097 ms).
    if (nb < 2) K = 0;
    if (env > 0) K = std::min(env, 4);
    for (; K > 0; --K) {
        const long long cap = walk_cap_for(d, K), keys = nb * K;
        const bool ok = cap <= gg::kIndexMaxCap && keys <= gg::kIndexMaxKeys &&
                        (K < 3 || (long long)e->rows * d * d * 4 <= (64ll << 20)) &&
                        (long long)e->rows * (cap + keys + 1) * 2 <= (1ll << 30);
        if (ok) break;
    }
    return K;
}

// walk_all_kernel for an evaluation of nb batches, or nullptr (a walk pass per
// batch): visited-set pull levels, 4096-source batches, degree 4 or 8, K <= 3, and
// the level-K rows of all nb batches within the GG_WALK_ALL_MB budget.  Grows
// d_vall as needed (a failed allocation falls back to the per-batch pass).
void *walk_all_for(gg_engine *e, int K, int nb) {
    if (!e->walk_vpull || e->nC != 32 || K < 1 || K > 3 || (e->d != 4 && e->d != 8)) return nullptr;
    const size_t bytes = (size_t)nb * e->items * sizeof(uint4);
    const size_t fbytes = (size_t)nb * ((e->items + 31) / 32) * sizeof(uint32_t);
    if ((long long)(bytes >> 20) > e->walk_all_mb) return nullptr;
    if ((size_t)nb > e->vall_batches) {
        invalidate_graph(e);
        cudaFree(e->d_vall); cudaFree(e->d_vall_fl);
        e->d_vall = nullptr;
        e->d_vall_fl = nullptr;
        e->vall_batches = 0;
        if (cudaMalloc(&e->d_vall, bytes) != cudaSuccess || cudaMalloc(&e->d_vall_fl, fbytes) != cudaSuccess) {
            cudaFree(e->d_vall); cudaFree(e->d_vall_fl);
            e->d_vall = nullptr;
            e->d_vall_fl = nullptr;
            (void)cudaGetLastError();
            return nullptr;
        }
        e->vall_batches = (size_t)nb;
    }
    void *k = nullptr;
    if (e->d == 8) k = K == 1 ? (void *)gg::walk_all_kernel<8, 1> : K == 2 ? (void *)gg::walk_all_kernel<8, 2> : (void *)gg::walk_all_kernel<8, 3>;
    else k = K == 1 ? (void *)gg::walk_all_kernel<4, 1> : K == 2 ? (void *)gg::walk_all_kernel<4, 2> : (void *)gg::walk_all_kernel<4, 3>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, gg::walk_all_smem(K)) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    return k;
}

void *index_kernel_for(int d) {
    switch (kernel_degree_slot(d)) {
        case 3: return (void *)gg::walk_index_kernel<3>;
        case 4: return (void *)gg::walk_index_kernel<4>;
        case 6: return (void *)gg::walk_index_kernel<6>;
        case 8: return (void *)gg::walk_index_kernel<8>;
        case 12: return (void *)gg::walk_index_kernel<12>;
        case 16: return (void *)gg::walk_index_kernel<16>;
        default: return (void *)gg::walk_index_kernel<0>;
    }
}

// Source-batch plan: batch width, chunks per row, grid size.
// gg_autotune's choices (batch width, resident blocks per SM, walk depth) are
// kept in the tuning cache under (GPU, form, rows, degree, sources).
std::string engine_tune_key(const gg_engine *e) {
    return gg::tune_key(e->device, "graph", {e->form, e->rows, e->d, (long long)e->reps.size()});
}

gg_status plan(gg_engine *e, int want_bits) {
    invalidate_graph(e);
    const int n_src = (int)e->reps.size();
    int bits;
    if (want_bits > 0) {
        bits = want_bits;
    } else {
        const int env = env_int("GG_BATCH_SOURCES", 0);
        std::vector<int> tuned;
        if (env > 0) {
            bits = env;
        } else if (gg::tune_get(engine_tune_key(e), &tuned) && tuned.size() >= 3 && tuned[0] > 0) {
            bits = tuned[0];
            e->bps_cap = tuned[1];
            e->walk_pref = tuned[2];
        } else {
            // The widest batch whose three bitsets (3 * rows * bits / 8 bytes)
            // stay within 3/4 of the L2, so that the gathers hit L2 rather than
            // HBM; at least 4096 sources (one 512-byte row segment per vertex)
            // when there are that many.
            int l2 = 0;
            if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, e->device) != cudaSuccess || l2 <= 0) {
                (void)cudaGetLastError();
                l2 = 64 << 20;
            }
            const double per_bit = 3.0 * e->rows / 8.0;
            long long fit = (long long)(0.75 * l2 / per_bit);
            fit = std::max<long long>(fit, 4096);
            bits = (int)std::min<long long>(fit, n_src);
            if (bits > 4096) bits = (bits / 4096) * 4096;
        }
    }
    bits = std::max(128, ((std::min(bits, std::max(n_src, 1)) + 127) / 128) * 128);
    const long long items = (long long)e->rows * (bits / 128);
    if (items >= (1ll << 31)) return fail(GG_BAD_ARG, "rows x batch width exceeds 2^31 uint4 chunks");
    if (bits != e->batch_bits) {
        free_batch_buffers(e);
        e->batch_bits = bits;
        e->nC = bits / 128;
        e->items = (uint32_t)items;
        const size_t vbytes = (size_t)items * sizeof(uint4);
        const size_t fwords = (size_t)((items + 31) / 32);
        GG_CK(cudaMalloc(&e->d_V, vbytes));
        GG_CK(cudaMalloc(&e->d_F0, vbytes));
        GG_CK(cudaMalloc(&e->d_F1, vbytes));
        GG_CK(cudaMalloc(&e->d_fl0, fwords * 4));
        GG_CK(cudaMalloc(&e->d_fl1, fwords * 4));
        GG_CK(cudaMalloc(&e->d_P0, vbytes));
        GG_CK(cudaMalloc(&e->d_P1, vbytes));
        GG_CK(cudaMalloc(&e->d_pf0, fwords * 4));
        GG_CK(cudaMalloc(&e->d_pf1, fwords * 4));
        GG_CK(cudaMalloc(&e->d_nf, fwords * 4));
        GG_CK(cudaMalloc(&e->d_nf2, fwords * 4));
        e->p_dirty = true;
    }
    // Walk pass: levels 1..K of each batch from the walk ends of every row.
    e->walk_K = walk_levels(e);
    e->walk_rpg = 1;
    size_t walk_bytes = 0;
    if (e->walk_K > 0) {
        int g = e->nC, b = 32;
        while (b) { const int t = g % b; g = b; b = t; }   // gcd(nC, 32)
        e->walk_rpg = 32 / g;
        walk_bytes = (size_t)(gg::kBlock / 32) * gg::walk_smem_per_warp(e->nC);
    }
    const size_t h2_need = e->walk_K >= 3 ? (size_t)e->rows * e->d * e->d : 0;
    if (h2_need != e->h2_elems) {
        cudaFree(e->d_h2);
        e->d_h2 = nullptr;
        e->h2_elems = 0;
        if (h2_need) {
            GG_CK(cudaMalloc(&e->d_h2, h2_need * sizeof(int32_t)));
            e->h2_elems = h2_need;
        }
    }
    // row stride of the index: the walk ends, rounded up to a multiple of 8 (rows start
    // 16-byte aligned: the index kernel writes them 16 bytes at a time)
    e->walk_cap = e->walk_K ? (int)((walk_cap_for(e->d, e->walk_K) + 7) & ~7ll) : 0;
    e->walk_off_stride = e->walk_K ? (int)(((long long)e->reps.size() + bits - 1) / bits) * e->walk_K + 1 : 0;
    const size_t went_need = (size_t)e->rows * e->walk_cap, woff_need = (size_t)e->rows * e->walk_off_stride;
    if (went_need != e->went_elems || woff_need != e->woff_elems) {
        cudaFree(e->d_went);
        cudaFree(e->d_woff);
        e->d_went = e->d_woff = nullptr;
        e->went_elems = e->woff_elems = 0;
        if (went_need) {
            GG_CK(cudaMalloc(&e->d_went, went_need * sizeof(uint16_t)));
            GG_CK(cudaMalloc(&e->d_woff, woff_need * sizeof(uint16_t)));
            e->went_elems = went_need;
            e->woff_elems = woff_need;
        }
    }
    int per_sm = 0, sms = 0;
    GG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device));
    GG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel_for(e->d), gg::kBlock, walk_bytes));
    if (per_sm < 1) return fail(GG_CUDA_ERROR, "BFS kernel cannot be resident");
    const long long tiles = ((long long)e->items + 31) / 32;
    const long long want = (tiles + (gg::kBlock / 32) - 1) / (gg::kBlock / 32);
    // Resident blocks per SM: at most what fits; GG_BLOCKS_PER_SM, else the tuned cap.
    const int cap_per_sm = env_int("GG_BLOCKS_PER_SM", e->bps_cap);
    if (cap_per_sm > 0) per_sm = std::min(per_sm, cap_per_sm);
    e->grid = (int)std::max<long long>(1, std::min<long long>((long long)per_sm * sms, want));
    // Shared-memory adjacency slice: a block's contiguous tile range spans at most
    // ceil(tiles/grid)*32/nC + 2 vertices.  Cached when it fits a small budget and
    // does not lower the number of resident blocks.
    e->adj_smem_rows = 0;
    e->smem_bytes = walk_bytes;
    e->walk_smem_off = 0;
    if (env_int("GG_ADJ_SMEM", 1) && e->d > 0) {
        const long long per_block = (tiles + e->grid - 1) / e->grid;
        const long long rows = per_block * 32 / e->nC + 2;
        const long long bytes = (rows * e->d * 4 + 15) / 16 * 16;
        // within 32 KB, and within the 48 KB a launch gets without opting in
        if (bytes <= 32 * 1024 && bytes + (long long)walk_bytes <= 48 * 1024) {
            int per_sm2 = 0;
            GG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, kernel_for(e->d), gg::kBlock,
                                                                (size_t)bytes + walk_bytes));
            if (per_sm2 >= per_sm) {
                e->adj_smem_rows = (int)rows;
                e->walk_smem_off = (unsigned)bytes;
                e->smem_bytes = (size_t)bytes + walk_bytes;
            }
        }
    }
    return GG_OK;
}

gg_status ensure_counters(gg_engine *e, int cap, int nb) {
    if (cap <= e->cap_alloc && nb <= e->nb_alloc) return GG_OK;
    cap = std::max(cap, e->cap_alloc);
    nb = std::max(nb, e->nb_alloc);
    invalidate_graph(e);
    free_counters(e);
    const size_t n = (size_t)(cap + 1) * nb;
    e->off_levels_run = 512;
    e->off_batch_ns = e->off_levels_run + (((size_t)nb * sizeof(int) + 15) & ~size_t(15));
    e->off_counts = e->off_batch_ns + (size_t)nb * 2 * sizeof(unsigned long long);
    const size_t bytes = e->off_counts + n * sizeof(unsigned long long);
    GG_CK(cudaMalloc(&e->d_status, bytes));
    GG_CK(cudaMallocHost(&e->h_status, bytes));
    e->d_ctl = reinterpret_cast<Ctl *>(e->d_status);
    e->h_ctl = reinterpret_cast<Ctl *>(e->h_status);
    e->d_bad = reinterpret_cast<int *>(e->d_status + sizeof(Ctl));
    e->h_bad = reinterpret_cast<int *>(e->h_status + sizeof(Ctl));
    e->d_asym = e->d_bad + 1;
    e->d_wasym = e->d_bad + 2;
    GG_CK(cudaMalloc(&e->d_vtot, (size_t)nb * 3 * sizeof(unsigned long long)));
    e->d_levels_run = reinterpret_cast<int *>(e->d_status + e->off_levels_run);
    e->h_levels_run = reinterpret_cast<int *>(e->h_status + e->off_levels_run);
    e->d_batch_ns = reinterpret_cast<unsigned long long *>(e->d_status + e->off_batch_ns);
    e->h_batch_ns = reinterpret_cast<unsigned long long *>(e->h_status + e->off_batch_ns);
    e->d_counts = reinterpret_cast<unsigned long long *>(e->d_status + e->off_counts);
    e->h_counts = reinterpret_cast<unsigned long long *>(e->h_status + e->off_counts);
    GG_CK(cudaMalloc(&e->d_masks, n * sizeof(unsigned)));
    GG_CK(cudaMallocHost(&e->h_masks, n * sizeof(unsigned)));
    GG_CK(cudaMalloc(&e->d_level_ns, (size_t)(cap + 1) * sizeof(unsigned long long)));
    GG_CK(cudaMallocHost(&e->h_level_ns, (size_t)(cap + 1) * sizeof(unsigned long long)));
    e->cap_alloc = cap;
    e->nb_alloc = nb;
    return GG_OK;
}

gg_status create_common(gg_engine *e) {
    if (fault("alloc")) return fail(GG_OUT_OF_MEMORY, "injected allocation failure");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        return fail(GG_NO_DEVICE, "no CUDA device");
    }
    if (e->device < 0 || e->device >= ndev) return fail(GG_NO_DEVICE, "device index out of range");
    GG_CK(cudaSetDevice(e->device));
    GG_CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    GG_CK(cudaEventCreate(&e->ev0));
    GG_CK(cudaEventCreate(&e->ev1));
    const size_t tb = std::max<size_t>(e->table_elems, 1) * sizeof(int32_t);
    GG_CK(cudaMalloc(&e->d_table, tb));
    GG_CK(cudaMallocHost(&e->h_table, tb));
    if (e->form == FORM_GRAPH) {
        e->d_adj = e->d_table;  // the graph table is the adjacency
    } else {
        GG_CK(cudaMalloc(&e->d_adj, std::max<size_t>((size_t)e->rows * e->d, 1) * sizeof(int32_t)));
    }
    // The kernel finds a chunk's source from its vertex: directly when the
    // sources are consecutive vertex ids, else through the inverse list.
    bool consecutive = true;
    for (size_t i = 0; i < e->reps.size() && consecutive; ++i)
        consecutive = e->reps[i] == e->reps[0] + (int32_t)i;
    e->src_first = e->reps.empty() ? 0 : e->reps[0];
    if (!consecutive) {
        std::vector<int32_t> inv((size_t)std::max(e->rows, 1), -1);
        for (size_t i = 0; i < e->reps.size(); ++i) {
            const int32_t v = e->reps[i];
            if (v < 0 || v >= e->rows || inv[(size_t)v] != -1)
                return fail(GG_BAD_ARG, "sources must be distinct vertices");
            inv[(size_t)v] = (int32_t)i;
        }
        GG_CK(cudaMalloc(&e->d_inv, inv.size() * sizeof(int32_t)));
        GG_CK(cudaMemcpy(e->d_inv, inv.data(), inv.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    }
    e->dense_w_ppm = env_int("GG_DENSE_W_PPM", e->dense_w_ppm);
    e->dense_r_ppm = env_int("GG_DENSE_R_PPM", e->dense_r_ppm);
    e->full_skip_ppm = env_int("GG_FULL_SKIP_PPM", e->full_skip_ppm);
    e->split_ppm = env_int("GG_SPLIT_PPM", e->split_ppm);
    e->walk_vpull = env_int("GG_VPULL", e->walk_vpull) != 0;
    e->walk_own_skip = env_int("GG_OWN_SKIP", e->walk_own_skip) != 0;
    e->walk_third = env_int("GG_WALK_THIRD", e->walk_third) != 0;
    e->walk_all_mb = env_int("GG_WALK_ALL_MB", (int)e->walk_all_mb);
    e->push_ppm = env_int("GG_PUSH_PPM", e->push_ppm);
    e->push_min_items = env_int("GG_PUSH_MIN_ITEMS", e->push_min_items);
    e->use_graph = env_int("GG_NO_GRAPH", 0) == 0;
    const int wait_ms = env_int("GG_WAIT_LIMIT_MS", 10000);
    e->wait_ns = (long long)std::max(wait_ms, 1) * 1000000ll;
    gg_status s = plan(e, 0);
    if (s != GG_OK) return s;
    return ensure_counters(e, 128, 1);
}

gg_status finish_create(gg_engine *e, gg_engine **out) {
    gg_status s = create_common(e);
    if (s != GG_OK) {
        destroy_all(e);
        *out = nullptr;
        return s;
    }
    *out = e;
    return GG_OK;
}

// Core evaluation with the table already on the device (d_table_in) on `st`.
gg_status run_eval(gg_engine *e, const int32_t *d_table_in, const gg_eval_opts *o, gg_result *r,
                   cudaStream_t st, const gg::EvalExtra *x = nullptr) {
    const int n_src_all = x && x->inv ? x->ns : (int)e->reps.size();
    int s0 = 0, s1 = n_src_all;
    if (x && x->inv && (n_src_all < 1 || n_src_all > e->rows)) return fail(GG_BAD_ARG, "bad source list");
    if (x && x->planes && (o && (o->src_begin || o->src_end))) return fail(GG_BAD_ARG, "planes need every source");
    if (o && (o->src_begin || o->src_end)) {
        s0 = o->src_begin;
        s1 = o->src_end;
        if (s0 < 0 || s1 > n_src_all || s0 >= s1) return fail(GG_BAD_ARG, "bad source range");
        if (o->want_wvc && (s0 % 32)) return fail(GG_BAD_ARG, "WVC needs a 32-aligned source range");
    }
    const int cap_req = (o && o->max_levels > 0) ? o->max_levels : std::max(e->rows, 1);
    const bool wvc = o && o->want_wvc;
    const bool want_ns = o && o->level_ns;
    const int ns_all = s1 - s0;
    const int nb = (ns_all + e->batch_bits - 1) / e->batch_bits;
    gg_status s = ensure_counters(e, cap_req, nb);
    if (s != GG_OK) return s;
    const int stride = cap_req + 1;      // counts of batch b at [b * stride, (b + 1) * stride)

    (void)cudaGetLastError();  // launch checks below must not see an earlier, unrelated error
    if (e->p_dirty) {
        // New buffers, or a launch that stopped early: the push buffers are
        // zero again only after these four writes.
        const size_t vbytes = (size_t)e->items * sizeof(uint4), fbytes = (size_t)((e->items + 31) / 32) * 4;
        GG_CK(cudaMemsetAsync(e->d_P0, 0, vbytes, st));
        GG_CK(cudaMemsetAsync(e->d_P1, 0, vbytes, st));
        GG_CK(cudaMemsetAsync(e->d_pf0, 0, fbytes, st));
        GG_CK(cudaMemsetAsync(e->d_pf1, 0, fbytes, st));
        e->p_dirty = false;
    }
    if (fault("launch")) return fail(GG_CUDA_ERROR, "injected launch failure");
    const unsigned extra = fault("barrier") ? 1u : 0u;
    const size_t lv = (size_t)cap_req + 1;
    uint64_t d2h = e->off_counts + (size_t)nb * stride * sizeof(unsigned long long);
    if (wvc) d2h += (size_t)nb * stride * sizeof(unsigned);
    if (want_ns) d2h += lv * sizeof(unsigned long long);
    // Walk pass for this evaluation: not with the WVC masks or the distance planes
    // (their per-level bookkeeping lives in the level loop), at most the level cap.
    const int walk_K = (wvc || (x && x->planes)) ? 0 : std::min(e->walk_K, cap_req);
    const int launches = 1 + ((long long)e->rows * e->d > 0 ? 1 : 0) + (walk_K > 0 ? 1 : 0) + (walk_K >= 3 ? 1 : 0);
    void *wall = walk_K > 0 ? walk_all_for(e, walk_K, nb) : nullptr;

    // Everything the GPU does for one evaluation, on `q`: status words zeroed,
    // table -> adjacency (checked), one cooperative launch for every source
    // batch, and one copy back of the status block.
    // The timing events are recorded here only when launching directly; a
    // replayed graph is timed by events recorded around its launch.
    auto enqueue = [&](cudaStream_t q, bool timed) -> gg_status {
        if (timed) GG_CK(cudaEventRecord(e->ev0, q));
        // control block, range-check and symmetry words
        GG_CK(cudaMemsetAsync(e->d_status, 0, sizeof(Ctl) + 3 * sizeof(int), q));   // ctl, bad, asym, wasym
        const long long n = (long long)e->rows * e->d;
        if (e->form == FORM_GRAPH) {
            if (d_table_in != e->d_table)
                GG_CK(cudaMemcpyAsync(e->d_table, d_table_in, e->table_elems * 4, cudaMemcpyDeviceToDevice, q));
            if (n > 0) {
                gg::check_table_kernel<<<(int)std::min<long long>((n + 255) / 256, 4096), 256, 0, q>>>(
                    e->d_table, n, e->rows, e->d_bad);
                GG_CK(cudaGetLastError());
            }
        } else if (n > 0) {
            ExpandArgs x{};
            x.table = d_table_in;
            x.adj = e->d_adj;
            x.form = (e->form == FORM_PART) ? 1 : (e->form == FORM_PIECE ? 2 : 3);
            x.rows = e->rows; x.d = e->d; x.N = e->N; x.M = e->M;
            x.Nx = e->dims[0]; x.Ny = e->dims[1]; x.Nz = e->dims[2];
            x.Mx = e->dims[3]; x.My = e->dims[4]; x.Mz = e->dims[5];
            gg::expand_kernel<<<(int)std::min<long long>((n + 255) / 256, 8192), 256, 0, q>>>(x);
            GG_CK(cudaGetLastError());
        }
        if (want_ns)
            GG_CK(cudaMemsetAsync(e->d_level_ns, 0, lv * sizeof(unsigned long long), q));
        if (walk_K > 0) {
            // blocks add the walk's level counts before any grid barrier
            GG_CK(cudaMemsetAsync(e->d_counts, 0, (size_t)nb * stride * sizeof(unsigned long long), q));
            GG_CK(cudaMemsetAsync(e->d_vtot, 0, (size_t)nb * 3 * sizeof(unsigned long long), q));
            // the walk of all batches needs the table's one-way flag first; h2_kernel
            // takes the check along when its warps see whole neighbour rows
            const long long nh = (long long)e->rows * e->d * e->d;
            const int qd = e->d / 4;
            const bool h2_checks = wall && walk_K >= 3 && e->d % 4 == 0 && (qd & (qd - 1)) == 0 && (nh / 4) % 32 == 0;
            if (walk_K >= 3) {
                gg::h2_kernel<<<(int)std::min<long long>((nh + 255) / 256, 8192), 256, 0, q>>>(
                    e->d_adj, e->d_h2, e->rows, e->d, e->form == FORM_GRAPH ? e->d_bad : nullptr,
                    h2_checks ? e->d_wasym : nullptr);
                GG_CK(cudaGetLastError());
            }
            // the walk index of this evaluation's sources and batches
            gg::WalkIndexArgs wi{};
            wi.adj = e->d_adj;
            wi.h2 = walk_K >= 3 ? e->d_h2 : nullptr;
            wi.inv = x && x->inv ? x->inv : e->d_inv;
            wi.src_first = x && x->inv ? 0 : e->src_first;
            wi.src_begin = s0;
            wi.ns_total = ns_all;
            wi.S = 128 * e->nC;
            wi.div_S = FastDiv((uint32_t)wi.S);
            wi.nb = nb;
            wi.K = walk_K;
            wi.rows = e->rows;
            wi.d = e->d;
            wi.cap = e->walk_cap;
            wi.ent = e->d_went;
            wi.off = e->d_woff;
            wi.off_stride = e->walk_off_stride;
            wi.bad = e->form == FORM_GRAPH ? e->d_bad : nullptr;
            wi.asym = e->walk_vpull && e->walk_own_skip ? e->d_wasym : nullptr;
            // one resident wave of blocks, each striding over the rows
            void *wk = wall ? wall : index_kernel_for(e->d);
            const size_t wsmem = wall ? (size_t)gg::walk_all_smem(walk_K) : 0;
            if (wall) {
                wi.vall = e->d_vall;
                wi.vall_fl = e->d_vall_fl;
                wi.counts = e->d_counts;
                wi.counts_stride = stride;
                // the table's one-way flag first: walk_all_kernel reads it to choose
                // how it counts, the level kernel whether dense levels read own chunks
                wi.asym = nullptr;
                wi.oneway = e->d_wasym;
                if (!h2_checks) {
                    const long long ne = (long long)e->rows * e->d;
                    gg::walk_check_kernel<<<(int)std::min<long long>((ne + 255) / 256, 8192), 256, 0, q>>>(
                        e->d_adj, e->rows, e->d, e->d_wasym, e->form == FORM_GRAPH ? e->d_bad : nullptr);
                    GG_CK(cudaGetLastError());
                }
            }
            int sms = 0, per_sm = 0;
            GG_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device));
            GG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wk, gg::kIndexBlock, wsmem));
            const int wgrid = (int)std::max<long long>(1, std::min<long long>(((long long)e->rows + 7) / 8,
                                                                              (long long)sms * std::max(per_sm, 1)));
            void *wargs[] = {&wi};
            GG_CK(cudaLaunchKernel(wk, dim3(wgrid), dim3(gg::kIndexBlock), wargs, wsmem, q));
        }
        BfsArgs a{};
        a.adj = e->d_adj;
        a.inv = x && x->inv ? x->inv : e->d_inv;
        a.src_first = x && x->inv ? 0 : e->src_first;
        if (x && x->planes) {
            a.planes = x->planes;
            a.nplanes = x->nplanes;
            a.plane_cols = (unsigned)(nb * e->nC);
            a.plane_stride = (unsigned long long)e->rows * a.plane_cols;
        }
        a.src_begin = s0;
        a.ns_total = ns_all;
        a.nb = nb;
        a.V = e->d_V; a.F0 = e->d_F0; a.F1 = e->d_F1;
        a.fl0 = e->d_fl0; a.fl1 = e->d_fl1;
        a.P0 = e->d_P0; a.P1 = e->d_P1; a.pf0 = e->d_pf0; a.pf1 = e->d_pf1;
        // Below ~1M chunks a pull level costs about one grid barrier anyway.
        a.push_ppm = (long long)e->items >= (long long)e->push_min_items ? e->push_ppm : 0;
        a.nf = e->d_nf;
        a.nf2 = e->d_nf2;
        a.asym = e->d_asym;
        a.counts = e->d_counts;
        a.masks = wvc ? e->d_masks : nullptr;
        a.stride = stride;
        a.levels_run = e->d_levels_run;
        a.level_ns = want_ns ? e->d_level_ns : nullptr;
        a.batch_ns = e->d_batch_ns;
        a.ctl = e->d_ctl;
        a.rows = e->rows; a.d = e->d; a.nC = e->nC; a.items = e->items;
        a.div_nc = FastDiv((uint32_t)e->nC);
        a.max_levels = cap_req;
        a.dense_w_ppm = e->dense_w_ppm;
        a.dense_r_ppm = e->dense_r_ppm;
        a.full_skip_ppm = e->full_skip_ppm;
        a.split_ppm = e->split_ppm;
        a.adj_smem_rows = e->adj_smem_rows;
        a.wait_ns = e->wait_ns;
        a.expected = (unsigned)e->grid + extra;
        a.bad = e->form == FORM_GRAPH ? e->d_bad : nullptr;
        a.walk_K = walk_K;
        a.walk_rpg = e->walk_rpg;
        a.walk_smem_off = e->walk_smem_off;
        a.walk_ent = e->d_went;
        a.walk_off = e->d_woff;
        a.walk_cap = e->walk_cap;
        a.walk_off_stride = e->walk_off_stride;
        a.walk_vpull = walk_K > 0 && !wvc ? e->walk_vpull : 0;
        a.walk_asym = a.walk_vpull && e->walk_own_skip ? e->d_wasym : nullptr;
        a.vtot = e->d_vtot;
        a.vall = wall ? e->d_vall : nullptr;
        a.vall_fl = wall ? e->d_vall_fl : nullptr;
        a.third = wall && e->walk_third ? e->d_F0 : nullptr;
        void *args[] = {&a};
        GG_CK(cudaLaunchCooperativeKernel(kernel_for(e->d, a.planes != nullptr), dim3(e->grid), dim3(gg::kBlock), args,
                                          wall ? (size_t)e->walk_smem_off : e->smem_bytes, q));
        if (timed) GG_CK(cudaEventRecord(e->ev1, q));
        // One copy back: control block, status words, per-batch levels and
        // times, and the counts of every batch (cap_req + 1 each).
        GG_CK(cudaMemcpyAsync(e->h_status, e->d_status, e->off_counts + (size_t)nb * stride * 8,
                              cudaMemcpyDeviceToHost, q));
        if (wvc)
            GG_CK(cudaMemcpyAsync(e->h_masks, e->d_masks, (size_t)nb * stride * sizeof(unsigned),
                                  cudaMemcpyDeviceToHost, q));
        if (want_ns)
            GG_CK(cudaMemcpyAsync(e->h_level_ns, e->d_level_ns, lv * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, q));
        return GG_OK;
    };

    // Repeated evaluations of one shape replay a captured CUDA graph of the
    // same work (one launch call instead of about eight).  Anything that
    // changes the work -- the table pointer, the source range, the level cap,
    // the outputs asked for, reallocated buffers -- captures a new graph.
    const EvalKey key{d_table_in, e->d_status, e->d_V, x ? (const void *)x->inv : nullptr,
                      x ? (const void *)x->planes : nullptr, s0, ns_all, cap_req, wvc, want_ns};
    e->p_dirty = true;  // until the launch is known to have finished cleanly
    bool replayed = false;
    if (e->use_graph && !extra && !(x && x->no_graph)) {
        if (!e->graph_exec || !(key == e->graph_key)) {
            if (e->graph_exec) { cudaGraphExecDestroy(e->graph_exec); e->graph_exec = nullptr; }
            cudaGraph_t g = nullptr;
            gg_status cs = GG_CUDA_ERROR;
            if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                cs = enqueue(st, false);
                const cudaError_t ce = cudaStreamEndCapture(st, &g);
                if (ce != cudaSuccess) cs = GG_CUDA_ERROR;
            }
            if (cs == GG_OK && g && cudaGraphInstantiate(&e->graph_exec, g, 0) == cudaSuccess) {
                e->graph_key = key;
            } else {
                e->graph_exec = nullptr;
                e->use_graph = false;   // this device or driver cannot capture it: launch directly
            }
            if (g) cudaGraphDestroy(g);
            (void)cudaGetLastError();
        }
        if (e->graph_exec) {
            GG_CK(cudaEventRecord(e->ev0, st));
            GG_CK(cudaGraphLaunch(e->graph_exec, st));
            GG_CK(cudaEventRecord(e->ev1, st));
            replayed = true;
        }
    }
    if (!replayed) {
        gg_status es = enqueue(st, true);
        if (es != GG_OK) return es;
    }
    e->last_d2h = d2h;
    GG_CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    GG_CK(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
    e->last_ms = ms;
    e->last_launches = launches;
    e->last_batches = nb;

    if (e->form == FORM_GRAPH && *e->h_bad)
        return fail(GG_BAD_ARG, "adjacency entry outside [0, N)");
    if (e->h_ctl->err)
        return fail(GG_TIMEOUT, "grid barrier wait exceeded its limit at level " +
                                    std::to_string(e->h_ctl->err_level));
    e->p_dirty = false;

    // Exact fold of the per-batch level counters.
    gg_result R{};
    R.scale = e->scale;
    R.pairs = (uint64_t)ns_all * (uint64_t)e->rows;
    R.n_sources = ns_all;
    R.batches = nb;
    R.wvc = -1;
    std::vector<int> lev(nb, 0);
    std::vector<unsigned long long> agg(cap_req + 1, 0ull);
    for (int b = 0; b < nb; ++b) {
        const unsigned long long *c = e->h_counts + (size_t)b * stride;
        const int run = e->h_levels_run[b];
        int last = 0;
        for (int L = 0; L <= run && L <= cap_req; ++L) {
            R.reached += c[L];
            R.total += (uint64_t)L * c[L];
            agg[L] += c[L];
            if (L > 0 && c[L]) last = L;
        }
        lev[b] = last;
        R.level_steps += run;
        R.levels = std::max(R.levels, last);
        if (run >= cap_req && c[cap_req]) R.capped = 1;
    }
    R.connected = (!R.capped && R.reached == R.pairs) ? 1 : 0;
    if (wvc) {
        // Lane-aggregated completion masks across batches: a batch's mask stays
        // at its final value after its last level.
        auto mask_at = [&](int L) {
            unsigned m = 0xffffffffu;
            for (int b = 0; b < nb; ++b)
                m &= e->h_masks[(size_t)b * stride + std::min(L, lev[b])];
            return m;
        };
        const int E = R.levels;
        R.wvc = E > 0 ? __builtin_popcount(mask_at(E - 1) ^ mask_at(E)) : 0;
    }
    if (o && o->level_counts)
        std::memcpy(o->level_counts, agg.data(), (size_t)(cap_req + 1) * sizeof(uint64_t));
    if (want_ns)
        std::memcpy(o->level_ns, e->h_level_ns, (size_t)(cap_req + 1) * sizeof(uint64_t));
    *r = R;
    return GG_OK;
}

// A host table into the pinned staging buffer, split over a few threads when it is
// large (one thread's copy bounded a 2 MiB table at about 0.1 ms a call).
void copy_to_pinned(void *dst, const void *src, size_t bytes) {
    constexpr size_t kPart = 256u << 10;
    const int parts = (int)std::min<size_t>(8, bytes / kPart);
    if (parts <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
#pragma omp parallel for num_threads(parts) schedule(static)
    for (int i = 0; i < parts; ++i) {
        const size_t lo = bytes * (size_t)i / (size_t)parts, hi = bytes * (size_t)(i + 1) / (size_t)parts;
        std::memcpy(static_cast<char *>(dst) + lo, static_cast<const char *>(src) + lo, hi - lo);
    }
}

gg_status eval_host(gg_engine *e, const int32_t *table, const gg_eval_opts *o, gg_result *r) {
    if (!e || !r) return fail(GG_BAD_ARG, "null engine or result");
    if (e->table_elems && !table) return fail(GG_BAD_ARG, "null table");
    GG_CK(cudaSetDevice(e->device));
    if (e->table_elems) {
        copy_to_pinned(e->h_table, table, e->table_elems * sizeof(int32_t));
        GG_CK(cudaMemcpyAsync(e->d_table, e->h_table, e->table_elems * sizeof(int32_t),
                              cudaMemcpyHostToDevice, e->stream));
    }
    gg_status s = run_eval(e, e->d_table, o, r, e->stream);
    e->last_h2d = e->table_elems * sizeof(int32_t);
    return s;
}

double aspl_of(uint64_t total, uint64_t scale, int N) {
    // total *= N/M; double(total)/(int64_t(N)*(N-1))  (cudaASPLconv.cu:241-242)
    const int64_t t = (int64_t)(total * scale);
    return double(t) / (int64_t(N) * (N - 1));
}

// The level loop `for(step=1; step<100; ...)` of cudaASPLconv::diameterASPL and
// its piece/box twins (cudaASPLconv.cu:208-242, cudaASPLpiece.cu:181-215,
// cudaASPLbox.cu:191-225).
gg_status lifted_diameter_aspl(gg_engine *e, const int32_t *table, int *diameter, double *aspl) {
    if (!diameter || !aspl) return fail(GG_BAD_ARG, "null output");
    gg_eval_opts o{};
    o.max_levels = 99;
    gg_result r;
    gg_status s = eval_host(e, table, &o, &r);
    if (s != GG_OK) return s;
    if (r.capped) {  // step 99 still found pairs: loop ends, diameter stays 1e8
        *diameter = kSentinel;
        *aspl = aspl_of(r.total, r.scale, e->N);
    } else if (!r.connected) {
        *diameter = kSentinel;
        *aspl = 100000000.0;
    } else {
        *diameter = r.levels;
        *aspl = aspl_of(r.total, r.scale, e->N);
    }
    return GG_OK;
}

}  // namespace

namespace gg {
gg_status engine_eval(gg_engine *e, const int32_t *d_table, const gg_eval_opts *o, gg_result *r,
                      cudaStream_t st, const EvalExtra *x) {
    if (!e || !r || !d_table) return fail(GG_BAD_ARG, "null argument");
    GG_CK(cudaSetDevice(e->device));
    return run_eval(e, d_table, o, r, st ? st : e->stream, x);
}
int engine_plane_cols(const gg_engine *e) {
    const int n_src = (int)e->reps.size();
    return ((n_src + e->batch_bits - 1) / e->batch_bits) * e->nC;
}
}  // namespace gg

extern "C" {

int gg_abi_version(void) { return GG_ABI_VERSION; }

const char *gg_status_str(gg_status s) {
    switch (s) {
        case GG_OK: return "ok";
        case GG_BAD_ARG: return "bad argument";
        case GG_CUDA_ERROR: return "CUDA error";
        case GG_TIMEOUT: return "bounded wait timed out";
        case GG_OUT_OF_MEMORY: return "out of memory";
        case GG_NO_DEVICE: return "no device";
    }
    return "unknown status";
}

const char *gg_last_error(void) { return g_err.c_str(); }

gg_status gg_graph_create(int N, int degree_max, int device, gg_engine **out) {
    if (!out) return fail(GG_BAD_ARG, "null out");
    *out = nullptr;
    if (N < 1 || degree_max < 0) return fail(GG_BAD_ARG, "need N >= 1, degree_max >= 0");
    gg_engine *e = new gg_engine();
    e->form = FORM_GRAPH; e->device = device;
    e->N = N; e->M = N; e->d = degree_max; e->rows = N; e->scale = 1;
    e->table_elems = (size_t)N * degree_max;
    e->reps.resize(N);
    for (int i = 0; i < N; ++i) e->reps[i] = i;
    return finish_create(e, out);
}

gg_status gg_conv_create(int N, int M, int degree, int device, gg_engine **out) {
    if (!out) return fail(GG_BAD_ARG, "null out");
    *out = nullptr;
    if (N < 1 || M < 1 || M > N || degree < 0) return fail(GG_BAD_ARG, "need 1 <= M <= N, degree >= 0");
    gg_engine *e = new gg_engine();
    e->form = FORM_PART; e->device = device;
    e->N = N; e->M = M; e->d = degree; e->rows = N; e->scale = (uint64_t)(N / M);
    e->table_elems = (size_t)M * degree;
    e->reps.resize(M);
    for (int i = 0; i < M; ++i) e->reps[i] = i;
    return finish_create(e, out);
}

gg_status gg_beamer_create(int N, int M, int degree, int device, gg_engine **out) {
    if (!out) return fail(GG_BAD_ARG, "null out");
    *out = nullptr;
    if (N < 1 || M < 1 || M > N || degree < 0 || N > kBeamerRows)
        return fail(GG_BAD_ARG, "need 1 <= M <= N <= 10^6, degree >= 0");
    gg_engine *e = new gg_engine();
    e->form = FORM_PART; e->device = device;
    e->N = N; e->M = M; e->d = degree; e->rows = kBeamerRows; e->scale = (uint64_t)(N / M);
    e->table_elems = (size_t)M * degree;
    e->reps.resize(M);
    for (int i = 0; i < M; ++i) e->reps[i] = i;
    return finish_create(e, out);
}

gg_status gg_piece_create(int Nx, int Ny, int Mx, int My, int degree, int device, gg_engine **out) {
    if (!out) return fail(GG_BAD_ARG, "null out");
    *out = nullptr;
    if (Nx < 1 || Ny < 1 || Mx < 1 || My < 1 || Mx > Nx || My > Ny || degree < 0 ||
        (long long)Nx * Ny >= (1ll << 31))
        return fail(GG_BAD_ARG, "need 1 <= Mx <= Nx, 1 <= My <= Ny, degree >= 0");
    gg_engine *e = new gg_engine();
    e->form = FORM_PIECE; e->device = device;
    e->dims[0] = Nx; e->dims[1] = Ny; e->dims[2] = 1; e->dims[3] = Mx; e->dims[4] = My; e->dims[5] = 1;
    e->N = Nx * Ny; e->M = Mx * My; e->d = degree; e->rows = e->N;
    e->scale = (uint64_t)(e->N / e->M);
    e->table_elems = (size_t)e->M * degree * 2;
    // representatives: corner tile, source index x*My+y (cudaASPLpiece.cu:23-29)
    for (int x = 0; x < Mx; ++x)
        for (int y = 0; y < My; ++y) e->reps.push_back(x * Ny + y);
    return finish_create(e, out);
}

gg_status gg_box_create(int Nx, int Ny, int Nz, int Mx, int My, int Mz, int degree, int device,
                        gg_engine **out) {
    if (!out) return fail(GG_BAD_ARG, "null out");
    *out = nullptr;
    if (Nx < 1 || Ny < 1 || Nz < 1 || Mx < 1 || My < 1 || Mz < 1 || Mx > Nx || My > Ny || Mz > Nz ||
        degree < 0 || (long long)Nx * Ny * Nz >= (1ll << 31))
        return fail(GG_BAD_ARG, "need 1 <= M* <= N*, degree >= 0");
    gg_engine *e = new gg_engine();
    e->form = FORM_BOX; e->device = device;
    e->dims[0] = Nx; e->dims[1] = Ny; e->dims[2] = Nz; e->dims[3] = Mx; e->dims[4] = My; e->dims[5] = Mz;
    e->N = Nx * Ny * Nz; e->M = Mx * My * Mz; e->d = degree; e->rows = e->N;
    e->scale = (uint64_t)(e->N / e->M);
    e->table_elems = (size_t)e->M * degree * 3;
    // representatives: corner tile, source index (x*My+y)*Mz+z (cudaASPLbox.cu:25-32)
    for (int x = 0; x < Mx; ++x)
        for (int y = 0; y < My; ++y)
            for (int z = 0; z < Mz; ++z) e->reps.push_back((x * Ny + y) * Nz + z);
    return finish_create(e, out);
}

gg_status gg_destroy(gg_engine *e) {
    destroy_all(e);
    return GG_OK;
}


gg_status gg_eval(gg_engine *e, const int32_t *table, const gg_eval_opts *opts, gg_result *out) {
    return eval_host(e, table, opts, out);
}

gg_status gg_eval_device(gg_engine *e, const int32_t *d_table, const gg_eval_opts *opts,
                         gg_result *out, void *stream) {
    if (!e || !out) return fail(GG_BAD_ARG, "null engine or result");
    if (e->table_elems && !d_table) return fail(GG_BAD_ARG, "null table");
    GG_CK(cudaSetDevice(e->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : e->stream;
    gg_status s = run_eval(e, d_table ? d_table : e->d_table, opts, out, st);
    e->last_h2d = 0;
    return s;
}

gg_status gg_last_transfer_bytes(gg_engine *e, uint64_t *h2d, uint64_t *d2h) {
    if (!e || !h2d || !d2h) return fail(GG_BAD_ARG, "null argument");
    *h2d = e->last_h2d;
    *d2h = e->last_d2h;
    return GG_OK;
}

gg_status gg_last_device_ms(gg_engine *e, double *ms) {
    if (!e || !ms) return fail(GG_BAD_ARG, "null argument");
    *ms = e->last_ms;
    return GG_OK;
}

gg_status gg_last_batch_ns(gg_engine *e, uint64_t *ns, int n) {
    if (!e || !ns || n < 0) return fail(GG_BAD_ARG, "bad arguments");
    for (int b = 0; b < n && b < e->last_batches; ++b) {
        ns[2 * b] = e->h_batch_ns[2 * b];
        ns[2 * b + 1] = e->h_batch_ns[2 * b + 1];
    }
    return GG_OK;
}

gg_status gg_last_launches(gg_engine *e, int *launches) {
    if (!e || !launches) return fail(GG_BAD_ARG, "null argument");
    *launches = e->last_launches;
    return GG_OK;
}

gg_status gg_set_batch_sources(gg_engine *e, int sources) {
    if (!e || sources < 0) return fail(GG_BAD_ARG, "bad batch width");
    GG_CK(cudaSetDevice(e->device));
    GG_CK(cudaStreamSynchronize(e->stream));
    return plan(e, sources);
}

gg_status gg_autotune(gg_engine *e, const int32_t *table, int trials, int *best_sources, double *best_ms) {
    if (!e || (e->table_elems && !table) || trials < 1) return fail(GG_BAD_ARG, "bad arguments");
    GG_CK(cudaSetDevice(e->device));
    GG_CK(cudaStreamSynchronize(e->stream));
    const int n_src = (int)e->reps.size();
    // the L2-resident width the default plan picks, and its neighbours
    int base = 0, max_bps = 0;
    {
        const int keep = e->batch_bits, keep_bps = e->bps_cap, keep_walk = e->walk_pref;
        e->bps_cap = 0;
        e->walk_pref = -1;
        gg_status s = plan(e, 0);
        if (s != GG_OK) return s;
        base = e->batch_bits;
        GG_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&max_bps, kernel_for(e->d), gg::kBlock,
                                                            e->smem_bytes));
        e->bps_cap = keep_bps;
        e->walk_pref = keep_walk;
        if (keep > 0) { s = plan(e, keep); if (s != GG_OK) return s; }
    }
    std::vector<int> widths;
    for (double f : {0.25, 0.5, 1.0, 2.0, 4.0}) {
        int w = (int)(base * f);
        w = std::max(128, std::min(((w + 127) / 128) * 128, ((n_src + 127) / 128) * 128));
        widths.push_back(w);
    }
    widths.push_back(((n_src + 127) / 128) * 128);
    std::sort(widths.begin(), widths.end());
    widths.erase(std::unique(widths.begin(), widths.end()), widths.end());
    std::vector<int> bps_opts;   // 0 = as many as fit, then one and two fewer
    bps_opts.push_back(0);
    for (int k = 1; k <= 2; ++k)
        if (max_bps - k >= 1) bps_opts.push_back(max_bps - k);
    if (e->table_elems) {
        copy_to_pinned(e->h_table, table, e->table_elems * sizeof(int32_t));
        GG_CK(cudaMemcpyAsync(e->d_table, e->h_table, e->table_elems * sizeof(int32_t),
                              cudaMemcpyHostToDevice, e->stream));
    }
    int best = 0, best_bps = 0, best_walk = -1;
    double best_t = 1e300;
    gg_result r;
    for (int w : widths) {
        if ((long long)e->rows * (w / 128) >= (1ll << 31)) continue;
        for (int bps : bps_opts) {
            bool auto_walks = true;
            for (int walk : {-1, 0}) {
                if (walk == 0 && !auto_walks) continue;   // the automatic plan has no walk already
                e->bps_cap = bps;
                e->walk_pref = walk;
                gg_status s = plan(e, w);
                if (s == GG_OUT_OF_MEMORY) { (void)cudaGetLastError(); break; }  // too wide for this device
                if (s != GG_OK) return s;
                if (walk == -1) auto_walks = e->walk_K > 0;
                s = run_eval(e, e->d_table, nullptr, &r, e->stream);  // warm
                if (s != GG_OK) return s;
                double t = 1e300;
                for (int k = 0; k < trials; ++k) {
                    s = run_eval(e, e->d_table, nullptr, &r, e->stream);
                    if (s != GG_OK) return s;
                    t = std::min(t, e->last_ms);
                }
                if (t < best_t) { best_t = t; best = w; best_bps = bps; best_walk = walk; }
            }
        }
    }
    if (!best) return fail(GG_OUT_OF_MEMORY, "no batch width fits");
    e->bps_cap = best_bps;
    e->walk_pref = best_walk;
    gg_status s = plan(e, best);
    if (s != GG_OK) return s;
    gg::tune_put(engine_tune_key(e), {best, best_bps, best_walk});
    if (best_sources) *best_sources = best;
    if (best_ms) *best_ms = best_t;
    return GG_OK;
}

gg_status gg_engine_plan(gg_engine *e, int *batch_sources, int *blocks_per_sm, int *walk_levels) {
    if (!e) return fail(GG_BAD_ARG, "null engine");
    if (batch_sources) *batch_sources = e->batch_bits;
    if (blocks_per_sm) *blocks_per_sm = e->grid;
    if (walk_levels) *walk_levels = e->walk_K;
    int sms = 0;
    if (blocks_per_sm && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device) == cudaSuccess &&
        sms > 0)
        *blocks_per_sm = (e->grid + sms - 1) / sms;
    else
        (void)cudaGetLastError();
    return GG_OK;
}

gg_status gg_set_wait_limit_ms(gg_engine *e, int ms) {
    if (!e || ms < 1) return fail(GG_BAD_ARG, "bad wait limit");
    e->wait_ns = (long long)ms * 1000000ll;
    invalidate_graph(e);
    return GG_OK;
}

// cudaASPLgraph::calc (cudaASPLgraph.cu:141-199)
gg_status gg_graph_calc(gg_engine *e, const int32_t *adj, int *diameter, int64_t *total) {
    if (!e || !diameter || !total) return fail(GG_BAD_ARG, "null argument");
    if (e->form != FORM_GRAPH) return fail(GG_BAD_ARG, "not a graph engine");
    gg_eval_opts o{};
    o.max_levels = 199;
    gg_result r;
    gg_status s = eval_host(e, adj, &o, &r);
    if (s != GG_OK) return s;
    if (!r.capped && r.connected) {
        *diameter = r.levels;
        *total = (int64_t)r.total;
        return GG_OK;
    }
    // Some source hits the 199-step limit or misses a vertex: the reference
    // answers for the first 1024-source chunk (in source order) that does
    // either, so resolve chunk by chunk with the table already on the device.
    for (int off = 0; off < e->N; off += 1024) {
        gg_eval_opts c{};
        c.max_levels = 199;
        c.src_begin = off;
        c.src_end = std::min(off + 1024, e->N);
        gg_result rc;
        s = run_eval(e, e->d_table, &c, &rc, e->stream);
        if (s != GG_OK) return s;
        if (rc.capped) { *diameter = -2; *total = -2; return GG_OK; }
        if (!rc.connected) { *diameter = -1; *total = -1; return GG_OK; }
    }
    return fail(GG_CUDA_ERROR, "inconsistent chunk resolution");
}

gg_status gg_conv_calc(gg_engine *e, const int32_t *diffs, double *aspl) {
    if (!e || !aspl) return fail(GG_BAD_ARG, "null argument");
    gg_eval_opts o{};
    o.max_levels = 99;
    gg_result r;
    gg_status s = eval_host(e, diffs, &o, &r);
    if (s != GG_OK) return s;
    if (!r.capped && !r.connected) *aspl = 1e9;  // cudaASPLconv.cu:182
    else *aspl = aspl_of(r.total, r.scale, e->N);
    return GG_OK;
}

gg_status gg_conv_diameter_aspl(gg_engine *e, const int32_t *diffs, int *diameter, double *aspl) {
    if (!e) return fail(GG_BAD_ARG, "null engine");
    if (e->form != FORM_PART) return fail(GG_BAD_ARG, "not a part engine");
    return lifted_diameter_aspl(e, diffs, diameter, aspl);
}

// cudaASPLconv::WVCdiameterASPL (cudaASPLconv.cu:244-308)
gg_status gg_conv_wvc_diameter_aspl(gg_engine *e, const int32_t *diffs, int *wvc, int *diameter,
                                    double *aspl) {
    if (!e || !wvc || !diameter || !aspl) return fail(GG_BAD_ARG, "null argument");
    if (e->form != FORM_PART) return fail(GG_BAD_ARG, "not a part engine");
    gg_eval_opts o{};
    o.max_levels = 100;
    o.want_wvc = 1;
    gg_result r;
    gg_status s = eval_host(e, diffs, &o, &r);
    if (s != GG_OK) return s;
    if (r.capped || !r.connected) {
        *wvc = kSentinel; *diameter = kSentinel; *aspl = 100000000.0;
    } else {
        *wvc = r.wvc; *diameter = r.levels; *aspl = aspl_of(r.total, r.scale, e->N);
    }
    return GG_OK;
}

gg_status gg_piece_diameter_aspl(gg_engine *e, const int32_t *vals, int *diameter, double *aspl) {
    if (!e) return fail(GG_BAD_ARG, "null engine");
    if (e->form != FORM_PIECE) return fail(GG_BAD_ARG, "not a piece engine");
    return lifted_diameter_aspl(e, vals, diameter, aspl);
}

gg_status gg_box_diameter_aspl(gg_engine *e, const int32_t *vals, int *diameter, double *aspl) {
    if (!e) return fail(GG_BAD_ARG, "null engine");
    if (e->form != FORM_BOX) return fail(GG_BAD_ARG, "not a box engine");
    return lifted_diameter_aspl(e, vals, diameter, aspl);
}

// cudaASPLbeamer::calc (cudaASPLbeamer.cu:71-84)
gg_status gg_beamer_calc(gg_engine *e, const int32_t *diffs, int regular, double *aspl) {
    if (!e || !aspl) return fail(GG_BAD_ARG, "null argument");
    if (e->form != FORM_PART || e->rows != kBeamerRows) return fail(GG_BAD_ARG, "not a beamer engine");
    if (!regular) { *aspl = 100000000; return GG_OK; }
    gg_eval_opts o{};
    o.max_levels = kBeamerLevels;
    gg_result r;
    gg_status s = eval_host(e, diffs, &o, &r);
    if (s != GG_OK) return s;
    *aspl = aspl_of(r.total, r.scale, e->N);
    return GG_OK;
}

}  // extern "C"
