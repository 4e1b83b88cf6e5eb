// gg_inc.cu -- incremental exact evaluation of 2-opt moves on one plain graph.
//
// A full evaluation of the current graph also writes its distance matrix as
// bit-planes (4 planes: distances up to 15).  A 2-opt move (remove (a,b), (c,d);
// add (a,p), (b,q)) changes the distances from source s only if
//   * a removed edge joins two consecutive BFS levels of s and its deeper end has
//     no other neighbour on the shallower level (else every vertex keeps a parent
//     one level up, and by induction over the levels no distance grows), or
//   * an added edge joins vertices whose distances from s differ by 2 or more
//     (else no path gets shorter).
// Only those sources are searched again, on the new graph.  The new total is the
// old total minus the old distance sums of those sources plus their new sums; the
// new diameter is the larger of their new eccentricities and the old
// eccentricities of the other sources.  Every source's distance sum and
// eccentricity are computed once per current graph from the planes (row
// reductions, gg_planes.cuh), so a move reads only the planes' columns of its
// endpoints.  Exact whenever the current graph is symmetric and connected with
// diameter <= 15; otherwise a call evaluates the moved graph in full.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "gg.h"
#include "gg_internal.h"
#include "gg_kernels.cuh"
#include "gg_planes.cuh"

namespace {

constexpr int kPlanes = 4;

struct IncStatus {
    unsigned long long old_sum;   // distance sum of the affected sources (current graph)
    unsigned count;               // affected sources
    unsigned max_other;           // largest distance from an unaffected source
};

__device__ __forceinline__ unsigned dist_of(const uint32_t *pw, unsigned long long pstride_w,
                                            unsigned cols4, unsigned x, unsigned s) {
    // u32 word of (vertex x, source s) in plane k: (k * pstride + x * cols) * 4 + s / 32
    const size_t base = (size_t)x * cols4 + (s >> 5);
    unsigned dv = 0;
#pragma unroll
    for (int k = 0; k < kPlanes; ++k) dv |= ((__ldg(pw + (size_t)k * pstride_w + base) >> (s & 31u)) & 1u) << k;
    return dv;
}

// One thread per source: the test above.  Gives each affected source a position
// in the list of affected sources (inv[s], -1 preset) and adds its old distance
// sum; the unaffected sources give the largest eccentricity that stays.
__global__ void affected_kernel(const uint32_t *planes, unsigned long long pstride_w, unsigned cols4,
                                const int32_t *adj, int n, int d, gg_swap sw, const unsigned *rowsum,
                                const unsigned *ecc, int32_t *inv, IncStatus *st) {
    const unsigned s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = s < (unsigned)n;
    bool aff = false;
    if (live) {
        const int a = sw.a, b = sw.b, c = sw.c, dd = sw.d;
        const int p = sw.mode ? dd : c, q = sw.mode ? c : dd;
        const int ends[2][2] = {{a, b}, {c, dd}};
        for (int e = 0; e < 2 && !aff; ++e) {
            const int x = ends[e][0], y = ends[e][1];
            const unsigned dx = dist_of(planes, pstride_w, cols4, x, s), dy = dist_of(planes, pstride_w, cols4, y, s);
            if (dx == dy) continue;
            const int lo = dx < dy ? x : y, hi = dx < dy ? y : x;
            const unsigned l = min(dx, dy);
            // another neighbour of hi one level up (the removed slot is the first
            // occurrence of lo in hi's row)
            bool other = false, skipped = false;
            for (int i = 0; i < d && !other; ++i) {
                const int z = __ldg(adj + (size_t)hi * d + i);
                if (z == lo && !skipped) { skipped = true; continue; }
                other = dist_of(planes, pstride_w, cols4, (unsigned)z, s) == l;
            }
            aff = !other;
        }
        if (!aff) {
            const unsigned da = dist_of(planes, pstride_w, cols4, a, s), dp = dist_of(planes, pstride_w, cols4, p, s);
            const unsigned db = dist_of(planes, pstride_w, cols4, b, s), dq = dist_of(planes, pstride_w, cols4, q, s);
            aff = (da > dp ? da - dp : dp - da) >= 2u || (db > dq ? db - dq : dq - db) >= 2u;
        }
    }
    // one set of atomics per warp
    const unsigned am = __ballot_sync(0xffffffffu, aff);
    const unsigned sum = __reduce_add_sync(0xffffffffu, aff ? __ldg(rowsum + s) : 0u);
    const unsigned mx = __reduce_max_sync(0xffffffffu, live && !aff ? __ldg(ecc + s) : 0u);
    const unsigned lane = threadIdx.x & 31u;
    unsigned first = 0;
    if (lane == 0) {
        if (am) {
            first = atomicAdd(&st->count, (unsigned)__popc(am));
            atomicAdd(&st->old_sum, (unsigned long long)sum);
        }
        atomicMax(&st->max_other, mx);
    }
    first = __shfl_sync(0xffffffffu, first, 0);
    if (aff) inv[s] = (int32_t)(first + __popc(am & ((1u << lane) - 1u)));
}

// The candidate's adjacency: the current rows with the four slots of the move
// replaced (first occurrence, as gg_swap specifies).
__global__ void apply_swap_kernel(int32_t *adj, int d, gg_swap sw) {
    const int i = threadIdx.x;
    if (i >= 4) return;
    const int rows[4] = {sw.a, sw.b, sw.c, sw.d};
    const int from[4] = {sw.b, sw.a, sw.d, sw.c};
    const int to0[4] = {sw.c, sw.d, sw.a, sw.b};
    const int to1[4] = {sw.d, sw.c, sw.b, sw.a};
    int32_t *row = adj + (size_t)rows[i] * d;
    for (int k = 0; k < d; ++k)
        if (row[k] == from[i]) { row[k] = sw.mode ? to1[i] : to0[i]; break; }
}

gg_status ifail(gg_status s, const std::string &m) {
    (void)cudaGetLastError();
    gg::set_last_error(m.c_str());
    return s;
}

#define GI_CK(call)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return ifail(e_ == cudaErrorMemoryAllocation ? GG_OUT_OF_MEMORY : GG_CUDA_ERROR, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));           \
    } while (0)

}  // namespace

struct gg_inc {
    int n = 0, d = 0, device = 0;
    gg_engine *eng = nullptr;         // full evaluations and searches from a source list
    cudaStream_t stream = nullptr;
    std::vector<int32_t> h_adj;       // current graph (host copy, validates moves)
    int32_t *d_adj = nullptr, *d_cand = nullptr, *d_inv = nullptr;
    unsigned *d_stats = nullptr;      // [2][n]: distance sum, eccentricity of each source
    int *d_asym = nullptr, *h_asym = nullptr;
    uint4 *d_planes = nullptr;
    unsigned cols = 0;                // plane columns (chunks of 128 sources)
    IncStatus *d_st = nullptr, *h_st = nullptr;
    bool planes_ok = false;           // symmetric, connected, diameter <= 15
    gg_result cur{};                  // current graph's exact counts
};

namespace {

void inc_free(gg_inc *h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->eng) gg_destroy(h->eng);
    cudaFree(h->d_adj); cudaFree(h->d_cand); cudaFree(h->d_inv); cudaFree(h->d_stats);
    cudaFree(h->d_planes); cudaFree(h->d_st); cudaFreeHost(h->h_st);
    cudaFree(h->d_asym); cudaFreeHost(h->h_asym);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

// Full evaluation of the current graph, writing the distance planes.
gg_status inc_rebuild(gg_inc *h) {
    gg_eval_opts o{};
    o.max_levels = 199;               // cudaASPLgraph's cap (cudaASPLgraph.cu:190)
    gg::EvalExtra x;
    x.planes = h->d_planes;
    x.nplanes = kPlanes;
    x.no_graph = true;
    gg_status s = gg::engine_eval(h->eng, h->d_adj, &o, &h->cur, h->stream, &x);
    if (s != GG_OK) return s;
    h->planes_ok = false;
    if (!h->cur.connected || h->cur.levels >= (1 << kPlanes)) return GG_OK;
    // the table passed the engine's range check; the row reductions need a
    // symmetric distance matrix
    const cudaStream_t st = h->stream;
    const long long ent = (long long)h->n * h->d;
    GI_CK(cudaMemsetAsync(h->d_asym, 0, sizeof(int), st));
    table_symmetry<<<(int)((ent + 255) / 256), 256, 0, st>>>(h->d_adj, h->n, h->d, h->d_asym);
    GI_CK(cudaGetLastError());
    int sms = 0;
    GI_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    plane_row_stats<kPlanes><<<plane_row_stats_grid(h->n, sms), 256, 0, st>>>(
        h->d_planes, (unsigned long long)h->n * h->cols, h->cols, h->n, h->d_stats, h->d_stats + h->n);
    GI_CK(cudaGetLastError());
    GI_CK(cudaMemcpyAsync(h->h_asym, h->d_asym, sizeof(int), cudaMemcpyDeviceToHost, st));
    GI_CK(cudaStreamSynchronize(st));
    h->planes_ok = *h->h_asym == 0;
    return GG_OK;
}

gg_status check_swap(const gg_inc *h, const gg_swap *sw) {
    const int v[4] = {sw->a, sw->b, sw->c, sw->d};
    for (int i = 0; i < 4; ++i)
        if (v[i] < 0 || v[i] >= h->n) return ifail(GG_BAD_ARG, "move vertex out of range");
    for (int i = 0; i < 4; ++i)
        for (int j = i + 1; j < 4; ++j)
            if (v[i] == v[j]) return ifail(GG_BAD_ARG, "move needs four distinct vertices");
    if (sw->mode != 0 && sw->mode != 1) return ifail(GG_BAD_ARG, "move mode must be 0 or 1");
    auto has = [&](int x, int y) {
        for (int k = 0; k < h->d; ++k)
            if (h->h_adj[(size_t)x * h->d + k] == y) return true;
        return false;
    };
    if (!has(sw->a, sw->b) || !has(sw->b, sw->a) || !has(sw->c, sw->d) || !has(sw->d, sw->c))
        return ifail(GG_BAD_ARG, "move removes an edge the graph does not have");
    return GG_OK;
}

void apply_host(std::vector<int32_t> &adj, int d, const gg_swap &sw) {
    const int rows[4] = {sw.a, sw.b, sw.c, sw.d};
    const int from[4] = {sw.b, sw.a, sw.d, sw.c};
    const int to0[4] = {sw.c, sw.d, sw.a, sw.b};
    const int to1[4] = {sw.d, sw.c, sw.b, sw.a};
    for (int i = 0; i < 4; ++i)
        for (int k = 0; k < d; ++k)
            if (adj[(size_t)rows[i] * d + k] == from[i]) {
                adj[(size_t)rows[i] * d + k] = sw.mode ? to1[i] : to0[i];
                break;
            }
}

}  // namespace

extern "C" {

gg_status gg_inc_create(int n, int degree, int device, gg_inc **out) {
    if (!out || n < 2 || degree < 1) return ifail(GG_BAD_ARG, "need n >= 2, degree >= 1");
    *out = nullptr;
    gg_inc *h = new gg_inc();
    h->n = n; h->d = degree; h->device = device;
    gg_status s = gg_graph_create(n, degree, device, &h->eng);
    if (s != GG_OK) { inc_free(h); return s; }
    if (cudaSetDevice(device) != cudaSuccess) { inc_free(h); return ifail(GG_NO_DEVICE, "cudaSetDevice failed"); }
    h->cols = (unsigned)gg::engine_plane_cols(h->eng);
    const size_t adj_b = (size_t)n * degree * sizeof(int32_t);
    const size_t plane_b = (size_t)kPlanes * n * h->cols * sizeof(uint4);
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_adj, adj_b);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_cand, adj_b);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_inv, (size_t)n * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_stats, 2 * (size_t)n * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_asym, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_asym, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_planes, plane_b);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_st, sizeof(IncStatus));
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_st, sizeof(IncStatus));
    if (e != cudaSuccess) {
        inc_free(h);
        return ifail(e == cudaErrorMemoryAllocation ? GG_OUT_OF_MEMORY : GG_CUDA_ERROR, cudaGetErrorString(e));
    }
    *out = h;
    return GG_OK;
}

gg_status gg_inc_set_graph(gg_inc *h, const int32_t *adj, gg_result *r) {
    if (!h || !adj) return ifail(GG_BAD_ARG, "null argument");
    GI_CK(cudaSetDevice(h->device));
    h->h_adj.assign(adj, adj + (size_t)h->n * h->d);
    GI_CK(cudaMemcpyAsync(h->d_adj, h->h_adj.data(), h->h_adj.size() * 4, cudaMemcpyHostToDevice, h->stream));
    gg_status s = inc_rebuild(h);
    if (s != GG_OK) return s;
    if (r) *r = h->cur;
    return GG_OK;
}

gg_status gg_inc_eval(gg_inc *h, const gg_swap *sw, gg_cand_result *out, int *affected) {
    if (!h || !sw || !out) return ifail(GG_BAD_ARG, "null argument");
    if (h->h_adj.empty()) return ifail(GG_BAD_ARG, "no graph set");
    gg_status s = check_swap(h, sw);
    if (s != GG_OK) return s;
    GI_CK(cudaSetDevice(h->device));
    const cudaStream_t st = h->stream;
    const size_t adj_b = h->h_adj.size() * sizeof(int32_t);
    GI_CK(cudaMemcpyAsync(h->d_cand, h->d_adj, adj_b, cudaMemcpyDeviceToDevice, st));
    apply_swap_kernel<<<1, 32, 0, st>>>(h->d_cand, h->d, *sw);
    GI_CK(cudaGetLastError());
    gg_eval_opts o{};
    o.max_levels = 199;
    gg_result r{};
    if (!h->planes_ok) {
        // distances of the current graph unknown: evaluate the moved graph in full
        gg::EvalExtra full;
        full.no_graph = true;
        s = gg::engine_eval(h->eng, h->d_cand, &o, &r, st, &full);
        if (s != GG_OK) return s;
        out->total = r.total; out->reached = r.reached; out->levels = r.levels; out->connected = r.connected;
        if (affected) *affected = h->n;
        return GG_OK;
    }
    GI_CK(cudaMemsetAsync(h->d_st, 0, sizeof(IncStatus), st));
    GI_CK(cudaMemsetAsync(h->d_inv, 0xff, (size_t)h->n * sizeof(int32_t), st));
    const unsigned long long pstride = (unsigned long long)h->n * h->cols;
    affected_kernel<<<(h->n + 255) / 256, 256, 0, st>>>(reinterpret_cast<const uint32_t *>(h->d_planes),
                                                        pstride * 4, h->cols * 4, h->d_adj, h->n, h->d, *sw,
                                                        h->d_stats, h->d_stats + h->n, h->d_inv, h->d_st);
    GI_CK(cudaGetLastError());
    GI_CK(cudaMemcpyAsync(h->h_st, h->d_st, sizeof(IncStatus), cudaMemcpyDeviceToHost, st));
    GI_CK(cudaStreamSynchronize(st));
    const IncStatus is = *h->h_st;
    if (affected) *affected = (int)is.count;
    if (is.count == 0) {
        // no distance changes
        out->total = h->cur.total; out->reached = h->cur.reached;
        out->levels = h->cur.levels; out->connected = h->cur.connected;
        return GG_OK;
    }
    gg::EvalExtra x;
    x.inv = h->d_inv;
    x.ns = (int)is.count;
    x.no_graph = true;   // the source count changes from call to call
    s = gg::engine_eval(h->eng, h->d_cand, &o, &r, st, &x);
    if (s != GG_OK) return s;
    out->total = h->cur.total - is.old_sum + r.total;
    out->reached = h->cur.reached - (uint64_t)is.count * h->n + r.reached;
    out->levels = std::max<int>((int)is.max_other, r.levels);
    out->connected = out->reached == (uint64_t)h->n * h->n;
    return GG_OK;
}

gg_status gg_inc_commit(gg_inc *h, const gg_swap *sw, gg_result *r) {
    if (!h || !sw) return ifail(GG_BAD_ARG, "null argument");
    if (h->h_adj.empty()) return ifail(GG_BAD_ARG, "no graph set");
    gg_status s = check_swap(h, sw);
    if (s != GG_OK) return s;
    GI_CK(cudaSetDevice(h->device));
    apply_host(h->h_adj, h->d, *sw);
    GI_CK(cudaMemcpyAsync(h->d_adj, h->h_adj.data(), h->h_adj.size() * 4, cudaMemcpyHostToDevice, h->stream));
    s = inc_rebuild(h);
    if (s != GG_OK) return s;
    if (r) *r = h->cur;
    return GG_OK;
}

gg_status gg_inc_destroy(gg_inc *h) {
    inc_free(h);
    return GG_OK;
}

}  // extern "C"
