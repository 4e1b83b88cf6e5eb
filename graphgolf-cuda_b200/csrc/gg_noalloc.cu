// gg_noalloc.cu -- gg_graph_eval_noalloc: the plain-graph evaluation for callers
// that must not allocate device memory.
//
// Who needs it: a search driver that hands the engine only device buffers it
// already owns -- for example a host process whose GPU memory is entirely held
// by another framework's pool, or a tight annealing loop that cannot afford the
// device-wide synchronisation that cudaFree implies -- cannot let a calculator
// cudaMalloc its bitsets the way gg_graph_create does.  This entry point takes
// the adjacency and the output counters as device pointers and keeps its working
// memory in one fixed device array compiled into the library.
//
// The scratch array below is GG_NOALLOC_SCRATCH_BYTES (8 MiB).  Every GPU that
// loads libggb200.so keeps that much device memory for it until the process
// exits, whether or not this entry point is ever called.  All calls share it:
// two calls whose work overlaps on the GPU (different streams, threads or
// processes sharing a context) race on it and both results are undefined.
// A call clears everything the BFS needs to start from zero (visited bits,
// frontier flags, level counters, barrier state) before the BFS runs, so the
// contents a previous call left behind never leak into a result.
#include "gg.h"
#include "gg_kernels.cuh"

#include <algorithm>
#include <mutex>

namespace gg {
void set_last_error(const char *msg);  // gg_engine.cu
}

namespace {

constexpr size_t kScratchBytes = GG_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 256;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices];

// Device address of the scratch array on the current device.  In host code the
// array's name is only a stand-in for the device symbol, so the address is asked
// of the runtime once per device (with that device current) and cached.
gg_status scratch_address(int dev, unsigned char **out) {
    if (dev < 0 || dev >= kMaxDevices) return GG_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            (void)cudaGetLastError();
            return GG_CUDA_ERROR;
        }
        g_scratch_addr[dev] = p;
    }
    *out = (unsigned char *)g_scratch_addr[dev];
    return GG_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Bytes of scratch one evaluation of an N-vertex graph uses (one batch of N sources).
size_t scratch_need(int N) {
    if (N < 1) return 0;
    const size_t nC = ((size_t)N + 127) / 128;
    const size_t items = (size_t)N * nC;
    const size_t fwords = (items + 31) / 32;
    return align256(sizeof(gg::Ctl)) + align256(sizeof(int)) + 3 * align256(items * 16) +
           2 * align256(fwords * 4);
}

gg_status noalloc_fail(gg_status s, const char *msg) {
    (void)cudaGetLastError();
    gg::set_last_error(msg);
    return s;
}

void *noalloc_kernel_for(int d) {
    switch (d) {
        case 3: return (void *)gg::bfs_batch_kernel<3, false>;
        case 4: return (void *)gg::bfs_batch_kernel<4, false>;
        case 6: return (void *)gg::bfs_batch_kernel<6, false>;
        case 8: return (void *)gg::bfs_batch_kernel<8, false>;
        case 12: return (void *)gg::bfs_batch_kernel<12, false>;
        case 16: return (void *)gg::bfs_batch_kernel<16, false>;
        default: return (void *)gg::bfs_batch_kernel<0, false>;
    }
}

}  // namespace

extern "C" gg_status gg_graph_eval_noalloc(const int32_t *d_adj, int N, int degree, int max_levels,
                                           uint64_t *d_level_counts, void *stream) {
    gg::set_last_error("");
    if (!d_adj && (long long)N * degree > 0) return noalloc_fail(GG_BAD_ARG, "null adjacency");
    if (!d_level_counts || N < 1 || degree < 0 || max_levels < 1)
        return noalloc_fail(GG_BAD_ARG, "need N >= 1, degree >= 0, max_levels >= 1, non-null outputs");
    if (scratch_need(N) > kScratchBytes)
        return noalloc_fail(GG_BAD_ARG, "N too large for the fixed scratch array (GG_NOALLOC_SCRATCH_BYTES)");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return noalloc_fail(GG_NO_DEVICE, "no current device");
    unsigned char *base = nullptr;
    if (scratch_address(dev, &base) != GG_OK)
        return noalloc_fail(GG_CUDA_ERROR, "cudaGetSymbolAddress of the scratch array failed");
    (void)cudaGetLastError();

    const int nC = (N + 127) / 128;
    const uint32_t items = (uint32_t)N * (uint32_t)nC;
    const size_t fwords = ((size_t)items + 31) / 32;
    unsigned char *p = base;
    gg::Ctl *ctl = (gg::Ctl *)p;           p += align256(sizeof(gg::Ctl));
    int *bad = (int *)p;                   p += align256(sizeof(int));
    uint4 *V = (uint4 *)p;                 p += align256((size_t)items * 16);
    uint4 *F0 = (uint4 *)p;                p += align256((size_t)items * 16);
    uint4 *F1 = (uint4 *)p;                p += align256((size_t)items * 16);
    uint32_t *fl0 = (uint32_t *)p;         p += align256(fwords * 4);
    uint32_t *fl1 = (uint32_t *)p;

    cudaStream_t st = (cudaStream_t)stream;
    void *kern = noalloc_kernel_for(degree);
    int per_sm = 0, sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, gg::kBlock, 0) != cudaSuccess ||
        per_sm < 1)
        return noalloc_fail(GG_CUDA_ERROR, "occupancy query failed");
    const long long tiles = ((long long)items + 31) / 32;
    const long long want = (tiles + gg::kBlock / 32 - 1) / (gg::kBlock / 32);
    const int grid = (int)std::max<long long>(1, std::min<long long>((long long)per_sm * sms, want));

    if (cudaMemsetAsync(ctl, 0, sizeof(gg::Ctl), st) != cudaSuccess ||
        cudaMemsetAsync(bad, 0, sizeof(int), st) != cudaSuccess)
        return noalloc_fail(GG_CUDA_ERROR, "cudaMemsetAsync on the scratch array failed");
    const long long nent = (long long)N * degree;
    if (nent > 0)
        gg::check_table_kernel<<<(int)std::min<long long>((nent + 255) / 256, 4096), 256, 0, st>>>(
            d_adj, nent, N, bad);
    if (cudaGetLastError() != cudaSuccess) return noalloc_fail(GG_CUDA_ERROR, "launch failed");

    gg::BfsArgs a{};
    a.adj = d_adj;
    a.inv = nullptr;              // source i is vertex i
    a.src_first = 0;
    a.src_begin = 0;
    a.ns_total = N;
    a.nb = 1;
    a.V = V; a.F0 = F0; a.F1 = F1; a.fl0 = fl0; a.fl1 = fl1;
    a.counts = (unsigned long long *)d_level_counts;
    a.masks = nullptr;
    a.stride = max_levels + 1;
    a.levels_run = &ctl->levels_run;
    a.ctl = ctl;
    a.bad = bad;
    a.expected = (unsigned)grid;
    a.div_nc = gg::FastDiv((uint32_t)nC);
    a.items = items;
    a.rows = N; a.d = degree; a.nC = nC;
    a.max_levels = max_levels;
    a.dense_w_ppm = 100;
    a.dense_r_ppm = 4000;
    a.full_skip_ppm = 995000;
    a.split_ppm = 850000;
    a.wait_ns = 10ll * 1000 * 1000 * 1000;
    void *args[] = {&a};
    if (cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(gg::kBlock), args, 0, st) != cudaSuccess)
        return noalloc_fail(GG_CUDA_ERROR, "cooperative launch failed");
    // Blocking like every other entry point: the range check and the barrier
    // status come back into host stack variables.
    gg::Ctl hctl{};
    int hbad = 0;
    if (cudaMemcpyAsync(&hctl, ctl, sizeof(hctl), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return noalloc_fail(GG_CUDA_ERROR, "status read-back failed");
    if (hbad) return noalloc_fail(GG_BAD_ARG, "adjacency entry outside [0, N)");
    if (hctl.err) return noalloc_fail(GG_TIMEOUT, "grid barrier wait exceeded its limit");
    return GG_OK;
}
