// gg_probe.cu -- gather-rate microbenchmark: the ceiling of a dense BFS level.
//
// A dense pull level of bfs_batch_kernel reads, for every vertex row of a source
// batch, the frontier rows of its d neighbours (random rows, each a contiguous
// 512-byte segment read by one warp as 32 x 16 bytes), its own visited row, and
// writes one row.  This kernel does exactly that access pattern and nothing else:
//   Y[v] = (OR_{i<d} X[idx[v][i]]) & ~Y0[v]
// over `rows` rows of 32 uint4 with a random index table, so its rate is the
// practical ceiling of a dense level for the same array sizes: with 64 MiB of
// arrays it measures the L2-resident gather rate, with arrays far larger than
// the L2 the HBM gather rate.  Bytes counted per row: (d + 1) reads and one
// write of 512 bytes; the index table (d * 4 bytes per row) is counted too.
#include "gg.h"
#include "gg_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

namespace {

constexpr int kProbeBlock = 256;
constexpr int kRowChunks = 32;  // uint4 per row: 512 bytes

template <int D>
__global__ void __launch_bounds__(kProbeBlock, 6)
gather_probe_kernel(const uint4 *__restrict__ X, const uint4 *__restrict__ Y0, uint4 *__restrict__ Y,
                    const int32_t *__restrict__ idx, int rows, int d) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
    const int dd = D > 0 ? D : d;
    for (unsigned v = warp; v < (unsigned)rows; v += nwarps) {
        const int32_t *row = idx + (size_t)v * dd;
        const uint4 own = __ldcg(Y0 + (size_t)v * kRowChunks + lane);
        uint4 acc = make_uint4(0u, 0u, 0u, 0u);
        if constexpr (D > 0) {
            unsigned u[D];
#pragma unroll
            for (int i = 0; i < D; ++i) u[i] = (unsigned)__ldg(row + i);
            uint4 x[D];
#pragma unroll
            for (int i = 0; i < D; ++i) x[i] = __ldcg(X + (size_t)u[i] * kRowChunks + lane);
#pragma unroll
            for (int i = 0; i < D; ++i) {
                acc.x |= x[i].x; acc.y |= x[i].y; acc.z |= x[i].z; acc.w |= x[i].w;
            }
        } else {
            for (int i = 0; i < dd; ++i) {
                const uint4 x = __ldcg(X + (size_t)(unsigned)__ldg(row + i) * kRowChunks + lane);
                acc.x |= x.x; acc.y |= x.y; acc.z |= x.z; acc.w |= x.w;
            }
        }
        Y[(size_t)v * kRowChunks + lane] =
            make_uint4(acc.x & ~own.x, acc.y & ~own.y, acc.z & ~own.z, acc.w & ~own.w);
    }
}

void *probe_kernel_for(int d) {
    switch (d) {
        case 4: return (void *)gather_probe_kernel<4>;
        case 8: return (void *)gather_probe_kernel<8>;
        case 16: return (void *)gather_probe_kernel<16>;
        default: return (void *)gather_probe_kernel<0>;
    }
}

uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" gg_status gg_gather_peak(int device, int rows, int degree, int iters, double *gbs,
                                    double *ms_per_pass) {
    if (rows < 1 || degree < 1 || degree > 64 || iters < 1 || !gbs)
        return (gg::set_last_error("gg_gather_peak: need rows >= 1, 1 <= degree <= 64, iters >= 1"),
                GG_BAD_ARG);
    if ((long long)rows * kRowChunks * 16 > (64ll << 30))
        return (gg::set_last_error("gg_gather_peak: arrays above 64 GiB"), GG_BAD_ARG);
    cudaError_t err = cudaSetDevice(device);
    if (err != cudaSuccess) {
        (void)cudaGetLastError();
        gg::set_last_error(cudaGetErrorString(err));
        return GG_NO_DEVICE;
    }
    const size_t abytes = (size_t)rows * kRowChunks * sizeof(uint4);
    uint4 *X = nullptr, *Y0 = nullptr, *Y = nullptr;
    int32_t *idx = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t st = nullptr;
    gg_status status = GG_OK;
    std::vector<int32_t> h((size_t)rows * degree);
    uint64_t seed = 0x5eedull + (uint64_t)rows * 131u + (uint64_t)degree;
    for (auto &x : h) x = (int32_t)(splitmix(seed) % (uint64_t)rows);
    auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && status == GG_OK) {
            (void)cudaGetLastError();
            gg::set_last_error((std::string("gg_gather_peak: ") + cudaGetErrorString(e)).c_str());
            status = e == cudaErrorMemoryAllocation ? GG_OUT_OF_MEMORY : GG_CUDA_ERROR;
        }
        return status == GG_OK;
    };
    float best = 1e30f;
    do {
        if (!ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking))) break;
        if (!ck(cudaMalloc(&X, abytes)) || !ck(cudaMalloc(&Y0, abytes)) || !ck(cudaMalloc(&Y, abytes)) ||
            !ck(cudaMalloc(&idx, h.size() * sizeof(int32_t))))
            break;
        if (!ck(cudaMemcpyAsync(idx, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st))) break;
        if (!ck(cudaMemsetAsync(X, 0x5a, abytes, st)) || !ck(cudaMemsetAsync(Y0, 0x0f, abytes, st))) break;
        if (!ck(cudaEventCreate(&e0)) || !ck(cudaEventCreate(&e1))) break;
        int per_sm = 0, sms = 0;
        void *k = probe_kernel_for(degree);
        if (!ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) ||
            !ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kProbeBlock, 0)))
            break;
        const long long want = ((long long)rows * 32 + kProbeBlock - 1) / kProbeBlock;
        const int grid = (int)std::max<long long>(1, std::min<long long>((long long)std::max(per_sm, 1) * sms, want));
        const uint4 *cX = X, *cY0 = Y0;
        const int32_t *cidx = idx;
        void *args[] = {(void *)&cX, (void *)&cY0, (void *)&Y, (void *)&cidx, (void *)&rows, (void *)&degree};
        for (int w = 0; w < 3 && status == GG_OK; ++w)  // warm-up: arrays into the L2 where they fit
            ck(cudaLaunchKernel(k, dim3(grid), dim3(kProbeBlock), args, 0, st));
        for (int it = 0; it < iters && status == GG_OK; ++it) {
            if (!ck(cudaEventRecord(e0, st)) || !ck(cudaLaunchKernel(k, dim3(grid), dim3(kProbeBlock), args, 0, st)) ||
                !ck(cudaEventRecord(e1, st)) || !ck(cudaEventSynchronize(e1)))
                break;
            float ms = 0.f;
            if (!ck(cudaEventElapsedTime(&ms, e0, e1))) break;
            best = std::min(best, ms);
        }
    } while (false);
    if (st) cudaStreamSynchronize(st);
    cudaFree(X); cudaFree(Y0); cudaFree(Y); cudaFree(idx);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    if (status != GG_OK) return status;
    const double bytes = (double)rows * ((degree + 2) * 512.0 + degree * 4.0);
    *gbs = bytes / (best * 1e-3) / 1e9;
    if (ms_per_pass) *ms_per_pass = best;
    return GG_OK;
}
