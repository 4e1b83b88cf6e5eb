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
//
// gg_level_probe runs the dense level loop itself outside the engine: one
// cooperative launch, `levels` levels of Y[v] = OR of 8 neighbour rows of X
// (X and Y ping-ponged), each row's popcount, flag and not-full words, one
// count per block, and the engine's grid barrier between levels, timed per
// level with device timestamps.  Variant 1 keeps a second row in flight a warp
// by gathering it with cp.async into shared memory.
#include "gg.h"
#include "gg_internal.h"
#include "gg_kernels.cuh"

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

constexpr int kLevelDeg = 8;      // neighbours a row in the level probe
constexpr int kLevelBlocks = 4;   // resident blocks a SM, as bfs_batch_kernel
constexpr int kSlotU4 = 8 * 32;   // variant 1: uint4 of one warp's staged row

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}

// Rows of CH uint4 (128 * CH sources); a tile is 32 uint4 = 32 / CH rows and
// lane l works on row t * (32 / CH) + l / CH, chunk l % CH.  Block b owns the
// balanced tile range [t_lo, t_hi) and its warps take tiles from a shared
// counter, as the engine's dense levels do.
template <int CH, int VAR>
__global__ void __launch_bounds__(kProbeBlock, kLevelBlocks)
level_probe_kernel(uint4 *B0, uint4 *B1, const int32_t *__restrict__ idx, unsigned ntiles, int levels,
                   gg::Ctl *ctl, unsigned long long *cnts, uint32_t *fl, uint32_t *nf,
                   unsigned long long *stamps, long long wait_ns) {
    extern __shared__ __align__(16) int32_t s_ladj[];
    __shared__ unsigned s_next;
    __shared__ unsigned s_sum[kProbeBlock / 32];
    constexpr unsigned kRpt = 32u / CH;   // rows a tile
    const unsigned lane = threadIdx.x & 31u;
    const unsigned t_lo = (unsigned)((unsigned long long)ntiles * blockIdx.x / gridDim.x);
    const unsigned t_hi = (unsigned)((unsigned long long)ntiles * (blockIdx.x + 1) / gridDim.x);
    const unsigned nadj = (t_hi - t_lo) * kRpt * kLevelDeg;
    for (unsigned k = threadIdx.x; k < nadj; k += blockDim.x) s_ladj[k] = idx[(size_t)t_lo * kRpt * kLevelDeg + k];
    uint4 *slot = reinterpret_cast<uint4 *>(s_ladj + (nadj + 3u) / 4u * 4u) + (threadIdx.x >> 5) * kSlotU4;
    __syncthreads();
    unsigned epoch = 0;
    for (int L = 0; L < levels; ++L) {
        const uint4 *X = (L & 1) ? B1 : B0;
        uint4 *Y = (L & 1) ? B0 : B1;
        unsigned cnt = 0u;
        if (threadIdx.x == 0) s_next = t_lo;
        __syncthreads();
        auto grab = [&]() {
            unsigned t = 0u;
            if (lane == 0) t = atomicAdd(&s_next, 1u);
            return __shfl_sync(0xffffffffu, t, 0);
        };
        auto nbr = [&](const unsigned t, const int i) {
            return (unsigned)s_ladj[((t - t_lo) * kRpt + lane / CH) * kLevelDeg + i] * CH + lane % CH;
        };
        auto finish = [&](const unsigned t, const uint4 a) {
            Y[((size_t)t * kRpt + lane / CH) * CH + lane % CH] = a;
            cnt += gg::u4popc(a);
            const unsigned fb = __ballot_sync(0xffffffffu, gg::u4any(a));
            const unsigned nb = __ballot_sync(0xffffffffu, !gg::u4full(a));
            if (lane == 0) {
                fl[t] = fb;
                nf[t] = nb;
            }
        };
        if constexpr (VAR == 0) {
            for (;;) {
                const unsigned t = grab();
                if (t >= t_hi) break;
                unsigned u[kLevelDeg];
#pragma unroll
                for (int i = 0; i < kLevelDeg; ++i) u[i] = nbr(t, i);
                uint4 x[kLevelDeg];
#pragma unroll
                for (int i = 0; i < kLevelDeg; ++i) x[i] = __ldcg(X + u[i]);
                uint4 q = x[0];
#pragma unroll
                for (int i = 1; i < kLevelDeg; ++i) gg::or_into(q, x[i]);
                finish(t, q);
            }
        } else {
            // tile a staged in this warp's slot (each lane copies and later reads
            // only its own 16-byte entries) while tile b is gathered into registers
            auto stage = [&](const unsigned t) {
#pragma unroll
                for (int i = 0; i < kLevelDeg; ++i) cp_async16(slot + i * 32 + lane, X + nbr(t, i));
                asm volatile("cp.async.commit_group;" ::: "memory");
            };
            unsigned ta = grab();
            if (ta < t_hi) stage(ta);
            while (ta < t_hi) {
                const unsigned tb = grab();
                uint4 x[kLevelDeg];
                if (tb < t_hi) {
                    unsigned u[kLevelDeg];
#pragma unroll
                    for (int i = 0; i < kLevelDeg; ++i) u[i] = nbr(tb, i);
#pragma unroll
                    for (int i = 0; i < kLevelDeg; ++i) x[i] = __ldcg(X + u[i]);
                }
                asm volatile("cp.async.wait_group 0;" ::: "memory");
                uint4 q = slot[lane];
#pragma unroll
                for (int i = 1; i < kLevelDeg; ++i) gg::or_into(q, slot[i * 32 + lane]);
                finish(ta, q);   // the slot's values are consumed before it is refilled
                if (tb >= t_hi) break;
                const unsigned tc = grab();
                if (tc < t_hi) stage(tc);
                q = x[0];
#pragma unroll
                for (int i = 1; i < kLevelDeg; ++i) gg::or_into(q, x[i]);
                finish(tb, q);
                ta = tc;
            }
        }
        const unsigned wsum = __reduce_add_sync(0xffffffffu, cnt);
        if (lane == 0) s_sum[threadIdx.x >> 5] = wsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long bs = 0ull;
            for (int w = 0; w < kProbeBlock / 32; ++w) bs += s_sum[w];
            atomicAdd(cnts + L, bs);
        }
        unsigned long long total = 0ull;
        if (!gg::grid_sync_value(ctl, gridDim.x, wait_ns, L, epoch, cnts + L, total)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) stamps[L] = gg::gtimer();
    }
}

void *level_kernel_for(int chunks, int variant) {
    if (chunks == 32) return variant ? (void *)level_probe_kernel<32, 1> : (void *)level_probe_kernel<32, 0>;
    return variant ? (void *)level_probe_kernel<16, 1> : (void *)level_probe_kernel<16, 0>;
}

// Dynamic shared memory of a level-probe block: its adjacency slice (rounded to
// 16 bytes) and, for variant 1, one staged row a warp.
size_t level_smem(unsigned ntiles, int grid, int chunks, int variant) {
    const size_t tiles = (ntiles + (unsigned)grid - 1u) / (unsigned)grid;
    const size_t ints = tiles * (size_t)(32 / chunks) * kLevelDeg;
    return (ints + 3u) / 4u * 16u + (variant ? (size_t)(kProbeBlock / 32) * kSlotU4 * sizeof(uint4) : 0u);
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

extern "C" gg_status gg_level_probe(int device, int rows, int chunks, int levels, int variant,
                                    double *us_per_level) {
    if (rows < 64 || rows > (1 << 18) || (chunks != 32 && chunks != 16) || (rows * chunks) % 32 != 0 ||
        levels < 12 || levels > 1024 || variant < 0 || variant > 1 || !us_per_level)
        return (gg::set_last_error("gg_level_probe: need 64 <= rows <= 262144, chunks 16 or 32 (rows even for 16), "
                                   "12 <= levels <= 1024, variant 0 or 1"),
                GG_BAD_ARG);
    cudaError_t err = cudaSetDevice(device);
    if (err != cudaSuccess) {
        (void)cudaGetLastError();
        gg::set_last_error(cudaGetErrorString(err));
        return GG_NO_DEVICE;
    }
    const unsigned ntiles = (unsigned)((long long)rows * chunks / 32);
    const size_t abytes = (size_t)rows * chunks * sizeof(uint4);
    uint4 *B0 = nullptr, *B1 = nullptr;
    int32_t *idx = nullptr;
    gg::Ctl *ctl = nullptr;
    unsigned long long *cnts = nullptr, *stamps = nullptr;
    uint32_t *fl = nullptr, *nf = nullptr;
    cudaStream_t st = nullptr;
    gg_status status = GG_OK;
    // kLevelDeg random permutations: every row is a neighbour kLevelDeg times,
    // as in a regular graph
    std::vector<int32_t> h((size_t)rows * kLevelDeg), perm(rows);
    uint64_t seed = 0x1e7e1ull + (uint64_t)rows * 977u;
    for (int i = 0; i < kLevelDeg; ++i) {
        for (int v = 0; v < rows; ++v) perm[v] = v;
        for (int v = rows - 1; v > 0; --v) std::swap(perm[v], perm[splitmix(seed) % (uint64_t)(v + 1)]);
        for (int v = 0; v < rows; ++v) h[(size_t)v * kLevelDeg + i] = perm[v];
    }
    auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && status == GG_OK) {
            (void)cudaGetLastError();
            gg::set_last_error((std::string("gg_level_probe: ") + cudaGetErrorString(e)).c_str());
            status = e == cudaErrorMemoryAllocation ? GG_OUT_OF_MEMORY : GG_CUDA_ERROR;
        }
        return status == GG_OK;
    };
    double best = 1e30;
    do {
        if (!ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking))) break;
        if (!ck(cudaMalloc(&B0, abytes)) || !ck(cudaMalloc(&B1, abytes)) ||
            !ck(cudaMalloc(&idx, h.size() * sizeof(int32_t))) || !ck(cudaMalloc(&ctl, sizeof(gg::Ctl))) ||
            !ck(cudaMalloc(&cnts, (size_t)levels * 8)) || !ck(cudaMalloc(&stamps, (size_t)levels * 8)) ||
            !ck(cudaMalloc(&fl, (size_t)ntiles * 4)) || !ck(cudaMalloc(&nf, (size_t)ntiles * 4)))
            break;
        if (!ck(cudaMemcpyAsync(idx, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st))) break;
        if (!ck(cudaMemsetAsync(B0, 0x21, abytes, st)) || !ck(cudaMemsetAsync(B1, 0x42, abytes, st))) break;
        void *k = level_kernel_for(chunks, variant);
        int sms = 0, per_sm = 0;
        if (!ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device))) break;
        // every block resident (cooperative launch): shrink the grid until the
        // shared memory its tile ranges need still allows it
        int grid = sms * kLevelBlocks;
        size_t smem = 0;
        for (;;) {
            smem = level_smem(ntiles, grid, chunks, variant);
            if (smem > 48u * 1024u) {
                if (!ck(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))) break;
            }
            if (!ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kProbeBlock, smem))) break;
            if (per_sm < 1) {
                gg::set_last_error("gg_level_probe: no block fits a SM");
                status = GG_BAD_ARG;
                break;
            }
            if (per_sm * sms >= grid) break;
            grid = per_sm * sms;
        }
        if (status != GG_OK) break;
        unsigned nt = ntiles;
        int lv = levels;
        long long wait_ns = 2000000000ll;
        void *args[] = {(void *)&B0, (void *)&B1, (void *)&idx, (void *)&nt, (void *)&lv, (void *)&ctl,
                        (void *)&cnts, (void *)&fl, (void *)&nf, (void *)&stamps, (void *)&wait_ns};
        std::vector<unsigned long long> t(levels);
        for (int rep = 0; rep < 4 && status == GG_OK; ++rep) {
            gg::Ctl hctl{};
            if (!ck(cudaMemsetAsync(ctl, 0, sizeof(gg::Ctl), st)) || !ck(cudaMemsetAsync(cnts, 0, (size_t)levels * 8, st)) ||
                !ck(cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kProbeBlock), args, smem, st)) ||
                !ck(cudaMemcpyAsync(t.data(), stamps, (size_t)levels * 8, cudaMemcpyDeviceToHost, st)) ||
                !ck(cudaMemcpyAsync(&hctl, ctl, sizeof(gg::Ctl), cudaMemcpyDeviceToHost, st)) ||
                !ck(cudaStreamSynchronize(st)))
                break;
            if (hctl.err) {
                gg::set_last_error("gg_level_probe: a grid-barrier wait ran out");
                status = GG_TIMEOUT;
                break;
            }
            // levels 10.. only: the first ones bring the arrays into the L2
            best = std::min(best, (double)(t[levels - 1] - t[9]) / 1000.0 / (levels - 10));
        }
    } while (false);
    if (st) cudaStreamSynchronize(st);
    cudaFree(B0); cudaFree(B1); cudaFree(idx); cudaFree(ctl);
    cudaFree(cnts); cudaFree(stamps); cudaFree(fl); cudaFree(nf);
    if (st) cudaStreamDestroy(st);
    if (status != GG_OK) return status;
    *us_per_level = best;
    return GG_OK;
}
