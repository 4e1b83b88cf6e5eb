// gg_planes.cuh -- per-source statistics of a distance matrix kept as bit-planes,
// and the symmetry test that makes them cheap.
//
// Plane layout (BfsArgs::planes in gg_kernels.cuh): bit s % 128 of
// planes[k * stride + v * cols + s / 128] is bit k of dist(source s, vertex v);
// bits of columns past the last source and of unreached pairs are 0.
//
// On a symmetric adjacency (u in adj[v] <=> v in adj[u]) the distance matrix is
// symmetric, so source s's distance sum and eccentricity are reductions along
// ROW v = s: a popcount of each plane weighted by 2^k, and a most-significant-
// plane-first search for the largest value.  One warp per row, coalesced 16-byte
// loads along it: one read of the planes, no transposition.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

template <int NP>
static __global__ void plane_row_stats(const uint4 *planes, unsigned long long stride, unsigned cols, int n,
                                       unsigned *rowsum, unsigned *ecc) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned long long nwarps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
    for (unsigned long long v = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < (unsigned)n;
         v += nwarps) {
        const uint4 *row = planes + v * cols;
        unsigned sum = 0, mx = 0;
#pragma unroll 2
        for (unsigned c = lane; c < cols; c += 32) {
            uint4 w[NP];
#pragma unroll
            for (int p = 0; p < NP; ++p) w[p] = __ldg(row + (size_t)p * stride + c);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                unsigned cand = 0xffffffffu, val = 0;
#pragma unroll
                for (int p = NP - 1; p >= 0; --p) {
                    const unsigned x = k == 0 ? w[p].x : k == 1 ? w[p].y : k == 2 ? w[p].z : w[p].w;
                    sum += (unsigned)__popc(x) << p;
                    const unsigned hit = cand & x;
                    if (hit) {
                        cand = hit;
                        val |= 1u << p;
                    }
                }
                mx = max(mx, val);
            }
        }
        sum = __reduce_add_sync(0xffffffffu, sum);
        mx = __reduce_max_sync(0xffffffffu, mx);
        if (lane == 0) {
            rowsum[v] = sum;
            ecc[v] = mx;
        }
    }
}

// 1 into *asym when some entry u of row v has no entry v in row u (one thread
// per entry; entries outside [0, n) are the caller's to reject first).
static __global__ void table_symmetry(const int32_t *adj, int n, int d, int *asym) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)n * d) return;
    const int v = (int)(k / d), u = adj[k];
    bool back = false;
    for (int j = 0; j < d && !back; ++j) back = adj[(size_t)u * d + j] == v;
    if (!back) *asym = 1;
}

// Launch shape of plane_row_stats: one warp per row, at most 8 blocks of 8
// warps per SM in flight.
static inline int plane_row_stats_grid(int n, int sms) {
    const long long blocks = ((long long)n + 7) / 8;
    return (int)(blocks < (long long)sms * 8 ? blocks : (long long)sms * 8);
}
