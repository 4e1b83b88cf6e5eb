// gg_surrogate.cu -- the surrogate ΔASPL ranker (gg_surrogate_* in gg.h).
//
// Every product rounds its operands to bf16 (round to nearest even) in shared
// memory and multiplies with mma.sync m16n8k16 (bf16 in, fp32 accumulate), on
// 64x64 output tiles of 128 threads.  The forward pass (graph embedding and swap
// readout) is one cooperative launch (surrogate_forward_kernel) with a bounded
// grid barrier per message-passing layer; the backward pass with the Adam step is
// another (surrogate_backward_kernel: weight gradients add each tile's partial
// product with fp32 atomics, scatters and elementwise steps in fp32).
#include "gg.h"
#include "gg_kernels.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace gg {
void set_last_error(const char *msg);  // gg_engine.cu
}

namespace {

constexpr int kH = 64;           // hidden width
constexpr int kZ = 3 * kH;       // swap readout width
constexpr int kLayers = 3;       // message-passing layers

__device__ __forceinline__ uint16_t bf16_bits(float x) {
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    return *reinterpret_cast<uint16_t *>(&h);
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ---------------------------------------------------------------------------
// swap readout helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ void partners(const gg_swap &s, int &p, int &q) {
    p = s.mode ? s.d : s.c;  // new edges (a,p), (b,q)
    q = s.mode ? s.c : s.d;
}

// Per-call scalars, written by the host before each replay: [0] 1/count of
// unmasked swaps, [1] learning rate, [2] 1 - beta1^t, [3] 1 - beta2^t.
enum { kHypInvCnt = 0, kHypLr = 1, kHypC1 = 2, kHypC2 = 3, kHypN = 4 };

// ---------------------------------------------------------------------------
// Fused forward: the graph embedding (H0 .. H3, with the neighbour means M0 .. M2
// kept for the backward pass) and the readout of P swaps (Z, O, y) in one
// cooperative launch of 128-thread blocks, with a bounded grid barrier after each
// layer (every block needs the whole previous layer for its neighbour means).
// A block owns 64-row tiles (vertices, then swaps).  For each tile it stages both
// operands as bf16 in shared memory -- A (64 x K) row-major, B transposed (64 x K)
// -- and multiplies with mma.sync m16n8k16 (fp32 accumulate), the arithmetic of
// every surrogate product; a layer's two products H Ws + M Wn run as one K = 128 product
// over [H | M] and [Ws ; Wn].
// ---------------------------------------------------------------------------
constexpr int kFwdBlock = 128;
constexpr int kFwdKmax = 256;              // in_features <= 256, 2 * kH, kZ all fit
constexpr int kFwdLd = kFwdKmax + 8;       // row stride (bf16): fragment loads spread over the banks

struct FwdArgs {
    const float *X;
    int F;
    const int32_t *adj;
    int n, d;
    const float *P;
    int o_win, o_bin, o_ws[kLayers], o_wn[kLayers], o_b[kLayers], o_wr1, o_br1, o_wr2, o_br2;
    float *H[kLayers + 1];
    float *M[kLayers];
    const gg_swap *sw;
    int n_sw;
    float *Z, *O, *y;
    gg::Ctl *ctl;
    unsigned expected;
    long long wait_ns;
};

// acc[8][4] of this warp's 16 rows x 64 columns = As (64 x K) * Bt^T, K % 16 == 0.
__device__ __forceinline__ void tile_mma(const uint16_t *As, const uint16_t *Bt, const int K, float acc[8][4]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tg = lane & 3;
    const int r = warp * 16;
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t a[4];
        a[0] = *reinterpret_cast<const uint32_t *>(As + (r + gid) * kFwdLd + k0 + 2 * tg);
        a[1] = *reinterpret_cast<const uint32_t *>(As + (r + gid + 8) * kFwdLd + k0 + 2 * tg);
        a[2] = *reinterpret_cast<const uint32_t *>(As + (r + gid) * kFwdLd + k0 + 2 * tg + 8);
        a[3] = *reinterpret_cast<const uint32_t *>(As + (r + gid + 8) * kFwdLd + k0 + 2 * tg + 8);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            uint32_t b[2];
            b[0] = *reinterpret_cast<const uint32_t *>(Bt + (8 * j + gid) * kFwdLd + k0 + 2 * tg);
            b[1] = *reinterpret_cast<const uint32_t *>(Bt + (8 * j + gid) * kFwdLd + k0 + 2 * tg + 8);
            mma_bf16(acc[j], a, b);
        }
    }
}

// Rows [row0, row0 + 64) of out (width kH) = relu(acc + bias); rows >= rows are dropped.
__device__ __forceinline__ void tile_store_relu(const float acc[8][4], const float *bias, float *out, int row0,
                                                int rows) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int m = row0 + warp * 16 + gid + ((h >> 1) << 3);
            const int c = 8 * j + 2 * tg + (h & 1);
            if (m < rows) {
                const float v = acc[j][h] + bias[c];
                out[(size_t)m * kH + c] = v > 0.f ? v : 0.f;
            }
        }
}

__global__ void __launch_bounds__(kFwdBlock) surrogate_forward_kernel(const FwdArgs a) {
    extern __shared__ __align__(16) uint16_t fsm[];
    uint16_t *As = fsm;                    // [64][kFwdLd]
    uint16_t *Bt = fsm + 64 * kFwdLd;      // [64][kFwdLd]
    __shared__ float s_o[64][kH + 1];
    const int tid = threadIdx.x;
    unsigned epoch = 0;
    float acc[8][4];
    const int nrb = (a.n + 63) / 64;
    if (a.n > 0) {
        // H0 = relu(X W_in + b_in); K = in_features padded to 16
        const int K0 = (a.F + 15) / 16 * 16;
        for (int e = tid; e < 64 * K0; e += kFwdBlock) {
            const int c = e / K0, k = e % K0;
            Bt[c * kFwdLd + k] = bf16_bits(k < a.F ? a.P[a.o_win + k * kH + c] : 0.f);
        }
        for (int rb = blockIdx.x; rb < nrb; rb += gridDim.x) {
            for (int e = tid; e < 64 * K0; e += kFwdBlock) {
                const int r = e / K0, k = e % K0, v = rb * 64 + r;
                As[r * kFwdLd + k] = bf16_bits(v < a.n && k < a.F ? a.X[(size_t)v * a.F + k] : 0.f);
            }
            __syncthreads();
            tile_mma(As, Bt, K0, acc);
            tile_store_relu(acc, a.P + a.o_bin, a.H[0], rb * 64, a.n);
            __syncthreads();
        }
        for (int l = 0; l < kLayers; ++l) {
            if (!gg::grid_sync(a.ctl, a.expected, a.wait_ns, l, epoch)) return;
            // Bt = [Ws ; Wn]^T (K = 128)
            for (int e = tid; e < 64 * 2 * kH; e += kFwdBlock) {
                const int c = e / (2 * kH), k = e % (2 * kH);
                const float w = k < kH ? a.P[a.o_ws[l] + k * kH + c] : a.P[a.o_wn[l] + (k - kH) * kH + c];
                Bt[c * kFwdLd + k] = bf16_bits(w);
            }
            const float inv = 1.f / (float)a.d;
            for (int rb = blockIdx.x; rb < nrb; rb += gridDim.x) {
                // A = [H_l | mean of the neighbours' H_l rows]; the means are kept in M_l
                for (int e = tid; e < 64 * kH; e += kFwdBlock) {
                    const int r = e / kH, c = e % kH, v = rb * 64 + r;
                    float h = 0.f, m = 0.f;
                    if (v < a.n) {
                        h = __ldcg(a.H[l] + (size_t)v * kH + c);
                        for (int i = 0; i < a.d; ++i)
                            m += __ldcg(a.H[l] + (size_t)__ldg(a.adj + (size_t)v * a.d + i) * kH + c);
                        m *= inv;
                        a.M[l][(size_t)v * kH + c] = m;
                    }
                    As[r * kFwdLd + c] = bf16_bits(h);
                    As[r * kFwdLd + kH + c] = bf16_bits(m);
                }
                __syncthreads();
                tile_mma(As, Bt, 2 * kH, acc);
                tile_store_relu(acc, a.P + a.o_b[l], a.H[l + 1], rb * 64, a.n);
                __syncthreads();
            }
        }
        if (!gg::grid_sync(a.ctl, a.expected, a.wait_ns, kLayers, epoch)) return;
    }
    // readout: Z = [Ha+Hb+Hc+Hd, Ha*Hb + Hc*Hd, Ha*Hp + Hb*Hq], O = relu(Z Wr1 + br1), y = O.wr2 + br2
    if (a.n_sw > 0) {
        for (int e = tid; e < 64 * kZ; e += kFwdBlock) {
            const int c = e / kZ, k = e % kZ;
            Bt[c * kFwdLd + k] = bf16_bits(a.P[a.o_wr1 + k * kH + c]);
        }
        const float *H3 = a.H[kLayers];
        const int ntb = (a.n_sw + 63) / 64;
        for (int tb = blockIdx.x; tb < ntb; tb += gridDim.x) {
            for (int e = tid; e < 64 * kH; e += kFwdBlock) {
                const int r = e / kH, j = e % kH, p = tb * 64 + r;
                float z0 = 0.f, z1 = 0.f, z2 = 0.f;
                if (p < a.n_sw) {
                    const gg_swap s = a.sw[p];
                    int pa, qb;
                    partners(s, pa, qb);
                    const float ha = __ldcg(H3 + (size_t)s.a * kH + j), hb = __ldcg(H3 + (size_t)s.b * kH + j);
                    const float hc = __ldcg(H3 + (size_t)s.c * kH + j), hd = __ldcg(H3 + (size_t)s.d * kH + j);
                    const float hp = __ldcg(H3 + (size_t)pa * kH + j), hq = __ldcg(H3 + (size_t)qb * kH + j);
                    z0 = ha + hb + hc + hd;
                    z1 = ha * hb + hc * hd;
                    z2 = ha * hp + hb * hq;
                    float *z = a.Z + (size_t)p * kZ;
                    z[j] = z0; z[kH + j] = z1; z[2 * kH + j] = z2;
                }
                As[r * kFwdLd + j] = bf16_bits(z0);
                As[r * kFwdLd + kH + j] = bf16_bits(z1);
                As[r * kFwdLd + 2 * kH + j] = bf16_bits(z2);
            }
            __syncthreads();
            tile_mma(As, Bt, kZ, acc);
            tile_store_relu(acc, a.P + a.o_br1, a.O, tb * 64, a.n_sw);
            {
                // the block's O rows, for the output dot products
                const int warp = tid >> 5, lane = tid & 31, gid = lane >> 2, tg = lane & 3;
#pragma unroll
                for (int j = 0; j < 8; ++j)
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const int r = warp * 16 + gid + ((h >> 1) << 3), c = 8 * j + 2 * tg + (h & 1);
                        const float v = acc[j][h] + a.P[a.o_br1 + c];
                        s_o[r][c] = v > 0.f ? v : 0.f;
                    }
            }
            __syncthreads();
            if (tid < 64 && tb * 64 + tid < a.n_sw) {
                float sum = 0.f;
                for (int j = 0; j < kH; ++j) sum += s_o[tid][j] * a.P[a.o_wr2 + j];
                a.y[tb * 64 + tid] = sum + a.P[a.o_br2];
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Fused backward (and Adam): the gradient of the masked MSE of P swap predictions with
// respect to every parameter, in one cooperative launch of 128-thread blocks with a
// bounded grid barrier between dependent stages:
//   1. swap tiles: dy, dO = dy w_r2 (O > 0), dZ = dO Wr1^T, dWr1 += Z^T dO, the output
//      biases and weights, and dZ scattered into dH3 (fp32 atomics);
//   2. per layer l = 2, 1, 0, vertex tiles: dPre = dH (H_{l+1} > 0), db_l, dWs_l += H_l^T
//      dPre, dWn_l += M_l^T dPre, dH_l = dPre Ws_l^T (rows) and G = dPre Wn_l^T; then,
//      after a barrier, dH_l += the neighbour mean of G (symmetric adjacency);
//   3. the input layer: dPre0 = dH (H0 > 0), db_in, dWin += X^T dPre0;
//   4. with `train`, Adam on every parameter.
// Products round both operands to bf16 in shared memory and multiply with mma.sync
// (fp32 accumulate), as the forward does; weight gradients add each tile's partial
// product with fp32 atomics; elementwise steps stay in fp32.  Data other blocks wrote
// earlier in the launch is read through the L2 (__ldcg).
// ---------------------------------------------------------------------------
struct BwdArgs {
    const float *X;
    int F;
    const int32_t *adj;
    int n, d;
    const float *P;
    float *Gd;
    int o_win, o_bin, o_ws[kLayers], o_wn[kLayers], o_b[kLayers], o_wr1, o_br1, o_wr2, o_br2;
    const float *H[kLayers + 1];
    const float *M[kLayers];
    const gg_swap *sw;
    int n_sw;
    const float *Z, *O, *y, *t;
    const int32_t *mask;
    const float *hyper;
    float *dO, *dZ, *dHa, *dHb, *Gt, *loss;
    float *adam_m, *adam_v;
    float *params;
    int n_params, train;
    gg::Ctl *ctl;
    unsigned expected;
    long long wait_ns;
};

// S[c][r] = bf16(src[(row0 + r) * ld + col0 + c]), c < 64 (columns past ncols: 0),
// r < 64 (rows past nrows: 0): the transposed tile
__device__ __forceinline__ void stage_cols(uint16_t *S, const float *src, long long ld, int row0, int nrows,
                                           int col0, int ncols) {
#pragma unroll 8
    for (int e = threadIdx.x; e < 64 * 64; e += kFwdBlock) {
        const int r = e >> 6, c = e & 63, m = row0 + r;
        S[c * kFwdLd + r] = bf16_bits(m < nrows && col0 + c < ncols ? src[(size_t)m * ld + col0 + c] : 0.f);
    }
}

// S[k][c] = bf16(W[(k0 + k) * ldw + c]), k, c < 64: a weight block, row k of W as row k of S
__device__ __forceinline__ void stage_wt(uint16_t *S, const float *W, int ldw, int k0) {
#pragma unroll 8
    for (int e = threadIdx.x; e < 64 * 64; e += kFwdBlock) {
        const int k = e >> 6, c = e & 63;
        S[k * kFwdLd + c] = bf16_bits(W[(size_t)(k0 + k) * ldw + c]);
    }
}

// dst[(r0 + m) * ld + c0 + c] (=|+= atomically) acc[m][c], m < mrows, c < ncols
template <bool ATOMIC>
__device__ __forceinline__ void tile_out(const float acc[8][4], float *dst, long long ld, int r0, int mrows, int c0,
                                         int ncols) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int m = warp * 16 + gid + ((h >> 1) << 3), c = 8 * j + 2 * tg + (h & 1);
            if (m < mrows && c < ncols) {
                float *q = dst + (size_t)(r0 + m) * ld + c0 + c;
                if (ATOMIC) atomicAdd(q, acc[j][h]); else *q = acc[j][h];
            }
        }
}

__global__ void __launch_bounds__(kFwdBlock) surrogate_backward_kernel(const BwdArgs a) {
    extern __shared__ __align__(16) uint16_t bsm[];
    uint16_t *As = bsm;                    // [64][kFwdLd]
    uint16_t *Bt = bsm + 64 * kFwdLd;      // [64][kFwdLd]
    const int tid = threadIdx.x, jc = tid & 63;   // elementwise loops: this thread's column
    unsigned epoch = 0;
    float acc[8][4];
    const float *Pm = a.P;
    float *Gd = a.Gd;
    // 1. swap tiles
    {
        const float inv_cnt = a.hyper[kHypInvCnt];
        float g_wr2 = 0.f, g_br1 = 0.f, g_br2 = 0.f;
        const float *H3 = a.H[kLayers];
        const int ntb = (a.n_sw + 63) / 64;
        for (int tb = blockIdx.x; tb < ntb; tb += gridDim.x) {
            const int p0 = tb * 64, prow = min(64, a.n_sw - p0);
#pragma unroll 8
            for (int e = tid; e < 64 * kH; e += kFwdBlock) {
                const int r = e / kH, j = e % kH, p = p0 + r;
                float v = 0.f;
                if (p < a.n_sw) {
                    const float m = a.mask[p] ? 1.f : 0.f;
                    const float err = (a.y[p] - a.t[p]) * m;
                    const float dyp = 2.f * err * inv_cnt;
                    const float o = a.O[(size_t)p * kH + j];
                    v = o > 0.f ? dyp * Pm[a.o_wr2 + j] : 0.f;
                    a.dO[(size_t)p * kH + j] = v;
                    g_wr2 += dyp * o;
                    g_br1 += v;
                    if (j == 0) {
                        g_br2 += dyp;
                        atomicAdd(a.loss, err * err * inv_cnt);
                    }
                }
                As[r * kFwdLd + j] = bf16_bits(v);
            }
            __syncthreads();
            // dZ = dO Wr1^T, 64 columns of Z at a time
            for (int zc = 0; zc < kZ / 64; ++zc) {
                stage_wt(Bt, Pm + a.o_wr1, kH, zc * 64);   // Bt[z][j] = Wr1[zc * 64 + z][j]
                __syncthreads();
                tile_mma(As, Bt, kH, acc);
                tile_out<false>(acc, a.dZ, kZ, p0, prow, zc * 64, 64);
                __syncthreads();
            }
            // dWr1 += Z^T dO
            stage_cols(Bt, a.dO, kH, p0, a.n_sw, 0, kH);   // Bt[j][r] = dO[p0 + r][j]
            for (int zc = 0; zc < kZ / 64; ++zc) {
                stage_cols(As, a.Z, kZ, p0, a.n_sw, zc * 64, kZ);   // As[z][r] = Z[p0 + r][zc * 64 + z]
                __syncthreads();
                tile_mma(As, Bt, 64, acc);
                tile_out<true>(acc, Gd + a.o_wr1, kH, zc * 64, 64, 0, kH);
                __syncthreads();
            }
            // dZ of this tile's swaps into dH3 (the readout's products, fp32 atomics)
#pragma unroll 8
            for (int e = tid; e < 64 * kH; e += kFwdBlock) {
                const int r = e / kH, j = e % kH, p = p0 + r;
                if (p >= a.n_sw) continue;
                const gg_swap w = a.sw[p];
                int pa, qb;
                partners(w, pa, qb);
                const float g0 = a.dZ[(size_t)p * kZ + j], g1 = a.dZ[(size_t)p * kZ + kH + j],
                            g2 = a.dZ[(size_t)p * kZ + 2 * kH + j];
                const float ha = H3[(size_t)w.a * kH + j], hb = H3[(size_t)w.b * kH + j];
                const float hc = H3[(size_t)w.c * kH + j], hd = H3[(size_t)w.d * kH + j];
                const float hp = H3[(size_t)pa * kH + j], hq = H3[(size_t)qb * kH + j];
                atomicAdd(a.dHa + (size_t)w.a * kH + j, g0 + g1 * hb + g2 * hp);
                atomicAdd(a.dHa + (size_t)w.b * kH + j, g0 + g1 * ha + g2 * hq);
                atomicAdd(a.dHa + (size_t)w.c * kH + j, g0 + g1 * hd);
                atomicAdd(a.dHa + (size_t)w.d * kH + j, g0 + g1 * hc);
                atomicAdd(a.dHa + (size_t)pa * kH + j, g2 * ha);
                atomicAdd(a.dHa + (size_t)qb * kH + j, g2 * hb);
            }
            __syncthreads();
        }
        atomicAdd(Gd + a.o_wr2 + jc, g_wr2);
        atomicAdd(Gd + a.o_br1 + jc, g_br1);
        if (jc == 0) atomicAdd(Gd + a.o_br2, g_br2);
    }
    // 2. layers 2, 1, 0 (dH holds dL/dH_{l+1}; dHn receives dL/dH_l)
    float *dH = a.dHa, *dHn = a.dHb;
    const int nrb = (a.n + 63) / 64;
    const long long gtid = (long long)blockIdx.x * blockDim.x + tid, nthr = (long long)gridDim.x * blockDim.x;
    for (int l = kLayers - 1; l >= 0; --l) {
        if (!gg::grid_sync(a.ctl, a.expected, a.wait_ns, 2 * (kLayers - 1 - l) + 1, epoch)) return;
        float g_b = 0.f;
        for (int rb = blockIdx.x; rb < nrb; rb += gridDim.x) {
            const int v0 = rb * 64, vrows = min(64, a.n - v0);
            // dPre = dH (H_{l+1} > 0), in place; As = dPre rows
#pragma unroll 8
            for (int e = tid; e < 64 * kH; e += kFwdBlock) {
                const int r = e / kH, c = e % kH, v = v0 + r;
                float q = 0.f;
                if (v < a.n) {
                    q = a.H[l + 1][(size_t)v * kH + c] > 0.f ? __ldcg(dH + (size_t)v * kH + c) : 0.f;
                    dH[(size_t)v * kH + c] = q;
                }
                g_b += q;
                As[r * kFwdLd + c] = bf16_bits(q);
            }
            __syncthreads();
            // dH_l rows = dPre Ws^T, G = dPre Wn^T
            stage_wt(Bt, Pm + a.o_ws[l], kH, 0);   // Bt[k][c] = Ws[k][c]
            __syncthreads();
            tile_mma(As, Bt, kH, acc);
            tile_out<false>(acc, dHn, kH, v0, vrows, 0, kH);
            __syncthreads();
            stage_wt(Bt, Pm + a.o_wn[l], kH, 0);
            __syncthreads();
            tile_mma(As, Bt, kH, acc);
            tile_out<false>(acc, a.Gt, kH, v0, vrows, 0, kH);
            __syncthreads();
            // dWs_l += H_l^T dPre, dWn_l += M_l^T dPre
            stage_cols(Bt, dH, kH, v0, a.n, 0, kH);       // Bt[c][r] = dPre[v0 + r][c]
            stage_cols(As, a.H[l], kH, v0, a.n, 0, kH);   // As[k][r] = H_l[v0 + r][k]
            __syncthreads();
            tile_mma(As, Bt, 64, acc);
            tile_out<true>(acc, Gd + a.o_ws[l], kH, 0, 64, 0, kH);
            __syncthreads();
            stage_cols(As, a.M[l], kH, v0, a.n, 0, kH);
            __syncthreads();
            tile_mma(As, Bt, 64, acc);
            tile_out<true>(acc, Gd + a.o_wn[l], kH, 0, 64, 0, kH);
            __syncthreads();
        }
        atomicAdd(Gd + a.o_b[l] + jc, g_b);
        if (!gg::grid_sync(a.ctl, a.expected, a.wait_ns, 2 * (kLayers - 1 - l) + 2, epoch)) return;
        // dH_l += the neighbour mean of G (a symmetric adjacency: the transpose of the mean)
        const float inv = 1.f / (float)a.d;
#pragma unroll 4
        for (long long t = gtid; t < (long long)a.n * kH; t += nthr) {
            const int v = (int)(t / kH), j = (int)(t % kH);
            float sum = 0.f;
            for (int i = 0; i < a.d; ++i) sum += __ldcg(a.Gt + (size_t)__ldg(a.adj + (size_t)v * a.d + i) * kH + j);
            dHn[t] = __ldcg(dHn + t) + sum * inv;
        }
        float *tmp = dH;
        dH = dHn;
        dHn = tmp;
    }
    // 3. the input layer: dPre0 = dH (H0 > 0), db_in, dWin += X^T dPre0
    if (!gg::grid_sync(a.ctl, a.expected, a.wait_ns, 2 * kLayers + 1, epoch)) return;
    {
        float g_b = 0.f;
        for (int rb = blockIdx.x; rb < nrb; rb += gridDim.x) {
            const int v0 = rb * 64;
#pragma unroll 8
            for (int e = tid; e < 64 * kH; e += kFwdBlock) {
                const int r = e / kH, c = e % kH, v = v0 + r;
                if (v < a.n) {
                    const float q = a.H[0][(size_t)v * kH + c] > 0.f ? __ldcg(dH + (size_t)v * kH + c) : 0.f;
                    dH[(size_t)v * kH + c] = q;
                    g_b += q;
                }
            }
            __syncthreads();
            stage_cols(Bt, dH, kH, v0, a.n, 0, kH);   // Bt[c][r] = dPre0[v0 + r][c]
            for (int f0 = 0; f0 < a.F; f0 += 64) {
                stage_cols(As, a.X, a.F, v0, a.n, f0, a.F);   // As[f][r] = X[v0 + r][f0 + f]
                __syncthreads();
                tile_mma(As, Bt, 64, acc);
                tile_out<true>(acc, Gd + a.o_win, kH, f0, min(64, a.F - f0), 0, kH);
                __syncthreads();
            }
        }
        atomicAdd(Gd + a.o_bin + jc, g_b);
    }
    // 4. Adam on every parameter
    if (a.train) {
        if (!gg::grid_sync(a.ctl, a.expected, a.wait_ns, 2 * kLayers + 2, epoch)) return;
        const float lr = a.hyper[kHypLr], c1 = a.hyper[kHypC1], c2 = a.hyper[kHypC2];
        for (long long i = gtid; i < a.n_params; i += nthr) {
            const float gi = __ldcg(Gd + i);
            const float b1 = 0.9f, b2 = 0.999f;
            const float mi = b1 * a.adam_m[i] + (1.f - b1) * gi;
            const float vi = b2 * a.adam_v[i] + (1.f - b2) * gi * gi;
            a.adam_m[i] = mi;
            a.adam_v[i] = vi;
            a.params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host object
// ---------------------------------------------------------------------------
struct gg_surrogate {
    int device = 0, n = 0, d = 0, F = 0;
    cudaStream_t st = nullptr;
    // parameter layout offsets (floats)
    int o_win = 0, o_bin = 0, o_ws[kLayers], o_wn[kLayers], o_b[kLayers], o_wr1 = 0, o_br1 = 0,
        o_wr2 = 0, o_br2 = 0, n_params = 0;
    float *params = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    int32_t *adj = nullptr;
    float *X = nullptr;
    float *Hs[kLayers + 1] = {};
    float *Ms[kLayers] = {};
    float *dH0 = nullptr, *dH1 = nullptr, *G = nullptr;
    // per-swap device buffers and their pinned host staging (capacity `cap`)
    int cap = 0;
    gg_swap *sw = nullptr, *h_sw = nullptr;
    float *Z = nullptr, *O = nullptr, *y = nullptr, *t = nullptr, *dO = nullptr, *dZ = nullptr;
    float *h_y = nullptr, *h_t = nullptr;
    int32_t *mask = nullptr, *h_mask = nullptr;
    float *loss = nullptr, *h_loss = nullptr;
    float *hyper = nullptr, *h_hyper = nullptr;
    gg::Ctl *ctl = nullptr;                // grid barrier of the fused forward launch
    int *h_err = nullptr;                  // its wait status, copied back after each call
    int fwd_per_sm = 0, bwd_per_sm = 0, sms = 0;
    bool fwd_valid = false, graph_set = false;
    long long adam_step = 0;
    // captured launch sequences, per swap count: predict (with the graph
    // forward), readout+backward (grad), readout+backward+Adam (train)
    struct Cached { int P; int kind; cudaGraphExec_t exec; };
    std::vector<Cached> graphs;
};

namespace {

gg_status sfail(gg_status s, const std::string &m) {
    (void)cudaGetLastError();
    gg::set_last_error(m.c_str());
    return s;
}

#define GS_CK(call)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return sfail(e_ == cudaErrorMemoryAllocation ? GG_OUT_OF_MEMORY : GG_CUDA_ERROR, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                \
    } while (0)


void drop_graphs(gg_surrogate *s) {
    for (auto &c : s->graphs) cudaGraphExecDestroy(c.exec);
    s->graphs.clear();
}

gg_status ensure_swaps(gg_surrogate *s, int P) {
    if (P <= s->cap) return GG_OK;
    const int cap = std::max(P, 2 * s->cap);
    drop_graphs(s);
    cudaFree(s->sw); cudaFree(s->Z); cudaFree(s->O); cudaFree(s->y); cudaFree(s->t);
    cudaFree(s->dO); cudaFree(s->dZ); cudaFree(s->mask);
    cudaFreeHost(s->h_sw); cudaFreeHost(s->h_y); cudaFreeHost(s->h_t); cudaFreeHost(s->h_mask);
    s->cap = 0;
    GS_CK(cudaMalloc(&s->sw, (size_t)cap * sizeof(gg_swap)));
    GS_CK(cudaMalloc(&s->Z, (size_t)cap * kZ * 4));
    GS_CK(cudaMalloc(&s->O, (size_t)cap * kH * 4));
    GS_CK(cudaMalloc(&s->y, (size_t)cap * 4));
    GS_CK(cudaMalloc(&s->t, (size_t)cap * 4));
    GS_CK(cudaMalloc(&s->dO, (size_t)cap * kH * 4));
    GS_CK(cudaMalloc(&s->dZ, (size_t)cap * kZ * 4));
    GS_CK(cudaMalloc(&s->mask, (size_t)cap * 4));
    GS_CK(cudaMallocHost(&s->h_sw, (size_t)cap * sizeof(gg_swap)));
    GS_CK(cudaMallocHost(&s->h_y, (size_t)cap * 4));
    GS_CK(cudaMallocHost(&s->h_t, (size_t)cap * 4));
    GS_CK(cudaMallocHost(&s->h_mask, (size_t)cap * 4));
    s->cap = cap;
    return GG_OK;
}

constexpr size_t kFwdSmem = 2 * 64 * kFwdLd * sizeof(uint16_t);

// One fused launch (surrogate_forward_kernel): the embeddings of the current graph
// when `graph` (H0 .. H3 and the neighbour means M0 .. M2), then the readout of the
// P swaps in s->sw (Z, O, y) when P > 0.  The barrier status goes to s->h_err.
void forward_fused(gg_surrogate *s, bool graph, int P) {
    FwdArgs a{};
    a.X = s->X; a.F = s->F; a.adj = s->adj; a.n = graph ? s->n : 0; a.d = s->d;
    a.P = s->params;
    a.o_win = s->o_win; a.o_bin = s->o_bin;
    for (int l = 0; l < kLayers; ++l) { a.o_ws[l] = s->o_ws[l]; a.o_wn[l] = s->o_wn[l]; a.o_b[l] = s->o_b[l]; }
    a.o_wr1 = s->o_wr1; a.o_br1 = s->o_br1; a.o_wr2 = s->o_wr2; a.o_br2 = s->o_br2;
    for (int l = 0; l <= kLayers; ++l) a.H[l] = s->Hs[l];
    for (int l = 0; l < kLayers; ++l) a.M[l] = s->Ms[l];
    a.sw = s->sw; a.n_sw = P; a.Z = s->Z; a.O = s->O; a.y = s->y;
    const int tiles = std::max((a.n + 63) / 64, (P + 63) / 64);
    const int grid = std::max(1, std::min(s->fwd_per_sm * s->sms, tiles));
    a.ctl = s->ctl;
    a.expected = (unsigned)grid;
    a.wait_ns = 10ll * 1000 * 1000 * 1000;
    cudaMemsetAsync(s->ctl, 0, sizeof(gg::Ctl), s->st);
    void *args[] = {&a};
    cudaLaunchCooperativeKernel((void *)surrogate_forward_kernel, dim3(grid), dim3(kFwdBlock), args, kFwdSmem, s->st);
    cudaMemcpyAsync(s->h_err, &s->ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s->st);
}

// Embeddings of the current graph: H0 .. H3 (and the neighbour means M0 .. M2).
void forward_graph(gg_surrogate *s) { forward_fused(s, true, 0); }

// Readout of the P swaps in s->sw: Z, O, y.
void forward_readout(gg_surrogate *s, int P) { forward_fused(s, false, P); }

// Loss and full gradient into s->grad (zeroed here) for the swaps/targets/mask on the
// device, and with `train` the Adam step: one fused launch (surrogate_backward_kernel).
// Its barrier status goes to s->h_err[1].
void backward(gg_surrogate *s, int P, bool train) {
    cudaMemsetAsync(s->grad, 0, (size_t)s->n_params * 4, s->st);
    cudaMemsetAsync(s->loss, 0, 4, s->st);
    cudaMemsetAsync(s->dH0, 0, (size_t)s->n * kH * 4, s->st);
    BwdArgs a{};
    a.X = s->X; a.F = s->F; a.adj = s->adj; a.n = s->n; a.d = s->d;
    a.P = s->params; a.Gd = s->grad;
    a.o_win = s->o_win; a.o_bin = s->o_bin;
    for (int l = 0; l < kLayers; ++l) { a.o_ws[l] = s->o_ws[l]; a.o_wn[l] = s->o_wn[l]; a.o_b[l] = s->o_b[l]; }
    a.o_wr1 = s->o_wr1; a.o_br1 = s->o_br1; a.o_wr2 = s->o_wr2; a.o_br2 = s->o_br2;
    for (int l = 0; l <= kLayers; ++l) a.H[l] = s->Hs[l];
    for (int l = 0; l < kLayers; ++l) a.M[l] = s->Ms[l];
    a.sw = s->sw; a.n_sw = P;
    a.Z = s->Z; a.O = s->O; a.y = s->y; a.t = s->t; a.mask = s->mask; a.hyper = s->hyper;
    a.dO = s->dO; a.dZ = s->dZ; a.dHa = s->dH0; a.dHb = s->dH1; a.Gt = s->G; a.loss = s->loss;
    a.adam_m = s->adam_m; a.adam_v = s->adam_v; a.params = s->params;
    a.n_params = s->n_params; a.train = train ? 1 : 0;
    // every resident block: the tile stages take one block a 64-row tile, the
    // neighbour means and Adam use them all
    const int grid = std::max(1, s->bwd_per_sm * s->sms);
    a.ctl = s->ctl;
    a.expected = (unsigned)grid;
    a.wait_ns = 10ll * 1000 * 1000 * 1000;
    cudaMemsetAsync(s->ctl, 0, sizeof(gg::Ctl), s->st);
    void *args[] = {&a};
    cudaLaunchCooperativeKernel((void *)surrogate_backward_kernel, dim3(grid), dim3(kFwdBlock), args, kFwdSmem, s->st);
    cudaMemcpyAsync(s->h_err + 1, &s->ctl->err, sizeof(int), cudaMemcpyDeviceToHost, s->st);
}

enum { kPredict = 0, kGrad = 1, kTrain = 2 };

// The launch sequence of one call kind for P swaps, staged from/to pinned memory.
void enqueue_kind(gg_surrogate *s, int kind, int P) {
    cudaMemcpyAsync(s->sw, s->h_sw, (size_t)P * sizeof(gg_swap), cudaMemcpyHostToDevice, s->st);
    if (kind == kPredict) {
        forward_fused(s, true, P);
        cudaMemcpyAsync(s->h_y, s->y, (size_t)P * 4, cudaMemcpyDeviceToHost, s->st);
        return;
    }
    cudaMemcpyAsync(s->t, s->h_t, (size_t)P * 4, cudaMemcpyHostToDevice, s->st);
    cudaMemcpyAsync(s->mask, s->h_mask, (size_t)P * 4, cudaMemcpyHostToDevice, s->st);
    cudaMemcpyAsync(s->hyper, s->h_hyper, kHypN * 4, cudaMemcpyHostToDevice, s->st);
    forward_readout(s, P);
    backward(s, P, kind == kTrain);
    cudaMemcpyAsync(s->h_loss, s->loss, 4, cudaMemcpyDeviceToHost, s->st);
}

// Replay (capturing on first use) the sequence `kind` for P swaps, then wait.
gg_status run_kind(gg_surrogate *s, int kind, int P) {
    cudaGraphExec_t exec = nullptr;
    for (auto &c : s->graphs)
        if (c.P == P && c.kind == kind) exec = c.exec;
    if (!exec) {
        GS_CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
        enqueue_kind(s, kind, P);
        cudaGraph_t g = nullptr;
        GS_CK(cudaStreamEndCapture(s->st, &g));
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        GS_CK(e);
        s->graphs.push_back({P, kind, exec});
    }
    GS_CK(cudaGraphLaunch(exec, s->st));
    GS_CK(cudaStreamSynchronize(s->st));
    if (s->h_err[0]) return sfail(GG_TIMEOUT, "grid barrier wait of the fused forward exceeded its limit");
    if (kind != kPredict && s->h_err[1])
        return sfail(GG_TIMEOUT, "grid barrier wait of the fused backward exceeded its limit");
    return GG_OK;
}

gg_status stage_swaps(gg_surrogate *s, int P, const gg_swap *swaps) {
    for (int i = 0; i < P; ++i) {
        const gg_swap &w = swaps[i];
        if (w.a < 0 || w.a >= s->n || w.b < 0 || w.b >= s->n || w.c < 0 || w.c >= s->n || w.d < 0 ||
            w.d >= s->n || (w.mode != 0 && w.mode != 1))
            return sfail(GG_BAD_ARG, "swap " + std::to_string(i) + " out of range");
    }
    gg_status r = ensure_swaps(s, P);
    if (r != GG_OK) return r;
    std::memcpy(s->h_sw, swaps, (size_t)P * sizeof(gg_swap));
    return GG_OK;
}

gg_status grad_common(gg_surrogate *s, int kind, int P, const gg_swap *swaps, const float *target,
                      const int32_t *mask, float lr, float *loss) {
    if (!s || P < 1 || !swaps || !target) return sfail(GG_BAD_ARG, "bad arguments");
    if (!s->graph_set) return sfail(GG_BAD_ARG, "no graph set");
    GS_CK(cudaSetDevice(s->device));
    gg_status r = stage_swaps(s, P, swaps);
    if (r != GG_OK) return r;
    int cnt = 0;
    for (int i = 0; i < P; ++i) {
        s->h_mask[i] = mask ? (mask[i] != 0) : 1;
        cnt += s->h_mask[i];
    }
    std::memcpy(s->h_t, target, (size_t)P * 4);
    s->h_hyper[kHypInvCnt] = cnt ? 1.f / (float)cnt : 0.f;
    s->h_hyper[kHypLr] = lr;
    if (kind == kTrain) {
        const long long t = s->adam_step + 1;
        s->h_hyper[kHypC1] = 1.f - std::pow(0.9f, (float)t);
        s->h_hyper[kHypC2] = 1.f - std::pow(0.999f, (float)t);
    }
    if (!s->fwd_valid) {  // embeddings of the current graph and parameters
        forward_graph(s);
        GS_CK(cudaGetLastError());
        GS_CK(cudaStreamSynchronize(s->st));
        if (*s->h_err) return sfail(GG_TIMEOUT, "grid barrier wait of the fused forward exceeded its limit");
        s->fwd_valid = true;
    }
    r = run_kind(s, kind, P);
    if (r != GG_OK) return r;
    if (kind == kTrain) {
        s->adam_step += 1;
        s->fwd_valid = false;
    }
    if (loss) *loss = *s->h_loss;
    return GG_OK;
}

}  // namespace

extern "C" {

gg_status gg_surrogate_create(int device, int n, int degree, int in_features, uint64_t seed,
                              gg_surrogate **out) {
    if (!out || n < 2 || degree < 1 || in_features < 1 || in_features > 256)
        return sfail(GG_BAD_ARG, "need n >= 2, degree >= 1, 1 <= in_features <= 256");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return sfail(GG_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return sfail(GG_NO_DEVICE, "device index out of range");
    gg_surrogate *s = new gg_surrogate();
    s->device = device; s->n = n; s->d = degree; s->F = in_features;
    int o = 0;
    s->o_win = o; o += in_features * kH;
    s->o_bin = o; o += kH;
    for (int l = 0; l < kLayers; ++l) {
        s->o_ws[l] = o; o += kH * kH;
        s->o_wn[l] = o; o += kH * kH;
        s->o_b[l] = o; o += kH;
    }
    s->o_wr1 = o; o += kZ * kH;
    s->o_br1 = o; o += kH;
    s->o_wr2 = o; o += kH;
    s->o_br2 = o; o += 1;
    s->n_params = o;
    // Glorot-uniform weights, zero biases, from a seeded host generator
    std::vector<float> p(o, 0.f);
    uint64_t x = seed * 0x9e3779b97f4a7c15ull + 1;
    auto unif = [&]() {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;  // xorshift64
        return (double)(x >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int fin, int fout) {
        const double a = std::sqrt(6.0 / (fin + fout));
        for (int i = 0; i < fin * fout; ++i) p[off + i] = (float)((2 * unif() - 1) * a);
    };
    fill(s->o_win, in_features, kH);
    for (int l = 0; l < kLayers; ++l) { fill(s->o_ws[l], kH, kH); fill(s->o_wn[l], kH, kH); }
    fill(s->o_wr1, kZ, kH);
    fill(s->o_wr2, kH, 1);
    auto bad = [&](gg_status st) { gg_surrogate_destroy(s); return st; };
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess)
        return bad(sfail(GG_CUDA_ERROR, "stream creation failed"));
    const size_t pb = (size_t)o * 4;
    bool ok = cudaMalloc(&s->params, pb) == cudaSuccess && cudaMalloc(&s->grad, pb) == cudaSuccess &&
              cudaMalloc(&s->adam_m, pb) == cudaSuccess && cudaMalloc(&s->adam_v, pb) == cudaSuccess &&
              cudaMalloc(&s->adj, (size_t)n * degree * 4) == cudaSuccess &&
              cudaMalloc(&s->X, (size_t)n * in_features * 4) == cudaSuccess &&
              cudaMalloc(&s->dH0, (size_t)n * kH * 4) == cudaSuccess &&
              cudaMalloc(&s->dH1, (size_t)n * kH * 4) == cudaSuccess &&
              cudaMalloc(&s->G, (size_t)n * kH * 4) == cudaSuccess &&
              cudaMalloc(&s->loss, 4) == cudaSuccess && cudaMalloc(&s->hyper, kHypN * 4) == cudaSuccess &&
              cudaMallocHost(&s->h_loss, 4) == cudaSuccess && cudaMallocHost(&s->h_hyper, kHypN * 4) == cudaSuccess &&
              cudaMalloc(&s->ctl, sizeof(gg::Ctl)) == cudaSuccess && cudaMallocHost(&s->h_err, 2 * sizeof(int)) == cudaSuccess;
    for (int l = 0; l <= kLayers && ok; ++l) ok = cudaMalloc(&s->Hs[l], (size_t)n * kH * 4) == cudaSuccess;
    for (int l = 0; l < kLayers && ok; ++l) ok = cudaMalloc(&s->Ms[l], (size_t)n * kH * 4) == cudaSuccess;
    if (!ok) return bad(sfail(GG_OUT_OF_MEMORY, "surrogate allocation failed"));
    std::memset(s->h_hyper, 0, kHypN * 4);
    s->h_err[0] = s->h_err[1] = 0;
    if (cudaFuncSetAttribute(surrogate_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->fwd_per_sm, surrogate_forward_kernel, kFwdBlock, kFwdSmem) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || s->fwd_per_sm < 1)
        return bad(sfail(GG_CUDA_ERROR, "fused forward cannot be resident"));
    if (cudaFuncSetAttribute(surrogate_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->bwd_per_sm, surrogate_backward_kernel, kFwdBlock, kFwdSmem) !=
            cudaSuccess ||
        s->bwd_per_sm < 1)
        return bad(sfail(GG_CUDA_ERROR, "fused backward cannot be resident"));
    if (cudaMemcpy(s->params, p.data(), pb, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(s->adam_m, 0, pb) != cudaSuccess || cudaMemset(s->adam_v, 0, pb) != cudaSuccess)
        return bad(sfail(GG_CUDA_ERROR, "surrogate initialisation failed"));
    *out = s;
    return GG_OK;
}

gg_status gg_surrogate_set_graph(gg_surrogate *s, const int32_t *adj, const float *features) {
    if (!s || !adj || !features) return sfail(GG_BAD_ARG, "null argument");
    for (long long k = 0; k < (long long)s->n * s->d; ++k)
        if (adj[k] < 0 || adj[k] >= s->n) return sfail(GG_BAD_ARG, "adjacency entry outside [0, n)");
    GS_CK(cudaSetDevice(s->device));
    GS_CK(cudaMemcpyAsync(s->adj, adj, (size_t)s->n * s->d * 4, cudaMemcpyHostToDevice, s->st));
    GS_CK(cudaMemcpyAsync(s->X, features, (size_t)s->n * s->F * 4, cudaMemcpyHostToDevice, s->st));
    s->graph_set = true;
    s->fwd_valid = false;
    GS_CK(cudaStreamSynchronize(s->st));
    return GG_OK;
}

gg_status gg_surrogate_predict(gg_surrogate *s, int P, const gg_swap *swaps, float *pred) {
    if (!s || P < 0 || (P && (!swaps || !pred))) return sfail(GG_BAD_ARG, "bad arguments");
    if (!s->graph_set) return sfail(GG_BAD_ARG, "no graph set");
    if (P == 0) return GG_OK;
    GS_CK(cudaSetDevice(s->device));
    gg_status r = stage_swaps(s, P, swaps);
    if (r != GG_OK) return r;
    r = run_kind(s, kPredict, P);  // recomputes the embeddings: they are valid afterwards
    if (r != GG_OK) return r;
    s->fwd_valid = true;
    std::memcpy(pred, s->h_y, (size_t)P * 4);
    return GG_OK;
}

gg_status gg_surrogate_grad(gg_surrogate *s, int P, const gg_swap *swaps, const float *target,
                            const int32_t *mask, float *grad, float *loss) {
    if (!grad) return sfail(GG_BAD_ARG, "null grad");
    gg_status r = grad_common(s, kGrad, P, swaps, target, mask, 0.f, loss);
    if (r != GG_OK) return r;
    GS_CK(cudaMemcpy(grad, s->grad, (size_t)s->n_params * 4, cudaMemcpyDeviceToHost));
    return GG_OK;
}

gg_status gg_surrogate_train(gg_surrogate *s, int P, const gg_swap *swaps, const float *target,
                             const int32_t *mask, float lr, float *loss) {
    return grad_common(s, kTrain, P, swaps, target, mask, lr, loss);
}

gg_status gg_surrogate_param_count(gg_surrogate *s, int *count) {
    if (!s || !count) return sfail(GG_BAD_ARG, "null argument");
    *count = s->n_params;
    return GG_OK;
}

gg_status gg_surrogate_get_params(gg_surrogate *s, float *params) {
    if (!s || !params) return sfail(GG_BAD_ARG, "null argument");
    GS_CK(cudaSetDevice(s->device));
    GS_CK(cudaMemcpy(params, s->params, (size_t)s->n_params * 4, cudaMemcpyDeviceToHost));
    return GG_OK;
}

gg_status gg_surrogate_set_params(gg_surrogate *s, const float *params) {
    if (!s || !params) return sfail(GG_BAD_ARG, "null argument");
    GS_CK(cudaSetDevice(s->device));
    GS_CK(cudaMemcpy(s->params, params, (size_t)s->n_params * 4, cudaMemcpyHostToDevice));
    s->fwd_valid = false;
    return GG_OK;
}

gg_status gg_surrogate_destroy(gg_surrogate *s) {
    if (!s) return GG_OK;
    cudaSetDevice(s->device);
    if (s->st) cudaStreamSynchronize(s->st);
    drop_graphs(s);
    cudaFree(s->params); cudaFree(s->grad); cudaFree(s->adam_m); cudaFree(s->adam_v);
    cudaFree(s->adj); cudaFree(s->X); cudaFree(s->dH0); cudaFree(s->dH1); cudaFree(s->G); cudaFree(s->loss);
    cudaFree(s->hyper); cudaFreeHost(s->h_loss); cudaFreeHost(s->h_hyper);
    cudaFree(s->ctl); cudaFreeHost(s->h_err);
    for (auto p : s->Hs) cudaFree(p);
    for (auto p : s->Ms) cudaFree(p);
    cudaFree(s->sw); cudaFree(s->Z); cudaFree(s->O); cudaFree(s->y); cudaFree(s->t);
    cudaFree(s->dO); cudaFree(s->dZ); cudaFree(s->mask);
    cudaFreeHost(s->h_sw); cudaFreeHost(s->h_y); cudaFreeHost(s->h_t); cudaFreeHost(s->h_mask);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
    return GG_OK;
}

}  // extern "C"
