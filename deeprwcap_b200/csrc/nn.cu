// Learned transition kernels: a small 3-D convolutional network on a cube's
// N^3 permittivity (N = 16, 21 or 23), with BF16 operands and FP32 accumulation on the
// tensor cores (tcgen05 GEMM tiles of umma.cuh), FP32 master weights and a
// hand-written backward pass and AdamW update.
//
//   input   X  [B, N^3]             eps / max eps of the cube, BF16
//   conv1   1 -> 16, 3^3, stride 2, pad 1, ReLU     A1 [B*D2^3, 16]
//   conv2  16 -> 32, 3^3, stride 2, pad 1, ReLU     A2 [B*D3^3, 32]
//   conv3  32 -> 64, 3^3, stride 2, pad 1, ReLU     A3 [B*D4^3, 64] = F [B, 64*D4^3]
//           (D_{l+1} = (D_l - 1) / 2 + 1: N = 16 -> 8, 4, 2; 21 -> 11, 6, 3;
//           23 -> 12, 6, 3)
//   heads   O = F Wd^T + bd  [B, DEC]: 6N^2 Poisson-kernel logits (softmax over
//           the panels, ggft panel order) and 1 confidence output (the
//           predicted log10 KL divergence to the FDM Green's function), DEC =
//           6N^2 + 1 rounded up to 16 (1552 at N = 16);
//           G = F Wg^T + bg  [B, GLD]: the 6N^2 centre-gradient surface values
//           along z (WVTZ), scaled, rows padded to GLD = 6N^2 rounded up to
//           16; other axes rotate the cube first.
//
// Layers are implicit GEMMs: rows are output positions (channels-last), K is
// (tap, input channel) with the channel fastest, so an 8-wide K chunk of a
// conv is one 16-byte load of 8 channels at one tap. The backward pass uses
// the same tile: weight gradients as split-K GEMMs over (batch x position),
// input gradients as transposed-convolution gathers. Inference (the forward
// entry points, the learned walker, the server) runs conv1 and conv2 fused
// in one CTA per group of cubes (stem.cuh), so A1 never reaches global
// memory; training runs every layer as a GEMM and keeps A1 for the backward
// pass.
//
// The architecture follows the learned-transition design of DeepRWCap
// (training_pytorch/src/architecture.py: small 3-D conv encoders on the
// normalised permittivity, per-sample max normalisation train.py:59-60,
// softmax-normalised Poisson outputs, KL loss train.py:69-120).
#include <cmath>
#include <cstring>
#include <random>
#include <type_traits>
#include <vector>

#include "host.cuh"
#include "nn.cuh"
#include "stem.cuh"
#include "umma_launch.cuh"
#include "umma_tma.cuh"

namespace drwc {

// Layer sizes of the network for cube resolution N.
template <int N>
struct NetDims {
    static constexpr int D1 = N, D2 = (D1 - 1) / 2 + 1, D3 = (D2 - 1) / 2 + 1,
                         D4 = (D3 - 1) / 2 + 1;
    static constexpr int P2 = D2 * D2 * D2, P3 = D3 * D3 * D3, P4 = D4 * D4 * D4;
    static constexpr int NP = 6 * N * N;               // panels
    static constexpr int DEC = (NP + 1 + 15) / 16 * 16; // Poisson logits + confidence, padded
    static constexpr int GLD = (NP + 15) / 16 * 16;     // gradient-head row stride
    static constexpr int FEAT = 64 * P4;
};

// Calls f(std::integral_constant<int, N>) for a served network resolution.
template <class F>
inline int net_dispatch(int N, F&& f) {
    switch (N) {
        case 16: return f(std::integral_constant<int, 16>{});
        case 21: return f(std::integral_constant<int, 21>{});
        case 23: return f(std::integral_constant<int, 23>{});
        default: return DRWC_ERR_INVALID;
    }
}

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------- loaders
// Conv input gather: input [B, D^3, C] channels-last (C = 1: the cube),
// output position row r = b * Do^3 + p, K index = tap * C + ci.
template <int D, int C>
struct ConvGather {
    const bf16* __restrict__ x;
    int rows;  // B * Do^3
    // with 8k input channels a chunk is 8 channels of one tap: 16 contiguous bytes
    static constexpr bool kChunks = C % 8 == 0;
    DRWC_DEV bool chunks_ok() const { return (reinterpret_cast<uintptr_t>(x) & 15) == 0; }
    DRWC_DEV const void* chunk(int r, int k8) const {
        constexpr int Do = (D - 1) / 2 + 1, P = Do * Do * Do, K = 27 * C;
        if (r >= rows || k8 >= K) return nullptr;
        const int b = r / P, p = r % P;
        const int pz = p / (Do * Do), py = (p / Do) % Do, px = p % Do;
        const int tap = k8 / C, ci = k8 % C;
        const int z = 2 * pz - 1 + tap / 9, y = 2 * py - 1 + (tap / 3) % 3, xx = 2 * px - 1 + tap % 3;
        if (z < 0 || z >= D || y < 0 || y >= D || xx < 0 || xx >= D) return nullptr;
        return x + ((((int64_t)b * D + z) * D + y) * D + xx) * C + ci;
    }
    DRWC_DEV void operator()(int r, int k8, uint4* out) const {
        constexpr int Do = (D - 1) / 2 + 1, P = Do * Do * Do, K = 27 * C;
        if (r >= rows || k8 >= K) { *out = make_uint4(0, 0, 0, 0); return; }
        const int b = r / P, p = r % P;
        const int pz = p / (Do * Do), py = (p / Do) % Do, px = p % Do;
        if constexpr (C % 8 == 0) {
            const int tap = k8 / C, ci = k8 % C;
            const int z = 2 * pz - 1 + tap / 9, y = 2 * py - 1 + (tap / 3) % 3, xx = 2 * px - 1 + tap % 3;
            if (z < 0 || z >= D || y < 0 || y >= D || xx < 0 || xx >= D) {
                *out = make_uint4(0, 0, 0, 0);
                return;
            }
            *out = *reinterpret_cast<const uint4*>(
                x + ((((int64_t)b * D + z) * D + y) * D + xx) * C + ci);
        } else {
            __align__(16) bf16 tmp[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int k = k8 + i;
                bf16 v = __float2bfloat16(0.f);
                if (k < K) {
                    const int tap = k / C, ci = k % C;
                    const int z = 2 * pz - 1 + tap / 9, y = 2 * py - 1 + (tap / 3) % 3,
                              xx = 2 * px - 1 + tap % 3;
                    if (z >= 0 && z < D && y >= 0 && y < D && xx >= 0 && xx < D)
                        v = x[((((int64_t)b * D + z) * D + y) * D + xx) * C + ci];
                }
                tmp[i] = v;
            }
            *out = *reinterpret_cast<const uint4*>(tmp);
        }
    }
};

// Weight-gradient operand: im2col(input)^T. Operand row = K index (tap, ci),
// operand column = output row r (b, p), 8 consecutive r per chunk.
template <int D, int C>
struct Im2colT {
    const bf16* __restrict__ x;
    int nrows;  // B * Do^3 (the reduction length)
    static constexpr bool kChunks = false;
    DRWC_DEV void operator()(int kk, int r8, uint4* out) const {
        constexpr int Do = (D - 1) / 2 + 1, P = Do * Do * Do, K = 27 * C;
        __align__(16) bf16 tmp[8];
        const int tap = kk / C, ci = kk % C;
        const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int r = r8 + i;
            bf16 v = __float2bfloat16(0.f);
            if (kk < K && r < nrows) {
                const int b = r / P, p = r % P;
                const int z = 2 * (p / (Do * Do)) - 1 + dz, y = 2 * ((p / Do) % Do) - 1 + dy,
                          xx = 2 * (p % Do) - 1 + dx;
                if (z >= 0 && z < D && y >= 0 && y < D && xx >= 0 && xx < D)
                    v = x[((((int64_t)b * D + z) * D + y) * D + xx) * C + ci];
            }
            tmp[i] = v;
        }
        *out = *reinterpret_cast<const uint4*>(tmp);
    }
};

// Input-gradient operand: for input position row (b, q) and K index
// (tap, co), the output gradient dZ[b, p, co] of the output position p that
// reads q through tap (2p - 1 + d = q on every axis), zero when none does.
template <int D, int CO>
struct ConvTGather {
    const bf16* __restrict__ dz;  // [B * Do^3, CO]
    int rows;                     // B * D^3
    static constexpr bool kChunks = false;
    DRWC_DEV void operator()(int r, int k8, uint4* out) const {
        constexpr int Do = (D - 1) / 2 + 1, P = Do * Do * Do, Q = D * D * D, K = 27 * CO;
        static_assert(CO % 8 == 0, "output channels per chunk");
        if (r >= rows || k8 >= K) { *out = make_uint4(0, 0, 0, 0); return; }
        const int b = r / Q, q = r % Q;
        const int qz = q / (D * D), qy = (q / D) % D, qx = q % D;
        const int tap = k8 / CO, co = k8 % CO;
        const int tz = qz + 1 - tap / 9, ty = qy + 1 - (tap / 3) % 3, tx = qx + 1 - tap % 3;
        if ((tz | ty | tx) & 1 || tz < 0 || ty < 0 || tx < 0) {
            *out = make_uint4(0, 0, 0, 0);
            return;
        }
        const int pz = tz >> 1, py = ty >> 1, px = tx >> 1;
        if (pz >= Do || py >= Do || px >= Do) { *out = make_uint4(0, 0, 0, 0); return; }
        *out = *reinterpret_cast<const uint4*>(dz + ((int64_t)b * P + (pz * Do + py) * Do + px) * CO + co);
    }
};

// Input-gradient weight operand: rows ci, K index (tap, co): W[co][tap*CI + ci].
template <int CI, int CO>
struct WeightT {
    const bf16* __restrict__ w;  // [CO][27*CI]
    static constexpr bool kChunks = false;
    DRWC_DEV void operator()(int ci, int k8, uint4* out) const {
        __align__(16) bf16 tmp[8];
        const int tap = k8 / CO, co0 = k8 % CO;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const bool in = ci < CI && k8 < 27 * CO;
            tmp[i] = in ? w[(int64_t)(co0 + i) * 27 * CI + tap * CI + ci] : __float2bfloat16(0.f);
        }
        *out = *reinterpret_cast<const uint4*>(tmp);
    }
};

// ---------------------------------------------------------------- epilogues
// bias + ReLU -> BF16 rows [rows, N].
struct EpiReluBf16 {
    bf16* __restrict__ out;
    const float* __restrict__ bias;
    int N;
    DRWC_DEV void operator()(int row, int col0, const float* v) const {
        bf16* dst = out + (int64_t)row * N;
        if (col0 + 32 <= N && ((reinterpret_cast<uintptr_t>(dst + col0) & 15) == 0)) {
            // 32 values = four 16-byte stores
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                __align__(16) __nv_bfloat162 h[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int i = 8 * q + 2 * e;
                    h[e] = __floats2bfloat162_rn(fmaxf(v[i] + bias[col0 + i], 0.f),
                                                 fmaxf(v[i + 1] + bias[col0 + i + 1], 0.f));
                }
                reinterpret_cast<uint4*>(dst + col0)[q] = *reinterpret_cast<const uint4*>(h);
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int c = col0 + i;
            if (c < N) dst[c] = __float2bfloat16(fmaxf(v[i] + bias[c], 0.f));
        }
    }
    // 4 consecutive columns (col a multiple of 4) of one row.
    DRWC_DEV void store4(int row, int col, float4 v) const {
        bf16* dst = out + (int64_t)row * N + col;
        if (col + 4 <= N && (reinterpret_cast<uintptr_t>(dst) & 7) == 0) {
            __align__(8) __nv_bfloat162 h[2];
            h[0] = __floats2bfloat162_rn(fmaxf(v.x + bias[col], 0.f), fmaxf(v.y + bias[col + 1], 0.f));
            h[1] = __floats2bfloat162_rn(fmaxf(v.z + bias[col + 2], 0.f), fmaxf(v.w + bias[col + 3], 0.f));
            *reinterpret_cast<uint2*>(dst) = *reinterpret_cast<const uint2*>(h);
            return;
        }
        const float e[4] = {v.x, v.y, v.z, v.w};
        for (int i = 0; i < 4 && col + i < N; ++i)
            dst[i] = __float2bfloat16(fmaxf(e[i] + bias[col + i], 0.f));
    }
};

// bias -> FP32 rows [rows, ld].
struct EpiF32 {
    float* __restrict__ out;
    const float* __restrict__ bias;
    int N;
    int64_t ld;
    const int* __restrict__ rowmap;  // output row = rowmap[row] when set
    DRWC_DEV void operator()(int row, int col0, const float* v) const {
        float* dst = out + (int64_t)(rowmap ? rowmap[row] : row) * ld;
        if (col0 + 32 <= N && ((reinterpret_cast<uintptr_t>(dst + col0) & 15) == 0)) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                float4 o;
                o.x = v[4 * q] + (bias ? bias[col0 + 4 * q] : 0.f);
                o.y = v[4 * q + 1] + (bias ? bias[col0 + 4 * q + 1] : 0.f);
                o.z = v[4 * q + 2] + (bias ? bias[col0 + 4 * q + 2] : 0.f);
                o.w = v[4 * q + 3] + (bias ? bias[col0 + 4 * q + 3] : 0.f);
                reinterpret_cast<float4*>(dst + col0)[q] = o;
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int c = col0 + i;
            if (c < N) dst[c] = v[i] + (bias ? bias[c] : 0.f);
        }
    }
    // 4 consecutive columns (col a multiple of 4) of one row.
    DRWC_DEV void store4(int row, int col, float4 v) const {
        float* dst = out + (int64_t)(rowmap ? rowmap[row] : row) * ld + col;
        if (col + 4 <= N && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
            if (bias) { v.x += bias[col]; v.y += bias[col + 1]; v.z += bias[col + 2]; v.w += bias[col + 3]; }
            *reinterpret_cast<float4*>(dst) = v;
            return;
        }
        const float e[4] = {v.x, v.y, v.z, v.w};
        for (int i = 0; i < 4 && col + i < N; ++i) dst[i] = e[i] + (bias ? bias[col + i] : 0.f);
    }
};

// Accumulate into FP32 [rows, N] with atomics (split-K weight gradients).
struct EpiAtomicF32 {
    float* __restrict__ out;
    int N;
    DRWC_DEV void operator()(int row, int col0, const float* v) const {
        float* dst = out + (int64_t)row * N;
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if (col0 + i < N) atomicAdd(dst + col0 + i, v[i]);
    }
};

// Input gradient through ReLU: dZ_in = dA * (A > 0) -> BF16.
struct EpiReluGrad {
    bf16* __restrict__ out;
    const bf16* __restrict__ act;  // the forward activation of this layer's input
    int N;
    DRWC_DEV void operator()(int row, int col0, const float* v) const {
        const int64_t base = (int64_t)row * N;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int c = col0 + i;
            if (c < N) {
                const float a = __bfloat162float(act[base + c]);
                out[base + c] = __float2bfloat16(a > 0.f ? v[i] : 0.f);
            }
        }
    }
};

// Split-K wrapper: the tile covers K range [z*kc, min((z+1)*kc, K)).
template <class L>
struct KSlice {
    L inner;
    int koff, kend;
    static constexpr bool kChunks = L::kChunks;
    DRWC_DEV bool chunks_ok() const {
        if constexpr (L::kChunks) return inner.chunks_ok() && koff % 8 == 0 && kend % 8 == 0;
        else return false;
    }
    DRWC_DEV const void* chunk(int r, int k8) const {
        if (k8 + koff >= kend) return nullptr;
        return loader_chunk(inner, r, k8 + koff);
    }
    DRWC_DEV void operator()(int r, int k8, uint4* out) const {
        const int k = k8 + koff;
        if (k >= kend) { *out = make_uint4(0, 0, 0, 0); return; }
        inner(r, k, out);
    }
};

template <int BN, class LA, class LB, class EPI>
__global__ void __launch_bounds__(128) umma_splitk_kernel(int M, int N, int K, int kc, LA la,
                                                          LB lb, EPI epi, int* err) {
    extern __shared__ __align__(1024) unsigned char umma_smem[];
    const int koff = blockIdx.z * kc;
    const int kend = min(K, koff + kc);
    KSlice<LA> sa{la, koff, kend};
    KSlice<LB> sb{lb, koff, kend};
    umma_gemm_tile<BN>(M, N, kend - koff, blockIdx.x * kUmmaM, blockIdx.y * BN, sa, sb, epi, err,
                       umma_smem);
}

template <int BN, class LA, class LB, class EPI>
static int launch_splitk(drwc_ctx* ctx, int M, int N, int K, int splits, const LA& la,
                         const LB& lb, const EPI& epi, int* err) {
    if (M <= 0 || N <= 0 || K <= 0) return DRWC_OK;
    static bool attr = false;
    if (!attr) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(umma_splitk_kernel<BN, LA, LB, EPI>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)umma_smem_bytes<BN>()));
        attr = true;
    }
    int kc = (K + splits - 1) / splits;
    kc = (kc + kUmmaBK - 1) / kUmmaBK * kUmmaBK;  // whole K tiles per slice
    splits = (K + kc - 1) / kc;
    dim3 grid((M + kUmmaM - 1) / kUmmaM, (N + BN - 1) / BN, splits);
    umma_splitk_kernel<BN, LA, LB, EPI><<<grid, 128, umma_smem_bytes<BN>(), ctx->stream>>>(
        M, N, K, kc, la, lb, epi, err);
    return launch_check(ctx);
}

// ------------------------------------------------------------ small kernels
__global__ void f32_to_bf16_kernel(const float* __restrict__ a, bf16* __restrict__ b, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        b[i] = __float2bfloat16(a[i]);
}

// Column sums of a [rows, N] BF16 matrix into FP32 (atomics over row chunks).
__global__ void colsum_bf16_kernel(const bf16* __restrict__ m, int rows, int N,
                                   float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int r0 = blockIdx.y * 256, r1 = min(rows, r0 + 256);
    float s = 0.f;
    for (int r = r0; r < r1; ++r) s += __bfloat162float(m[(int64_t)r * N + c]);
    atomicAdd(out + c, s);
}

// Loss and output gradients for one batch. Per row b:
//   Poisson: softmax over O[b, 0:1536] vs target t (sums to 1), CE loss and
//            dO = (s - t) / B; KL(t || s) is the confidence target
//            c* = log10(KL + 1e-8), dO[b, 1536] = 2 wc (O - c*) / B.
//   Gradient (when G given): dG = 2 wg (G - T) / (B * 1536).
// loss[0..2] += CE, confidence MSE, gradient MSE (means over the batch).
__global__ void loss_kernel(int B, int kNP, int kDecRows, int gld, const float* __restrict__ O,
                            const float* __restrict__ T, const float* __restrict__ G,
                            const float* __restrict__ TG, float wc, float wg,
                            bf16* __restrict__ dO, bf16* __restrict__ dG,
                            float* __restrict__ loss, float* __restrict__ kl_out) {
    const int b = blockIdx.x;
    if (b >= B) return;
    __shared__ float red[32];
    __shared__ float bcast[2];
    const float* o = O + (int64_t)b * kDecRows;
    const float* t = T + (int64_t)b * kNP;
    float mx = -1e30f;
    for (int j = threadIdx.x; j < kNP; j += blockDim.x) mx = fmaxf(mx, o[j]);
    for (int s = 16; s > 0; s >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, s));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        float m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, red[w]);
        bcast[0] = m;
    }
    __syncthreads();
    mx = bcast[0];
    float se = 0.f;
    for (int j = threadIdx.x; j < kNP; j += blockDim.x) se += __expf(o[j] - mx);
    for (int s = 16; s > 0; s >>= 1) se += __shfl_xor_sync(0xffffffffu, se, s);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = se;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        bcast[1] = logf(s) + mx;  // log-sum-exp
    }
    __syncthreads();
    const float lse = bcast[1];
    float ce = 0.f, kl = 0.f;
    for (int j = threadIdx.x; j < kNP; j += blockDim.x) {
        const float logs = o[j] - lse;
        const float tj = t[j];
        ce -= tj * logs;
        if (tj > 0.f) kl += tj * (logf(tj) - logs);
        dO[(int64_t)b * kDecRows + j] = __float2bfloat16((__expf(logs) - tj) / B);
    }
    for (int s = 16; s > 0; s >>= 1) {
        ce += __shfl_xor_sync(0xffffffffu, ce, s);
        kl += __shfl_xor_sync(0xffffffffu, kl, s);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = ce; red[16 + (threadIdx.x >> 5)] = kl; }
    __syncthreads();
    if (threadIdx.x == 0) {
        float c = 0.f, k = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { c += red[w]; k += red[16 + w]; }
        const float cstar = log10f(fmaxf(k, 0.f) + 1e-8f);
        const float cp = o[kNP];
        dO[(int64_t)b * kDecRows + kNP] = __float2bfloat16(2.f * wc * (cp - cstar) / B);
        for (int j = kNP + 1; j < kDecRows; ++j) dO[(int64_t)b * kDecRows + j] = __float2bfloat16(0.f);
        atomicAdd(loss + 0, c / B);
        atomicAdd(loss + 1, (cp - cstar) * (cp - cstar) / B);
        if (kl_out) kl_out[b] = k;
    }
    if (G) {
        const float* g = G + (int64_t)b * gld;
        const float* tg = TG + (int64_t)b * kNP;
        float sq = 0.f;
        for (int j = threadIdx.x; j < kNP; j += blockDim.x) {
            const float d = g[j] - tg[j];
            sq += d * d;
            dG[(int64_t)b * kNP + j] = __float2bfloat16(2.f * wg * d / ((float)B * kNP));
        }
        for (int s = 16; s > 0; s >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, s);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
        __syncthreads();
        if (threadIdx.x == 0) {
            float s = 0.f;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
            atomicAdd(loss + 2, s / ((float)B * kNP));
        }
    }
}

// AdamW on a flat FP32 parameter vector; refreshes the BF16 working copy.
__global__ void adamw_kernel(float* __restrict__ p, const float* __restrict__ g,
                             float* __restrict__ m, float* __restrict__ v, bf16* __restrict__ pb,
                             int64_t n, float lr, float b1, float b2, float eps, float wd,
                             float c1, float c2, float clip_scale) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i] * clip_scale;
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float upd = (mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i];
        const float pi = p[i] - lr * upd;
        p[i] = pi;
        pb[i] = __float2bfloat16(pi);
    }
}

__global__ void relu_mask_kernel(const float* __restrict__ d, const bf16* __restrict__ a,
                                 bf16* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __float2bfloat16(__bfloat162float(a[i]) > 0.f ? d[i] : 0.f);
}

__global__ void sumsq_kernel(const float* __restrict__ g, int64_t n, float* __restrict__ out) {
    float s = 0.f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        s += g[i] * g[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// ----------------------------------------------------------------- the net
struct ParamLayout {
    int64_t w1 = 0, b1 = 0, w2 = 0, b2 = 0, w3 = 0, b3 = 0, wd = 0, bd = 0, wg = 0, bg = 0, total = 0;
    ParamLayout() = default;
    ParamLayout(int kNP, int kDecRows, int kFeat) {
        int64_t o = 0;
        auto take = [&](int64_t n) { int64_t r = o; o += (n + 63) / 64 * 64; return r; };
        w1 = take(16 * 27); b1 = take(16);
        w2 = take(32 * 27 * 16); b2 = take(32);
        w3 = take(64 * 27 * 32); b3 = take(64);
        wd = take((int64_t)kDecRows * kFeat); bd = take(kDecRows);
        wg = take((int64_t)kNP * kFeat); bg = take(kNP);
        total = o;
    }
};

}  // namespace drwc

using namespace drwc;

struct drwc_net {
    drwc_ctx* ctx = nullptr;
    int N = 16;                          // cube resolution
    int np = 0, dec = 0, gld = 0, feat = 0, p2 = 0, p3 = 0, p4 = 0;  // NetDims<N>
    ParamLayout L;
    float* p = nullptr;    // FP32 master weights
    bf16* pb = nullptr;    // BF16 working copy
    float* g = nullptr;    // gradients
    float* m = nullptr;    // Adam first moment
    float* v = nullptr;    // Adam second moment
    int64_t step = 0;
    // activations / gradients for the current batch capacity
    int cap = 0;
    bf16 *a1 = nullptr, *a2 = nullptr, *a3 = nullptr;
    bf16 *dO = nullptr, *dG = nullptr, *dF = nullptr, *dz2 = nullptr, *dz1 = nullptr;
    float* tmpf = nullptr;  // FP32 scratch (dF accumulation, losses)
    float* O = nullptr;
    float* G = nullptr;
    int* err = nullptr;
    int holders = 0;  // servers whose captured graphs point at the activations
};

namespace drwc {

static int net_reserve(drwc_net* n, int B) {
    if (B <= n->cap) return DRWC_OK;
    if (n->holders > 0) return DRWC_ERR_INVALID;  // a server's graph uses the buffers
    auto fr = [](void* q) { if (q) cudaFree(q); };
    fr(n->a1); fr(n->a2); fr(n->a3); fr(n->dO); fr(n->dG); fr(n->dF); fr(n->dz2); fr(n->dz1);
    fr(n->tmpf); fr(n->O); fr(n->G);
    const int cap = std::max(B, 64);
    auto al = [&](void** q, size_t bytes) { return cudaMalloc(q, bytes) == cudaSuccess; };
    bool ok = al((void**)&n->a1, (size_t)cap * n->p2 * 16 * 2) && al((void**)&n->a2, (size_t)cap * n->p3 * 32 * 2) &&
              al((void**)&n->a3, (size_t)cap * n->p4 * 64 * 2) && al((void**)&n->dO, (size_t)cap * n->dec * 2) &&
              al((void**)&n->dG, (size_t)cap * n->np * 2) && al((void**)&n->dF, (size_t)cap * n->feat * 2) &&
              al((void**)&n->dz2, (size_t)cap * n->p3 * 32 * 2) && al((void**)&n->dz1, (size_t)cap * n->p2 * 16 * 2) &&
              al((void**)&n->tmpf, (size_t)cap * n->feat * 4 + 256) && al((void**)&n->O, (size_t)cap * n->dec * 4) &&
              al((void**)&n->G, (size_t)cap * n->gld * 4);
    if (!ok) { cudaGetLastError(); n->cap = 0; return DRWC_ERR_NOMEM; }
    n->cap = cap;
    return DRWC_OK;
}

// Encoder: X [B, N^3] BF16 -> A3 [B, FEAT] BF16.
template <int N>
static int net_encode_t(drwc_net* n, int B, const bf16* X) {
    using S = NetDims<N>;
    drwc_ctx* ctx = n->ctx;
    const bf16* pb = n->pb;
    int rc;
    rc = launch_umma<16>(ctx, B * S::P2, 16, 27, ConvGather<S::D1, 1>{X, B * S::P2},
                         RowsBf16{pb + n->L.w1, 16, 27, 27, nullptr},
                         EpiReluBf16{n->a1, n->p + n->L.b1, 16}, n->err);
    if (rc) return rc;
    rc = launch_umma<32>(ctx, B * S::P3, 32, 27 * 16, ConvGather<S::D2, 16>{n->a1, B * S::P3},
                         RowsBf16{pb + n->L.w2, 32, 27 * 16, 27 * 16, nullptr},
                         EpiReluBf16{n->a2, n->p + n->L.b2, 32}, n->err);
    if (rc) return rc;
    return launch_umma<64>(ctx, B * S::P4, 64, 27 * 32, ConvGather<S::D3, 32>{n->a2, B * S::P4},
                           RowsBf16{pb + n->L.w3, 64, 27 * 32, 27 * 32, nullptr},
                           EpiReluBf16{n->a3, n->p + n->L.b3, 64}, n->err);
}

static int net_encode(drwc_net* n, int B, const bf16* X) {
    return net_dispatch(n->N, [&](auto nc) { return net_encode_t<decltype(nc)::value>(n, B, X); });
}

static int net_heads(drwc_net* n, int rows, const int* rowmap, float* O, float* G,
                     const int* rowmap_g, int rows_g) {
    drwc_ctx* ctx = n->ctx;
    const int kNP = n->np, kDecRows = n->dec, kFeat = n->feat;
    int rc = DRWC_OK;
    if (O) {
        rc = rowmap ? DRWC_ERR_INVALID
                    : launch_umma_tma<DRWC_TMA_BN>(ctx, rows, nullptr, 1, kDecRows, kFeat, n->a3, kFeat,
                                           n->pb + n->L.wd, kFeat,
                                           EpiF32{O, n->p + n->L.bd, kDecRows, kDecRows, nullptr},
                                           n->err);
        if (rc == DRWC_ERR_INVALID)
            rc = launch_umma<128>(ctx, rows, kDecRows, kFeat,
                                  RowsBf16{n->a3, rows, kFeat, kFeat, rowmap},
                                  RowsBf16{n->pb + n->L.wd, kDecRows, kFeat, kFeat, nullptr},
                                  EpiF32{O, n->p + n->L.bd, kDecRows, kDecRows, rowmap}, n->err);
        if (rc) return rc;
    }
    if (G && rows_g > 0) {
        rc = launch_umma<128>(ctx, rows_g, kNP, kFeat,
                              RowsBf16{n->a3, rows_g, kFeat, kFeat, rowmap_g},
                              RowsBf16{n->pb + n->L.wg, kNP, kFeat, kFeat, nullptr},
                              EpiF32{G, n->p + n->L.bg, kNP, n->gld, nullptr}, n->err);
    }
    return rc;
}

// Inference stem: the cubes of X (BF16 [B][N^3]) through conv1 and conv2 on
// the tensor cores inside one CTA per group of cubes (stem.cuh), conv2's
// activations to a2. Training keeps the per-layer GEMMs: its backward pass
// needs conv1's activations.
template <int N>
__global__ void __launch_bounds__(StemDims<N>::NT, StemDims<N>::CTAS)
    stem_cubes_kernel(const bf16* __restrict__ X, int B, NetStem W) {
    using D = StemDims<N>;
    extern __shared__ __align__(1024) unsigned char stem_smem[];
    if ((int)blockIdx.x * D::CUBES >= B) return;
    Stem<N> st{stem_smem};
    st.begin(W);
    bool ok = true;
    for (int grp = blockIdx.x; ok && grp * D::CUBES < B; grp += gridDim.x) {
        const int g0 = grp * D::CUBES, nc = min(D::CUBES, B - g0);
        for (int cb = 0; ok && cb < nc; ++cb) {
            const bf16* src = X + (size_t)(g0 + cb) * (N * N * N);
            bf16* xs = st.xs();
            for (int v = threadIdx.x; v < N * N * N; v += blockDim.x) xs[v] = src[v];
            __syncthreads();
            ok = st.conv1(cb, W.err);
        }
        if (ok) ok = st.conv2(nc, W.a2 + (size_t)g0 * D::P3 * 32, W.err);
    }
    st.end();
}

// Encoder for inference: fused stem, then conv3 as a tile GEMM.
template <int N>
static int net_infer_encode_t(drwc_net* n, int B, const bf16* X) {
    using S = NetDims<N>;
    using D = StemDims<N>;
    drwc_ctx* ctx = n->ctx;
    static int per_sm = 0;  // resident stem CTAs per SM (one instantiation per N)
    if (!per_sm) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(stem_cubes_kernel<N>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, D::BYTES));
        DRWC_CUDA_TRY(cudaFuncSetAttribute(stem_cubes_kernel<N>,
                                           cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        DRWC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stem_cubes_kernel<N>,
                                                                    D::NT, D::BYTES));
        if (per_sm < 1) { per_sm = 0; return DRWC_ERR_INVALID; }
    }
    const int groups = (B + D::CUBES - 1) / D::CUBES;
    const int resident = std::max(per_sm, D::CTAS) * ctx->sm_count;
    stem_cubes_kernel<N><<<std::min(groups, resident), D::NT, D::BYTES, ctx->stream>>>(
        X, B, net_stem_operands(n));
    int rc = launch_check(ctx);
    if (rc) return rc;
    return launch_umma<64>(ctx, B * S::P4, 64, 27 * 32, ConvGather<S::D3, 32>{n->a2, B * S::P4},
                           RowsBf16{n->pb + n->L.w3, 64, 27 * 32, 27 * 32, nullptr},
                           EpiReluBf16{n->a3, n->p + n->L.b3, 64}, n->err);
}

static int net_infer_encode(drwc_net* n, int B, const bf16* X) {
    return net_dispatch(n->N, [&](auto nc) { return net_infer_encode_t<decltype(nc)::value>(n, B, X); });
}

int net_forward_locked(drwc_net* n, int B, const bf16* X, float* O, float* G) {
    int rc = net_reserve(n, B);
    if (rc) return rc;
    rc = net_infer_encode(n, B, X);
    if (rc) return rc;
    return net_heads(n, B, nullptr, O, G, nullptr, B);
}

int net_forward_mapped(drwc_net* n, int B, const bf16* X, float* O, float* G, const int* gmap,
                       int rows_g) {
    int rc = net_reserve(n, B);
    if (rc) return rc;
    rc = net_infer_encode(n, B, X);
    if (rc) return rc;
    return net_heads(n, B, nullptr, O, G, gmap, rows_g);
}

template <int N>
static int net_forward_dyn_t(drwc_net* n, int Bmax, const unsigned* nrows, const bf16* X,
                             float* O, float* G, const int* gmap, const unsigned* nrows_g) {
    using S = NetDims<N>;
    drwc_ctx* ctx = n->ctx;
    const bf16* pb = n->pb;
    int rc = DRWC_OK;
    if (X) {  // else conv2's activations are already in a2 (net_stem_operands)
        rc = launch_umma_dyn<16>(ctx, Bmax * S::P2, nrows, S::P2, 16, 27,
                                 ConvGather<S::D1, 1>{X, Bmax * S::P2},
                                 RowsBf16{pb + n->L.w1, 16, 27, 27, nullptr},
                                 EpiReluBf16{n->a1, n->p + n->L.b1, 16}, n->err);
        if (rc) return rc;
        rc = launch_umma_dyn<32>(ctx, Bmax * S::P3, nrows, S::P3, 32, 27 * 16,
                                 ConvGather<S::D2, 16>{n->a1, Bmax * S::P3},
                                 RowsBf16{pb + n->L.w2, 32, 27 * 16, 27 * 16, nullptr},
                                 EpiReluBf16{n->a2, n->p + n->L.b2, 32}, n->err);
        if (rc) return rc;
    }
    rc = launch_umma_dyn<64>(ctx, Bmax * S::P4, nrows, S::P4, 64, 27 * 32,
                             ConvGather<S::D3, 32>{n->a2, Bmax * S::P4},
                             RowsBf16{pb + n->L.w3, 64, 27 * 32, 27 * 32, nullptr},
                             EpiReluBf16{n->a3, n->p + n->L.b3, 64}, n->err);
    if (rc) return rc;
    rc = launch_umma_tma<DRWC_TMA_BN>(ctx, Bmax, nrows, 1, S::DEC, S::FEAT, n->a3, S::FEAT,
                              n->pb + n->L.wd, S::FEAT,
                              EpiF32{O, n->p + n->L.bd, S::DEC, S::DEC, nullptr}, n->err);
    if (rc == DRWC_ERR_INVALID)
        rc = launch_umma_dyn<128>(ctx, Bmax, nrows, 1, S::DEC, S::FEAT,
                                  RowsBf16{n->a3, Bmax, S::FEAT, S::FEAT, nullptr},
                                  RowsBf16{n->pb + n->L.wd, S::DEC, S::FEAT, S::FEAT, nullptr},
                                  EpiF32{O, n->p + n->L.bd, S::DEC, S::DEC, nullptr}, n->err);
    if (rc) return rc;
    return launch_umma_dyn<128>(ctx, Bmax, nrows_g, 1, S::NP, S::FEAT,
                                RowsBf16{n->a3, Bmax, S::FEAT, S::FEAT, gmap},
                                RowsBf16{n->pb + n->L.wg, S::NP, S::FEAT, S::FEAT, nullptr},
                                EpiF32{G, n->p + n->L.bg, S::NP, S::GLD, nullptr}, n->err);
}

int net_forward_dyn(drwc_net* n, int Bmax, const unsigned* nrows, const bf16* X, float* O,
                    float* G, const int* gmap, const unsigned* nrows_g) {
    if (Bmax > n->cap) return DRWC_ERR_INVALID;  // reserve first (not during capture)
    return net_dispatch(n->N, [&](auto nc) {
        return net_forward_dyn_t<decltype(nc)::value>(n, Bmax, nrows, X, O, G, gmap, nrows_g);
    });
}

int net_reserve_rows(drwc_net* n, int B) { return net_reserve(n, B); }

NetStem net_stem_operands(drwc_net* n) {
    return NetStem{n->pb + n->L.w1, n->p + n->L.b1, n->pb + n->L.w2, n->p + n->L.b2, n->a2,
                   n->err};
}

void net_hold(drwc_net* n, int delta) { n->holders += delta; }

drwc_ctx* net_context(drwc_net* n) { return n->ctx; }

int net_size(drwc_net* n) { return n->N; }

}  // namespace drwc

extern "C" {

DRWC_API int drwc_net_create(drwc_ctx* ctx, int N, uint64_t seed, drwc_net** out) {
    if (!ctx || !out || (N != 16 && N != 21 && N != 23)) return DRWC_ERR_INVALID;
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    drwc_net* n = new drwc_net();
    n->ctx = ctx;
    n->N = N;
    net_dispatch(N, [&](auto nc) {
        using S = NetDims<decltype(nc)::value>;
        n->np = S::NP; n->dec = S::DEC; n->gld = S::GLD; n->feat = S::FEAT;
        n->p2 = S::P2; n->p3 = S::P3; n->p4 = S::P4;
        return DRWC_OK;
    });
    n->L = ParamLayout(n->np, n->dec, n->feat);
    const int kNP = n->np, kFeat = n->feat;
    const int64_t T = n->L.total;
    bool ok = cudaMalloc(&n->p, T * 4) == cudaSuccess && cudaMalloc(&n->pb, T * 2) == cudaSuccess &&
              cudaMalloc(&n->g, T * 4) == cudaSuccess && cudaMalloc(&n->m, T * 4) == cudaSuccess &&
              cudaMalloc(&n->v, T * 4) == cudaSuccess && cudaMalloc(&n->err, 64) == cudaSuccess;
    if (!ok) { cudaGetLastError(); delete n; return DRWC_ERR_NOMEM; }
    // Kaiming-uniform convolutions, 1/sqrt(fan_in) heads, zero biases.
    std::vector<float> h(T, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int64_t off, int64_t cnt, double bound) {
        std::uniform_real_distribution<double> U(-bound, bound);
        for (int64_t i = 0; i < cnt; ++i) h[off + i] = (float)U(rng);
    };
    fill(n->L.w1, 16 * 27, std::sqrt(6.0 / 27));
    fill(n->L.w2, 32 * 432, std::sqrt(6.0 / 432));
    fill(n->L.w3, 64 * 864, std::sqrt(6.0 / 864));
    fill(n->L.wd, (int64_t)(kNP + 1) * kFeat, std::sqrt(1.0 / kFeat));
    fill(n->L.wg, (int64_t)kNP * kFeat, std::sqrt(1.0 / kFeat));
    DRWC_CUDA_TRY(cudaMemcpy(n->p, h.data(), T * 4, cudaMemcpyHostToDevice));
    DRWC_CUDA_TRY(cudaMemset(n->m, 0, T * 4));
    DRWC_CUDA_TRY(cudaMemset(n->v, 0, T * 4));
    DRWC_CUDA_TRY(cudaMemset(n->err, 0, 64));
    f32_to_bf16_kernel<<<256, 256, 0, ctx->stream>>>(n->p, n->pb, T);
    int rc = launch_check(ctx);
    if (rc) return rc;
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *out = n;
    return DRWC_OK;
}

DRWC_API int drwc_net_destroy(drwc_net* n) {
    if (!n || n->holders > 0) return DRWC_ERR_INVALID;  // destroy its servers first
    cudaSetDevice(n->ctx->device);
    cudaStreamSynchronize(n->ctx->stream);
    void* ps[] = {n->p, n->pb, n->g, n->m, n->v, n->err, n->a1, n->a2, n->a3, n->dO, n->dG,
                  n->dF, n->dz2, n->dz1, n->tmpf, n->O, n->G};
    for (void* q : ps)
        if (q) cudaFree(q);
    delete n;
    return DRWC_OK;
}

DRWC_API int drwc_net_dims(drwc_net* n, int32_t* N, int32_t* panels, int32_t* out_row,
                           int32_t* grad_row, int32_t* features) {
    if (!n) return DRWC_ERR_INVALID;
    if (N) *N = n->N;
    if (panels) *panels = n->np;
    if (out_row) *out_row = n->dec;
    if (grad_row) *grad_row = n->gld;
    if (features) *features = n->feat;
    return DRWC_OK;
}

DRWC_API int drwc_net_param_count(drwc_net* n, int64_t* count) {
    if (!n || !count) return DRWC_ERR_INVALID;
    *count = n->L.total;
    return DRWC_OK;
}

DRWC_API int drwc_net_get_params(drwc_net* n, float* host) {
    if (!n || !host) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    DRWC_CUDA_TRY(cudaStreamSynchronize(n->ctx->stream));
    DRWC_CUDA_TRY(cudaMemcpy(host, n->p, n->L.total * 4, cudaMemcpyDeviceToHost));
    return DRWC_OK;
}

DRWC_API int drwc_net_set_params(drwc_net* n, const float* host) {
    if (!n || !host) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    drwc_ctx* ctx = n->ctx;
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    DRWC_CUDA_TRY(cudaMemcpy(n->p, host, n->L.total * 4, cudaMemcpyHostToDevice));
    f32_to_bf16_kernel<<<256, 256, 0, ctx->stream>>>(n->p, n->pb, n->L.total);
    int rc = launch_check(ctx);
    if (rc) return rc;
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return DRWC_OK;
}

DRWC_API int drwc_net_gradients(drwc_net* n, float* host) {
    if (!n || !host) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    DRWC_CUDA_TRY(cudaStreamSynchronize(n->ctx->stream));
    DRWC_CUDA_TRY(cudaMemcpy(host, n->g, n->L.total * 4, cudaMemcpyDeviceToHost));
    return DRWC_OK;
}

// Forward: X [B, N^3] BF16 (device) -> O [B, out_row] FP32 (Poisson logits +
// confidence) and, when G is set, G [B, grad_row] FP32 (gradient head).
DRWC_API int drwc_net_forward(drwc_net* n, int B, const void* X, float* O, float* G) {
    if (!n || B < 0 || (B > 0 && !X)) return DRWC_ERR_INVALID;
    if (B == 0) return DRWC_OK;
    std::lock_guard<std::mutex> lock(n->ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(n->ctx->device));
    return net_forward_locked(n, B, (const bf16*)X, O, G);
}

// One training step on a batch: X [B, 4096] BF16, T [B, 1536] FP32 target
// Green's functions (each row sums to 1), TG [B, 1536] FP32 scaled gradient
// targets (nullable). Computes the losses, backpropagates, clips the global
// gradient norm to clip (<= 0: no clipping) and applies AdamW.
// loss_out (host, 3 floats): CE, confidence MSE, gradient MSE.
DRWC_API int drwc_net_train_step(drwc_net* n, int B, const void* X, const float* T,
                                 const float* TG, float lr, float weight_decay, float clip,
                                 float w_conf, float w_grad, int apply, float* loss_out) {
    if (!n || B <= 0 || !X || !T) return DRWC_ERR_INVALID;
    drwc_ctx* ctx = n->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    int rc = net_reserve(n, B);
    if (rc) return rc;
    const bf16* x = (const bf16*)X;
    const ParamLayout& L = n->L;
    const int kNP = n->np, kDecRows = n->dec, kFeat = n->feat;
    // ---- forward
    rc = net_encode(n, B, x);
    if (rc) return rc;
    rc = net_heads(n, B, nullptr, n->O, TG ? n->G : nullptr, nullptr, B);
    if (rc) return rc;
    float* loss = n->tmpf + (size_t)n->cap * kFeat;  // 3 floats + norm
    DRWC_CUDA_TRY(cudaMemsetAsync(loss, 0, 64, ctx->stream));
    DRWC_CUDA_TRY(cudaMemsetAsync(n->g, 0, L.total * 4, ctx->stream));
    loss_kernel<<<B, 256, 0, ctx->stream>>>(B, kNP, kDecRows, n->gld, n->O, T,
                                             TG ? n->G : nullptr, TG, w_conf, w_grad, n->dO, n->dG,
                                             loss, nullptr);
    if ((rc = launch_check(ctx))) return rc;
    rc = net_dispatch(n->N, [&](auto nc) -> int {
    using S = NetDims<decltype(nc)::value>;
    int rc = DRWC_OK;
    // ---- heads: weight / bias gradients, dF
    const int spl = std::max(1, std::min(64, B / 64));
    rc = launch_splitk<128>(ctx, kDecRows, kFeat, B, spl, ColsBf16{n->dO, kDecRows, B, kDecRows},
                            ColsBf16{n->a3, kFeat, B, kFeat}, EpiAtomicF32{n->g + L.wd, kFeat},
                            n->err);
    if (rc) return rc;
    colsum_bf16_kernel<<<dim3((kDecRows + 255) / 256, (B + 255) / 256), 256, 0, ctx->stream>>>(
        n->dO, B, kDecRows, n->g + L.bd);
    if ((rc = launch_check(ctx))) return rc;
    // dF (FP32) = dO Wd (+ dG Wg), then BF16
    float* dF32 = n->tmpf;
    DRWC_CUDA_TRY(cudaMemsetAsync(dF32, 0, (size_t)B * kFeat * 4, ctx->stream));
    rc = launch_splitk<128>(ctx, B, kFeat, kDecRows, 1, RowsBf16{n->dO, B, kDecRows, kDecRows, nullptr},
                            ColsBf16{n->pb + L.wd, kFeat, kDecRows, kFeat},
                            EpiAtomicF32{dF32, kFeat}, n->err);
    if (rc) return rc;
    if (TG) {
        rc = launch_splitk<128>(ctx, kNP, kFeat, B, spl, ColsBf16{n->dG, kNP, B, kNP},
                                ColsBf16{n->a3, kFeat, B, kFeat}, EpiAtomicF32{n->g + L.wg, kFeat},
                                n->err);
        if (rc) return rc;
        colsum_bf16_kernel<<<dim3((kNP + 255) / 256, (B + 255) / 256), 256, 0, ctx->stream>>>(
            n->dG, B, kNP, n->g + L.bg);
        if ((rc = launch_check(ctx))) return rc;
        rc = launch_splitk<128>(ctx, B, kFeat, kNP, 1, RowsBf16{n->dG, B, kNP, kNP, nullptr},
                                ColsBf16{n->pb + L.wg, kFeat, kNP, kFeat},
                                EpiAtomicF32{dF32, kFeat}, n->err);
        if (rc) return rc;
    }
    // dZ3 = dF * (A3 > 0) -> BF16 [B*8, 64] (same element order as F)
    relu_mask_kernel<<<(int)std::min<int64_t>(4096, ((int64_t)B * kFeat + 255) / 256), 256, 0,
                       ctx->stream>>>(dF32, n->a3, n->dF, (int64_t)B * kFeat);
    if ((rc = launch_check(ctx))) return rc;
    const bf16* dz3 = n->dF;  // [B*8, 64]
    // ---- conv3: dW3, db3, dZ2
    const int r3 = B * S::P4, r2 = B * S::P3, r1 = B * S::P2;
    rc = launch_splitk<128>(ctx, 64, 27 * 32, r3, std::max(1, std::min(128, r3 / 256)),
                            ColsBf16{dz3, 64, r3, 64}, Im2colT<S::D3, 32>{n->a2, r3},
                            EpiAtomicF32{n->g + L.w3, 27 * 32}, n->err);
    if (rc) return rc;
    colsum_bf16_kernel<<<dim3(1, (r3 + 255) / 256), 64, 0, ctx->stream>>>(dz3, r3, 64, n->g + L.b3);
    if ((rc = launch_check(ctx))) return rc;
    rc = launch_umma<32>(ctx, r2, 32, 27 * 64, ConvTGather<S::D3, 64>{dz3, r2},
                         WeightT<32, 64>{n->pb + L.w3}, EpiReluGrad{n->dz2, n->a2, 32}, n->err);
    if (rc) return rc;
    // ---- conv2: dW2, db2, dZ1
    rc = launch_splitk<32>(ctx, 32, 27 * 16, r2, std::max(1, std::min(256, r2 / 512)),
                           ColsBf16{n->dz2, 32, r2, 32}, Im2colT<S::D2, 16>{n->a1, r2},
                           EpiAtomicF32{n->g + L.w2, 27 * 16}, n->err);
    // note: M = 32 output channels -> a 128-row tile with 96 zero rows
    if (rc) return rc;
    colsum_bf16_kernel<<<dim3(1, (r2 + 255) / 256), 32, 0, ctx->stream>>>(n->dz2, r2, 32, n->g + L.b2);
    if ((rc = launch_check(ctx))) return rc;
    rc = launch_umma<16>(ctx, r1, 16, 27 * 32, ConvTGather<S::D2, 32>{n->dz2, r1},
                         WeightT<16, 32>{n->pb + L.w2}, EpiReluGrad{n->dz1, n->a1, 16}, n->err);
    if (rc) return rc;
    // ---- conv1: dW1, db1
    rc = launch_splitk<32>(ctx, 16, 27, r1, std::max(1, std::min(512, r1 / 1024)),
                           ColsBf16{n->dz1, 16, r1, 16}, Im2colT<S::D1, 1>{x, r1},
                           EpiAtomicF32{n->g + L.w1, 27}, n->err);
    if (rc) return rc;
    colsum_bf16_kernel<<<dim3(1, (r1 + 255) / 256), 32, 0, ctx->stream>>>(n->dz1, r1, 16, n->g + L.b1);
    return launch_check(ctx);
    });
    if (rc) return rc;
    // ---- clip + AdamW
    float host_loss[4] = {0, 0, 0, 0};
    sumsq_kernel<<<512, 256, 0, ctx->stream>>>(n->g, L.total, loss + 3);
    if ((rc = launch_check(ctx))) return rc;
    DRWC_CUDA_TRY(cudaMemcpyAsync(host_loss, loss, 16, cudaMemcpyDeviceToHost, ctx->stream));
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (loss_out) {
        loss_out[0] = host_loss[0];
        loss_out[1] = host_loss[1];
        loss_out[2] = host_loss[2];
    }
    if (apply) {
        const float gn = std::sqrt(host_loss[3]);
        const float scale = (clip > 0 && gn > clip) ? clip / gn : 1.f;
        n->step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)n->step), c2 = 1.f - std::pow(b2, (float)n->step);
        adamw_kernel<<<1024, 256, 0, ctx->stream>>>(n->p, n->g, n->m, n->v, n->pb, L.total, lr, b1,
                                                    b2, 1e-8f, weight_decay, c1, c2, scale);
        if ((rc = launch_check(ctx))) return rc;
    }
    int herr = 0;
    DRWC_CUDA_TRY(cudaMemcpyAsync(&herr, n->err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return herr ? DRWC_ERR_TIMEOUT : DRWC_OK;
}

}  // extern "C"

