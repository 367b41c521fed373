// Plain BF16 GEMM on the tcgen05 building block (umma.cuh), exposed through
// the C ABI as drwc_gemm_bf16: C[M,N] (FP32) = act(A[M,K] * B[N,K]^T + bias).
// It is the primitive the learned transition kernels are made of, and the
// unit the tensor-core tests check against an FP32 reference.
#include <type_traits>

#include "host.cuh"
#include "umma.cuh"
#include "umma_tma.cuh"

namespace drwc {

struct RowLoader {
    const __nv_bfloat16* __restrict__ p;
    int rows, cols;
    int64_t ld;
    static constexpr bool kChunks = true;
    DRWC_DEV bool chunks_ok() const {
        return cols % 8 == 0 && ld % 8 == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0;
    }
    DRWC_DEV const void* chunk(int r, int k8) const {
        if (r >= rows || k8 >= cols) return nullptr;
        return p + (int64_t)r * ld + k8;
    }
    DRWC_DEV void operator()(int r, int k8, uint4* out) const {
        if (r >= rows || k8 >= cols) { *out = make_uint4(0, 0, 0, 0); return; }
        const __nv_bfloat16* src = p + (int64_t)r * ld + k8;
        if (k8 + 8 <= cols && ((reinterpret_cast<uintptr_t>(src) & 15) == 0)) {
            *out = *reinterpret_cast<const uint4*>(src);
            return;
        }
        __align__(16) __nv_bfloat16 tmp[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) tmp[i] = (k8 + i < cols) ? src[i] : __float2bfloat16(0.f);
        *out = *reinterpret_cast<const uint4*>(tmp);
    }
};

struct StoreF32 {
    float* __restrict__ c;
    const float* __restrict__ bias;
    int N;
    int64_t ldc;
    int act;  // 0 none, 1 relu
    DRWC_DEV void operator()(int row, int col0, const float* v) const {
        float* dst = c + (int64_t)row * ldc;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int col = col0 + i;
            if (col < N) {
                float x = v[i] + (bias ? bias[col] : 0.f);
                if (act == 1) x = fmaxf(x, 0.f);
                dst[col] = x;
            }
        }
    }
    // 4 consecutive columns (col a multiple of 4) of one row.
    DRWC_DEV void store4(int row, int col, float4 v) const {
        float* dst = c + (int64_t)row * ldc + col;
        float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (col + i < N) {
                e[i] += bias ? bias[col + i] : 0.f;
                if (act == 1) e[i] = fmaxf(e[i], 0.f);
            }
        }
        if (col + 4 <= N && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
            *reinterpret_cast<float4*>(dst) = make_float4(e[0], e[1], e[2], e[3]);
            return;
        }
        for (int i = 0; i < 4 && col + i < N; ++i) dst[i] = e[i];
    }
};

template <int BN>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(int M, int N, int K, RowLoader la,
                                                        RowLoader lb, StoreF32 st, int* err) {
    extern __shared__ __align__(1024) unsigned char umma_smem[];
    umma_gemm_tile<BN>(M, N, K, blockIdx.x * kUmmaM, blockIdx.y * BN, la, lb, st, err, umma_smem);
}

}  // namespace drwc

using namespace drwc;

extern "C" {

DRWC_API int drwc_gemm_bf16(drwc_ctx* ctx, int M, int N, int K, const void* A, int64_t lda,
                            const void* B, int64_t ldb, float* C, int64_t ldc, const float* bias,
                            int act, int* err_flag) {
    if (!ctx || M < 0 || N < 0 || K < 0 || act < 0 || act > 1) return DRWC_ERR_INVALID;
    if (M == 0 || N == 0) return DRWC_OK;
    if (!A || !B || !C || lda < K || ldb < K || ldc < N) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    RowLoader la{(const __nv_bfloat16*)A, M, K, lda};
    RowLoader lb{(const __nv_bfloat16*)B, N, K, ldb};
    StoreF32 st{C, bias, N, ldc, act};
    constexpr int BN = 128;
    // TMA-fed, warp-specialised tiles when the operands allow it
    const int rt = launch_umma_tma<DRWC_TMA_BN>(ctx, M, nullptr, 1, N, K, (const __nv_bfloat16*)A, lda,
                                       (const __nv_bfloat16*)B, ldb, st, err_flag);
    if (rt != DRWC_ERR_INVALID) return rt;
    static bool attr = false;
    if (!attr) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(gemm_bf16_kernel<BN>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)umma_smem_bytes<BN>()));
        attr = true;
    }
    dim3 grid((M + kUmmaM - 1) / kUmmaM, (N + BN - 1) / BN);
    gemm_bf16_kernel<BN><<<grid, 128, umma_smem_bytes<BN>(), ctx->stream>>>(M, N, K, la, lb, st,
                                                                            err_flag);
    return launch_check(ctx);
}

}  // extern "C"
