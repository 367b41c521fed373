// Host-side launcher for umma_kernel (the tcgen05 GEMM tile).
#pragma once

#include "host.cuh"
#include "umma.cuh"

namespace drwc {

template <int BN, class LA, class LB, class EPI>
inline int launch_umma(drwc_ctx* ctx, int M, int N, int K, const LA& la, const LB& lb,
                       const EPI& epi, int* err) {
    if (M <= 0 || N <= 0) return DRWC_OK;
    static bool attr = false;  // one instantiation per (BN, LA, LB, EPI)
    if (!attr) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(umma_kernel<BN, LA, LB, EPI>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)umma_smem_bytes<BN>()));
        attr = true;
    }
    dim3 grid((M + kUmmaM - 1) / kUmmaM, (N + BN - 1) / BN);
    umma_kernel<BN, LA, LB, EPI><<<grid, 128, umma_smem_bytes<BN>(), ctx->stream>>>(
        M, N, K, la, lb, epi, err);
    return launch_check(ctx);
}

}  // namespace drwc
