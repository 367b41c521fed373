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

// Operand rows at or beyond M read as zeros (M known on the device only).
template <class L>
struct RowClamp {
    L inner;
    int M;
    static constexpr bool kChunks = L::kChunks;
    DRWC_DEV bool chunks_ok() const {
        if constexpr (L::kChunks) return inner.chunks_ok();
        else return false;
    }
    DRWC_DEV const void* chunk(int r, int k8) const {
        if (r >= M) return nullptr;
        return loader_chunk(inner, r, k8);
    }
    DRWC_DEV void operator()(int r, int k8, uint4* out) const {
        if (r >= M) { *out = make_uint4(0, 0, 0, 0); return; }
        inner(r, k8, out);
    }
};

// GEMM whose row count is read on the device: M = min(Mmax, *mcount * mmul).
// The grid covers Mmax; tiles past M return before touching shared or tensor
// memory, so the launch can sit in a CUDA graph while M changes per replay.
template <int BN, class LA, class LB, class EPI>
__global__ void __launch_bounds__(128) umma_dyn_kernel(int Mmax, const unsigned* __restrict__ mcount,
                                                       int mmul, int N, int K, LA la, LB lb,
                                                       EPI epi, int* err) {
    extern __shared__ __align__(1024) unsigned char umma_smem[];
    const long long m = (long long)(*mcount) * mmul;
    const int M = m < Mmax ? (int)m : Mmax;
    if ((int)blockIdx.x * kUmmaM >= M) return;
    RowClamp<LA> ca{la, M};
    umma_gemm_tile<BN>(M, N, K, blockIdx.x * kUmmaM, blockIdx.y * BN, ca, lb, epi, err, umma_smem);
}

template <int BN, class LA, class LB, class EPI>
inline int launch_umma_dyn(drwc_ctx* ctx, int Mmax, const unsigned* mcount, int mmul, int N,
                           int K, const LA& la, const LB& lb, const EPI& epi, int* err) {
    if (Mmax <= 0 || N <= 0) return DRWC_OK;
    static bool attr = false;
    if (!attr) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(umma_dyn_kernel<BN, LA, LB, EPI>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)umma_smem_bytes<BN>()));
        attr = true;
    }
    dim3 grid((Mmax + kUmmaM - 1) / kUmmaM, (N + BN - 1) / BN);
    umma_dyn_kernel<BN, LA, LB, EPI><<<grid, 128, umma_smem_bytes<BN>(), ctx->stream>>>(
        Mmax, mcount, mmul, N, K, la, lb, epi, err);
    return launch_check(ctx);
}

}  // namespace drwc
