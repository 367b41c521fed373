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
        DRWC_CUDA_TRY(cudaFuncSetAttribute(umma_kernel<BN, LA, LB, EPI>,
                                           cudaFuncAttributePreferredSharedMemoryCarveout, 100));
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
// A grid of a few CTAs per SM walks the 128-row tiles (tile = blockIdx.x,
// +gridDim.x, ...); each tile runs the whole tile routine, so the launch can
// sit in a CUDA graph while M changes per replay without paying for a grid
// sized to Mmax when few rows are present.
template <int BN, class LA, class LB, class EPI>
__global__ void __launch_bounds__(128) umma_dyn_kernel(int Mmax, const unsigned* __restrict__ mcount,
                                                       int mmul, int N, int K, LA la, LB lb,
                                                       EPI epi, int* err) {
    extern __shared__ __align__(1024) unsigned char umma_smem[];
    const long long m = (long long)(*mcount) * mmul;
    const int M = m < Mmax ? (int)m : Mmax;
    const int ntiles = (M + kUmmaM - 1) / kUmmaM;
    if ((int)blockIdx.x >= ntiles) return;
    RowClamp<LA> ca{la, M};
    const uint32_t tmem = umma_tmem_alloc<BN>(umma_tslot<BN>(umma_smem));
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
        umma_gemm_tile<BN>(M, N, K, tile * kUmmaM, blockIdx.y * BN, ca, lb, epi, err, umma_smem,
                           tmem);
    umma_tmem_free<BN>(tmem);
}

template <int BN, class LA, class LB, class EPI>
inline int launch_umma_dyn(drwc_ctx* ctx, int Mmax, const unsigned* mcount, int mmul, int N,
                           int K, const LA& la, const LB& lb, const EPI& epi, int* err) {
    if (Mmax <= 0 || N <= 0) return DRWC_OK;
    static int per_sm = 0;
    if (!per_sm) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(umma_dyn_kernel<BN, LA, LB, EPI>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)umma_smem_bytes<BN>()));
        DRWC_CUDA_TRY(cudaFuncSetAttribute(umma_dyn_kernel<BN, LA, LB, EPI>,
                                           cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        DRWC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, umma_dyn_kernel<BN, LA, LB, EPI>, 128, umma_smem_bytes<BN>()));
        if (per_sm < 1) per_sm = 1;
    }
    const int ntiles = (Mmax + kUmmaM - 1) / kUmmaM, ncol = (N + BN - 1) / BN;
    // about four CTAs per SM over the whole grid (the column tiles share the
    // SMs); CTAs beyond the resident ones wait for a slot, so the number only
    // sets how finely the tiles are dealt out
    const int target = std::max(per_sm, 4) * ctx->sm_count;
    const int gx = std::max(1, std::min(ntiles, (target + ncol - 1) / ncol));
    umma_dyn_kernel<BN, LA, LB, EPI><<<dim3(gx, ncol), 128, umma_smem_bytes<BN>(), ctx->stream>>>(
        Mmax, mcount, mmul, N, K, la, lb, epi, err);
    return launch_check(ctx);
}

}  // namespace drwc
