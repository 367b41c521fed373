// Warp-specialised tcgen05 GEMM with TMA operand loads, for dense row-major
// operands: C[M, N] = epi(A[M, K] * B[N, K]^T), BF16 in, FP32 accumulation in
// tensor memory.
//
// A CTA of 192 threads walks output tiles (128 x BN) blockIdx.x, +gridDim.x,
// ... in m-fastest order:
//   warp 0 (one thread)  producer: for every K stage of 64, arms the stage's
//                        "full" mbarrier with the byte count and issues one
//                        2D TMA load (cp.async.bulk.tensor, no multicast) per
//                        operand: a box of 64 columns (128 B) x 128 rows of A
//                        and x BN rows of B with the 128-byte swizzle, i.e.
//                        the K-major SWIZZLE_128B layout the tensor cores read
//                        (8-row atoms of 1024 B); it waits on the stage's
//                        "empty" mbarrier before reusing it;
//   warp 1 (one thread)  MMA issuer: waits "full", issues four
//                        tcgen05.mma.kind::f16 (K = 16 each) into one of two
//                        TMEM accumulators, commits to "empty" (the stage is
//                        free once those MMAs are done) and, after the tile's
//                        last stage, to the accumulator's "full" barrier;
//   warps 2-5            epilogue: wait for an accumulator, read it with
//                        tcgen05.ld (warp w owns TMEM lanes 32 (w mod 4) ..),
//                        hand rows to the epilogue functor, release the
//                        accumulator (its "empty" barrier counts four warps).
// Two accumulators let the MMAs of tile i + 1 run while tile i drains.
// Every wait is bounded (mbar_wait); a timeout raises the error flag and an
// abort flag that every role checks, and the CTA still waits (bounded) for
// its outstanding TMA loads and MMAs before it frees the tensor memory.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "host.cuh"
#include "umma.cuh"

namespace drwc {

constexpr int kTmaThreads = 192;

template <int BN>
constexpr int tma_stages() {
    return BN >= 256 ? 4 : BN >= 128 ? 3 : 4;
}

// Output columns per tile of the TMA GEMM for dense heads and drwc_gemm_bf16:
// 256 (one CTA per SM, 4 stages of 48 KB, both 256-column accumulators in
// the SM's 512 TMEM columns) runs 1.7x the 128-column tile at 8192^3.
#ifndef DRWC_TMA_BN
#define DRWC_TMA_BN 256
#endif

// Per epilogue warp, one staged 32 x 32 block (epi_block_store).
constexpr int kTmaStageFloats = kEpiStageFloats;

template <int BN>
constexpr size_t tma_smem_bytes() {
    return (size_t)tma_stages<BN>() * (kUmmaM + BN) * kUmmaBK * 2 + 256 + 4 * kTmaStageFloats * 4;
}



DRWC_DEV void tma_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}

DRWC_DEV void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Shared-memory descriptor of a K-major SWIZZLE_128B operand: 8-row atoms
// 1024 B apart (stride byte offset), layout type 2 in bits 61-63; a K step
// of 16 BF16 advances the start address by 32 B inside the 128-byte rows.
DRWC_DEV uint64_t umma_smem_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);      // start address >> 4
    d |= (uint64_t)1u << 16;                       // leading byte offset (unused here) = 16 B
    d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32; // stride byte offset: 1024 B between atoms
    d |= (uint64_t)1u << 46;                       // descriptor version 1
    d |= (uint64_t)2u << 61;                       // layout: SWIZZLE_128B
    return d;
}

DRWC_DEV void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int BN, class EPI>
__global__ void __launch_bounds__(kTmaThreads) umma_tma_kernel(const __grid_constant__ CUtensorMap ta,
                                                               const __grid_constant__ CUtensorMap tb,
                                                               int Mmax, const unsigned* mcount,
                                                               int mmul, int N, int K, EPI epi,
                                                               int* err) {
    extern __shared__ __align__(1024) unsigned char umma_smem[];
    constexpr int S = tma_stages<BN>();
    constexpr int SA = kUmmaM * kUmmaBK * 2, SB = BN * kUmmaBK * 2;
    constexpr uint32_t TCOLS = 2 * BN < 32 ? 32 : 2 * BN;  // two accumulators
    int M = Mmax;
    if (mcount) {
        const long long m = (long long)(*mcount) * mmul;
        M = m < Mmax ? (int)m : Mmax;
    }
    const int mt = (M + kUmmaM - 1) / kUmmaM, nt = (N + BN - 1) / BN, tiles = mt * nt;
    if ((int)blockIdx.x >= tiles) return;
    const int ktiles = (K + kUmmaBK - 1) / kUmmaBK;
    unsigned char* sA = umma_smem;
    unsigned char* sB = umma_smem + S * SA;
    uint64_t* full = reinterpret_cast<uint64_t*>(umma_smem + S * (SA + SB));
    uint64_t* empty = full + S;
    uint64_t* accf = empty + S;   // 2
    uint64_t* acce = accf + 2;    // 2
    uint64_t* spare = acce + 2;   // MMA drain
    uint32_t* tslot = reinterpret_cast<uint32_t*>(spare + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    int* issued = const_cast<int*>(abort_flag) + 1;    // stages armed by the producer
    int* consumed = issued + 1;                          // stages waited on by the MMA thread
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int q = 0; q < S; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], 1);
        }
        mbar_init(&accf[0], 1);
        mbar_init(&accf[1], 1);
        mbar_init(&acce[0], 4);
        mbar_init(&acce[1], 4);
        mbar_init(spare, 1);
        *abort_flag = 0;
        *issued = 0;
        *consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tslot)), "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int mine = (tiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    auto fail = [&]() {
        *abort_flag = 1;
        if (err) atomicExch(err, 1);
    };

    if (warp == 0) {
        if (lane == 0) {  // producer
            int g = 0;
            for (int i = 0; i < mine && !*abort_flag; ++i) {
                const int tile = (int)blockIdx.x + i * (int)gridDim.x;
                const int m0 = (tile % mt) * kUmmaM, n0 = (tile / mt) * BN;
                for (int kt = 0; kt < ktiles && !*abort_flag; ++kt, ++g) {
                    const int s = g % S, r = g / S;
                    if (r > 0 && !mbar_wait(&empty[s], (r - 1) & 1)) { fail(); break; }
                    mbar_arrive_expect(&full[s], SA + SB);
                    const uint32_t fb = smem_u32(&full[s]);
                    tma_load_2d(smem_u32(sA + s * SA), &ta, kt * kUmmaBK, m0, fb);
                    tma_load_2d(smem_u32(sB + s * SB), &tb, kt * kUmmaBK, n0, fb);
                    *issued = g + 1;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            int g = 0;
            for (int i = 0; i < mine && !*abort_flag; ++i) {
                const int ab = i & 1, r = i >> 1;
                if (r > 0 && !mbar_wait(&acce[ab], (r - 1) & 1)) { fail(); break; }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(ab * BN);
                bool ok = true;
                for (int kt = 0; kt < ktiles; ++kt, ++g) {
                    const int s = g % S;
                    if (!mbar_wait(&full[s], (g / S) & 1)) { ok = false; break; }
                    *consumed = g + 1;
                    tc_fence_after();
                    const int k0 = kt * kUmmaBK;
                    const int ksteps = min(kUmmaBK, K - k0 + 15) / 16;
                    for (int ks = 0; ks < ksteps && ks < kUmmaBK / 16; ++ks) {
                        const uint64_t da = umma_smem_desc_sw128(smem_u32(sA + s * SA + 32 * ks));
                        const uint64_t db = umma_smem_desc_sw128(smem_u32(sB + s * SB + 32 * ks));
                        umma_bf16(d, da, db, umma_idesc_bf16<BN>(), (kt > 0 || ks > 0) ? 1u : 0u);
                    }
                    umma_commit(&empty[s]);
                }
                if (!ok) { fail(); break; }
                umma_commit(&accf[ab]);
            }
            // every MMA this thread issued is complete before the memory is freed
            umma_commit(spare);
            if (!mbar_wait(spare, 0)) fail();
        }
    } else {  // epilogue warps 2..5
        const int q = warp & 3;
        float* stg = reinterpret_cast<float*>(umma_smem + S * (SA + SB) + 256) + q * kTmaStageFloats;
        for (int i = 0; i < mine; ++i) {
            if (*abort_flag) break;
            const int ab = i & 1, r = i >> 1;
            if (!mbar_wait(&accf[ab], r & 1)) { fail(); break; }
            tc_fence_after();
            const int tile = (int)blockIdx.x + i * (int)gridDim.x;
            const int m0 = (tile % mt) * kUmmaM, n0 = (tile / mt) * BN;
            const int row = m0 + q * 32 + lane;
            for (int c = 0; c < BN; c += 32) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * BN + c), v);
                if constexpr (EpiHasStore4<EPI>::value) {
                    if (n0 + c < N) epi_block_store(epi, stg, v, m0 + q * 32, n0 + c, M, N);
                } else {
                    if (row < M && n0 + c < N) epi(row, n0 + c, v);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[ab]);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) {
        // loads armed but never consumed must land before the CTA exits
        for (int g = *consumed; g < *issued; ++g) mbar_wait(&full[g % S], (g / S) & 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
}

// ---------------------------------------------------------------- host side
using TensorMapEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                       const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                       const cuuint32_t*, CUtensorMapInterleave,
                                       CUtensorMapSwizzle, CUtensorMapL2promotion,
                                       CUtensorMapFloatOOBfill);

inline TensorMapEncodeFn tensor_map_encoder() {
    static TensorMapEncodeFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", reinterpret_cast<void**>(&fn),
                                    cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
    }
    return fn;
}

// 2D map of a row-major BF16 matrix [rows, cols] (leading dimension ld
// elements): boxes of 64 columns (128 B) x box_rows rows with the 128-byte
// swizzle, zero fill outside.
inline bool tensor_map_rows(CUtensorMap* map, const void* base, int64_t rows, int64_t cols,
                            int64_t ld, int box_rows) {
    TensorMapEncodeFn enc = tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(base) & 15) || (ld % 8) || rows < 1 || cols < 1)
        return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kUmmaBK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
               box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

// Launch when both operands suit TMA (16-byte aligned bases, ld and K
// multiples of 8); returns DRWC_ERR_INVALID otherwise so the caller can take
// the gathering tile instead. mcount: row count on the device (nullable).
template <int BN, class EPI>
inline int launch_umma_tma(drwc_ctx* ctx, int Mmax, const unsigned* mcount, int mmul, int N, int K,
                           const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B,
                           int64_t ldb, const EPI& epi, int* err) {
    if (Mmax <= 0 || N <= 0) return DRWC_OK;
    if (K <= 0 || K % 8) return DRWC_ERR_INVALID;
    CUtensorMap ta, tb;
    if (!tensor_map_rows(&ta, A, Mmax, K, lda, kUmmaM) || !tensor_map_rows(&tb, B, N, K, ldb, BN))
        return DRWC_ERR_INVALID;
    static int per_sm = 0;
    auto kern = umma_tma_kernel<BN, EPI>;
    if (!per_sm) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)tma_smem_bytes<BN>()));
        DRWC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        DRWC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTmaThreads,
                                                                    tma_smem_bytes<BN>()));
        if (per_sm < 1) per_sm = 1;
    }
    const int tiles = ((Mmax + kUmmaM - 1) / kUmmaM) * ((N + BN - 1) / BN);
    const int grid = std::max(1, std::min(tiles, per_sm * ctx->sm_count));
    kern<<<grid, kTmaThreads, tma_smem_bytes<BN>(), ctx->stream>>>(ta, tb, Mmax, mcount, mmul, N, K,
                                                                   epi, err);
    return launch_check(ctx);
}

}  // namespace drwc
