// Blackwell (sm_100a) tensor-core GEMM building block: C = A * B^T with A
// [M, K] and B [N, K] in BF16, FP32 accumulation in tensor memory (TMEM).
//
// One CTA of 128 threads owns a 128 x BN tile of C. Operand tiles are
// produced by the threads through loader functors (plain matrices or the
// implicit-GEMM gathers of the 3-D convolutions) and written to shared memory
// in the canonical K-major, no-swizzle UMMA layout: 8-row x 16-byte core
// matrices, the two 8-element K halves of a 16-wide K step 128 B apart (LBO)
// and consecutive 8-row groups 256 B apart (SBO). One thread issues
// tcgen05.mma.cta_group::1.kind::f16 (M = 128, N = BN, K = 16 per
// instruction) for each K step and commits to an mbarrier; two shared-memory
// stages let the threads fill one while the tensor cores read the other. The
// epilogue reads the accumulator with tcgen05.ld (32 lanes x 32 columns per
// warp access) and hands rows to an epilogue functor.
//
// Bit layouts of the shared-memory and instruction descriptors follow the
// public CUTLASS definitions (cute/arch/mma_sm100_desc.hpp: SmemDescriptor,
// InstrDescriptor). Every wait is bounded: on timeout the kernel raises an
// error flag, still waits (bounded) for its own MMAs and frees its TMEM.
#pragma once

#include <cuda_bf16.h>

#include <type_traits>

#include "common.cuh"

namespace drwc {

constexpr int kUmmaM = 128;
constexpr int kUmmaThreads = 128;                // threads of a GEMM-tile CTA
constexpr int kUmmaBK = 64;                      // K per shared-memory stage (4 MMAs)
constexpr long long kWaitCycles = 4000000000LL;  // bounded wait: about 2 s of SM clock

DRWC_DEV uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle, K-major canonical layout.
DRWC_DEV uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);              // [0,14)  start address >> 4
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;    // [16,30) leading byte offset >> 4
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;    // [32,46) stride byte offset >> 4
    d |= (uint64_t)1u << 46;                               // [46,48) descriptor version 1
    return d;                                              // base offset 0, no swizzle
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, both K-major.
template <int BN>
DRWC_DEV constexpr uint32_t umma_idesc_bf16() {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M=128");
    return (1u << 4)                          // D format F32
           | (1u << 7)                        // A format BF16
           | (1u << 10)                       // B format BF16
           | ((uint32_t)(BN >> 3) << 17)      // N >> 3
           | ((uint32_t)(kUmmaM >> 4) << 24); // M >> 4
}

DRWC_DEV void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Bounded wait on phase `parity`; returns false on timeout. try_wait without
// a suspend-time hint returns as soon as the phase completes (or after a
// short system-defined slice), so the loop reacts at once; the cycle count
// bounds the total.
DRWC_DEV bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kWaitCycles) return false;
    }
}

DRWC_DEV void umma_fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
DRWC_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
DRWC_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

DRWC_DEV void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

DRWC_DEV void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar)) : "memory");
}

DRWC_DEV void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Offset (bytes) of element (row, k) of a [rows x 64] stage tile in the
// canonical layout: K step s = k/16 holds rows*32 bytes; inside it, row group
// g = row/8 at g*256, K half h = (k%16)/8 at h*128, row-in-group at 16 B.
DRWC_DEV uint32_t umma_tile_off(int row, int k, int rows) {
    return (uint32_t)((k >> 4) * rows * 32 + (row >> 3) * 256 + ((k >> 3) & 1) * 128 +
                      (row & 7) * 16 + (k & 7) * 2);
}

// Epilogue functors that can store 4 consecutive columns of one row
// (store4) get coalesced stores: each warp writes its 32 x 32 accumulator
// block back through shared memory, four rows per store instruction (eight
// lanes per row), instead of one row segment per lane.
template <class EPI, class = void>
struct EpiHasStore4 : std::false_type {};
template <class EPI>
struct EpiHasStore4<EPI, std::void_t<decltype(&EPI::store4)>> : std::true_type {};

// The block's floats per warp in shared memory: rows padded to 33 floats,
// so the row-per-lane writes and the column reads are free of bank conflicts.
constexpr int kEpiStageFloats = 32 * 33;

// Rows row0 .. row0+31 (lane = row) x columns col0 .. col0+31 of a warp's
// accumulator values v, through the warp's staging block stg.
template <class EPI>
DRWC_DEV void epi_block_store(const EPI& epi, float* stg, const float* v, int row0, int col0,
                              int M, int N) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int e = 0; e < 32; ++e) stg[lane * 33 + e] = v[e];
    __syncwarp();
#pragma unroll
    for (int it = 0; it < 8; ++it) {
        const int rr = it * 4 + (lane >> 3), cc = (lane & 7) * 4;
        const float* src = stg + rr * 33 + cc;
        if (row0 + rr < M && col0 + cc < N)
            epi.store4(row0 + rr, col0 + cc, make_float4(src[0], src[1], src[2], src[3]));
    }
    __syncwarp();
}

// Shared-memory stages of a tile: enough K stages in flight to cover the
// global latency at two CTAs per SM.
template <int BN>
constexpr int umma_stages() {
    return BN >= 128 ? 3 : 4;
}

// Shared memory a CTA of umma_gemm<BN> needs: the stages, their mbarriers
// and the TMEM address slot.
template <int BN>
constexpr size_t umma_smem_bytes() {
    return (size_t)umma_stages<BN>() * (kUmmaM + BN) * kUmmaBK * 2 + 8 * 8 + 16;
}

DRWC_DEV void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
DRWC_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
DRWC_DEV void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// A valid global address for zero-filled copies (no byte is read from it).
static __device__ __align__(16) uint4 umma_zero16;

// Loader protocol. Every loader is a functor (row, k8, uint4* out) writing the
// 8 BF16 values of columns k8..k8+7 of an operand row (zeros outside). A
// loader whose every such chunk is 16 contiguous, 16-byte aligned bytes of
// global memory (or all zeros) also sets kChunks = true and provides
// chunk(row, k8) -> source address or nullptr (zeros) and chunks_ok() (its
// run-time alignment conditions); tiles whose two loaders both qualify fill
// their stages with cp.async instead of through registers.
template <class L>
DRWC_DEV const void* loader_chunk(const L& l, int r, int k8) {
    if constexpr (L::kChunks) return l.chunk(r, k8);
    else return nullptr;
}

// C tile = A[m0:m0+128, :] * B[n0:n0+BN, :]^T.
//   la(row, k8, out) / lb(row, k8, out): loaders (above).
//   epi(row, col0, v[32]): consume 32 FP32 accumulator values of one row.
// err: device flag set on a wait timeout.
// tmem_cols: the TMEM columns one tile needs (allocated with tcgen05.alloc).
template <int BN>
constexpr uint32_t umma_tmem_cols() {
    return BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
}

// TMEM allocation of a CTA (warp 0 allocates and gives up the permit to
// allocate again, which lets the SM place further CTAs); all threads read the
// address back from the shared slot.
template <int BN>
DRWC_DEV uint32_t umma_tmem_alloc(uint32_t* tslot) {
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(tslot)), "r"(umma_tmem_cols<BN>()));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *tslot;
}

template <int BN>
DRWC_DEV void umma_tmem_free(uint32_t tmem) {
    tc_fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(umma_tmem_cols<BN>()));
}

// Address of the TMEM slot inside a tile CTA's shared memory.
template <int BN>
DRWC_DEV uint32_t* umma_tslot(unsigned char* smem) {
    return reinterpret_cast<uint32_t*>(smem + umma_stages<BN>() * (kUmmaM + BN) * kUmmaBK * 2 + 8 * 8);
}

// tmem_given: a TMEM accumulator the caller allocated (umma_tmem_alloc) and
// keeps across tiles; 0xffffffff: this call allocates and frees its own.
template <int BN, class LA, class LB, class EPI>
DRWC_DEV void umma_gemm_tile(int M, int N, int K, int m0, int n0, const LA& la, const LB& lb,
                             const EPI& epi, int* err, unsigned char* smem,
                             uint32_t tmem_given = 0xffffffffu) {
    constexpr int S = umma_stages<BN>();
    constexpr int STAGE_A = kUmmaM * kUmmaBK * 2, STAGE_B = BN * kUmmaBK * 2;
    auto stA = [&](int st) { return smem + st * (STAGE_A + STAGE_B); };
    auto stB = [&](int st) { return smem + st * (STAGE_A + STAGE_B) + STAGE_A; };
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + S * (STAGE_A + STAGE_B));
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 8);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;

    if (t == 0) {
        for (int q = 0; q < S; ++q) mbar_init(&bar[q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const bool own = tmem_given == 0xffffffffu;
    uint32_t tmem = tmem_given;
    if (own) tmem = umma_tmem_alloc<BN>(tslot);  // (synchronises the CTA)
    else __syncthreads();                         // barriers initialised before use

    const int ktiles = (K + kUmmaBK - 1) / kUmmaBK;
    uint32_t uses[S];
#pragma unroll
    for (int q = 0; q < S; ++q) uses[q] = 0;
    bool ok = true;
    // Operand chunks of a K stage: A 128 rows x 8 chunks of 8 BF16, B BN rows x
    // 8 chunks, spread over the 128 threads.
    constexpr int AV = kUmmaM * 8 / kUmmaThreads, BV = (BN * 8 + kUmmaThreads - 1) / kUmmaThreads;
    auto mma_stage = [&](int kt, int st) {  // thread 0
        tc_fence_after();
        const int k0 = kt * kUmmaBK;
        const int ksteps = min(kUmmaBK, K - k0 + 15) / 16;  // K steps with data
        for (int ks = 0; ks < ksteps && ks < kUmmaBK / 16; ++ks) {
            const uint64_t da = umma_smem_desc(smem_u32(stA(st) + ks * kUmmaM * 32), 128, 256);
            const uint64_t db = umma_smem_desc(smem_u32(stB(st) + ks * BN * 32), 128, 256);
            umma_bf16(tmem, da, db, umma_idesc_bf16<BN>(), (kt > 0 || ks > 0) ? 1u : 0u);
        }
        umma_commit(&bar[st]);
    };
    bool async_path = false;
    if constexpr (LA::kChunks && LB::kChunks) async_path = la.chunks_ok() && lb.chunks_ok();
    if (async_path) {
        // cp.async pipeline: S - 1 stages in flight ahead of the MMAs; a stage
        // is refilled once the MMAs that read it have committed.
        auto issue = [&](int kt) {
            const int st = kt % S, k0 = kt * kUmmaBK;
#pragma unroll
            for (int i = 0; i < AV; ++i) {
                const int v = t + i * kUmmaThreads;
                const void* src = loader_chunk(la, m0 + (v >> 3), k0 + (v & 7) * 8);
                cp_async16(smem_u32(stA(st) + umma_tile_off(v >> 3, (v & 7) * 8, kUmmaM)),
                           src ? src : (const void*)&umma_zero16, src ? 16u : 0u);
            }
#pragma unroll
            for (int i = 0; i < BV; ++i) {
                const int v = t + i * kUmmaThreads;
                if (v < BN * 8) {
                    const void* src = loader_chunk(lb, n0 + (v >> 3), k0 + (v & 7) * 8);
                    cp_async16(smem_u32(stB(st) + umma_tile_off(v >> 3, (v & 7) * 8, BN)),
                               src ? src : (const void*)&umma_zero16, src ? 16u : 0u);
                }
            }
        };
#pragma unroll
        for (int kt = 0; kt < S - 1; ++kt) {
            if (kt < ktiles) issue(kt);
            cp_async_commit();
        }
        for (int kt = 0; kt < ktiles; ++kt) {
            const int st = kt % S;
            cp_async_wait<S - 2>();  // this thread's copies of stage kt have landed
            umma_fence_proxy_async();
            __syncthreads();
            if (t == 0) mma_stage(kt, st);
            uses[st] += 1;
            const int kn = kt + S - 1;  // refill the stage tile kt - 1 used
            if (kn < ktiles) {
                const int sn = kn % S;
                if (uses[sn] > 0) ok &= mbar_wait(&bar[sn], (uses[sn] - 1) & 1);
                issue(kn);
            }
            cp_async_commit();
        }
        cp_async_wait<0>();
    } else {
        // register path: the next stage is gathered into registers while the
        // MMAs of this one run; two stages alternate
        uint4 ra[AV], rb[BV];
        auto gather = [&](int kt) {
            const int k0 = kt * kUmmaBK;
#pragma unroll
            for (int i = 0; i < AV; ++i) {
                const int v = t + i * kUmmaThreads;
                la(m0 + (v >> 3), k0 + (v & 7) * 8, &ra[i]);
            }
#pragma unroll
            for (int i = 0; i < BV; ++i) {
                const int v = t + i * kUmmaThreads;
                if (v < BN * 8) lb(n0 + (v >> 3), k0 + (v & 7) * 8, &rb[i]);
            }
        };
        if (ktiles > 0) gather(0);
        for (int kt = 0; kt < ktiles; ++kt) {
            const int st = kt & 1;
            // the MMAs that last read this stage must be done before refilling it
            if (uses[st] > 0) ok &= mbar_wait(&bar[st], (uses[st] - 1) & 1);
#pragma unroll
            for (int i = 0; i < AV; ++i) {
                const int v = t + i * kUmmaThreads;
                *reinterpret_cast<uint4*>(stA(st) + umma_tile_off(v >> 3, (v & 7) * 8, kUmmaM)) = ra[i];
            }
#pragma unroll
            for (int i = 0; i < BV; ++i) {
                const int v = t + i * kUmmaThreads;
                if (v < BN * 8)
                    *reinterpret_cast<uint4*>(stB(st) + umma_tile_off(v >> 3, (v & 7) * 8, BN)) = rb[i];
            }
            umma_fence_proxy_async();
            __syncthreads();
            if (t == 0) mma_stage(kt, st);
            uses[st] += 1;
            if (kt + 1 < ktiles) gather(kt + 1);
        }
    }
    // all MMAs done: wait for the last commit of every stage used (at most one
    // phase of each barrier is outstanding)
#pragma unroll
    for (int q = 0; q < S; ++q)
        if (uses[q] > 0) ok &= mbar_wait(&bar[q], (uses[q] - 1) & 1);
    tc_fence_after();
    if (!ok && err) atomicExch(err, 1);
    // epilogue: warp w reads accumulator lanes (rows) 32w .. 32w+31; the
    // stages are idle now and stage the coalesced stores
    const int row = m0 + warp * 32 + lane;
    for (int c = 0; c < BN; c += 32) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
        if constexpr (EpiHasStore4<EPI>::value) {
            if (ok && n0 + c < N)
                epi_block_store(epi, reinterpret_cast<float*>(smem) + warp * kEpiStageFloats, v,
                                m0 + warp * 32, n0 + c, M, N);
        } else {
            if (ok && row < M && n0 + c < N) epi(row, n0 + c, v);
        }
    }
    if (own) umma_tmem_free<BN>(tmem);
    else {
        tc_fence_before();
        __syncthreads();  // the accumulator is read before the next tile's MMAs
    }
}

}  // namespace drwc

namespace drwc {

// Generic launchable GEMM kernel: one CTA per 128 x BN tile of C.
template <int BN, class LA, class LB, class EPI>
__global__ void __launch_bounds__(128) umma_kernel(int M, int N, int K, LA la, LB lb, EPI epi,
                                                   int* err) {
    extern __shared__ __align__(1024) unsigned char umma_smem[];
    umma_gemm_tile<BN>(M, N, K, blockIdx.x * kUmmaM, blockIdx.y * BN, la, lb, epi, err,
                       umma_smem);
}

// Loader of a row-major BF16 matrix [rows, cols] with leading dimension ld;
// optional row map (operand row r reads matrix row map[r]).
struct RowsBf16 {
    const __nv_bfloat16* __restrict__ p;
    int rows, cols;
    int64_t ld;
    const int* __restrict__ map;
    static constexpr bool kChunks = true;
    DRWC_DEV bool chunks_ok() const {
        return cols % 8 == 0 && ld % 8 == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0;
    }
    DRWC_DEV const void* chunk(int r, int k8) const {
        if (r >= rows || k8 >= cols) return nullptr;
        return p + (map ? (int64_t)map[r] : (int64_t)r) * ld + k8;
    }
    DRWC_DEV void operator()(int r, int k8, uint4* out) const {
        if (r >= rows || k8 >= cols) { *out = make_uint4(0, 0, 0, 0); return; }
        const int64_t rr = map ? map[r] : r;
        const __nv_bfloat16* src = p + rr * ld + k8;
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

// Loader of the transpose of a row-major BF16 matrix S [K_rows, R_cols]:
// operand row r, columns k8..k8+7 are S[k8..k8+7][r] (strided gather).
struct ColsBf16 {
    const __nv_bfloat16* __restrict__ p;
    int rows, cols;      // operand shape (rows = S columns, cols = S rows)
    int64_t ld;          // S leading dimension
    static constexpr bool kChunks = false;
    DRWC_DEV void operator()(int r, int k8, uint4* out) const {
        __align__(16) __nv_bfloat16 tmp[8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
            tmp[i] = (r < rows && k8 + i < cols) ? p[(int64_t)(k8 + i) * ld + r]
                                                 : __float2bfloat16(0.f);
        *out = *reinterpret_cast<const uint4*>(tmp);
    }
};

}  // namespace drwc
