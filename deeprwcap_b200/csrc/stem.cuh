// Stem of the learned transition network (conv1 and conv2) on the tensor
// cores, inside the CTA that voxelised the cube, so neither the voxel grid
// nor conv1's activations leave shared memory.
//
// A group is the set of cubes whose conv2 rows fill one 128-row MMA tile
// (two cubes at N = 16: 4^3 = 64 rows each) or a single cube (N = 21, 23:
// 6^3 = 216 rows over two tiles). Per cube, conv1 (1 -> 16 channels, 3^3,
// stride 2, zero padding) is an implicit GEMM [D2^3 x 32] x [32 x 16]: the
// threads write the im2col rows of up to four (N = 16) or eight (N = 21,
// 23) 128-row M tiles (taps 27..31 zero) into a staging area in the
// canonical K-major no-swizzle layout, one thread issues two tcgen05.mma
// (K = 16) per tile into its own 16 TMEM columns, and the epilogue
// (tcgen05.ld, bias, ReLU, BF16) writes the rows into the group's conv1
// activations [cube][D2^3][16] in shared memory. conv2 (16 -> 32 channels)
// then gathers its im2col rows from there, nine taps (K steps) of every
// tile of the group per staging fill, accumulates each 128-row tile in 32
// TMEM columns and writes its activations [row][32] (BF16, channels last)
// to global memory, where the tile GEMMs of conv3 and the heads read them.
//
// Operands are the BF16 values the stand-alone convolution GEMMs read and
// each MMA sums in FP32, so a row's result does not depend on the other rows
// of its tile or on how rows are grouped. Phases are serialised inside the
// CTA (fill, barrier, MMA, bounded mbarrier wait, epilogue); co-resident CTAs
// overlap one another's phases. A wait that runs out raises the error flag,
// every thread leaves at the next barrier, and the CTA still waits (bounded)
// for its MMAs before it frees its tensor memory.
#pragma once

#include <cuda_bf16.h>

#include "nn.cuh"
#include "umma.cuh"

namespace drwc {

template <int N>
struct StemDims {
    static constexpr int D2 = (N - 1) / 2 + 1, P2 = D2 * D2 * D2;  // conv1 output
    static constexpr int D3 = (D2 - 1) / 2 + 1, P3 = D3 * D3 * D3;  // conv2 output
    static constexpr int CUBES = P3 <= 64 ? kUmmaM / P3 : 1;        // cubes per group
    static_assert(CUBES == 1 || CUBES * P3 == kUmmaM, "a group's conv2 rows fill whole tiles");
    static constexpr int ROWS2 = CUBES * P3;                         // conv2 rows per group
    static constexpr int MT2 = (ROWS2 + kUmmaM - 1) / kUmmaM;       // conv2 M tiles
    static constexpr int MT1 = (P2 + kUmmaM - 1) / kUmmaM;          // conv1 M tiles per cube
    static constexpr int NT = N <= 16 ? 256 : 512;
    static constexpr int CTAS = N <= 16 ? 2 : 1;
    // conv1 M tiles per MMA batch (16 TMEM columns each): N = 21 / 23 cubes
    // (11 / 14 tiles) take eight, so a cube needs two batches
    static constexpr int R1 = N <= 16 ? 4 : 8;
    static constexpr int TAPS = 9;         // conv2 taps (K steps of 16) per MMA batch
    static constexpr int MT2B = NT / 256;  // conv2 M tiles per batch: one per 256 threads
    static_assert(MT2 <= MT2B, "one conv2 batch holds every tile of a group");
    static constexpr int C2 = 16 * R1;     // first TMEM column of the conv2 accumulators
    static constexpr uint32_t TCOLS = N <= 16 ? 128 : 256;
    static_assert(C2 + 32 * MT2 <= (int)TCOLS, "conv2 accumulators after conv1's columns");
    // dynamic shared memory (bytes); every operand block is 1024-aligned
    static constexpr int OPA =
        R1 * 8192 > MT2B * TAPS * 4096 ? R1 * 8192 : MT2B * TAPS * 4096;
    static constexpr int W2B = 27 * 32 * 32;  // conv2 weights: 27 K steps x 32 rows x 32 B
    static constexpr int W1B = 2 * 16 * 32;   // conv1 weights: 2 K steps x 16 rows x 32 B
    static constexpr int A1B = CUBES * P2 * 32;
    static constexpr int XSB = (N * N * N * 2 + 15) / 16 * 16;
    static constexpr int MATB = (N * N * N + 15) / 16 * 16;
    static constexpr int O_W2 = OPA, O_W1 = O_W2 + W2B, O_A1 = O_W1 + W1B, O_XS = O_A1 + A1B,
                         O_MAT = O_XS + XSB, O_B1 = O_MAT + MATB, O_B2 = O_B1 + 16 * 4,
                         O_BAR = O_B2 + 32 * 4, O_TSLOT = O_BAR + 8, O_ABORT = O_TSLOT + 4,
                         BYTES = (O_ABORT + 4 + 15) / 16 * 16;
};

// 16 columns of the warp's 32 TMEM lanes.
DRWC_DEV void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ReLU(v + b) of 16 channels as BF16, two 16-byte stores.
DRWC_DEV void stem_store16(const float* v, const float* b, __nv_bfloat16* dst) {
    __align__(16) __nv_bfloat162 o[8];
#pragma unroll
    for (int q = 0; q < 8; ++q)
        o[q] = __floats2bfloat162_rn(fmaxf(v[2 * q] + b[2 * q], 0.f),
                                     fmaxf(v[2 * q + 1] + b[2 * q + 1], 0.f));
    uint4* d = reinterpret_cast<uint4*>(dst);
    d[0] = reinterpret_cast<const uint4*>(o)[0];
    d[1] = reinterpret_cast<const uint4*>(o)[1];
}

template <int N>
struct Stem {
    using S = StemDims<N>;
    unsigned char* sm;
    uint32_t tmem = 0;
    uint32_t phase = 0;
    bool pending = false;  // MMAs committed and not yet seen complete

    DRWC_DEV unsigned char* opa() const { return sm; }
    DRWC_DEV __nv_bfloat16* xs() const { return reinterpret_cast<__nv_bfloat16*>(sm + S::O_XS); }
    DRWC_DEV uint8_t* mat() const { return sm + S::O_MAT; }
    DRWC_DEV __nv_bfloat16* a1(int cube) const {
        return reinterpret_cast<__nv_bfloat16*>(sm + S::O_A1) + (size_t)cube * S::P2 * 16;
    }
    DRWC_DEV const float* b1() const { return reinterpret_cast<const float*>(sm + S::O_B1); }
    DRWC_DEV const float* b2() const { return reinterpret_cast<const float*>(sm + S::O_B2); }
    DRWC_DEV uint64_t* bar() const { return reinterpret_cast<uint64_t*>(sm + S::O_BAR); }
    DRWC_DEV volatile int* abort_flag() const {
        return reinterpret_cast<volatile int*>(sm + S::O_ABORT);
    }
    DRWC_DEV bool aborted() const { return *abort_flag() != 0; }

    // Weights in the canonical K-major layout, biases, barrier, TMEM.
    DRWC_DEV void begin(const NetStem& w) {
        const int t = threadIdx.x;
        for (int e = t; e < 16 * 32; e += blockDim.x) {
            const int co = e >> 5, k = e & 31;
            *reinterpret_cast<__nv_bfloat16*>(sm + S::O_W1 + umma_tile_off(co, k, 16)) =
                k < 27 ? w.w1[co * 27 + k] : __float2bfloat16(0.f);
        }
        for (int e = t; e < 32 * 432; e += blockDim.x) {
            const int co = e / 432, k = e % 432;
            *reinterpret_cast<__nv_bfloat16*>(sm + S::O_W2 + umma_tile_off(co, k, 32)) =
                w.w2[co * 432 + k];
        }
        if (t < 16) reinterpret_cast<float*>(sm + S::O_B1)[t] = w.b1[t];
        if (t < 32) reinterpret_cast<float*>(sm + S::O_B2)[t] = w.b2[t];
        if (t == 0) {
            mbar_init(bar(), 1);
            *abort_flag() = 0;
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + S::O_TSLOT);
        if ((t >> 5) == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                         ::"r"(smem_u32(tslot)), "r"(S::TCOLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        tmem = *tslot;
    }

    // The staging area is written: make it visible to the tensor cores and
    // meet at a barrier; false when a wait has run out (every thread agrees).
    DRWC_DEV bool staged() {
        umma_fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        return !aborted();
    }

    // After thread 0 committed: warp 0 waits for the MMAs (bounded), the
    // other warps at the CTA barrier, which leaves their issue slots to the
    // co-resident CTA; the barrier orders the accumulator reads after the
    // MMAs' completion.
    DRWC_DEV void complete(int* err) {
        if (threadIdx.x < 32) {
            const bool done = mbar_wait(bar(), phase);
            if (!done && threadIdx.x == 0) {
                *abort_flag() = 1;
                if (err) atomicExch(err, 1);
            }
        }
        phase ^= 1;
        __syncthreads();
        tc_fence_after();
        pending = aborted();  // after a timeout the MMAs may still be in flight
    }

    // Class of a conv1 output index along an axis whose input values do not
    // vary: which of its three taps fall outside the grid (0: the first, 1:
    // none, 2: the last). Rows of equal class along both such axes and the
    // same index along the varying axis have the same 27 taps.
    static constexpr DRWC_DEV int c1_class(int p) { return p == 0 ? 0 : (2 * p + 1 >= N ? 2 : 1); }
    // The same for a conv2 output index: its three taps read conv1 indices
    // 2q - 1 .. 2q + 1 (or the zero padding), and those classes (0, 1, 1 at
    // q = 0; 1, 1, 1 inside; at the last index of an odd N either 1, 1, 2 or
    // 1, 2, padding) fix the row; rep2 is an index of each class.
    static constexpr DRWC_DEV int c2_class(int q) {
        return q == 0 ? 0 : (q == S::D3 - 1 && (N & 1) ? 2 : 1);
    }
    static constexpr DRWC_DEV int c2_rep(int c) { return c == 2 ? S::D3 - 1 : c; }
    static constexpr int c2_sig(int q) {  // the conv1 classes (3: padding) of q's taps
        int sg = 0;
        for (int d = 0; d < 3; ++d) {
            const int p = 2 * q - 1 + d;
            sg = 4 * sg + ((p < 0 || p >= S::D2) ? 3 : c1_class(p));
        }
        return sg;
    }
    static constexpr bool c2_classes_exact() {
        for (int a = 0; a < S::D3; ++a) {
            if (c2_sig(a) != c2_sig(c2_rep(c2_class(a)))) return false;
            for (int b = 0; b < S::D3; ++b)
                if ((c2_class(a) == c2_class(b)) != (c2_sig(a) == c2_sig(b))) return false;
        }
        return true;
    }
    static_assert(c2_classes_exact(), "conv2 classes group exactly the rows with equal taps");

    // conv1 of a cube whose values vary along uaxis alone: its D2 x 3 x 3
    // distinct rows (index along uaxis; class along the other two axes in
    // z, y, x order) fill one M tile and stay at the start of a1(cube), where
    // conv2 reads a row's values from its class row. A row's result does not
    // depend on the other rows of its tile, so these are the values the full
    // convolution writes, from one MMA batch instead of MT1 tiles.
    DRWC_DEV bool conv1_uaxis(int cube, int* err, int uaxis,
                              const __nv_bfloat16* __restrict__ pv) {
        static_assert(9 * S::D2 <= kUmmaM, "the class rows fit one tile");
        const int t = threadIdx.x, w = t >> 5, lane = t & 31, q = w & 3, sub = w >> 2;
        // the class rows stay at the start of a1(cube): conv2_uaxis /
        // conv2_pair gather from them
        __nv_bfloat16* a1c = a1(cube);
        auto rep = [](int c) { return c == 2 ? S::D2 - 1 : c; };  // an index of each class
        if (t < kUmmaM) {
            const int r = t;
            uint32_t pk[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) pk[i] = 0u;
            if (r < 9 * S::D2) {
                const int pu = r / 9, ca = rep((r / 3) % 3), cb = rep(r % 3);
                const int pz = uaxis == 2 ? pu : ca;
                const int py = uaxis == 2 ? ca : uaxis == 1 ? pu : cb;
                const int px = uaxis == 0 ? pu : cb;
                const int z0 = 2 * pz - 1, y0 = 2 * py - 1, x0 = 2 * px - 1;
                const int u0 = uaxis == 2 ? z0 : uaxis == 1 ? y0 : x0;
                uint32_t uv[3], ok[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    uv[d] = (unsigned)(u0 + d) < (unsigned)N
                                ? (uint32_t)__bfloat16_as_ushort(pv[u0 + d]) : 0u;
                    ok[d] = ((unsigned)(x0 + d) < (unsigned)N ? 1u : 0u) |
                            ((unsigned)(y0 + d) < (unsigned)N ? 2u : 0u) |
                            ((unsigned)(z0 + d) < (unsigned)N ? 4u : 0u);
                }
#pragma unroll
                for (int tap = 0; tap < 27; ++tap) {
                    const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
                    const bool in = (ok[dx] & 1u) && (ok[dy] & 2u) && (ok[dz] & 4u);
                    const uint32_t v = uaxis == 2 ? uv[dz] : uaxis == 1 ? uv[dy] : uv[dx];
                    pk[tap >> 1] |= (in ? v : 0u) << (16 * (tap & 1));
                }
            }
            unsigned char* base = opa() + (r >> 3) * 256 + (r & 7) * 16;
#pragma unroll
            for (int c = 0; c < 4; ++c)
                *reinterpret_cast<uint4*>(base + (c >> 1) * 4096 + (c & 1) * 128) =
                    make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
        }
        if (!staged()) return false;
        if (t == 0) {
            for (int k = 0; k < 2; ++k)
                umma_bf16(tmem, umma_smem_desc(smem_u32(opa() + k * 4096), 128, 256),
                          umma_smem_desc(smem_u32(sm + S::O_W1 + k * 512), 128, 256),
                          umma_idesc_bf16<16>(), (uint32_t)k);
            umma_commit(bar());
        }
        complete(err);
        if (sub == 0) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * q) << 16), v);
            const int r = 32 * q + lane;
            if (r < 9 * S::D2) stem_store16(v, b1(), a1c + (size_t)r * 16);
        }
        tc_fence_before();  // the next MMAs overwrite these columns
        __syncthreads();  // class rows complete; every thread sees the same abort flag
        return !aborted();
    }

    // conv1 of the cube into a1(cube), up to R1 M tiles per batch, from the
    // voxels in xs() or, with uaxis >= 0, from pv: the cube's values then
    // vary along that index alone (0 = x, 1 = y, 2 = z; pv[t] is the value
    // at index t), so a row's 27 taps come from three values and the grid
    // bounds (the same values xs would hold), and conv1_uaxis computes it.
    DRWC_DEV bool conv1(int cube, int* err, int uaxis = -1,
                        const __nv_bfloat16* __restrict__ pv = nullptr) {
        if (uaxis >= 0) return conv1_uaxis(cube, err, uaxis, pv);
        const __nv_bfloat16* x = xs();
        const int t = threadIdx.x, w = t >> 5, lane = t & 31, q = w & 3, sub = w >> 2;
        for (int m0 = 0; m0 < S::MT1; m0 += S::R1) {
            const int nb = min(S::R1, S::MT1 - m0);
            for (int it = t; it < nb * kUmmaM; it += S::NT) {
                const int j = it >> 7, r = it & 127, p = (m0 + j) * kUmmaM + r;
                uint32_t pk[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) pk[i] = 0u;
                if (p < S::P2) {
                    const int pz = p / (S::D2 * S::D2), py = (p / S::D2) % S::D2, px = p % S::D2;
                    const int z0 = 2 * pz - 1, y0 = 2 * py - 1, x0 = 2 * px - 1;
                    if (uaxis >= 0) {
                        const int u0 = uaxis == 2 ? z0 : uaxis == 1 ? y0 : x0;
                        uint32_t uv[3], ok[3];  // values along the axis; in-grid bits per axis
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            uv[d] = (unsigned)(u0 + d) < (unsigned)N
                                        ? (uint32_t)__bfloat16_as_ushort(pv[u0 + d]) : 0u;
                            ok[d] = ((unsigned)(x0 + d) < (unsigned)N ? 1u : 0u) |
                                    ((unsigned)(y0 + d) < (unsigned)N ? 2u : 0u) |
                                    ((unsigned)(z0 + d) < (unsigned)N ? 4u : 0u);
                        }
#pragma unroll
                        for (int tap = 0; tap < 27; ++tap) {
                            const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
                            const bool in = (ok[dx] & 1u) && (ok[dy] & 2u) && (ok[dz] & 4u);
                            const uint32_t v = uaxis == 2 ? uv[dz] : uaxis == 1 ? uv[dy] : uv[dx];
                            pk[tap >> 1] |= (in ? v : 0u) << (16 * (tap & 1));
                        }
                    } else {
#pragma unroll
                        for (int tap = 0; tap < 27; ++tap) {
                            const int z = z0 + tap / 9, y = y0 + (tap / 3) % 3, xx = x0 + tap % 3;
                            const bool in = (unsigned)z < (unsigned)N &&
                                            (unsigned)y < (unsigned)N && (unsigned)xx < (unsigned)N;
                            const uint32_t v =
                                in ? (uint32_t)__bfloat16_as_ushort(x[(z * N + y) * N + xx]) : 0u;
                            pk[tap >> 1] |= v << (16 * (tap & 1));
                        }
                    }
                }
                unsigned char* base = opa() + j * 8192 + (r >> 3) * 256 + (r & 7) * 16;
#pragma unroll
                for (int c = 0; c < 4; ++c)  // taps 8c .. 8c + 7: K step c / 2, half c % 2
                    *reinterpret_cast<uint4*>(base + (c >> 1) * 4096 + (c & 1) * 128) =
                        make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
            }
            if (!staged()) return false;
            if (t == 0) {
                for (int j = 0; j < nb; ++j)
                    for (int s = 0; s < 2; ++s)
                        umma_bf16(tmem + 16 * j,
                                  umma_smem_desc(smem_u32(opa() + j * 8192 + s * 4096), 128, 256),
                                  umma_smem_desc(smem_u32(sm + S::O_W1 + s * 512), 128, 256),
                                  umma_idesc_bf16<16>(), (uint32_t)s);
                umma_commit(bar());
            }
            complete(err);
            __nv_bfloat16* dst = a1(cube);
            for (int j = sub; j < nb; j += S::NT / 128) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + 16 * j, v);
                const int p = (m0 + j) * kUmmaM + 32 * q + lane;
                if (p < S::P2) stem_store16(v, b1(), dst + (size_t)p * 16);
            }
            tc_fence_before();  // the next batch's MMAs overwrite these columns
        }
        __syncthreads();  // a1 complete; every thread sees the same abort flag
        return !aborted();
    }

    // conv2 of the group's nc cubes (a1(0 .. nc-1)) -> a2 rows [g0 * P3, ..).
    DRWC_DEV bool conv2(int nc, __nv_bfloat16* __restrict__ a2, int* err) {
        const int t = threadIdx.x, w = t >> 5, lane = t & 31, q = w & 3, sub = w >> 2;
        static_assert(S::TAPS == 9 && S::NT % 256 == 0, "a fill is one dz plane of taps");
        // every thread keeps one (row, channel half) of one tile (256 threads
        // per tile) and walks the taps of each fill: the row's position is
        // decoded once; a batch holds every tile of the group
        const int pr = t & 255, r = pr >> 1, h = pr & 1, mt = t >> 8;
        unsigned char* dst =
            opa() + mt * (S::TAPS * 4096) + (r >> 3) * 256 + h * 128 + (r & 7) * 16;
        {
            const int R = mt * kUmmaM + r;
            const int cube = R / S::P3, p = R % S::P3;
            const bool row_ok = mt < S::MT2 && R < S::ROWS2 && cube < nc;
            const int z0 = 2 * (p / (S::D3 * S::D3)) - 1, y0 = 2 * ((p / S::D3) % S::D3) - 1,
                      x0 = 2 * (p % S::D3) - 1;
            unsigned yx_ok = 0;  // bit dy * 3 + dx: that tap's (y, x) lies inside the grid
#pragma unroll
            for (int k = 0; k < 9; ++k)
                if ((unsigned)(y0 + k / 3) < (unsigned)S::D2 && (unsigned)(x0 + k % 3) < (unsigned)S::D2)
                    yx_ok |= 1u << k;
            const __nv_bfloat16* src0 = a1(row_ok ? cube : 0) + 8 * h;
            for (int cc = 0; cc < 3; ++cc) {  // fill cc holds the taps with dz = cc
                const int z = z0 + cc;
                const bool z_ok = row_ok && (unsigned)z < (unsigned)S::D2;
                if (mt < S::MT2) {
#pragma unroll
                    for (int ti = 0; ti < 9; ++ti) {
                        uint4 val = make_uint4(0u, 0u, 0u, 0u);
                        if (z_ok && ((yx_ok >> ti) & 1u))
                            val = *reinterpret_cast<const uint4*>(
                                src0 + (size_t)((z * S::D2 + y0 + ti / 3) * S::D2 + x0 + ti % 3) * 16);
                        *reinterpret_cast<uint4*>(dst + ti * 4096) = val;
                    }
                }
                if (!staged()) return false;
                if (t == 0) {
                    for (int j = 0; j < S::MT2; ++j)
                        for (int ti = 0; ti < S::TAPS; ++ti)
                            umma_bf16(tmem + S::C2 + 32 * j,
                                      umma_smem_desc(smem_u32(opa() + j * (S::TAPS * 4096) + ti * 4096),
                                                     128, 256),
                                      umma_smem_desc(
                                          smem_u32(sm + S::O_W2 + (cc * S::TAPS + ti) * 1024), 128, 256),
                                      umma_idesc_bf16<32>(), (cc | ti) ? 1u : 0u);
                    umma_commit(bar());
                }
                complete(err);
            }
        }
        // epilogue: (tile, 16-column half) tasks over the warp quarters
        for (int task = sub; task < 2 * S::MT2; task += S::NT / 128) {
            const int mt = task >> 1, half = task & 1;
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + S::C2 + 32 * mt + 16 * half, v);
            const int R = mt * kUmmaM + 32 * q + lane;
            if (R < S::ROWS2 && R / S::P3 < nc)
                stem_store16(v, b2() + 16 * half, a2 + (size_t)R * 32 + 16 * half);
        }
        tc_fence_before();
        __syncthreads();
        return !aborted();
    }

    // conv2 of a one-cube group whose cube varies along uaxis alone (conv1_uaxis
    // left its class rows at a1(0)): the D3 x 3 x 3 class rows (index along
    // uaxis, conv2 class along the other two) in one M tile, their taps
    // gathered from conv1's class rows; the epilogue stages them in shared
    // memory and every a2 row of the cube is copied from its class row. Same
    // operands per row as conv2, so the same a2.
    DRWC_DEV bool conv2_uaxis(int uaxis, __nv_bfloat16* __restrict__ a2, int* err) {
        static_assert(S::CUBES == 1 && 9 * S::D3 <= kUmmaM, "one cube, class rows in one tile");
        const int t = threadIdx.x, w = t >> 5, lane = t & 31, q = w & 3, sub = w >> 2;
        const __nv_bfloat16* a1c = a1(0);
        constexpr int NR = 9 * S::D3;
        const int pr = t & 255, r = pr >> 1, h = pr & 1;
        const bool filler = t < 256;  // one (row, channel half) of the tile each
        unsigned char* dst = opa() + (r >> 3) * 256 + h * 128 + (r & 7) * 16;
        int qz = 0, qy = 0, qx = 0;
        const bool row_ok = filler && r < NR;
        if (row_ok) {
            const int qu = r / 9, ca = c2_rep((r / 3) % 3), cb = c2_rep(r % 3);
            qz = uaxis == 2 ? qu : ca;
            qy = uaxis == 2 ? ca : uaxis == 1 ? qu : cb;
            qx = uaxis == 0 ? qu : cb;
        }
        const int z0 = 2 * qz - 1, y0 = 2 * qy - 1, x0 = 2 * qx - 1;
        for (int cc = 0; cc < 3; ++cc) {  // fill cc holds the taps with dz = cc
            if (filler) {
                const int z = z0 + cc;
#pragma unroll
                for (int ti = 0; ti < 9; ++ti) {
                    const int y = y0 + ti / 3, x = x0 + ti % 3;
                    uint4 val = make_uint4(0u, 0u, 0u, 0u);
                    if (row_ok && (unsigned)z < (unsigned)S::D2 && (unsigned)y < (unsigned)S::D2 &&
                        (unsigned)x < (unsigned)S::D2) {
                        const int pu = uaxis == 2 ? z : uaxis == 1 ? y : x;
                        const int ca1 = c1_class(uaxis == 2 ? y : z), cb1 = c1_class(uaxis == 0 ? y : x);
                        val = *reinterpret_cast<const uint4*>(a1c + (size_t)(pu * 9 + ca1 * 3 + cb1) * 16 +
                                                              8 * h);
                    }
                    *reinterpret_cast<uint4*>(dst + ti * 4096) = val;
                }
            }
            if (!staged()) return false;
            if (t == 0) {
                for (int ti = 0; ti < S::TAPS; ++ti)
                    umma_bf16(tmem + S::C2,
                              umma_smem_desc(smem_u32(opa() + ti * 4096), 128, 256),
                              umma_smem_desc(smem_u32(sm + S::O_W2 + (cc * S::TAPS + ti) * 1024), 128, 256),
                              umma_idesc_bf16<32>(), (cc | ti) ? 1u : 0u);
                umma_commit(bar());
            }
            complete(err);
        }
        // epilogue: the class rows (two 16-column halves) into shared memory
        // (the operand area, free once the MMAs completed) ...
        __nv_bfloat16* a2c = reinterpret_cast<__nv_bfloat16*>(opa());
        if (sub < 2) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + S::C2 + 16 * sub, v);
            const int R = 32 * q + lane;
            if (R < NR) stem_store16(v, b2() + 16 * sub, a2c + (size_t)R * 32 + 16 * sub);
        }
        tc_fence_before();
        __syncthreads();
        // ... then every row of the cube from its class row (four 16-byte parts)
        for (int e = t; e < 4 * S::P3; e += S::NT) {
            const int p = e >> 2, k = e & 3;
            const int pz = p / (S::D3 * S::D3), py = (p / S::D3) % S::D3, px = p % S::D3;
            const int qu = uaxis == 2 ? pz : uaxis == 1 ? py : px;
            const int ca = c2_class(uaxis == 2 ? py : pz), cb = c2_class(uaxis == 0 ? py : px);
            *reinterpret_cast<uint4*>(a2 + (size_t)p * 32 + 8 * k) =
                *reinterpret_cast<const uint4*>(a2c + (size_t)(qu * 9 + ca * 3 + cb) * 32 + 8 * k);
        }
        __syncthreads();  // the operand area is reused by the next group
        return !aborted();
    }

    // conv2 of a two-cube group (N = 16) of which at least one cube varies
    // along one axis alone (ux0 / ux1 >= 0; -1: a full cube): a class cube
    // uses its D3 x 3 x 3 class rows at the start of its 64-row part of the
    // tile, gathered from conv1's class rows, a full cube its 64 rows. The
    // epilogue stages the tile in shared memory, then writes each a2 row of
    // the group, a class cube's from its class row.
    DRWC_DEV bool conv2_pair(int nc, __nv_bfloat16* __restrict__ a2, int* err, int ux0, int ux1) {
        static_assert(S::CUBES == 2 && S::MT2 == 1 && S::NT == 256 && 9 * S::D3 <= S::P3,
                      "two cubes in one tile, class rows inside a cube's part");
        const int t = threadIdx.x, w = t >> 5, lane = t & 31, q = w & 3, sub = w >> 2;
        const int r = t >> 1, h = t & 1;  // one (row, channel half) of the tile each
        unsigned char* dst = opa() + (r >> 3) * 256 + h * 128 + (r & 7) * 16;
        const int cube = r / S::P3, p = r % S::P3;
        const int ux = cube == 0 ? ux0 : ux1;
        const bool cls = ux >= 0;
        const bool row_ok = cube < nc && (!cls || p < 9 * S::D3);
        int qz, qy, qx;
        if (cls) {
            const int qu = p / 9, ca = c2_rep((p / 3) % 3), cb = c2_rep(p % 3);
            qz = ux == 2 ? qu : ca;
            qy = ux == 2 ? ca : ux == 1 ? qu : cb;
            qx = ux == 0 ? qu : cb;
        } else {
            qz = p / (S::D3 * S::D3);
            qy = (p / S::D3) % S::D3;
            qx = p % S::D3;
        }
        const int z0 = 2 * qz - 1, y0 = 2 * qy - 1, x0 = 2 * qx - 1;
        const __nv_bfloat16* A1 = a1(cube < nc ? cube : 0) + 8 * h;
        for (int cc = 0; cc < 3; ++cc) {  // fill cc holds the taps with dz = cc
            const int z = z0 + cc;
#pragma unroll
            for (int ti = 0; ti < 9; ++ti) {
                const int y = y0 + ti / 3, x = x0 + ti % 3;
                uint4 val = make_uint4(0u, 0u, 0u, 0u);
                if (row_ok && (unsigned)z < (unsigned)S::D2 && (unsigned)y < (unsigned)S::D2 &&
                    (unsigned)x < (unsigned)S::D2) {
                    int idx;
                    if (cls) {
                        const int pu = ux == 2 ? z : ux == 1 ? y : x;
                        idx = pu * 9 + c1_class(ux == 2 ? y : z) * 3 + c1_class(ux == 0 ? y : x);
                    } else {
                        idx = (z * S::D2 + y) * S::D2 + x;
                    }
                    val = *reinterpret_cast<const uint4*>(A1 + (size_t)idx * 16);
                }
                *reinterpret_cast<uint4*>(dst + ti * 4096) = val;
            }
            if (!staged()) return false;
            if (t == 0) {
                for (int ti = 0; ti < S::TAPS; ++ti)
                    umma_bf16(tmem + S::C2,
                              umma_smem_desc(smem_u32(opa() + ti * 4096), 128, 256),
                              umma_smem_desc(smem_u32(sm + S::O_W2 + (cc * S::TAPS + ti) * 1024), 128, 256),
                              umma_idesc_bf16<32>(), (cc | ti) ? 1u : 0u);
                umma_commit(bar());
            }
            complete(err);
        }
        // epilogue: the tile's rows (two 16-column halves) into shared memory
        // (the operand area, free once the MMAs completed) ...
        __nv_bfloat16* a2s = reinterpret_cast<__nv_bfloat16*>(opa());
        {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + S::C2 + 16 * sub, v);
            stem_store16(v, b2() + 16 * sub, a2s + (size_t)(32 * q + lane) * 32 + 16 * sub);
        }
        tc_fence_before();
        __syncthreads();
        // ... then the group's a2 rows (four 16-byte parts each)
        for (int e = t; e < 4 * nc * S::P3; e += S::NT) {
            const int row = e >> 2, k = e & 3;
            const int cb2 = row / S::P3, pp = row % S::P3;
            const int u = cb2 == 0 ? ux0 : ux1;
            int src = pp;
            if (u >= 0) {
                const int pz = pp / (S::D3 * S::D3), py = (pp / S::D3) % S::D3, px = pp % S::D3;
                const int qu = u == 2 ? pz : u == 1 ? py : px;
                src = qu * 9 + c2_class(u == 2 ? py : pz) * 3 + c2_class(u == 0 ? py : px);
            }
            *reinterpret_cast<uint4*>(a2 + (size_t)row * 32 + 8 * k) =
                *reinterpret_cast<const uint4*>(a2s + (size_t)(cb2 * S::P3 + src) * 32 + 8 * k);
        }
        __syncthreads();  // the operand area is reused by the next group
        return !aborted();
    }

    // Wait (bounded) for MMAs still in flight after a timeout, free TMEM.
    DRWC_DEV void end() {
        if (threadIdx.x == 0 && pending) mbar_wait(bar(), phase ^ 1);
        tc_fence_before();
        __syncthreads();
        if ((threadIdx.x >> 5) == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                         "r"(S::TCOLS));
    }
};

}  // namespace drwc
