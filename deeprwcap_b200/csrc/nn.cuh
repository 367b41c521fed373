// Internal host API of the learned transition network (nn.cu) for the
// learned walker (walker.cu). Not part of the C ABI.
#pragma once

#include <cuda_bf16.h>

#include "host.cuh"

#define DRWC_DEV_INLINE __device__ __forceinline__

struct drwc_net;

namespace drwc {

// Scale of the gradient head: outputs are WVTZ surface values times this.
constexpr float kGradScale = 64.0f;

// Encoder + heads on B rows of X (BF16 [B, 4096], device): O [B, 1552] and G
// [B, 1536] (either nullable). Launches on the net's context stream; the
// caller holds the context lock.
int net_forward_locked(drwc_net* n, int B, const __nv_bfloat16* X, float* O, float* G);
// Same, with the gradient head only on rows_g feature rows (gmap[r] is the
// encoder row of gradient output row r).
int net_forward_mapped(drwc_net* n, int B, const __nv_bfloat16* X, float* O, float* G,
                       const int* gmap, int rows_g);
// Same on row counts read on the device (*nrows rows of X, *nrows_g rows
// of the gradient head), for CUDA-graph replay: every launch covers Bmax
// rows and tiles past the count exit at once. Call net_reserve_rows(Bmax)
// beforehand (it allocates). X = nullptr starts at conv2: the caller has
// written conv1's activations (see conv1_cube below) into the net's a1.
int net_forward_dyn(drwc_net* n, int Bmax, const unsigned* nrows, const __nv_bfloat16* X,
                    float* O, float* G, const int* gmap, const unsigned* nrows_g);
int net_reserve_rows(drwc_net* n, int B);
// A held network keeps its activation buffers: calls that would need larger
// ones fail with DRWC_ERR_INVALID until every holder lets go.
void net_hold(drwc_net* n, int delta);
drwc_ctx* net_context(drwc_net* n);
int net_size(drwc_net* n);  // cube resolution N of the network

// conv1 operands: BF16 weights [16][27] (tap = dz*9 + dy*3 + dx), FP32 bias,
// and the activation buffer a1 [rows * 512][16] (channels last).
struct NetConv1 {
    const __nv_bfloat16* w1;
    const float* b1;
    __nv_bfloat16* a1;
};
NetConv1 net_conv1_operands(drwc_net* n);

// conv1 of one D^3 cube on the CUDA cores, CTA-wide: x (shared, BF16 eps /
// max eps), w4 (shared, FP32 copies of the BF16 weights, tap-major: w4[tap *
// 4 + g] holds output channels 4g..4g+3 of that tap), b (shared, bias) ->
// a1 rows [Do^3][16] BF16 = ReLU(b + sum over taps of w * x), zero padding,
// stride 2 (Do = (D - 1) / 2 + 1). The operands are the BF16 values the
// tensor-core layer reads and every product is exact in FP32; only the FP32
// summation order differs. With one input channel its GEMM has K = 27, too
// thin for the tensor cores, while the FMAs run next to the voxelisation
// that produced x.
template <int D>
DRWC_DEV_INLINE void conv1_cube(const __nv_bfloat16* x, const float4* w4, const float* b,
                                __nv_bfloat16* __restrict__ a1) {
    constexpr int Do = (D - 1) / 2 + 1, P = Do * Do * Do;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const int pz = p / (Do * Do), py = (p / Do) % Do, px = p % Do;
        float acc[16];
#pragma unroll
        for (int co = 0; co < 16; ++co) acc[co] = 0.f;
#pragma unroll 3
        for (int tap = 0; tap < 27; ++tap) {  // partly unrolled: weights stream from shared
            const int z = 2 * pz - 1 + tap / 9, y = 2 * py - 1 + (tap / 3) % 3,
                      xx = 2 * px - 1 + tap % 3;
            const bool in = z >= 0 && z < D && y >= 0 && y < D && xx >= 0 && xx < D;
            const float xv = in ? __bfloat162float(x[(z * D + y) * D + xx]) : 0.f;
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                const float4 w = w4[tap * 4 + g];
                acc[4 * g] = fmaf(w.x, xv, acc[4 * g]);
                acc[4 * g + 1] = fmaf(w.y, xv, acc[4 * g + 1]);
                acc[4 * g + 2] = fmaf(w.z, xv, acc[4 * g + 2]);
                acc[4 * g + 3] = fmaf(w.w, xv, acc[4 * g + 3]);
            }
        }
        __align__(16) __nv_bfloat162 out[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
            out[q] = __floats2bfloat162_rn(fmaxf(acc[2 * q] + b[2 * q], 0.f),
                                           fmaxf(acc[2 * q + 1] + b[2 * q + 1], 0.f));
        uint4* dst = reinterpret_cast<uint4*>(a1 + (size_t)p * 16);
        dst[0] = reinterpret_cast<const uint4*>(out)[0];
        dst[1] = reinterpret_cast<const uint4*>(out)[1];
    }
}


}  // namespace drwc
