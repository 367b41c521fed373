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
// beforehand (it allocates). X = nullptr starts at conv3: the caller has
// written conv2's activations into the net's a2 (see NetStem below).
int net_forward_dyn(drwc_net* n, int Bmax, const unsigned* nrows, const __nv_bfloat16* X,
                    float* O, float* G, const int* gmap, const unsigned* nrows_g);
int net_reserve_rows(drwc_net* n, int B);
// A held network keeps its activation buffers: calls that would need larger
// ones fail with DRWC_ERR_INVALID until every holder lets go.
void net_hold(drwc_net* n, int delta);
drwc_ctx* net_context(drwc_net* n);
int net_size(drwc_net* n);  // cube resolution N of the network

// Operands of the network's stem (conv1 and conv2) for a caller that runs it
// itself: BF16 weights w1 [16][27] (tap = dz*9 + dy*3 + dx) and w2 [32][27 *
// 16] (K index = tap * 16 + input channel), FP32 biases, the conv2
// activation buffer a2 [rows * Do2^3][32] (BF16, channels last) that
// net_forward_dyn reads when called without X, and the net's error flag.
struct NetStem {
    const __nv_bfloat16* w1;
    const float* b1;
    const __nv_bfloat16* w2;
    const float* b2;
    __nv_bfloat16* a2;
    int* err;
};
NetStem net_stem_operands(drwc_net* n);

}  // namespace drwc
