// Host-side plumbing shared by the entry points: the context, device
// workspaces that grow on demand, error handling and launch accounting.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <vector>

#include "../../include/drwc.h"

struct drwc_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;                       // one call at a time per context
    std::atomic<int64_t> launches{0};    // kernels launched by this context
    // grow-only device workspaces
    void* ws[8] = {nullptr};
    size_t ws_bytes[8] = {0};
    // pinned host staging
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // uniform-permittivity solutions per N and solver code (warm starts)
    double* warm[DRWC_N_MAX + 1][4] = {};
};

namespace drwc {

enum Workspace { WS_SCRATCH = 0, WS_IN = 1, WS_OUT = 2, WS_AUX = 3, WS_AUX2 = 4, WS_RES = 5 };

#define DRWC_CUDA_TRY(expr)                                                       \
    do {                                                                          \
        cudaError_t e_ = (expr);                                                  \
        if (e_ != cudaSuccess) {                                                  \
            std::fprintf(stderr, "drwc: %s failed: %s (%s:%d)\n", #expr,         \
                         cudaGetErrorString(e_), __FILE__, __LINE__);             \
            return DRWC_ERR_CUDA;                                                 \
        }                                                                         \
    } while (0)

inline int ws_get(drwc_ctx* ctx, int slot, size_t bytes, void** out) {
    if (ctx->ws_bytes[slot] < bytes) {
        if (ctx->ws[slot]) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ctx->ws[slot]);
            ctx->ws[slot] = nullptr;
            ctx->ws_bytes[slot] = 0;
        }
        size_t want = bytes < 4096 ? 4096 : bytes + bytes / 4;
        if (cudaMalloc(&ctx->ws[slot], want) != cudaSuccess) {
            cudaGetLastError();
            return DRWC_ERR_NOMEM;
        }
        ctx->ws_bytes[slot] = want;
    }
    *out = ctx->ws[slot];
    return DRWC_OK;
}

inline int pinned_get(drwc_ctx* ctx, size_t bytes, void** out) {
    if (ctx->pinned_bytes < bytes) {
        if (ctx->pinned) {
            cudaStreamSynchronize(ctx->stream);
            cudaFreeHost(ctx->pinned);
            ctx->pinned = nullptr;
            ctx->pinned_bytes = 0;
        }
        size_t want = bytes < 65536 ? 65536 : bytes + bytes / 4;
        if (cudaMallocHost(&ctx->pinned, want) != cudaSuccess) {
            cudaGetLastError();
            return DRWC_ERR_NOMEM;
        }
        ctx->pinned_bytes = want;
    }
    *out = ctx->pinned;
    return DRWC_OK;
}

inline int launch_check(drwc_ctx* ctx) {
    ctx->launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "drwc: kernel launch failed: %s\n", cudaGetErrorString(e));
        return DRWC_ERR_CUDA;
    }
    return DRWC_OK;
}

inline bool n_supported(int N) { return N >= DRWC_N_MIN && N <= DRWC_N_MAX; }

// Fills warm[0..3] with the context's uniform-permittivity solutions for N
// (computed on the device the first time they are asked for). warm.cu.
int warm_tables(drwc_ctx* ctx, int N, const double* warm[4]);

// Calls f(std::integral_constant<int, N>) for a runtime N in the supported set.
template <class F>
inline int dispatch_N(int N, F&& f) {
    switch (N) {
#define DRWC_CASE(n) case n: return f(std::integral_constant<int, n>{});
        DRWC_CASE(4) DRWC_CASE(5) DRWC_CASE(6) DRWC_CASE(7) DRWC_CASE(8) DRWC_CASE(9)
        DRWC_CASE(10) DRWC_CASE(11) DRWC_CASE(12) DRWC_CASE(13) DRWC_CASE(14) DRWC_CASE(15)
        DRWC_CASE(16) DRWC_CASE(17) DRWC_CASE(18) DRWC_CASE(19) DRWC_CASE(20) DRWC_CASE(21)
        DRWC_CASE(22) DRWC_CASE(23)
#undef DRWC_CASE
        default: return DRWC_ERR_INVALID;
    }
}

}  // namespace drwc
