// Library identity, status strings and the per-device context.
#include <cstring>

#include "host.cuh"

namespace drwc {
int noalloc_prepare(drwc_ctx* ctx);  // fdm_noalloc.cu
}

extern "C" {

DRWC_API const char* drwc_version(void) { return "deeprwcap-b200 0.1.0 (sm_100a)"; }

DRWC_API const char* drwc_status_string(int s) {
    switch (s) {
        case DRWC_OK: return "ok";
        case DRWC_ERR_INVALID: return "invalid argument";
        case DRWC_ERR_CUDA: return "CUDA runtime error";
        case DRWC_ERR_NOMEM: return "out of memory";
        case DRWC_ERR_NOT_CONVERGED: return "solve did not converge";
        case DRWC_ERR_NO_DEVICE: return "no usable sm_100 device";
        case DRWC_ERR_TIMEOUT: return "bounded wait ran out";
        case DRWC_ERR_SHUTDOWN: return "shutting down";
        case DRWC_ERR_GEOMETRY: return "structure rejected";
        default: return "unknown status";
    }
}

DRWC_API int drwc_ctx_create(int device, drwc_ctx** out) {
    if (!out) return DRWC_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return DRWC_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    DRWC_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return DRWC_ERR_NO_DEVICE;  // kernels are built for sm_100a only
    DRWC_CUDA_TRY(cudaSetDevice(device));
    drwc_ctx* c = new drwc_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return DRWC_ERR_CUDA;
    }
    // the no-allocation solver's static arrays, set up here rather than in
    // its first call (once per device)
    const int rc = drwc::noalloc_prepare(c);
    if (rc) {
        cudaStreamDestroy(c->stream);
        delete c;
        return rc;
    }
    *out = c;
    return DRWC_OK;
}

DRWC_API int drwc_ctx_destroy(drwc_ctx* ctx) {
    if (!ctx) return DRWC_ERR_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < 8; ++i)
        if (ctx->ws[i]) cudaFree(ctx->ws[i]);
    for (int n = 0; n <= DRWC_N_MAX; ++n)
        for (int c = 0; c < 4; ++c)
            if (ctx->warm[n][c]) cudaFree(ctx->warm[n][c]);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return DRWC_OK;
}

DRWC_API int drwc_ctx_stream(drwc_ctx* ctx, void** stream_out) {
    if (!ctx || !stream_out) return DRWC_ERR_INVALID;
    *stream_out = (void*)ctx->stream;
    return DRWC_OK;
}

DRWC_API int drwc_ctx_synchronize(drwc_ctx* ctx) {
    if (!ctx) return DRWC_ERR_INVALID;
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return DRWC_OK;
}

DRWC_API int drwc_ctx_launch_count(drwc_ctx* ctx, int64_t* count_out) {
    if (!ctx || !count_out) return DRWC_ERR_INVALID;
    *count_out = ctx->launches.load();
    return DRWC_OK;
}

}  // extern "C"
