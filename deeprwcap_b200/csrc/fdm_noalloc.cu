// Batched FDM surface Green's functions without any device allocation.
//
// Some callers cannot allocate device memory when they call us: a host
// application that hands all GPU memory to its own pool at start-up and
// forbids driver allocations afterwards, or a latency-critical loop where a
// cudaMalloc (which may synchronise the device) is not allowed. For them,
// drwc_fdm_solve_noalloc solves a batch of same-N cubes using only the
// caller's input/output buffers plus a fixed scratch area that lives in this
// file as a statically sized __device__ array: the library allocates nothing
// per call (no cudaMalloc / cudaFree, no pinned or pooled memory).
//
// The scratch array (kNoAllocScratchBytes) and the warm-start tables beside
// it (kNoAllocWarmDoubles) are part of the loaded module, so every GPU that
// loads the library holds them until the process exits. The module is loaded
// and both arrays are set up when a context is created on the device
// (drwc_ctx_create calls noalloc_prepare), not inside a solve: a caller that
// creates its context before handing the GPU's memory to its own pool never
// has this entry point allocate or load anything later. All calls share the
// scratch: it keeps the last call's contents (the solver overwrites every
// value it reads before reading it, so nothing needs clearing), and calls
// that overlap on the GPU — on different streams, or from several host
// threads on one device — race on it. Issue them on one stream.
#include <mutex>
#include <type_traits>

#include "fdm_cube.cuh"
#include "host.cuh"

namespace drwc {

FdmParams make_params(const drwc_fdm_opts* o, int N);

// 16 MiB: per resident CTA the solver needs 12 bytes per cell (FP64 y and
// FP32 Jacobi scale), so N = 16 fits 341 CTAs (more than the 296 that are
// resident) and N = 23 fits 114.
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Warm starts (the uniform-permittivity solution per N and solver code, as
// the regular entry points use): 4 * N^3 doubles for every N in
// [DRWC_N_MIN, DRWC_N_MAX], 2.4 MB in all, solved once per device at set-up.
constexpr size_t warm_offset(int N) {  // doubles before resolution N's tables
    size_t o = 0;
    for (int n = DRWC_N_MIN; n < N; ++n) o += 4 * (size_t)n * n * n;
    return o;
}
constexpr size_t kNoAllocWarmDoubles = warm_offset(DRWC_N_MAX + 1);
static __device__ __align__(256) double g_noalloc_warm[kNoAllocWarmDoubles];

// One CTA per solver code: the uniform-permittivity solve (the same solve,
// with the same parameters, as the per-context warm tables of warm.cu).
template <int N>
__global__ void __launch_bounds__(Cube<N>::NT)
noalloc_uniform_kernel(double* __restrict__ warm, float* __restrict__ scratch_s, FdmParams prm) {
    const int code = blockIdx.x;
    double* out = warm + (size_t)code * Cube<N>::NNN;
    FdmStats st;
    cube_solve<N>(EpsUniform{}, out, scratch_s + (size_t)code * Cube<N>::NNN, code, prm, &st);
    if constexpr (Cube<N>::YSMEM) {
        const double* y = cube_y<N>(out);
        for (int c = threadIdx.x; c < Cube<N>::NNN; c += blockDim.x) out[c] = y[c];
    }
}

// Cube c reads eps + c*N^3 and writes out + c*6N^2 (packed, same N).
template <int N>
__global__ void __launch_bounds__(Cube<N>::NT)
fdm_noalloc_kernel(int ncubes, const double* __restrict__ eps, const int32_t* __restrict__ code,
                   double* __restrict__ out, int32_t* __restrict__ iters,
                   int32_t* __restrict__ status, FdmParams prm,
                   unsigned char* __restrict__ scratch) {
    extern __shared__ __align__(128) unsigned char drwc_dyn_smem[];
    unsigned char* smem = drwc_dyn_smem;
    using D = Cube<N>;
    const CubeSmem<N> sm = CubeSmem<N>::carve(smem);
    double* ys = reinterpret_cast<double*>(scratch) + (size_t)blockIdx.x * D::NNN;
    float* ss = reinterpret_cast<float*>(scratch + (size_t)gridDim.x * D::NNN * sizeof(double)) +
                (size_t)blockIdx.x * D::NNN;
    for (int c = blockIdx.x; c < ncubes; c += gridDim.x) {
        const double* e = eps + (size_t)c * D::NNN;
        const int cd = code ? code[c] : DRWC_GFT;
        FdmStats st;
        if (cd < DRWC_GFT || cd > DRWC_WVTY) {  // not a solver code: status 2, zero rows
            st.status = 2; st.iters = 0; st.sweeps = 0; st.relres = CUDART_NAN;
            st.escalated = 0;
        } else if (planar_cube<N>(e)) {  // one permittivity per z plane
            cube_solve_planar<N>(EpsGlobalPlanar<N>{e}, ys, cd, prm, &st);
        } else {
            cube_solve<N>(EpsGlobal{e}, ys, ss, cd, prm, &st);
        }
        double* o = out + (size_t)c * 6 * D::NN;
        if (st.status == 2) {
            for (int b = threadIdx.x; b < 6 * D::NN; b += blockDim.x) o[b] = 0.0;
        } else {
            for_each_panel<N>(EpsGlobal{e}, cube_y<N>(ys), [&](int b, double v) { o[b] = v; });
        }
        if (threadIdx.x == 0) {
            if (iters) iters[c] = st.iters;
            if (status) status[c] = st.status;
        }
        __syncthreads();
    }
}

// Per-device set-up, done once per device when the first context on it is
// created: the device addresses of the scratch and warm-table arrays and, per
// N, the kernel's shared-memory limit, its resident CTAs per SM and the warm
// tables.
struct NoAllocDevice {
    bool ready = false;
    unsigned char* scratch = nullptr;
    double* warm = nullptr;
    int per_sm[DRWC_N_MAX + 1] = {0};
};
constexpr int kMaxDevices = 64;
static NoAllocDevice g_noalloc_dev[kMaxDevices];
static std::mutex g_noalloc_mu;

// Set-up for ctx's device, once per device (ctx's device is current).
static int noalloc_setup(drwc_ctx* ctx, NoAllocDevice** out) {
    const int device = ctx->device;
    if (device < 0 || device >= kMaxDevices) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[device];
    if (!d.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            std::fprintf(stderr, "drwc: cudaGetSymbolAddress(no-alloc scratch) failed: %s\n",
                         cudaGetErrorString(e));
            cudaGetLastError();
            return DRWC_ERR_CUDA;
        }
        void* pw = nullptr;
        e = cudaGetSymbolAddress(&pw, g_noalloc_warm);
        if (e != cudaSuccess || pw == nullptr) {
            std::fprintf(stderr, "drwc: cudaGetSymbolAddress(no-alloc warm tables) failed: %s\n",
                         cudaGetErrorString(e));
            cudaGetLastError();
            return DRWC_ERR_CUDA;
        }
        for (int n = DRWC_N_MIN; n <= DRWC_N_MAX; ++n) {
            const int rc = dispatch_N(n, [&](auto nc) -> int {
                constexpr int NC = decltype(nc)::value;
                using Dm = Cube<NC>;
                DRWC_CUDA_TRY(cudaFuncSetAttribute(fdm_noalloc_kernel<NC>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)Dm::kSmemBytes));
                int nb = 0;
                DRWC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &nb, fdm_noalloc_kernel<NC>, Dm::NT, Dm::kSmemBytes));
                d.per_sm[NC] = nb < 1 ? 1 : nb;
                // warm-start tables of this N (scratch: the Jacobi scales)
                DRWC_CUDA_TRY(cudaFuncSetAttribute(noalloc_uniform_kernel<NC>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)Dm::kSmemBytes));
                FdmParams prm{};
                prm.tol = 1e-13;
                prm.inner_tol = 1e-6f;
                prm.max_outer = 12;
                prm.max_inner = 8 * NC * NC;
                noalloc_uniform_kernel<NC><<<4, Dm::NT, Dm::kSmemBytes, ctx->stream>>>(
                    static_cast<double*>(pw) + warm_offset(NC), static_cast<float*>(p), prm);
                int rc2 = launch_check(ctx);
                if (rc2) return rc2;
                // one launch with no cubes, so that the driver sizes the
                // kernel's local memory now and not in a later solve
                fdm_noalloc_kernel<NC><<<1, Dm::NT, Dm::kSmemBytes, ctx->stream>>>(
                    0, nullptr, nullptr, nullptr, nullptr, nullptr, prm,
                    static_cast<unsigned char*>(p));
                return launch_check(ctx);
            });
            if (rc) return rc;
        }
        DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        d.scratch = static_cast<unsigned char*>(p);
        d.warm = static_cast<double*>(pw);
        d.ready = true;
    }
    if (out) *out = &d;
    return DRWC_OK;
}

int noalloc_prepare(drwc_ctx* ctx) { return noalloc_setup(ctx, nullptr); }

}  // namespace drwc

using namespace drwc;

extern "C" {

DRWC_API int drwc_fdm_solve_noalloc(drwc_ctx* ctx, int N, int ncubes, const double* eps,
                                    const int32_t* code, const drwc_fdm_opts* opts, double* out,
                                    int32_t* iters, int32_t* status) {
    if (!ctx || ncubes < 0) return DRWC_ERR_INVALID;
    if (!n_supported(N)) {
        std::fprintf(stderr, "drwc_fdm_solve_noalloc: N=%d outside [%d, %d]\n", N, DRWC_N_MIN,
                     DRWC_N_MAX);
        return DRWC_ERR_INVALID;
    }
    const size_t slot = (size_t)N * N * N * (sizeof(double) + sizeof(float));
    if (slot > kNoAllocScratchBytes) {
        std::fprintf(stderr,
                     "drwc_fdm_solve_noalloc: one cube of N=%d needs %zu scratch bytes, more "
                     "than the %zu-byte static scratch\n", N, slot, kNoAllocScratchBytes);
        return DRWC_ERR_INVALID;
    }
    if (ncubes == 0) return DRWC_OK;
    if (!eps || !out) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    NoAllocDevice* d = nullptr;
    int rc = noalloc_setup(ctx, &d);  // done already when the context was created
    if (rc) return rc;
    const size_t fit = kNoAllocScratchBytes / slot;
    size_t grid = (size_t)d->per_sm[N] * ctx->sm_count;
    if (grid > fit) grid = fit;
    if (grid > (size_t)ncubes) grid = (size_t)ncubes;
    return dispatch_N(N, [&](auto nc) -> int {
        constexpr int NC = decltype(nc)::value;
        using Dm = Cube<NC>;
        FdmParams prm = make_params(opts, NC);
        if (!opts || opts->warm_start)
            for (int c = 0; c < 4; ++c) prm.warm[c] = d->warm + warm_offset(NC) + c * Dm::NNN;
        fdm_noalloc_kernel<NC><<<(int)grid, Dm::NT, Dm::kSmemBytes, ctx->stream>>>(
            ncubes, eps, code, out, iters, status, prm, d->scratch);
        return launch_check(ctx);
    });
}

}  // extern "C"
