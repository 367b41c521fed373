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
// The scratch array (kNoAllocScratchBytes) is part of the loaded module, so
// every GPU that loads the library holds it until the process exits. All
// calls share it: it keeps the last call's contents (the solver overwrites
// every value it reads before reading it, so nothing needs clearing), and
// calls that overlap on the GPU — on different streams, or from several host
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
        cube_solve<N>(EpsGlobal{e}, ys, ss, cd, prm, &st);
        double* o = out + (size_t)c * 6 * D::NN;
        if (st.status == 2) {
            for (int b = threadIdx.x; b < 6 * D::NN; b += blockDim.x) o[b] = 0.0;
        } else {
            for_each_panel<N>(EpsGlobal{e}, ys, [&](int b, double v) { o[b] = v; });
        }
        if (threadIdx.x == 0) {
            if (iters) iters[c] = st.iters;
            if (status) status[c] = st.status;
        }
        __syncthreads();
    }
}

// Per-device set-up, done once by the first call on that device: the device
// address of the scratch array and, per N, the kernel's shared-memory limit
// and its resident CTAs per SM.
struct NoAllocDevice {
    bool ready = false;
    unsigned char* scratch = nullptr;
    int per_sm[DRWC_N_MAX + 1] = {0};
};
constexpr int kMaxDevices = 64;
static NoAllocDevice g_noalloc_dev[kMaxDevices];
static std::mutex g_noalloc_mu;

static int noalloc_setup(int device, NoAllocDevice** out) {
    if (device < 0 || device >= kMaxDevices) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[device];
    if (!d.ready) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            std::fprintf(stderr, "drwc: cudaGetSymbolAddress(no-alloc scratch) failed: %s\n",
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
                return DRWC_OK;
            });
            if (rc) return rc;
        }
        d.scratch = static_cast<unsigned char*>(p);
        d.ready = true;
    }
    *out = &d;
    return DRWC_OK;
}

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
    int rc = noalloc_setup(ctx->device, &d);
    if (rc) return rc;
    const size_t fit = kNoAllocScratchBytes / slot;
    size_t grid = (size_t)d->per_sm[N] * ctx->sm_count;
    if (grid > fit) grid = fit;
    if (grid > (size_t)ncubes) grid = (size_t)ncubes;
    return dispatch_N(N, [&](auto nc) -> int {
        constexpr int NC = decltype(nc)::value;
        using Dm = Cube<NC>;
        fdm_noalloc_kernel<NC><<<(int)grid, Dm::NT, Dm::kSmemBytes, ctx->stream>>>(
            ncubes, eps, code, out, iters, status, make_params(opts, NC), d->scratch);
        return launch_check(ctx);
    });
}

}  // extern "C"
