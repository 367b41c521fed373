// Warm starts: the uniform-permittivity solution of each cube resolution and
// solver code, solved once per context on the device. ggft does the same in
// its constructor (bootstrap_solve, ggft_solver.cpp:83-135) and starts every
// later solve from it (solveWithGuess, :554-560); a cube whose permittivity
// is uniform then converges at the first residual check.
#include <type_traits>

#include "fdm_cube.cuh"
#include "host.cuh"

namespace drwc {

// One CTA per code; writes x = eps .* y (= y, eps = 1) into out[code].
template <int N>
__global__ void __launch_bounds__(Cube<N>::NT)
uniform_kernel(double* __restrict__ out0, double* __restrict__ out1, double* __restrict__ out2,
               double* __restrict__ out3, float* __restrict__ scratch_s, FdmParams prm) {
    double* outs[4] = {out0, out1, out2, out3};
    const int code = blockIdx.x;
    FdmStats st;
    cube_solve<N>(EpsUniform{}, outs[code], scratch_s + (size_t)code * Cube<N>::NNN, code, prm,
                  &st);
    if constexpr (Cube<N>::YSMEM) {  // the solution is in shared memory
        const double* y = cube_y<N>(outs[code]);
        for (int c = threadIdx.x; c < Cube<N>::NNN; c += blockDim.x) outs[code][c] = y[c];
    }
}

int warm_tables(drwc_ctx* ctx, int N, const double* warm[4]) {
    if (!n_supported(N)) return DRWC_ERR_INVALID;
    if (!ctx->warm[N][0]) {
        const size_t nnn = (size_t)N * N * N;
        double* t[4] = {nullptr, nullptr, nullptr, nullptr};
        float* sscr = nullptr;
        for (int c = 0; c < 4; ++c)
            if (cudaMalloc(&t[c], nnn * sizeof(double)) != cudaSuccess) {
                cudaGetLastError();
                for (int d = 0; d < 4; ++d) if (t[d]) cudaFree(t[d]);
                return DRWC_ERR_NOMEM;
            }
        if (cudaMalloc(&sscr, 4 * nnn * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            for (int d = 0; d < 4; ++d) cudaFree(t[d]);
            return DRWC_ERR_NOMEM;
        }
        const int rc = dispatch_N(N, [&](auto nc) -> int {
            constexpr int NC = decltype(nc)::value;
            using D = Cube<NC>;
            DRWC_CUDA_TRY(cudaFuncSetAttribute(uniform_kernel<NC>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)D::kSmemBytes));
            FdmParams prm{};
            prm.tol = 1e-13;
            prm.inner_tol = 1e-6f;
            prm.max_outer = 12;
            prm.max_inner = 8 * NC * NC;
            uniform_kernel<NC><<<4, D::NT, D::kSmemBytes, ctx->stream>>>(t[0], t[1], t[2], t[3],
                                                                       sscr, prm);
            return launch_check(ctx);
        });
        cudaStreamSynchronize(ctx->stream);
        cudaFree(sscr);
        if (rc) {
            for (int d = 0; d < 4; ++d) cudaFree(t[d]);
            return rc;
        }
        for (int c = 0; c < 4; ++c) ctx->warm[N][c] = t[c];
    }
    for (int c = 0; c < 4; ++c) warm[c] = ctx->warm[N][c];
    return DRWC_OK;
}

}  // namespace drwc
