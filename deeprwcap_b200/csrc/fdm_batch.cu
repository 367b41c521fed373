// Batched FDM surface Green's functions: the ggft replacement.
//
//   drwc_ggft_solve              ggft_solver::solve + gft (ggft_solver.cpp:521-636)
//   drwc_fdm_solve_batch[_device] many cubes of mixed N in one call
//
// One persistent CTA per SM slot walks the cubes of one resolution; cubes are
// grouped by N on the host (one launch per N present) because the
// register-resident columns are compiled per N.
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "fdm_cube.cuh"
#include "host.cuh"

namespace drwc {

// Per-cube input is FP64 permittivity in global memory, read by the set-up
// passes of cube_solve and by its FP64 residual sweeps.
template <int N>
__global__ void __launch_bounds__(Cube<N>::NT, CubeTraits<N>::kMinBlocks)
fdm_batch_kernel(int nsel, const int32_t* __restrict__ sel, const double* __restrict__ eps,
                 const int64_t* __restrict__ eps_off, const int32_t* __restrict__ code,
                 const int64_t* __restrict__ out_off, double* __restrict__ out,
                 int32_t* __restrict__ iters, int32_t* __restrict__ sweeps,
                 double* __restrict__ relres, int32_t* __restrict__ status, FdmParams prm,
                 double* __restrict__ scratch_y,
                 float* __restrict__ scratch_s) {
    extern __shared__ __align__(128) unsigned char drwc_dyn_smem[];
    unsigned char* smem = drwc_dyn_smem;
    using D = Cube<N>;
    const CubeSmem<N> sm = CubeSmem<N>::carve(smem);
    double* ys = scratch_y + (size_t)blockIdx.x * D::NNN;
    float* ss = scratch_s + (size_t)blockIdx.x * D::NNN;
    for (int q = blockIdx.x; q < nsel; q += gridDim.x) {
        const int c = sel[q];
        const double* e = eps + eps_off[c];
        const int cd = code ? code[c] : DRWC_GFT;
        FdmStats st;
        if (planar_cube<N>(e))  // one permittivity per z plane: the per-plane solver
            cube_solve_planar<N>(EpsGlobalPlanar<N>{e}, ys, cd, prm, &st);
        else
            cube_solve<N>(EpsGlobal{e}, ys, ss, cd, prm, &st);
        double* o = out + out_off[c];
        if (st.status == 2) {
            for (int b = threadIdx.x; b < 6 * D::NN; b += blockDim.x) o[b] = 0.0;
        } else {
            for_each_panel<N>(EpsGlobal{e}, cube_y<N>(ys), [&](int b, double v) { o[b] = v; });
        }
        if (threadIdx.x == 0) {
            if (iters) iters[c] = st.iters;
            if (sweeps) sweeps[c] = st.sweeps;
            if (relres) relres[c] = st.relres;
            if (status) status[c] = st.status;
        }
        __syncthreads();
    }
}

struct LaunchShape {
    int grid_per_sm = 0;
};

template <int N>
static int fdm_shape(LaunchShape* s) {
    static LaunchShape cached;
    static bool init = false;
    if (!init) {
        using D = Cube<N>;
        DRWC_CUDA_TRY(cudaFuncSetAttribute(fdm_batch_kernel<N>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)D::kSmemBytes));
        int nb = 0;
        DRWC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fdm_batch_kernel<N>,
                                                                    D::NT, D::kSmemBytes));
        cached.grid_per_sm = nb < 1 ? 1 : nb;
        init = true;
    }
    *s = cached;
    return DRWC_OK;
}

FdmParams make_params(const drwc_fdm_opts* o, int N) {
    drwc_fdm_opts d;
    drwc_fdm_opts_default(&d);
    if (!o) o = &d;
    FdmParams p;
    p.tol = o->tol > 0 ? o->tol : d.tol;
    p.inner_tol = (float)(o->inner_tol > 0 ? o->inner_tol : d.inner_tol);
    p.max_outer = o->max_outer > 0 ? o->max_outer : d.max_outer;
    p.max_inner = o->max_inner > 0 ? o->max_inner : 4 * N * N;
    p.extra_outer = o->extra_outer > 0 ? o->extra_outer : 0;
    for (int c = 0; c < 4; ++c) p.warm[c] = nullptr;  // set by the caller (warm_tables)
    return p;
}

}  // namespace drwc

using namespace drwc;

extern "C" {

DRWC_API void drwc_fdm_opts_default(drwc_fdm_opts* opts) {
    if (!opts) return;
    opts->tol = 1e-10;
    opts->inner_tol = 1e-5;
    opts->max_outer = 8;
    opts->max_inner = 0;
    opts->warm_start = 1;
    opts->extra_outer = 8;
}

DRWC_API int drwc_fdm_solve_batch_device(drwc_ctx* ctx, int ncubes, const int32_t* N,
                                         const int64_t* eps_off, const double* eps,
                                         const int32_t* code, const drwc_fdm_opts* opts,
                                         const int64_t* out_off, double* out, int32_t* iters,
                                         int32_t* sweeps, double* relres, int32_t* status) {
    if (!ctx || ncubes < 0 || (ncubes > 0 && (!N || !eps_off || !eps || !out_off || !out)))
        return DRWC_ERR_INVALID;
    if (ncubes == 0) return DRWC_OK;
    for (int c = 0; c < ncubes; ++c) {
        if (!n_supported(N[c])) return DRWC_ERR_INVALID;
        if (code && (code[c] < DRWC_GFT || code[c] > DRWC_WVTY)) return DRWC_ERR_INVALID;
        if (eps_off[c] < 0 || out_off[c] < 0) return DRWC_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    // Group cubes by N; upload selection lists, offsets and codes.
    std::vector<int32_t> order(ncubes);
    for (int c = 0; c < ncubes; ++c) order[c] = c;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return N[a] < N[b]; });
    const size_t meta_bytes = sizeof(int32_t) * ncubes * 2 + sizeof(int64_t) * ncubes * 2;
    void* meta = nullptr;
    int rc = ws_get(ctx, WS_AUX, meta_bytes, &meta);
    if (rc) return rc;
    int64_t* d_eoff = (int64_t*)meta;
    int64_t* d_ooff = d_eoff + ncubes;
    int32_t* d_sel = (int32_t*)(d_ooff + ncubes);
    int32_t* d_code = d_sel + ncubes;
    // Pageable source: the copy is staged before cudaMemcpyAsync returns, so the
    // vector may go away while the transfer is still queued on the stream.
    std::vector<unsigned char> hmeta(meta_bytes);
    std::memcpy(hmeta.data(), eps_off, sizeof(int64_t) * ncubes);
    std::memcpy(hmeta.data() + sizeof(int64_t) * ncubes, out_off, sizeof(int64_t) * ncubes);
    std::memcpy(hmeta.data() + sizeof(int64_t) * 2 * ncubes, order.data(), sizeof(int32_t) * ncubes);
    if (code)
        std::memcpy(hmeta.data() + sizeof(int64_t) * 2 * ncubes + sizeof(int32_t) * ncubes, code,
                    sizeof(int32_t) * ncubes);
    DRWC_CUDA_TRY(cudaMemcpyAsync(meta, hmeta.data(), meta_bytes, cudaMemcpyHostToDevice,
                                  ctx->stream));
    // scratch: per resident CTA one cube of y (FP64) and S (FP32)
    size_t scratch_need = 0;
    struct Group { int n, first, count; };
    std::vector<Group> groups;
    for (int a = 0; a < ncubes;) {
        int b = a;
        while (b < ncubes && N[order[b]] == N[order[a]]) ++b;
        groups.push_back({N[order[a]], a, b - a});
        a = b;
    }
    for (auto& g : groups) {
        LaunchShape sh;
        rc = dispatch_N(g.n, [&](auto nc) { return fdm_shape<decltype(nc)::value>(&sh); });
        if (rc) return rc;
        const size_t grid = std::min<size_t>(g.count, (size_t)sh.grid_per_sm * ctx->sm_count);
        scratch_need = std::max(scratch_need, grid * (size_t)g.n * g.n * g.n * 12);
    }
    void* scratch = nullptr;
    rc = ws_get(ctx, WS_SCRATCH, scratch_need, &scratch);
    if (rc) return rc;
    for (auto& g : groups) {
        rc = dispatch_N(g.n, [&](auto nc) -> int {
            constexpr int NC = decltype(nc)::value;
            using D = Cube<NC>;
            LaunchShape sh;
            int r2 = fdm_shape<NC>(&sh);
            if (r2) return r2;
            const int grid = (int)std::min<size_t>(g.count, (size_t)sh.grid_per_sm * ctx->sm_count);
            double* sy = (double*)scratch;
            float* sf = (float*)(sy + (size_t)grid * D::NNN);
            FdmParams prm = make_params(opts, NC);
            if (!opts || opts->warm_start) {
                const int rw = warm_tables(ctx, NC, prm.warm);
                if (rw) return rw;
            }
            fdm_batch_kernel<NC><<<grid, D::NT, D::kSmemBytes, ctx->stream>>>(
                g.count, d_sel + g.first, eps, d_eoff, code ? d_code : nullptr, d_ooff, out,
                iters, sweeps, relres, status, prm, sy, sf);
            return launch_check(ctx);
        });
        if (rc) return rc;
    }
    return DRWC_OK;
}

DRWC_API int drwc_fdm_solve_batch(drwc_ctx* ctx, int ncubes, const int32_t* N,
                                  const int64_t* eps_off, const double* eps, const int32_t* code,
                                  const drwc_fdm_opts* opts, const int64_t* out_off, double* out,
                                  int32_t* iters, double* relres, int32_t* status) {
    if (!ctx || ncubes < 0 || (ncubes > 0 && (!N || !eps_off || !eps || !out_off || !out)))
        return DRWC_ERR_INVALID;
    if (ncubes == 0) return DRWC_OK;
    size_t ein = 0, oout = 0;
    for (int c = 0; c < ncubes; ++c) {
        if (!n_supported(N[c])) return DRWC_ERR_INVALID;
        ein = std::max<size_t>(ein, eps_off[c] + (size_t)N[c] * N[c] * N[c]);
        oout = std::max<size_t>(oout, out_off[c] + (size_t)6 * N[c] * N[c]);
    }
    void *d_in = nullptr, *d_out = nullptr, *d_res = nullptr;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
        int rc = ws_get(ctx, WS_IN, ein * sizeof(double), &d_in);
        if (rc) return rc;
        rc = ws_get(ctx, WS_OUT, oout * sizeof(double), &d_out);
        if (rc) return rc;
        rc = ws_get(ctx, WS_RES, (size_t)ncubes * 16, &d_res);
        if (rc) return rc;
        DRWC_CUDA_TRY(cudaMemcpyAsync(d_in, eps, ein * sizeof(double), cudaMemcpyHostToDevice,
                                      ctx->stream));
    }
    // [relres: ncubes doubles][iters: ncubes int32][status: ncubes int32]
    double* d_rr = (double*)d_res;
    int32_t* d_it = (int32_t*)(d_rr + ncubes);
    int32_t* d_st = d_it + ncubes;
    int rc = drwc_fdm_solve_batch_device(ctx, ncubes, N, eps_off, (const double*)d_in, code, opts,
                                         out_off, (double*)d_out, d_it, nullptr, d_rr, d_st);
    if (rc) return rc;
    std::vector<int32_t> st(ncubes);
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        DRWC_CUDA_TRY(cudaMemcpyAsync(out, d_out, oout * sizeof(double), cudaMemcpyDeviceToHost,
                                      ctx->stream));
        DRWC_CUDA_TRY(cudaMemcpyAsync(st.data(), d_st, ncubes * sizeof(int32_t),
                                      cudaMemcpyDeviceToHost, ctx->stream));
        if (iters)
            DRWC_CUDA_TRY(cudaMemcpyAsync(iters, d_it, ncubes * sizeof(int32_t),
                                          cudaMemcpyDeviceToHost, ctx->stream));
        if (relres)
            DRWC_CUDA_TRY(cudaMemcpyAsync(relres, d_rr, ncubes * sizeof(double),
                                          cudaMemcpyDeviceToHost, ctx->stream));
        DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    if (status) std::memcpy(status, st.data(), ncubes * sizeof(int32_t));
    for (int c = 0; c < ncubes; ++c)
        if (st[c] != 0) return DRWC_ERR_NOT_CONVERGED;
    return DRWC_OK;
}

DRWC_API int drwc_ggft_solve(drwc_ctx* ctx, int N, const double* eps, int code, double tol,
                             double* gft_out, int32_t* iters_out) {
    if (!ctx || !eps || !gft_out || !n_supported(N) || code < DRWC_GFT || code > DRWC_WVTY)
        return DRWC_ERR_INVALID;
    drwc_fdm_opts o;
    drwc_fdm_opts_default(&o);
    if (tol > 0) o.tol = tol;
    const int32_t n = N, cd = code;
    const int64_t zero = 0;
    return drwc_fdm_solve_batch(ctx, 1, &n, &zero, eps, &cd, &o, &zero, gft_out, iters_out,
                                nullptr, nullptr);
}

}  // extern "C"
