// dnnsolver drop-ins: structureConstruction, DNNSolverPoisson::sample and
// DNNSolverGrad::sample (inference_cpp/src/dnn_solver*.cpp), with the FDM
// surface Green's function in place of the TensorRT networks.
//
// One CTA per query: the query's 15 layers / 15 cuboids are staged in shared
// memory, the cube is voxelised with the reference fill rule
// (cuda_kernels.cu:21-84: last layer with min_z <= z, first containing cuboid
// with inclusive bounds overrides, padding -9999 ends each list) after the
// per-query max normalisation (dnn_solver.cpp:274-285), the FDM system is
// solved on chip, and one panel is drawn from the surface values.
#include <cstring>
#include <type_traits>
#include <vector>

#include "fdm_cube.cuh"
#include "host.cuh"
#include "sample.cuh"

namespace drwc {

FdmParams make_params(const drwc_fdm_opts* o, int N);

constexpr int kL = DRWC_MAX_LAYERS, kC = DRWC_MAX_CUBOIDS;

// Stage a query, normalise by its max permittivity (float32, as ATen's amax
// + div_ in the reference); returns the max.
DRWC_DEV float stage_query(const float* __restrict__ layers, const float* __restrict__ cuboids,
                           int normalise, float* lay, float* cub) {
    const int t = threadIdx.x;
    for (int v = t; v < 2 * kL; v += blockDim.x) lay[v] = layers[v];
    for (int v = t; v < 7 * kC; v += blockDim.x) cub[v] = cuboids[v];
    __syncthreads();
    float m = lay[1];
    for (int l = 0; l < kL; ++l) m = fmaxf(m, lay[2 * l + 1]);
    for (int c = 0; c < kC; ++c) m = fmaxf(m, cub[7 * c + 6]);
    __syncthreads();
    if (normalise) {
        if (t < kL) lay[2 * t + 1] = lay[2 * t + 1] / m;
        if (t < kC) cub[7 * t + 6] = cub[7 * t + 6] / m;
    }
    __syncthreads();
    return m;
}

// fill_structure_kernel's per-voxel rule (cuda_kernels.cu:39-83), float32.
DRWC_DEV float fill_voxel(int N, int x, int y, int z, const float* lay, const float* cub) {
    const float xc = (2.0f * (float)x + 1.0f) / (float)N - 1.0f;
    const float yc = (2.0f * (float)y + 1.0f) / (float)N - 1.0f;
    const float zc = (2.0f * (float)z + 1.0f) / (float)N - 1.0f;
    int li = 0;
    for (int l = 0; l < kL; ++l) {
        const float mz = lay[2 * l];
        if (mz == DRWC_PADDING) break;
        if (zc >= mz) li = l;
        else break;
    }
    float val = lay[2 * li + 1];
    for (int c = 0; c < kC; ++c) {
        const float* q = cub + 7 * c;
        if (q[0] == DRWC_PADDING) break;
        if (xc >= q[0] && xc <= q[3] && yc >= q[1] && yc <= q[4] && zc >= q[2] && zc <= q[5]) {
            val = q[6];
            break;
        }
    }
    return val;
}

__global__ void structure_kernel(int n, int N, const float* __restrict__ layers,
                                 const float* __restrict__ cuboids, int normalise,
                                 float* __restrict__ eps_out, float* __restrict__ max_out) {
    __shared__ float lay[2 * kL], cub[7 * kC];
    const int NNN = N * N * N;
    for (int q = blockIdx.x; q < n; q += gridDim.x) {
        const float m = stage_query(layers + (size_t)q * 2 * kL, cuboids + (size_t)q * 7 * kC,
                                    normalise, lay, cub);
        if (threadIdx.x == 0 && max_out) max_out[q] = m;
        float* o = eps_out + (size_t)q * NNN;
        for (int c = threadIdx.x; c < NNN; c += blockDim.x)
            o[c] = fill_voxel(N, c % N, (c / N) % N, c / (N * N), lay, cub);
        __syncthreads();
    }
}

// GRAD = false: transition (GFT, sample by G, out 3 floats);
// GRAD = true:  first hop (WVT along axis, sample by |g|, out 5 floats).
template <int N, bool GRAD>
__global__ void __launch_bounds__(Cube<N>::NT)
query_kernel(int n, const float* __restrict__ layers, const float* __restrict__ cuboids,
             const int32_t* __restrict__ axis, uint64_t seed, uint64_t stream, FdmParams prm,
             double* __restrict__ scratch_e, double* __restrict__ scratch_y,
             float* __restrict__ scratch_s, float* __restrict__ out, int32_t* __restrict__ status) {
    extern __shared__ __align__(128) unsigned char drwc_dyn_smem[];
    unsigned char* smem = drwc_dyn_smem;
    __shared__ float lay[2 * kL], cub[7 * kC];
    using D = Cube<N>;
    const CubeSmem<N> sm = CubeSmem<N>::carve(smem);
    double* es = scratch_e + (size_t)blockIdx.x * D::NNN;
    double* ys = scratch_y + (size_t)blockIdx.x * D::NNN;
    float* ss = scratch_s + (size_t)blockIdx.x * D::NNN;
    constexpr int M = 6 * D::NN;
    constexpr int OUTW = GRAD ? 5 : 3;
    for (int q = blockIdx.x; q < n; q += gridDim.x) {
        const float m = stage_query(layers + (size_t)q * 2 * kL, cuboids + (size_t)q * 7 * kC, 1,
                                    lay, cub);
        for (int c = threadIdx.x; c < D::NNN; c += blockDim.x)
            es[c] = (double)fill_voxel(N, c % N, (c / N) % N, c / (N * N), lay, cub);
        __syncthreads();
        int code = DRWC_GFT;
        if (GRAD) {
            const int a = axis[q];
            code = a == 0 ? DRWC_WVTX : a == 1 ? DRWC_WVTY : DRWC_WVTZ;
        }
        FdmStats st;
        if (planar_cube<N>(es))  // no cuboid reaches a cell centre: the per-plane solver
            cube_solve_planar<N>(EpsGlobalPlanar<N>{es}, ys, code, prm, &st);
        else
            cube_solve<N>(EpsGlobal{es}, ys, ss, code, prm, &st);
        double* w = reinterpret_cast<double*>(sm.stage());  // 6N^2 doubles over p|cx|cy|cz
        for_each_panel<N>(EpsGlobal{es}, cube_y<N>(ys), [&](int b, double v) { w[b] = v; });
        __syncthreads();
        const double u = philox_uniform2(seed, stream + (uint64_t)q, 0, 0).x;
        double tot = 0.0;
        const int b = (st.status == 2) ? -1 : cta_sample<D::NT>(w, M, GRAD, u, sm.red, &tot);
        if (threadIdx.x == 0) {
            float* o = out + (size_t)q * OUTW;
            if (b < 0) {
                for (int v = 0; v < OUTW; ++v) o[v] = 0.f;
            } else {
                float pos[3];
                locate_f32(N, b, pos);
                o[0] = pos[0]; o[1] = pos[1]; o[2] = pos[2];
                if (GRAD) {
                    o[3] = (float)(w[b] < 0.0 ? -tot : tot);
                    o[4] = (float)(center_diel<N>(EpsGlobal{es}, code) * (double)m);
                }
            }
            if (status) status[q] = b < 0 ? 2 : st.status;
        }
        __syncthreads();
    }
}

template <int N, bool GRAD>
static int query_launch(drwc_ctx* ctx, int n, const float* d_lay, const float* d_cub,
                        const int32_t* d_axis, uint64_t seed, uint64_t stream, float* d_out,
                        int32_t* d_status) {
    using D = Cube<N>;
    static int per_sm = 0;
    if (!per_sm) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(query_kernel<N, GRAD>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)D::kSmemBytes));
        DRWC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, query_kernel<N, GRAD>, D::NT, D::kSmemBytes));
        if (per_sm < 1) per_sm = 1;
    }
    const int grid = std::min(n, per_sm * ctx->sm_count);
    void* scratch = nullptr;
    int rc = ws_get(ctx, WS_SCRATCH, (size_t)grid * D::NNN * 20, &scratch);
    if (rc) return rc;
    double* se = (double*)scratch;
    double* sy = se + (size_t)grid * D::NNN;
    float* sf = (float*)(sy + (size_t)grid * D::NNN);
    FdmParams prm = make_params(nullptr, N);
    rc = warm_tables(ctx, N, prm.warm);
    if (rc) return rc;
    query_kernel<N, GRAD><<<grid, D::NT, D::kSmemBytes, ctx->stream>>>(
        n, d_lay, d_cub, d_axis, seed, stream, prm, se, sy, sf, d_out, d_status);
    return launch_check(ctx);
}

// Shared body of the two sampling drop-ins (host buffers, synchronous).
static int query_batch(drwc_ctx* ctx, bool grad, int n, int N, const float* layers,
                       const float* cuboids, const int32_t* axis, uint64_t seed,
                       uint64_t stream, float* out) {
    if (!ctx || n < 0 || !n_supported(N)) return DRWC_ERR_INVALID;
    if (n == 0) return DRWC_OK;
    if (!layers || !cuboids || !out) return DRWC_ERR_INVALID;
    if (grad) {
        if (!axis) return DRWC_ERR_INVALID;  // dnn_solver_gradient.cpp:40-47
        for (int q = 0; q < n; ++q)
            if (axis[q] < 0 || axis[q] > 2) return DRWC_ERR_INVALID;
    }
    const int outw = grad ? 5 : 3;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t lay_b = sizeof(float) * n * 2 * kL, cub_b = sizeof(float) * n * 7 * kC;
    const size_t ax_b = grad ? sizeof(int32_t) * n : 0, out_b = sizeof(float) * n * outw,
                 st_b = sizeof(int32_t) * n;
    void *d_in = nullptr, *d_out = nullptr;
    int rc = ws_get(ctx, WS_IN, lay_b + cub_b + ax_b + 64, &d_in);
    if (rc) return rc;
    rc = ws_get(ctx, WS_OUT, out_b + st_b + 64, &d_out);
    if (rc) return rc;
    float* d_lay = (float*)d_in;
    float* d_cub = d_lay + (size_t)n * 2 * kL;
    int32_t* d_axis = (int32_t*)(d_cub + (size_t)n * 7 * kC);
    DRWC_CUDA_TRY(cudaMemcpyAsync(d_lay, layers, lay_b, cudaMemcpyHostToDevice, ctx->stream));
    DRWC_CUDA_TRY(cudaMemcpyAsync(d_cub, cuboids, cub_b, cudaMemcpyHostToDevice, ctx->stream));
    if (grad)
        DRWC_CUDA_TRY(cudaMemcpyAsync(d_axis, axis, ax_b, cudaMemcpyHostToDevice, ctx->stream));
    float* d_o = (float*)d_out;
    int32_t* d_st = (int32_t*)(d_o + (size_t)n * outw);
    rc = dispatch_N(N, [&](auto nc) -> int {
        constexpr int NC = decltype(nc)::value;
        return grad ? query_launch<NC, true>(ctx, n, d_lay, d_cub, d_axis, seed, stream, d_o, d_st)
                    : query_launch<NC, false>(ctx, n, d_lay, d_cub, nullptr, seed, stream, d_o,
                                              d_st);
    });
    if (rc) return rc;
    std::vector<int32_t> st(n);
    DRWC_CUDA_TRY(cudaMemcpyAsync(out, d_o, out_b, cudaMemcpyDeviceToHost, ctx->stream));
    DRWC_CUDA_TRY(cudaMemcpyAsync(st.data(), d_st, st_b, cudaMemcpyDeviceToHost, ctx->stream));
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int q = 0; q < n; ++q) {
        if (st[q] == 2) return DRWC_ERR_INVALID;
        if (st[q] != 0) return DRWC_ERR_NOT_CONVERGED;
    }
    return DRWC_OK;
}

}  // namespace drwc

using namespace drwc;

extern "C" {

DRWC_API int drwc_structure_construction(drwc_ctx* ctx, int n, int N, const float* layers,
                                         const float* cuboids, int normalise, float* eps_out,
                                         float* max_out) {
    if (!ctx || n < 0 || N < 1 || N > 64) return DRWC_ERR_INVALID;
    if (n == 0) return DRWC_OK;
    if (!layers || !cuboids || !eps_out) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t lay_b = sizeof(float) * n * 2 * kL, cub_b = sizeof(float) * n * 7 * kC;
    const size_t eps_b = sizeof(float) * n * N * N * N, max_b = sizeof(float) * n;
    void *d_in = nullptr, *d_out = nullptr;
    int rc = ws_get(ctx, WS_IN, lay_b + cub_b, &d_in);
    if (rc) return rc;
    rc = ws_get(ctx, WS_OUT, eps_b + max_b, &d_out);
    if (rc) return rc;
    float* d_lay = (float*)d_in;
    float* d_cub = d_lay + (size_t)n * 2 * kL;
    float* d_eps = (float*)d_out;
    float* d_max = d_eps + (size_t)n * N * N * N;
    DRWC_CUDA_TRY(cudaMemcpyAsync(d_lay, layers, lay_b, cudaMemcpyHostToDevice, ctx->stream));
    DRWC_CUDA_TRY(cudaMemcpyAsync(d_cub, cuboids, cub_b, cudaMemcpyHostToDevice, ctx->stream));
    const int grid = std::min(n, ctx->sm_count * 8);
    structure_kernel<<<grid, 256, 0, ctx->stream>>>(n, N, d_lay, d_cub, normalise, d_eps, d_max);
    rc = launch_check(ctx);
    if (rc) return rc;
    DRWC_CUDA_TRY(cudaMemcpyAsync(eps_out, d_eps, eps_b, cudaMemcpyDeviceToHost, ctx->stream));
    if (max_out)
        DRWC_CUDA_TRY(cudaMemcpyAsync(max_out, d_max, max_b, cudaMemcpyDeviceToHost, ctx->stream));
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return DRWC_OK;
}

DRWC_API int drwc_transition_batch(drwc_ctx* ctx, int n, int N, const float* layers,
                                   const float* cuboids, uint64_t seed, uint64_t stream,
                                   float* out_pos) {
    return query_batch(ctx, false, n, N, layers, cuboids, nullptr, seed, stream, out_pos);
}

DRWC_API int drwc_first_hop_batch(drwc_ctx* ctx, int n, int N, const float* layers,
                                  const float* cuboids, const int32_t* axis, uint64_t seed,
                                  uint64_t stream, float* out) {
    return query_batch(ctx, true, n, N, layers, cuboids, axis, seed, stream, out);
}

}  // extern "C"
