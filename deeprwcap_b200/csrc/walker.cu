// Device-resident floating-random-walk capacitance extraction (the role of
// the reference's closed walker, executable/librwcapall.so) with every hop's
// transition kernel from the on-chip FDM solve.
//
// Walk w (job seed s): Philox4x32-10 key s, counter (w, hop, draw, 0).
//   hop 0: a point on the Gaussian surface (the master's bounding box grown
//          by gauss_offset) chosen by area, the largest conductor-free cube
//          around it, the centre-gradient surface values along the face
//          normal (WVTX/Y/Z), a panel drawn with probability |g_b| / sum|g|
//          and the walk weight
//             w = -s_out * A_gauss * eps_w * sum|g| * sign(g_b) / a0 * eps0
//          (dnn_solver_gradient.cpp:143-162 gives sum|g| * sign and the
//          centre permittivity; the area, the half-width a0 and the outward
//          sign s_out turn the normalised gradient into charge);
//   hop h: the largest conductor-free cube around the walker, its surface
//          Green's function (GFT), a panel drawn with probability G_b;
//   end:   when the L-infinity distance to the nearest conductor or
//          enclosure wall is below stop_dist; the walk adds w to the entry
//          of the net it ends on.
// One CTA carries one walk at a time from start to end (persistent grid,
// walks claimed with an atomic counter) and writes its record; capacitance
// sums are reduced afterwards in a fixed order, so results do not depend on
// scheduling. Geometry uses explicitly rounded FP64 operations so the walk
// visits exactly the points a non-contracted CPU evaluation visits.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "geom.cuh"

namespace drwc {

struct WalkState {
    double r[3];
    double a;
    double omega;
    int net;
    int hops;
    int code;
    int done;
    long long walk;
    double sgn_out;
    int lm[DRWC_N_MAX];  // layer material per z index (structures without blocks)
};

template <int N>
__global__ void __launch_bounds__(Cube<N>::NT, CubeTraits<N>::kMinBlocks)
walk_kernel(DevGeom g, Gauss G, WalkParams W, long long walk0, long long nwalks,
            unsigned long long* __restrict__ next, unsigned long long* __restrict__ stats,
            int32_t* __restrict__ end_out,
            int32_t* __restrict__ hops_out, double* __restrict__ w_out,
            double* __restrict__ scratch_y, float* __restrict__ scratch_s) {
    extern __shared__ __align__(128) unsigned char drwc_dyn_smem[];
    unsigned char* smem = drwc_dyn_smem;
    __shared__ WalkState S;
    using D = Cube<N>;
    constexpr int M = 6 * D::NN;
    const CubeSmem<N> sm = CubeSmem<N>::carve(smem);
    const int P = g.n_mat;
    unsigned char* xs = smem + D::kSmemBytes;
    uint8_t* mat = xs;
    double* tco = reinterpret_cast<double*>(xs + ((size_t)D::NNN + 15) / 16 * 16);
    double* pal = tco + N;
    double* palinv = pal + P;
    double* pair64 = palinv + P;
    float* pair32 = reinterpret_cast<float*>(pair64 + P * P);
    for (int v = threadIdx.x; v < P; v += blockDim.x) {
        pal[v] = g.pal[v];
        palinv[v] = 1.0 / g.pal[v];
    }
    for (int v = threadIdx.x; v < P * P; v += blockDim.x) {
        pair64[v] = g.pair64[v];
        pair32[v] = g.pair32[v];
    }
    centre_offsets<N>(tco);
    const EpsPalette E{mat, pal, palinv, pair64, pair32, P};
    double* ys = scratch_y + (size_t)blockIdx.x * D::NNN;
    float* ss = scratch_s + (size_t)blockIdx.x * D::NNN;
    __syncthreads();
    const int t = threadIdx.x;
    unsigned long long my_hops = 0, my_iters = 0, my_sweeps = 0, my_esc = 0, my_fail = 0;
    for (;;) {
        if (t == 0) S.walk = (long long)atomicAdd(next, 1ull);
        __syncthreads();
        const long long idx = S.walk;
        if (idx >= nwalks) break;
        const uint64_t w = (uint64_t)(walk0 + idx);
        // ---- start point on the Gaussian surface
        if (t == 0) {
            walk_start_point(G, g, W.seed, w, S.r, &S.sgn_out, &S.code);
            S.hops = 0;
            S.done = 0;
            S.omega = 0.0;
        }
        __syncthreads();
        for (;;) {
            // ---- distance to the nearest conductor: cube size / absorption
            if (t < 32) {
                double d;
                int net;
                double r[3] = {S.r[0], S.r[1], S.r[2]};
                nearest(g, r, &d, &net);
                if (t == 0) {
                    S.a = d;
                    S.net = net;
                    if (d < W.stop) S.done = 1;
                    else if (S.hops >= W.max_hops) { S.done = 1; S.net = -1; }
                }
            }
            __syncthreads();
            if (S.done) break;
            const double c[3] = {S.r[0], S.r[1], S.r[2]};
            const double a = S.a;
            const bool first = S.hops == 0;
            const int code = first ? S.code : DRWC_GFT;
            if (W.log && t == 0) {
                const unsigned int li = atomicAdd(W.log_count, 1u);
                if (li < W.log_cap) {
                    W.log[4 * (size_t)li + 0] = c[0];
                    W.log[4 * (size_t)li + 1] = c[1];
                    W.log[4 * (size_t)li + 2] = c[2];
                    W.log[4 * (size_t)li + 3] = a;
                    W.log_code[li] = code;
                }
            }
            // a stratified cube (no dielectric block reaches it) is solved by
            // the per-plane solver from its layer materials alone
            const int* lm = nullptr;
            if (g.n_diel > 0) {  // separable: per-axis index ranges of the blocks
                VoxScratch<N>& vs = *reinterpret_cast<VoxScratch<N>*>(
                    smem + (WalkSmem<N>::base(P) + 15) / 16 * 16);
                vox_prepare<N>(g, c, a, tco, vs);
                if (vs.nrel == 0) {
                    lm = vs.lm;
                } else {
                    for (int v = t; v < D::NNN; v += blockDim.x)
                        mat[v] = (uint8_t)vox_material<N>(g, vs, c, a, tco, v % N, (v / N) % N,
                                                          v / D::NN, 0);
                }
            } else {
                plane_layers<N>(g, c, a, tco, S.lm);
                lm = S.lm;
            }
            __syncthreads();
            FdmStats st;
            double* wv = reinterpret_cast<double*>(sm.stage());
            const EpsPlanar<N> EP{lm, pal, palinv, pair64, pair32, P};
            // each thread writes the panel chunk it samples from (no barrier
            // before the draw; cta_sample's own barriers order the rest)
            if (lm) {
                cube_solve_planar<N>(EP, ys, code, W.prm, &st);
                for_each_panel_chunked<N, D::NT>(EP, cube_y<N>(ys), [&](int b, double v) { wv[b] = v; });
            } else {
                cube_solve<N>(E, ys, ss, code, W.prm, &st);
                for_each_panel_chunked<N, D::NT>(E, cube_y<N>(ys), [&](int b, double v) { wv[b] = v; });
            }
            const double2 u = first ? philox_uniform2(W.seed, w, 0, 1)
                                    : philox_uniform2(W.seed, w, (uint32_t)S.hops, 0);
            const double ud = first ? u.y : u.x;
            double tot = 0.0;
            // the hop's closing barrier comes before red is written again
            const int b = cta_sample<D::NT, false>(wv, M, first, ud, sm.red, &tot);
            if (t == 0) {
                my_hops += 1;
                my_iters += (unsigned long long)st.iters;
                my_sweeps += (unsigned long long)st.sweeps;
                my_esc += (unsigned long long)st.escalated;
                my_fail += st.status == 1;
                if (b < 0 || st.status != 0) {
                    // no transition possible, or the cube's solve did not
                    // converge even after escalation: the walk is lost
                    S.net = -1;
                    S.done = 2;
                } else {
                    if (first)
                        S.omega = first_hop_weight(
                            G, S.sgn_out, lm ? center_diel<N>(EP, code) : center_diel<N>(E, code),
                            tot, wv[b], a);
                    double loc[3];
                    locate_f64(N, b, loc);
                    for (int d = 0; d < 3; ++d) S.r[d] = dadd(S.r[d], dmul(a, loc[d]));
                    S.hops += 1;
                }
            }
            __syncthreads();
            if (S.done) break;
        }
        if (t == 0) {
            end_out[idx] = S.net;
            hops_out[idx] = S.hops;
            w_out[idx] = S.omega;
        }
        __syncthreads();
    }
    if (t == 0 && stats) {
        atomicAdd(stats + 0, my_hops);
        atomicAdd(stats + 1, my_iters);
        atomicAdd(stats + 2, my_sweeps);
        atomicAdd(stats + 3, my_esc);
        atomicAdd(stats + 4, my_fail);
    }
}

// Per-entry sums of one batch of walk records: block e sums entry e.
__global__ void __launch_bounds__(256) reduce_kernel(int n_entries, long long nw,
                                                     const int32_t* __restrict__ end,
                                                     const double* __restrict__ w,
                                                     double* __restrict__ out) {
    reduce_entry(blockIdx.x, n_entries, nw, end, w, out);
}

__global__ void hop_sum_kernel(long long nw, const int32_t* __restrict__ hops,
                               unsigned long long* __restrict__ out) {
    unsigned long long s = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nw;
         i += (long long)gridDim.x * blockDim.x)
        s += (unsigned long long)hops[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// ------------------------------------------------------------------ host side
// Resident CTAs per SM for a given palette size (the shared-memory request
// grows with it); the attribute is set once for the largest palette.
template <int N>
static int walk_shape(int P, bool vox, int* per_sm) {
    static bool attr = false;
    static int cache[2][kMaxMaterials + 1] = {{0}};
    if (!attr) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(walk_kernel<N>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)WalkSmem<N>::bytes(kMaxMaterials, true)));
        attr = true;
    }
    if (!cache[vox][P]) {
        int nb = 0;
        DRWC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &nb, walk_kernel<N>, Cube<N>::NT, WalkSmem<N>::bytes(P, vox)));
        cache[vox][P] = nb < 1 ? 1 : nb;
    }
    *per_sm = cache[vox][P];
    return DRWC_OK;
}

// Device buffers for one batch of walk records.
struct WalkBuffers {
    int32_t* end;
    int32_t* hops;
    double* w;
    unsigned long long* counter;  // [0] claim counter, [1] hop sum, [2..6] solver stats
    double* sums;                 // 3 * (n_entries + 1)
};

static int launch_walks(drwc_ctx* ctx, const HostGeom& hg, const Gauss& G, const WalkParams& P,
                        long long walk0, long long nw, WalkBuffers& wb) {
    return dispatch_N(P.N, [&](auto nc) -> int {
        constexpr int NC = decltype(nc)::value;
        using D = Cube<NC>;
        const int nmat = hg.dev.n_mat;
        int per_sm = 0;
        const bool vox = hg.dev.n_diel > 0;
        int rc = walk_shape<NC>(nmat, vox, &per_sm);
        if (rc) return rc;
        const int grid = (int)std::min<long long>(nw, (long long)per_sm * ctx->sm_count);
        void* scratch = nullptr;
        rc = ws_get(ctx, WS_SCRATCH, (size_t)grid * D::NNN * 12, &scratch);
        if (rc) return rc;
        double* sy = (double*)scratch;
        float* sf = (float*)(sy + (size_t)grid * D::NNN);
        DRWC_CUDA_TRY(cudaMemsetAsync(wb.counter, 0, 8 * sizeof(unsigned long long), ctx->stream));
        walk_kernel<NC><<<grid, D::NT, WalkSmem<NC>::bytes(nmat, vox), ctx->stream>>>(
            hg.dev, G, P, walk0, nw, wb.counter, wb.counter + 2, wb.end, wb.hops, wb.w, sy, sf);
        return launch_check(ctx);
    });
}

static int walk_buffers(drwc_ctx* ctx, long long nw, int n_entries, WalkBuffers* wb) {
    const size_t bytes = nw * (4 + 4 + 8) + 64 + 8 * 3 * (n_entries + 2) + 1024;
    void* d = nullptr;
    int rc = ws_get(ctx, WS_RES, bytes, &d);
    if (rc) return rc;
    unsigned char* b = (unsigned char*)d;
    wb->w = (double*)b;
    wb->sums = (double*)(b + nw * 8);
    wb->counter = (unsigned long long*)(wb->sums + 3 * (n_entries + 2));
    wb->end = (int32_t*)(wb->counter + 8);
    wb->hops = wb->end + nw;
    return DRWC_OK;
}

}  // namespace drwc

using namespace drwc;

extern "C" {

DRWC_API void drwc_job_params_default(drwc_job_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->master = 0;
    p->N = 16;
    p->gauss_offset = 0.05;
    p->stop_dist = 1e-5;
    p->p_tol = 0.01;
    p->c_tol = 0.01;
    p->c_ratio = 0.95;
    p->min_walks = 4096;
    p->max_walks = 1LL << 26;
    p->batch_walks = 1LL << 16;
    p->max_hops = 10000;
    p->seed = 1;
    drwc_fdm_opts_default(&p->fdm);
}

}  // extern "C"

// A prepared job: validated structure uploaded once, walk buffers reusable.
struct drwc_job {
    drwc_ctx* ctx;
    HostGeom hg;
    Gauss G;
    WalkParams P;
    int n_entries;
    int64_t h2d_bytes;
};

extern "C" {

DRWC_API int drwc_job_create(drwc_ctx* ctx, const drwc_structure* s, const drwc_job_params* p,
                             drwc_job** out) {
    if (!ctx || !out) return DRWC_ERR_INVALID;
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    drwc_job* j = new drwc_job();
    j->ctx = ctx;
    int rc = prepare(ctx, s, p, &j->hg, &j->G, &j->P);
    if (rc) { delete j; return rc; }
    // the job owns its geometry copy (the context workspace is shared)
    void* own = nullptr;
    if (cudaMalloc(&own, j->hg.blob.size()) != cudaSuccess) {
        cudaGetLastError();
        delete j;
        return DRWC_ERR_NOMEM;
    }
    DRWC_CUDA_TRY(cudaMemcpyAsync(own, j->hg.blob.data(), j->hg.blob.size(),
                                  cudaMemcpyHostToDevice, ctx->stream));
    bind_geom(&j->hg, own);
    j->n_entries = s->n_nets + 1;
    j->h2d_bytes = (int64_t)(j->hg.box.size() * 8 + j->hg.net.size() * 4 + j->hg.zlo.size() * 8 +
                             j->hg.lmat.size() * 4 + j->hg.dmat.size() * 4 +
                             j->hg.pal.size() * 8 + j->hg.pair64.size() * 12 +
                             j->hg.diel.size() * 8 +
                             j->hg.gstart.size() * 4 + j->hg.gitems.size() * 4);
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *out = j;
    return DRWC_OK;
}

DRWC_API int drwc_job_destroy(drwc_job* j) {
    if (!j) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lock(j->ctx->mu);
    cudaSetDevice(j->ctx->device);
    cudaStreamSynchronize(j->ctx->stream);
    if (j->hg.dbuf) cudaFree(j->hg.dbuf);
    delete j;
    return DRWC_OK;
}

DRWC_API int drwc_job_walks_device(drwc_job* j, int64_t walk0, int64_t nwalks, int32_t* end_net,
                                   int32_t* hops, double* weight, int64_t* solver_stats) {
    if (!j || walk0 < 0 || nwalks < 0) return DRWC_ERR_INVALID;
    if (nwalks == 0) return DRWC_OK;
    if (!end_net || !hops || !weight) return DRWC_ERR_INVALID;
    drwc_ctx* ctx = j->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    WalkBuffers wb;
    void* d = nullptr;
    int rc = ws_get(ctx, WS_AUX, 64 * sizeof(unsigned long long), &d);
    if (rc) return rc;
    wb.counter = (unsigned long long*)d;
    wb.end = end_net;
    wb.hops = hops;
    wb.w = weight;
    wb.sums = nullptr;
    rc = launch_walks(ctx, j->hg, j->G, j->P, walk0, nwalks, wb);
    if (rc) return rc;
    if (solver_stats) {
        // stats are (hops, FP32 iterations, FP64 sweeps, escalated solves,
        // failed solves) as unsigned 64-bit
        DRWC_CUDA_TRY(cudaMemcpyAsync(solver_stats, wb.counter + 2, 5 * sizeof(int64_t),
                                      cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return DRWC_OK;
}

DRWC_API int drwc_job_h2d_bytes(drwc_job* j, int64_t* bytes) {
    if (!j || !bytes) return DRWC_ERR_INVALID;
    *bytes = j->h2d_bytes;
    return DRWC_OK;
}

DRWC_API int drwc_frw_walks(drwc_ctx* ctx, const drwc_structure* s, const drwc_job_params* p,
                            int64_t walk0, int64_t nwalks, int32_t* end_net, int32_t* hops,
                            double* weight, int64_t* solver_stats) {
    if (!ctx || walk0 < 0 || nwalks < 0) return DRWC_ERR_INVALID;
    if (nwalks == 0) return DRWC_OK;
    if (!end_net || !hops || !weight) return DRWC_ERR_INVALID;
    drwc_job* j = nullptr;
    int rc = drwc_job_create(ctx, s, p, &j);
    if (rc) return rc;
    void* d = nullptr;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        rc = ws_get(ctx, WS_RES, (size_t)nwalks * 16 + 64, &d);
    }
    if (rc) { drwc_job_destroy(j); return rc; }
    double* d_w = (double*)d;
    int32_t* d_end = (int32_t*)(d_w + nwalks);
    int32_t* d_hops = d_end + nwalks;
    int64_t* d_st = (int64_t*)(((uintptr_t)(d_hops + nwalks) + 7) & ~(uintptr_t)7);
    rc = drwc_job_walks_device(j, walk0, nwalks, d_end, d_hops, d_w, d_st);
    if (rc) { drwc_job_destroy(j); return rc; }
    int64_t st[5] = {0, 0, 0, 0, 0};
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        DRWC_CUDA_TRY(cudaMemcpyAsync(end_net, d_end, nwalks * 4, cudaMemcpyDeviceToHost, ctx->stream));
        DRWC_CUDA_TRY(cudaMemcpyAsync(hops, d_hops, nwalks * 4, cudaMemcpyDeviceToHost, ctx->stream));
        DRWC_CUDA_TRY(cudaMemcpyAsync(weight, d_w, nwalks * 8, cudaMemcpyDeviceToHost, ctx->stream));
        DRWC_CUDA_TRY(cudaMemcpyAsync(st, d_st, sizeof st, cudaMemcpyDeviceToHost, ctx->stream));
        DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    if (solver_stats) {
        solver_stats[0] = st[0];
        solver_stats[1] = st[1];
        solver_stats[2] = st[2];
        solver_stats[3] = st[0] * p->N * p->N * p->N;
        solver_stats[4] = st[3];
        solver_stats[5] = st[4];
    }
    return drwc_job_destroy(j);
}

DRWC_API int drwc_frw_run(drwc_ctx* ctx, const drwc_structure* s, const drwc_job_params* p,
                          drwc_job_result* out) {
    if (!ctx || !out) return DRWC_ERR_INVALID;
    const auto t0 = std::chrono::steady_clock::now();
    drwc_job* job = nullptr;
    int rc = drwc_job_create(ctx, s, p, &job);
    if (rc) return rc;
    struct JobGuard { drwc_job* j; ~JobGuard() { drwc_job_destroy(j); } } guard{job};
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    const HostGeom& hg = job->hg;
    const Gauss& G = job->G;
    const WalkParams& P = job->P;
    const int ne = s->n_nets + 1;  // nets + ground
    const long long batch = std::max<long long>(1, p->batch_walks);
    WalkBuffers wb;
    rc = walk_buffers(ctx, batch, ne, &wb);
    if (rc) return rc;
    // Neumaier-compensated FP64 accumulators per entry
    std::vector<double> S(ne + 1, 0.0), Sc(ne + 1, 0.0), S2(ne + 1, 0.0), S2c(ne + 1, 0.0);
    auto kadd = [](double& s, double& c, double v) {
        const double t = s + v;
        if (std::fabs(s) >= std::fabs(v)) c += (s - t) + v;
        else c += (v - t) + s;
        s = t;
    };
    long long walks = 0, lost = 0, escalated = 0, failed = 0;
    unsigned long long hops_total = 0;
    std::vector<double> sums(3 * (ne + 1));
    int converged = 0;
    std::memset(out, 0, sizeof(*out));
    while (walks < p->max_walks) {
        const long long nw = std::min<long long>(batch, p->max_walks - walks);
        rc = launch_walks(ctx, hg, G, P, walks, nw, wb);
        if (rc) return rc;
        reduce_kernel<<<ne + 1, 256, 0, ctx->stream>>>(ne, nw, wb.end, wb.w, wb.sums);
        rc = launch_check(ctx);
        if (rc) return rc;
        hop_sum_kernel<<<std::max(1, std::min<int>((int)((nw + 255) / 256), 1024)), 256, 0,
                         ctx->stream>>>(nw, wb.hops, wb.counter + 1);
        rc = launch_check(ctx);
        if (rc) return rc;
        unsigned long long hsum[7] = {0};  // [1] hop sum, [5] escalated, [6] failed solves
        DRWC_CUDA_TRY(cudaMemcpyAsync(sums.data(), wb.sums, sums.size() * 8,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        DRWC_CUDA_TRY(cudaMemcpyAsync(hsum, wb.counter, sizeof hsum, cudaMemcpyDeviceToHost,
                                      ctx->stream));
        DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        for (int e = 0; e <= ne; ++e) {
            kadd(S[e], Sc[e], sums[3 * e]);
            kadd(S2[e], S2c[e], sums[3 * e + 1]);
        }
        lost += (long long)sums[3 * ne + 2];
        hops_total += hsum[1];
        escalated += (long long)hsum[5];
        failed += (long long)hsum[6];
        walks += nw;
        if (walks < p->min_walks) continue;
        // convergence: relative 1-sigma of the self term <= p_tol, and of every
        // significant coupling (ground included) <= c_tol, where the
        // significant couplings are the largest ones that together make up
        // c_ratio of the summed coupling magnitude.
        const double n = (double)walks;
        auto mean = [&](int e) { return (S[e] + Sc[e]) / n; };
        auto sem = [&](int e) {
            const double m = mean(e);
            const double var = std::max(0.0, (S2[e] + S2c[e]) / n - m * m);
            return std::sqrt(var / n);
        };
        const double cs = mean(p->master);
        bool ok = cs != 0.0 && sem(p->master) <= p->p_tol * std::fabs(cs);
        std::vector<std::pair<double, int>> cpl;
        double ctot = 0.0;
        for (int e = 0; e < ne; ++e) {
            if (e == p->master) continue;
            cpl.push_back({std::fabs(mean(e)), e});
            ctot += std::fabs(mean(e));
        }
        std::sort(cpl.begin(), cpl.end(), [](auto& a, auto& b) { return a.first > b.first; });
        double acc = 0.0;
        for (auto& ce : cpl) {
            if (acc >= p->c_ratio * ctot) break;
            acc += ce.first;
            if (!(ce.first > 0.0) || sem(ce.second) > p->c_tol * ce.first) { ok = false; break; }
        }
        if (ok) { converged = 1; break; }
    }
    const double n = (double)std::max(1LL, walks);
    out->n_entries = ne;
    out->converged = converged;
    out->walks = walks;
    out->hops = (int64_t)hops_total;
    out->lost = lost;
    out->solves_escalated = escalated;
    out->solves_failed = failed;
    for (int e = 0; e < ne; ++e) {
        const double m = (S[e] + Sc[e]) / n;
        out->cap[e] = m;
        const double var = std::max(0.0, (S2[e] + S2c[e]) / n - m * m);
        out->stderr_[e] = std::sqrt(var / n);
    }
    out->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return DRWC_OK;
}

}  // extern "C"

// =========================================================================
// Training data and the learned walker.
// =========================================================================
#include "nn.cuh"

namespace drwc {

// Hop-log records -> network inputs (and FP64 permittivity for the FDM
// targets). Records of first hops are voxelised in the rotated frame of
// their gradient axis, so their target is always WVTZ.
template <int N>
__global__ void __launch_bounds__(256) records_kernel(DevGeom g, int n, const double* __restrict__ rec,
                                                      const int* __restrict__ code,
                                                      __nv_bfloat16* __restrict__ X,
                                                      double* __restrict__ eps64) {
    __shared__ double tco[N];
    __shared__ double pal[kMaxMaterials];
    __shared__ uint8_t mat[N * N * N];
    __shared__ float red[32];
    __shared__ VoxScratch<N> vs;
    for (int v = threadIdx.x; v < g.n_mat; v += blockDim.x) pal[v] = g.pal[v];
    centre_offsets<N>(tco);
    __syncthreads();
    for (int r = blockIdx.x; r < n; r += gridDim.x) {
        const double c[3] = {rec[4 * (size_t)r], rec[4 * (size_t)r + 1], rec[4 * (size_t)r + 2]};
        const double a = rec[4 * (size_t)r + 3];
        voxelise_net<N>(g, c, a, rot_of_code(code[r]), tco, pal, mat, X + (size_t)r * N * N * N,
                        eps64 ? eps64 + (size_t)r * N * N * N : nullptr, red, vs);
    }
}

// Random transition cubes of the batched-FDM generator (1-4 layers along a
// random axis, eps ~ U[2,8], 0-2 boxes eps ~ U[2,8], a quarter of the voxels
// of noisy cubes eps log-uniform in [1,12]), drawn from Philox per cube.
template <int N>
__global__ void __launch_bounds__(256) random_cubes_kernel(int n, uint64_t seed, float noise_frac,
                                                           __nv_bfloat16* __restrict__ X,
                                                           double* __restrict__ eps64) {
    constexpr int NNN = N * N * N;
    __shared__ double cut[4], val[4], box[2][7];
    __shared__ int nl, nb, axis, noisy;
    __shared__ float red[32];
    for (int q = blockIdx.x; q < n; q += gridDim.x) {
        if (threadIdx.x == 0) {
            double2 u = philox_uniform2(seed, (uint64_t)q, 0, 0);
            nl = 1 + (int)(u.x * 4.0);
            nb = (int)(u.y * 3.0);
            u = philox_uniform2(seed, (uint64_t)q, 0, 1);
            axis = (int)(u.x * 3.0);
            noisy = u.y < noise_frac;
            double cs[4];
            for (int l = 0; l < 4; ++l) {
                const double2 w = philox_uniform2(seed, (uint64_t)q, 1, l);
                cs[l] = l == 0 ? -1.0 : -1.0 + 2.0 * w.x;
                val[l] = 2.0 + 6.0 * w.y;
            }
            for (int l = 1; l < nl; ++l)  // sort the cuts
                for (int m2 = l + 1; m2 < nl; ++m2)
                    if (cs[m2] < cs[l]) { const double tmp = cs[l]; cs[l] = cs[m2]; cs[m2] = tmp; }
            for (int l = 0; l < 4; ++l) cut[l] = cs[l];
            for (int b = 0; b < 2; ++b) {
                double lo[3], hi[3];
                for (int d = 0; d < 3; ++d) {
                    const double2 w = philox_uniform2(seed, (uint64_t)q, 2 + b, d);
                    const double p0 = -1.0 + 2.0 * w.x, p1 = -1.0 + 2.0 * w.y;
                    lo[d] = fmin(p0, p1);
                    hi[d] = fmax(p0, p1);
                }
                const double2 w = philox_uniform2(seed, (uint64_t)q, 2 + b, 3);
                for (int d = 0; d < 3; ++d) { box[b][d] = lo[d]; box[b][3 + d] = hi[d]; }
                box[b][6] = 2.0 + 6.0 * w.x;
            }
        }
        __syncthreads();
        float mx = 0.f;
        for (int v = threadIdx.x; v < NNN; v += blockDim.x) {
            const int ix[3] = {v % N, (v / N) % N, v / (N * N)};
            double p[3];
            for (int d = 0; d < 3; ++d) p[d] = (2.0 * ix[d] + 1.0) / N - 1.0;
            const double zc = p[axis];
            int li = 0;
            for (int l = 0; l < nl; ++l)
                if (zc >= cut[l]) li = l;
            double e = val[li];
            for (int b = 0; b < nb; ++b) {
                if (p[0] >= box[b][0] && p[0] <= box[b][3] && p[1] >= box[b][1] && p[1] <= box[b][4] &&
                    p[2] >= box[b][2] && p[2] <= box[b][5]) { e = box[b][6]; break; }
            }
            if (noisy) {
                const double2 w = philox_uniform2(seed ^ 0x9E3779B97F4A7C15ull, (uint64_t)q, 8, v);
                if (w.x < 0.25) e = exp(w.y * log(12.0));
            }
            eps64[(size_t)q * NNN + v] = e;
            mx = fmaxf(mx, (float)e);
        }
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
        __syncthreads();
        float m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, red[w]);
        const float inv = 1.f / m;
        for (int v = threadIdx.x; v < NNN; v += blockDim.x)
            X[(size_t)q * NNN + v] = __float2bfloat16((float)eps64[(size_t)q * NNN + v] * inv);
        __syncthreads();
    }
}

}  // namespace drwc

extern "C" {

DRWC_API int drwc_frw_harvest(drwc_ctx* ctx, const drwc_structure* s, const drwc_job_params* p,
                              int64_t walk0, int64_t nwalks, int32_t cap, double* rec,
                              int32_t* code, int32_t* count) {
    if (!ctx || walk0 < 0 || nwalks <= 0 || cap <= 0 || !rec || !code || !count)
        return DRWC_ERR_INVALID;
    drwc_job* j = nullptr;
    int rc = drwc_job_create(ctx, s, p, &j);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
        WalkBuffers wb;
        void* d = nullptr;
        rc = ws_get(ctx, WS_RES, (size_t)nwalks * 16 + 256, &d);
        if (!rc) {
            wb.w = (double*)d;
            wb.end = (int32_t*)(wb.w + nwalks);
            wb.hops = wb.end + nwalks;
            unsigned int* cnt = (unsigned int*)(wb.hops + nwalks + 8);
            void* dc = nullptr;
            rc = ws_get(ctx, WS_AUX, 64 * sizeof(unsigned long long), &dc);
            if (!rc) {
                wb.counter = (unsigned long long*)dc;
                WalkParams P = j->P;
                P.log = rec;
                P.log_code = code;
                P.log_count = cnt;
                P.log_cap = (unsigned int)cap;
                DRWC_CUDA_TRY(cudaMemsetAsync(cnt, 0, 4, ctx->stream));
                rc = launch_walks(ctx, j->hg, j->G, P, walk0, nwalks, wb);
                unsigned int hc = 0;
                DRWC_CUDA_TRY(cudaMemcpyAsync(&hc, cnt, 4, cudaMemcpyDeviceToHost, ctx->stream));
                DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
                *count = (int32_t)std::min<unsigned int>(hc, (unsigned int)cap);
            }
        }
    }
    drwc_job_destroy(j);
    return rc;
}

DRWC_API int drwc_records_voxelise(drwc_ctx* ctx, const drwc_structure* s, int N, int n,
                                   const double* rec, const int32_t* code, void* X,
                                   double* eps64) {
    if (!ctx || n < 0 || (n > 0 && (!rec || !code || !X))) return DRWC_ERR_INVALID;
    if (N != 16 && N != 21 && N != 23) return DRWC_ERR_INVALID;
    if (n == 0) return DRWC_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    int rc = validate(s);
    if (rc) return rc;
    HostGeom hg;
    rc = upload_geom(ctx, s, &hg);
    if (rc) return rc;
    const int grid = std::min(n, ctx->sm_count * 8);
    if (N == 16)
        records_kernel<16><<<grid, 256, 0, ctx->stream>>>(hg.dev, n, rec, code, (__nv_bfloat16*)X, eps64);
    else if (N == 21)
        records_kernel<21><<<grid, 256, 0, ctx->stream>>>(hg.dev, n, rec, code, (__nv_bfloat16*)X, eps64);
    else
        records_kernel<23><<<grid, 256, 0, ctx->stream>>>(hg.dev, n, rec, code, (__nv_bfloat16*)X, eps64);
    rc = launch_check(ctx);
    if (rc) return rc;
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return DRWC_OK;
}

DRWC_API int drwc_cubes_random(drwc_ctx* ctx, int N, int n, uint64_t seed, float noise_frac,
                               void* X, double* eps64) {
    if (!ctx || n < 0 || (n > 0 && (!X || !eps64))) return DRWC_ERR_INVALID;
    if (N != 16 && N != 21 && N != 23) return DRWC_ERR_INVALID;
    if (n == 0) return DRWC_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    const int grid = std::min(n, ctx->sm_count * 8);
    __nv_bfloat16* x = (__nv_bfloat16*)X;
    if (N == 16) random_cubes_kernel<16><<<grid, 256, 0, ctx->stream>>>(n, seed, noise_frac, x, eps64);
    else if (N == 21) random_cubes_kernel<21><<<grid, 256, 0, ctx->stream>>>(n, seed, noise_frac, x, eps64);
    else random_cubes_kernel<23><<<grid, 256, 0, ctx->stream>>>(n, seed, noise_frac, x, eps64);
    return launch_check(ctx);
}

}  // extern "C"

// ------------------------------------------------------------ learned walker
// Batched walker: S slots each carry one walk at a time. A step runs, for
// every active slot at once: geometry (claim a walk, nearest conductor,
// absorption) -> voxelise into the network input -> network (tensor cores)
// -> draw the next point from the predicted Poisson kernel (or, on first
// hops, from the predicted gradient in the rotated frame). Slots whose
// confidence output says the prediction is off, and a Philox-chosen fraction
// of all hops (audits), take the hop through the FDM solve instead; audits
// also record the KL divergence between the FDM and the network's kernel.
// Walk w draws its uniforms from the same Philox counters as the FDM walker.
namespace drwc {

constexpr int kDecRowsLw = DRWC_NET_OUT;  // network output row (logits + confidence)

struct LwState {
    double *px, *py, *pz, *omega, *sgn, *a, *epsw;
    long long* walk;
    int *hops, *mode, *code, *act, *grow;
};

struct LwArgs {
    int S;
    long long nwalks;        // walks [walk0, walk0 + nwalks)
    long long walk0;
    DevGeom g;
    Gauss G;
    WalkParams W;
    LwState st;
    unsigned long long* ctr;  // [0] claimed, [1] finished, [2] nn hops, [3] fdm hops,
                              // [4] fallbacks, [5] audits
    int32_t* end_out;
    int32_t* hops_out;
    double* w_out;
    float conf_thresh;
    float audit_frac;
    int* fdm_list;
    int* fdm_kind;
    unsigned int* fdm_count;
    double* audit_kl;         // [0] sum KL, [1] count
    const float* O;           // network rows, compact over the active list
    const float* Gh;          // gradient rows, compact over the first-hop list
    __nv_bfloat16* X;         // network input rows, compact over the active list
    int* alist;               // active slots this step
    unsigned int* na;
    int* frow;                // network row of each first-hop entry
    unsigned int* nf;
};

DRWC_DEV void lw_start(const LwArgs& A, int slot, long long w) {
    double r[3], sgn;
    int code;
    walk_start_point(A.G, A.g, A.W.seed, (uint64_t)w, r, &sgn, &code);
    A.st.px[slot] = r[0]; A.st.py[slot] = r[1]; A.st.pz[slot] = r[2];
    A.st.sgn[slot] = sgn;
    A.st.code[slot] = code;
    A.st.hops[slot] = 0;
    A.st.omega[slot] = 0.0;
    A.st.walk[slot] = w;
    A.st.mode[slot] = 1;
}

DRWC_DEV void lw_finish(const LwArgs& A, int slot, int net) {
    const long long i = A.st.walk[slot] - A.walk0;
    A.end_out[i] = net;
    A.hops_out[i] = A.st.hops[slot];
    A.w_out[i] = A.st.omega[slot];
    atomicAdd(A.ctr + 1, 1ull);
    A.st.mode[slot] = 0;
}

// One warp per slot.
__global__ void lw_prepare_kernel(LwArgs A) {
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (slot >= A.S) return;
    int act = 0;
    for (int tries = 0; tries < 4; ++tries) {
        int mode = A.st.mode[slot];
        if (mode == 0) {
            long long w = 0;
            if (lane == 0) {
                w = (long long)atomicAdd(A.ctr + 0, 1ull);
                if (w < A.nwalks) lw_start(A, slot, A.walk0 + w);
                else A.st.mode[slot] = 2;
            }
            __syncwarp();
            mode = A.st.mode[slot];
        }
        if (mode == 2) break;
        double r[3] = {A.st.px[slot], A.st.py[slot], A.st.pz[slot]};
        double d;
        int net;
        nearest(A.g, r, &d, &net);
        if (lane == 0) {
            if (d < A.W.stop) {
                lw_finish(A, slot, net);
            } else if (A.st.hops[slot] >= A.W.max_hops) {
                lw_finish(A, slot, -1);
            } else {
                A.st.a[slot] = d;
                act = 1;
            }
        }
        act = __shfl_sync(0xffffffffu, act, 0);
        __syncwarp();
        if (act) break;
    }
    if (lane == 0) {
        A.st.act[slot] = act;
        if (act) {
            const unsigned int idx = atomicAdd(A.na, 1u);
            A.alist[idx] = slot;
            if (A.st.hops[slot] == 0) {
                const unsigned int f = atomicAdd(A.nf, 1u);
                A.frow[f] = (int)idx;
                A.st.grow[slot] = (int)f;
            }
        }
    }
}

// One CTA (256 threads) per slot: network input.
__global__ void __launch_bounds__(256) lw_voxelise_kernel(LwArgs A) {
    constexpr int N = 16;
    __shared__ double tco[N];
    __shared__ double pal[kMaxMaterials];
    __shared__ uint8_t mat[N * N * N];
    __shared__ float red[32];
    __shared__ VoxScratch<N> vs;
    for (int v = threadIdx.x; v < A.g.n_mat; v += blockDim.x) pal[v] = A.g.pal[v];
    centre_offsets<N>(tco);
    __syncthreads();
    const int na = (int)*A.na;
    for (int row = blockIdx.x; row < na; row += gridDim.x) {
        const int slot = A.alist[row];
        const bool first = A.st.hops[slot] == 0;
        const int rot = first ? rot_of_code(A.st.code[slot]) : 0;
        const double c[3] = {A.st.px[slot], A.st.py[slot], A.st.pz[slot]};
        voxelise_net<N>(A.g, c, A.st.a[slot], rot, tco, pal, mat, A.X + (size_t)row * N * N * N,
                        nullptr, red, vs);
        if (first && threadIdx.x == 0) {
            // centre permittivity of the gradient convention, in the rotated
            // frame where the gradient axis is z
            const EpsPalette E{mat, pal, nullptr, nullptr, nullptr, 0};
            A.st.epsw[slot] = center_diel<N>(E, DRWC_WVTZ);
        }
        __syncthreads();
    }
}

// One CTA (256 threads) per slot: draw from the network's prediction, or
// route the hop to the FDM solve.
__global__ void __launch_bounds__(256) lw_sample_kernel(LwArgs A) {
    constexpr int N = 16, M = 6 * N * N, NT = 256;
    __shared__ double wv[M];
    __shared__ double red[2 * (NT / 32) + 16];
    __shared__ int route;
    const int na = (int)*A.na;
    for (int row = blockIdx.x; row < na; row += gridDim.x) {
        const int slot = A.alist[row];
        const long long w = A.st.walk[slot];
        const int h = A.st.hops[slot];
        const bool first = h == 0;
        if (threadIdx.x == 0) {
            const float conf = A.O[(size_t)row * kDecRowsLw + 1536];
            const bool audit = philox_uniform2(A.W.seed, (uint64_t)w, (uint32_t)h, 2).x <
                               (double)A.audit_frac;
            const bool fallback = conf > A.conf_thresh;  // cube judged hard: FDM
            route = 0;
            if (audit || fallback) {
                const unsigned int idx = atomicAdd(A.fdm_count, 1u);
                A.fdm_list[idx] = slot;
                A.fdm_kind[idx] = (audit ? 1 : 0) | (row << 1);
                route = 1;
                atomicAdd(A.ctr + (audit ? 5 : 4), 1ull);
            }
        }
        __syncthreads();
        if (route) { __syncthreads(); continue; }
        double tot = 0.0;
        int b;
        if (first) {
            const float* g = A.Gh + (size_t)A.st.grow[slot] * M;
            for (int j = threadIdx.x; j < M; j += NT) wv[j] = (double)g[j] / (double)kGradScale;
            __syncthreads();
            const double u = philox_uniform2(A.W.seed, (uint64_t)w, 0, 1).y;
            b = cta_sample<NT>(wv, M, true, u, red, &tot);
        } else {
            const float* o = A.O + (size_t)row * kDecRowsLw;
            float mx = -1e30f;
            for (int j = threadIdx.x; j < M; j += NT) mx = fmaxf(mx, o[j]);
            for (int s = 16; s > 0; s >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, s));
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
            __syncthreads();
            float m = (float)red[0];
            for (int q = 1; q < NT / 32; ++q) m = fmaxf(m, (float)red[q]);
            __syncthreads();
            for (int j = threadIdx.x; j < M; j += NT) wv[j] = (double)__expf(o[j] - m);
            __syncthreads();
            const double u = philox_uniform2(A.W.seed, (uint64_t)w, (uint32_t)h, 0).x;
            b = cta_sample<NT>(wv, M, false, u, red, &tot);
        }
        if (threadIdx.x == 0 && b >= 0) {
            const double a = A.st.a[slot];
            double loc[3], mv[3];
            locate_f64(N, b, loc);
            if (first) {
                const int rot = rot_of_code(A.st.code[slot]);
                unrotate(rot, loc, mv);
                A.st.omega[slot] =
                    first_hop_weight(A.G, A.st.sgn[slot], A.st.epsw[slot], tot, wv[b], a);
            } else {
                mv[0] = loc[0]; mv[1] = loc[1]; mv[2] = loc[2];
            }
            A.st.px[slot] = dadd(A.st.px[slot], dmul(a, mv[0]));
            A.st.py[slot] = dadd(A.st.py[slot], dmul(a, mv[1]));
            A.st.pz[slot] = dadd(A.st.pz[slot], dmul(a, mv[2]));
            A.st.hops[slot] = h + 1;
            atomicAdd(A.ctr + 2, 1ull);
        }
        if (threadIdx.x == 0 && b < 0) lw_finish(A, slot, -1);  // no transition: lost
        __syncthreads();
    }
}

// The hops routed to the FDM solve (fallbacks and audits), one persistent CTA
// per SM slot over the routed list; same arithmetic as walk_kernel's hop.
template <int N>
__global__ void __launch_bounds__(Cube<N>::NT, CubeTraits<N>::kMinBlocks)
lw_fdm_kernel(LwArgs A, double* __restrict__ scratch_y, float* __restrict__ scratch_s) {
    extern __shared__ __align__(128) unsigned char drwc_dyn_smem[];
    unsigned char* smem = drwc_dyn_smem;
    using D = Cube<N>;
    constexpr int M = 6 * D::NN;
    const CubeSmem<N> sm = CubeSmem<N>::carve(smem);
    const DevGeom& g = A.g;
    const int P = g.n_mat;
    unsigned char* xs = smem + D::kSmemBytes;
    uint8_t* mat = xs;
    double* tco = reinterpret_cast<double*>(xs + ((size_t)D::NNN + 15) / 16 * 16);
    double* pal = tco + N;
    double* palinv = pal + P;
    double* pair64 = palinv + P;
    float* pair32 = reinterpret_cast<float*>(pair64 + P * P);
    for (int v = threadIdx.x; v < P; v += blockDim.x) {
        pal[v] = g.pal[v];
        palinv[v] = 1.0 / g.pal[v];
    }
    for (int v = threadIdx.x; v < P * P; v += blockDim.x) {
        pair64[v] = g.pair64[v];
        pair32[v] = g.pair32[v];
    }
    centre_offsets<N>(tco);
    const EpsPalette E{mat, pal, palinv, pair64, pair32, P};
    double* ys = scratch_y + (size_t)blockIdx.x * D::NNN;
    float* ss = scratch_s + (size_t)blockIdx.x * D::NNN;
    __syncthreads();
    const unsigned int count = *A.fdm_count;
    __shared__ int lm[N];  // layer material per z index (structures without blocks)
    VoxScratch<N>& vs =   // separable voxeliser (structures with blocks)
        *reinterpret_cast<VoxScratch<N>*>(smem + (WalkSmem<N>::base(P) + 15) / 16 * 16);
    for (unsigned int idx = blockIdx.x; idx < count; idx += gridDim.x) {
        const int slot = A.fdm_list[idx];
        const int audit = A.fdm_kind[idx] & 1;
        const int nrow = A.fdm_kind[idx] >> 1;
        const long long w = A.st.walk[slot];
        const int h = A.st.hops[slot];
        const bool first = h == 0;
        const int code = first ? A.st.code[slot] : DRWC_GFT;
        const double c[3] = {A.st.px[slot], A.st.py[slot], A.st.pz[slot]};
        const double a = A.st.a[slot];
        const int* lmc = nullptr;  // stratified cube: the per-plane solver
        if (g.n_diel > 0) {
            vox_prepare<N>(g, c, a, tco, vs);
            if (vs.nrel == 0) {
                lmc = vs.lm;
            } else {
                for (int v = threadIdx.x; v < D::NNN; v += blockDim.x)
                    mat[v] = (uint8_t)vox_material<N>(g, vs, c, a, tco, v % N, (v / N) % N,
                                                      v / D::NN, 0);
            }
        } else {
            plane_layers<N>(g, c, a, tco, lm);
            lmc = lm;
        }
        __syncthreads();
        FdmStats st;
        double* wv = reinterpret_cast<double*>(sm.stage());
        const EpsPlanar<N> EP{lmc, pal, palinv, pair64, pair32, P};
        if (lmc) {
            cube_solve_planar<N>(EP, ys, code, A.W.prm, &st);
            for_each_panel<N>(EP, cube_y<N>(ys), [&](int b, double v) { wv[b] = v; });
        } else {
            cube_solve<N>(E, ys, ss, code, A.W.prm, &st);
            for_each_panel<N>(E, cube_y<N>(ys), [&](int b, double v) { wv[b] = v; });
        }
        __syncthreads();
        if (audit && !first) {
            // KL(FDM || network) over the panels
            const float* o = A.O + (size_t)nrow * kDecRowsLw;
            const double ls = block_lse<D::NW>(o, M, sm.red);
            __syncthreads();
            double kl = 0.0, gs = 0.0;
            for (int j = threadIdx.x; j < M; j += blockDim.x) {
                const double gj = fmax(wv[j], 0.0);
                gs += gj;
                if (gj > 0.0) kl += gj * (log(gj) - ((double)o[j] - ls));
            }
            kl = block_sum_d<D::NW>(kl, sm.red, 1);
            if (threadIdx.x == 0) {
                atomicAdd(A.audit_kl + 0, kl);
                atomicAdd(A.audit_kl + 1, 1.0);
            }
            __syncthreads();
        }
        const double2 u2 = first ? philox_uniform2(A.W.seed, (uint64_t)w, 0, 1)
                                 : philox_uniform2(A.W.seed, (uint64_t)w, (uint32_t)h, 0);
        const double ud = first ? u2.y : u2.x;
        double tot = 0.0;
        const int b = cta_sample<D::NT>(wv, M, first, ud, sm.red, &tot);
        if (threadIdx.x == 0 && b >= 0 && st.status == 0) {
            if (first)
                A.st.omega[slot] = first_hop_weight(
                    A.G, A.st.sgn[slot], lmc ? center_diel<N>(EP, code) : center_diel<N>(E, code),
                    tot, wv[b], a);
            double loc[3];
            locate_f64(N, b, loc);
            A.st.px[slot] = dadd(A.st.px[slot], dmul(a, loc[0]));
            A.st.py[slot] = dadd(A.st.py[slot], dmul(a, loc[1]));
            A.st.pz[slot] = dadd(A.st.pz[slot], dmul(a, loc[2]));
            A.st.hops[slot] = h + 1;
            atomicAdd(A.ctr + 3, 1ull);
        }
        // lost: no transition, or the solve stayed unconverged after escalation
        if (threadIdx.x == 0 && (b < 0 || st.status != 0)) lw_finish(A, slot, -1);
        __syncthreads();
    }
}

}  // namespace drwc

extern "C" {

DRWC_API void drwc_learned_opts_default(drwc_learned_opts* o) {
    if (!o) return;
    o->slots = 65536;
    o->conf_threshold = -1.5f;
    o->audit_frac = 0.01f;
    o->use_graph = 1;
    o->max_steps = 200000;
}

DRWC_API int drwc_frw_walks_learned(drwc_ctx* ctx, const drwc_structure* s,
                                    const drwc_job_params* p, drwc_net* net,
                                    const drwc_learned_opts* opts, int64_t walk0, int64_t nwalks,
                                    int32_t* end_net, int32_t* hops, double* weight,
                                    double* stats) {
    if (!ctx || !net || walk0 < 0 || nwalks <= 0 || !end_net || !hops || !weight)
        return DRWC_ERR_INVALID;
    if (net_context(net) != ctx || !p || p->N != DRWC_NET_N || net_size(net) != DRWC_NET_N)
        return DRWC_ERR_INVALID;
    drwc_learned_opts o;
    drwc_learned_opts_default(&o);
    if (opts) o = *opts;
    const int S = (int)std::min<int64_t>(std::max(1, o.slots), nwalks);
    drwc_job* j = nullptr;
    int rc = drwc_job_create(ctx, s, p, &j);
    if (rc) return rc;
    struct JobGuard { drwc_job* j; ~JobGuard() { drwc_job_destroy(j); } } guard{j};
    std::lock_guard<std::mutex> lock(ctx->mu);
    DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
    constexpr int N = DRWC_NET_N;
    using D = Cube<N>;
    const int nmat = j->hg.dev.n_mat;
    int per_sm = 0;
    const bool vox = j->hg.dev.n_diel > 0;
    rc = walk_shape<N>(nmat, vox, &per_sm);  // same shared memory as the FDM walk
    if (rc) return rc;
    static bool lw_attr = false;
    if (!lw_attr) {
        DRWC_CUDA_TRY(cudaFuncSetAttribute(lw_fdm_kernel<N>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)WalkSmem<N>::bytes(kMaxMaterials, true)));
        lw_attr = true;
    }
    const int fdm_grid = per_sm * ctx->sm_count;
    // one allocation for everything this run needs
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t r = off; off += (bytes + 255) / 256 * 256; return r; };
    const size_t o_px = take(8 * (size_t)S * 7), o_walk = take(8 * (size_t)S), o_int = take(4 * (size_t)S * 8),
                 o_X = take(2 * (size_t)S * N * N * N), o_O = take(4 * (size_t)S * DRWC_NET_OUT),
                 o_G = take(4 * (size_t)S * DRWC_NET_PANELS), o_list = take(4 * (size_t)S * 2),
                 o_ctr = take(256), o_rec = take(16 * (size_t)nwalks),
                 o_sy = take(8 * (size_t)fdm_grid * D::NNN), o_ss = take(4 * (size_t)fdm_grid * D::NNN);
    void* buf = nullptr;
    rc = ws_get(ctx, WS_RES, off, &buf);
    if (rc) return rc;
    unsigned char* B8 = (unsigned char*)buf;
    LwArgs A{};
    A.S = S;
    A.nwalks = nwalks;
    A.walk0 = walk0;
    A.g = j->hg.dev;
    A.G = j->G;
    A.W = j->P;
    double* dd = (double*)(B8 + o_px);
    A.st.px = dd; A.st.py = dd + S; A.st.pz = dd + 2 * S; A.st.omega = dd + 3 * S;
    A.st.sgn = dd + 4 * S; A.st.a = dd + 5 * S; A.st.epsw = dd + 6 * S;
    A.st.walk = (long long*)(B8 + o_walk);
    int* ii = (int*)(B8 + o_int);
    A.st.hops = ii; A.st.mode = ii + S; A.st.code = ii + 2 * S; A.st.act = ii + 3 * S;
    A.st.grow = ii + 4 * S;
    A.alist = ii + 5 * S;
    A.frow = ii + 6 * S;
    A.X = (__nv_bfloat16*)(B8 + o_X);
    float* Ob = (float*)(B8 + o_O);
    float* Gb = (float*)(B8 + o_G);
    A.O = Ob;
    A.Gh = Gb;
    A.fdm_list = (int*)(B8 + o_list);
    A.fdm_kind = A.fdm_list + S;
    unsigned long long* ctr = (unsigned long long*)(B8 + o_ctr);
    A.ctr = ctr;
    A.fdm_count = (unsigned int*)(ctr + 8);
    A.na = A.fdm_count + 1;
    A.nf = A.fdm_count + 2;
    A.audit_kl = (double*)(ctr + 10);
    A.conf_thresh = o.conf_threshold;
    A.audit_frac = o.audit_frac;
    double* rw = (double*)(B8 + o_rec);
    A.w_out = rw;
    A.end_out = (int32_t*)(rw + nwalks);
    A.hops_out = A.end_out + nwalks;
    double* sy = (double*)(B8 + o_sy);
    float* ss = (float*)(B8 + o_ss);
    DRWC_CUDA_TRY(cudaMemsetAsync(A.st.mode, 0, 4 * (size_t)S, ctx->stream));
    DRWC_CUDA_TRY(cudaMemsetAsync(A.st.hops, 0, 4 * (size_t)S, ctx->stream));
    DRWC_CUDA_TRY(cudaMemsetAsync(ctr, 0, 256, ctx->stream));
    // Each step reads back the number of active slots (and first hops) so the
    // voxeliser, the network and the sampler run on exactly those rows.
    unsigned int hcnt[3] = {0, 0, 0};
    auto step = [&]() -> int {
        DRWC_CUDA_TRY(cudaMemsetAsync(A.fdm_count, 0, 12, ctx->stream));
        lw_prepare_kernel<<<(S * 32 + 255) / 256, 256, 0, ctx->stream>>>(A);
        int r = launch_check(ctx);
        if (r) return r;
        DRWC_CUDA_TRY(cudaMemcpyAsync(hcnt, A.fdm_count, 12, cudaMemcpyDeviceToHost, ctx->stream));
        DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        const int na = (int)hcnt[1], nf = (int)hcnt[2];
        if (na == 0) return DRWC_OK;
        const int g2 = std::min(na, ctx->sm_count * 16);
        lw_voxelise_kernel<<<g2, 256, 0, ctx->stream>>>(A);
        if ((r = launch_check(ctx))) return r;
        r = net_forward_mapped(net, na, A.X, Ob, Gb, A.frow, nf);
        if (r) return r;
        lw_sample_kernel<<<g2, 256, 0, ctx->stream>>>(A);
        if ((r = launch_check(ctx))) return r;
        lw_fdm_kernel<N><<<fdm_grid, D::NT, WalkSmem<N>::bytes(nmat, vox), ctx->stream>>>(A, sy, ss);
        return launch_check(ctx);
    };
    const auto t0 = std::chrono::steady_clock::now();
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int steps = 0;
    unsigned long long h_ctr[8] = {0};
    while (steps < o.max_steps) {
        for (int k = 0; k < 8 && steps < o.max_steps; ++k, ++steps) {
            rc = step();
            if (rc) break;
        }
        if (rc) break;
        DRWC_CUDA_TRY(cudaMemcpyAsync(h_ctr, ctr, sizeof h_ctr, cudaMemcpyDeviceToHost, ctx->stream));
        DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if ((long long)h_ctr[1] >= nwalks) break;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (rc) return rc;
    double akl[2] = {0, 0};
    DRWC_CUDA_TRY(cudaMemcpyAsync(akl, A.audit_kl, 16, cudaMemcpyDeviceToHost, ctx->stream));
    DRWC_CUDA_TRY(cudaMemcpyAsync(end_net, A.end_out, 4 * nwalks, cudaMemcpyDeviceToHost, ctx->stream));
    DRWC_CUDA_TRY(cudaMemcpyAsync(hops, A.hops_out, 4 * nwalks, cudaMemcpyDeviceToHost, ctx->stream));
    DRWC_CUDA_TRY(cudaMemcpyAsync(weight, A.w_out, 8 * nwalks, cudaMemcpyDeviceToHost, ctx->stream));
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (stats) {
        stats[0] = (double)h_ctr[2];                     // network hops
        stats[1] = (double)h_ctr[3];                     // FDM hops (fallback + audit)
        stats[2] = (double)h_ctr[4];                     // fallbacks
        stats[3] = (double)h_ctr[5];                     // audits
        stats[4] = akl[1] > 0 ? akl[0] / akl[1] : 0.0;   // mean audited KL(FDM || net)
        stats[5] = (double)steps;
        stats[6] = secs;
        stats[7] = (double)h_ctr[1];                     // walks finished
    }
    return (long long)h_ctr[1] >= nwalks ? DRWC_OK : DRWC_ERR_TIMEOUT;
}

}  // extern "C"
