// CTA-wide inverse-CDF sampling over one cube's 6N^2 surface values.
//
// Replaces the reference's two torch::multinomial draws (face, then tile:
// dnn_solver_poisson.cpp:92,107; dnn_solver_gradient.cpp:132,137), which
// together draw panel b with probability w_b / sum(w): here one uniform is
// inverted through the FP64 running sum of all 6N^2 weights. Each thread owns
// a contiguous chunk of panels; chunk sums are scanned with warp shuffles and
// one pass over the warp totals, so the draw is deterministic for a given
// uniform.
#pragma once

#include "common.cuh"

namespace drwc {

DRWC_DEV double warp_incl_scan_d(double v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// w: M weights in shared memory. Weight of panel b is |w_b| (use_abs) or
// max(w_b, 0). red: scratch of >= NW + 4 doubles. Returns the panel (all
// threads), -1 when every weight is zero; *total receives sum of weights.
// TAIL = false leaves out the closing barrier (the one that lets the caller
// write red again) for a caller that meets at a barrier of its own first.
template <int NT, bool TAIL = true>
DRWC_DEV int cta_sample(const double* w, int M, bool use_abs, double u, double* red,
                        double* total) {
    constexpr int NW = NT / 32;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int chunk = (M + NT - 1) / NT;
    const int b0 = min(t * chunk, M), b1 = min(b0 + chunk, M);
    double s = 0.0;
    int last = -1;
    for (int b = b0; b < b1; ++b) {
        const double v = use_abs ? fabs(w[b]) : fmax(w[b], 0.0);
        s += v;
        if (v > 0.0) last = b;
    }
    const double incl = warp_incl_scan_d(s);
    if (lane == 31) red[warp] = incl;
    // last non-zero panel (fallback when rounding leaves the target past the end)
    int lastw = last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lastw = max(lastw, __shfl_xor_sync(0xffffffffu, lastw, o));
    int* ired = reinterpret_cast<int*>(red + NW + 2);
    if (lane == 0) ired[warp] = lastw;
    __syncthreads();
    double before = 0.0, tot = 0.0;
    int lastall = -1;
#pragma unroll
    for (int q = 0; q < NW; ++q) {
        const double v = red[q];
        if (q < warp) before += v;
        tot += v;
        lastall = max(lastall, ired[q]);
    }
    const double excl = before + incl - s;  // running sum before this thread's chunk
    const double target = u * tot;
    int pick = 0x7fffffff;
    if (s > 0.0 && excl + s > target) {
        double run = excl;
        for (int b = b0; b < b1; ++b) {
            const double v = use_abs ? fabs(w[b]) : fmax(w[b], 0.0);
            run += v;
            if (run > target && v > 0.0) { pick = b; break; }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pick = min(pick, __shfl_xor_sync(0xffffffffu, pick, o));
    __syncthreads();  // everyone has read red / ired
    if (lane == 0) ired[warp] = pick;
    __syncthreads();
    int best = 0x7fffffff;
#pragma unroll
    for (int q = 0; q < NW; ++q) best = min(best, ired[q]);
    if constexpr (TAIL) __syncthreads();
    if (total) *total = tot;
    if (best == 0x7fffffff) best = lastall;
    return best;
}

// Panel -> point on the surface of [-1,1]^3 (locate_index_simple_kernel,
// cuda_kernels.cu:219-264), FP32 as the reference.
DRWC_DEV void locate_f32(int N, int panel, float out[3]) {
    const int NN = N * N;
    const int f = panel / NN, t = panel % NN;
    const int a = t % N, b = t / N;
    const float t0 = (2.0f * a + 1.0f) / N - 1.0f;
    const float t1 = (2.0f * b + 1.0f) / N - 1.0f;
    switch (f) {
        case 0: out[0] = t0; out[1] = t1; out[2] = -1.0f; break;
        case 1: out[0] = t0; out[1] = t1; out[2] = 1.0f; break;
        case 2: out[0] = t0; out[1] = -1.0f; out[2] = t1; break;
        case 3: out[0] = t0; out[1] = 1.0f; out[2] = t1; break;
        case 4: out[0] = -1.0f; out[1] = t0; out[2] = t1; break;
        default: out[0] = 1.0f; out[1] = t0; out[2] = t1; break;
    }
}

// FP64 form used by the walker: ((2a+1)/N - 1) computed as in the CPU walk.
DRWC_DEV void locate_f64(int N, int panel, double out[3]) {
    const int NN = N * N;
    const int f = panel / NN, t = panel % NN;
    const int a = t % N, b = t / N;
    const double t0 = dsub(ddiv(dadd(dmul(2.0, (double)a), 1.0), (double)N), 1.0);
    const double t1 = dsub(ddiv(dadd(dmul(2.0, (double)b), 1.0), (double)N), 1.0);
    switch (f) {
        case 0: out[0] = t0; out[1] = t1; out[2] = -1.0; break;
        case 1: out[0] = t0; out[1] = t1; out[2] = 1.0; break;
        case 2: out[0] = t0; out[1] = -1.0; out[2] = t1; break;
        case 3: out[0] = t0; out[1] = 1.0; out[2] = t1; break;
        case 4: out[0] = -1.0; out[1] = t0; out[2] = t1; break;
        default: out[0] = 1.0; out[1] = t0; out[2] = t1; break;
    }
}

}  // namespace drwc
