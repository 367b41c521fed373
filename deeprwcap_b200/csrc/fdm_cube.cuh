// CTA-resident mixed-precision solve of one transition cube's FDM system.
//
// The reference's operator (ggft/src/ggft_solver.cpp:447-518 through
// update_matrix :276-290) is A = K * diag(1/eps) with K symmetric positive
// definite:  K_pq = -g_pq, g_pq = eps_p eps_q / (eps_p + eps_q) for face
// neighbours, K_pp = sum_q g_pq + eps_p * (cube faces touched by p).
// ggft's `inner` = eps .* y with K y = e, and gft = A13*inner (:594-596)
// reads eps_c * y_c under each boundary panel. Right-hand sides e restate
// update_ek (:137-274).
//
// One CTA owns one cube; the whole FP32 iteration state stays on chip:
//   each z-column (i, j) is owned by one thread, or by two threads that own
//   its lower and upper halves (N^2 or 2N^2 threads); a thread keeps its
//   cells of r, x, q = K~p (and p) in registers (fully unrolled over k);
//   shared memory holds the search direction p and the three scaled link
//   coefficients cx, cy, cz (cell -> +x/+y/+z neighbour), each padded with N
//   zero guard cells on both ends so the 7-point stencil needs no branches:
//   a link that leaves the cube has coefficient 0, and the neighbour read at
//   c-1 / c-N / c+1 / c+N of a boundary cell lands on a guard or on a cell
//   whose coefficient toward it is 0.
// The inner solve is Jacobi-scaled CG on K~ = S K S (S = diag(K)^-1/2, so
// K~_pp = 1) in FP32. Accuracy comes from FP64 iterative refinement: the
// residual e - K y is evaluated in FP64 from the FP64 permittivity, the FP32
// solve corrects y (kept in FP64 in global scratch), repeated until
// ||e - K y|| <= tol ||e||.
#pragma once

#include "common.cuh"

namespace drwc {

struct FdmParams {
    double tol;        // FP64 relative residual target
    float inner_tol;   // relative residual reduction per FP32 sweep
    int max_outer;     // FP64 refinement sweeps
    int max_inner;     // FP32 CG iterations per sweep
    // Escalation: a cube still above tol after max_outer sweeps gets up to
    // extra_outer more, each with 4 * max_inner iterations, before it is
    // reported not converged (ggft falls back to a direct solve when its
    // iterative one fails, ggft_solver.cpp:565-589).
    int extra_outer;
    // Warm start per solver code (GFT, WVTZ, WVTX, WVTY): the cube solution
    // x = eps .* y of the uniform-permittivity problem (N^3 doubles), or null
    // for a cold start. ggft starts every solve from the same uniform
    // solutions (bootstrap_solve, ggft_solver.cpp:83-135, used by
    // solveWithGuess at :554-560).
    const double* warm[4];
};

// Per-cube solve outcome.
struct FdmStats {
    int iters;       // FP32 CG iterations (all sweeps); for stratified cubes the
                     // FP32 direct solves (cube_solve_planar)
    int sweeps;      // FP64 residual evaluations (refinement sweeps + final check)
    double relres;   // final ||e - K y|| / ||e||
    int status;      // 0 converged, 1 not converged, 2 invalid permittivity
    int escalated;   // 1 when sweeps beyond max_outer were needed
};

#ifndef DRWC_CG_ONE_REDUCTION
#define DRWC_CG_ONE_REDUCTION 0
#endif
#ifndef DRWC_SPLIT_MAX_N
#define DRWC_SPLIT_MAX_N 0
#endif
// Largest N whose FP64 solution y lives in shared memory during the solve
// (8 B per cell more; at N = 16 two cube CTAs still fit on one SM). Larger
// cubes keep y in the caller's global scratch.
#ifndef DRWC_YSMEM_MAX_N
#define DRWC_YSMEM_MAX_N 16
#endif

template <int N>
struct Cube {
    static constexpr int NN = N * N;
    static constexpr int NNN = N * N * N;
    static constexpr bool YSMEM = N <= DRWC_YSMEM_MAX_N;
    // Threads per z-column: two (each owning half of the column) while 2*N^2
    // threads fit in a CTA, else one.
    static constexpr int SPLIT = (N <= DRWC_SPLIT_MAX_N && 2 * NN <= 1024) ? 2 : 1;
    static constexpr int KH = (N + SPLIT - 1) / SPLIT;    // cells per thread
    static constexpr int NT = ((SPLIT * NN + 31) / 32) * 32;  // threads per CTA
    static constexpr int NW = NT / 32;
    static constexpr int PAD = N;                      // guard cells per side
    static constexpr int LEN = NNN + 2 * PAD;
    // dynamic shared memory: [red: 2*NW+8 doubles][rhs: 8 int + 8 double]
    //                        [flags: 8 int][p | cx | cy | cz : LEN floats each]
    //                        [y: N^3 doubles, when YSMEM]
    static constexpr size_t kRedOff = 0;
    static constexpr size_t kRhsIdxOff = kRedOff + sizeof(double) * (2 * NW + 8);
    static constexpr size_t kRhsValOff = kRhsIdxOff + sizeof(int) * kMaxRhs;
    static constexpr size_t kFlagOff = kRhsValOff + sizeof(double) * kMaxRhs;
    static constexpr size_t kArrOff = ((kFlagOff + sizeof(int) * 8 + 127) / 128) * 128;
    static constexpr size_t kArrBytes = ((sizeof(float) * LEN + 15) / 16) * 16;
    // The stratified-cube solver (cube_solve_planar) uses the p|cx|cy|cz
    // region as one block: two transform buffers of N planes x N rows of TS
    // floats (rows 16-byte aligned and padded) and its per-plane tables.
    static constexpr int TS = (N + 3) / 4 * 4 + 4;
    static constexpr size_t kTBuf = (size_t)N * N * TS;            // floats per buffer
    static constexpr size_t kPlanarTables = 16 * 3 * N + 16 * N + 4 * NN + 4 * N + 64;
    static constexpr size_t kPlanarBytes = 2 * kTBuf * sizeof(float) + kPlanarTables;
    static constexpr size_t kArrTotal =
        4 * kArrBytes > kPlanarBytes ? 4 * kArrBytes : (kPlanarBytes + 15) / 16 * 16;
    static constexpr size_t kYOff = kArrOff + kArrTotal;
    static constexpr size_t kSmemBytes = kYOff + (YSMEM ? sizeof(double) * NNN : 0);
    static_assert(kSmemBytes <= 227 * 1024, "cube does not fit in shared memory");
};

template <int N>
struct CubeSmem {
    double* red;     // 2*NW+8 doubles: partial sums / sampling scratch
    int* rhs_idx;
    double* rhs_val;
    int* flags;      // [0] rhs count, [1] invalid-eps flag
    float* p;        // each points at cell 0 (PAD guard cells before it)
    float* cx;
    float* cy;
    float* cz;
    double* y;       // the FP64 solution (YSMEM), else null
    DRWC_DEV static CubeSmem carve(unsigned char* base) {
        using D = Cube<N>;
        CubeSmem s;
        s.red = reinterpret_cast<double*>(base + D::kRedOff);
        s.rhs_idx = reinterpret_cast<int*>(base + D::kRhsIdxOff);
        s.rhs_val = reinterpret_cast<double*>(base + D::kRhsValOff);
        s.flags = reinterpret_cast<int*>(base + D::kFlagOff);
        float* a = reinterpret_cast<float*>(base + D::kArrOff);
        const size_t stride = D::kArrBytes / sizeof(float);
        s.p = a + D::PAD;
        s.cx = a + stride + D::PAD;
        s.cy = a + 2 * stride + D::PAD;
        s.cz = a + 3 * stride + D::PAD;
        s.y = D::YSMEM ? reinterpret_cast<double*>(base + D::kYOff) : nullptr;
        return s;
    }
    // Raw start of the p|cz region (2 arrays) for staging FP64 input.
    DRWC_DEV unsigned char* stage() const { return reinterpret_cast<unsigned char*>(p - Cube<N>::PAD); }
};

// ---------------------------------------------------------------- reductions
// Block sum of a float (all threads receive the result). `slot` selects one of
// two partial buffers so back-to-back reductions need only one barrier each.
template <int NW>
DRWC_DEV float block_sum_f(float v, double* red, int slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[slot * NW + warp] = (double)v;
    __syncthreads();
    double s = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) s += red[slot * NW + w];
    return (float)s;
}

// Two sums in one barrier (slot s uses red[2*s*NW .. 2*s*NW + 2*NW)).
template <int NW>
DRWC_DEV float2 block_sum_f2(float a, float b, double* red, int slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float2* r2 = reinterpret_cast<float2*>(red) + slot * NW;
    if (lane == 0) r2[warp] = make_float2(a, b);
    __syncthreads();
    float sa = 0.f, sb = 0.f;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const float2 v = r2[w];
        sa += v.x;
        sb += v.y;
    }
    return make_float2(sa, sb);
}

template <int NW>
DRWC_DEV double block_sum_d(double v, double* red, int slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[slot * NW + warp] = v;
    __syncthreads();
    double s = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) s += red[slot * NW + w];
    return s;
}

// ----------------------------------------------------------- permittivity
// Where a cube's permittivity comes from. Both sources give the FP64 value of
// a cell, the FP64 conductance g = e_p e_q / (e_p + e_q) of a face link and
// its FP32 counterpart for the inner solve.
//
// EpsGlobal: an arbitrary FP64 array in global memory (the ggft drop-in and
// the batched solver); conductances are computed per use.
struct EpsGlobal {
    const double* __restrict__ eps;
    DRWC_DEV double e64(int c) const { return eps[c]; }
    DRWC_DEV double inv64(int c) const { return 1.0 / eps[c]; }
    DRWC_DEV float e32(int c) const { return (float)eps[c]; }
    DRWC_DEV double g64(int c, int q) const {
        const double a = eps[c], b = eps[q];
        return a * b / (a + b);
    }
    DRWC_DEV float g32(int c, int q) const {
        const float a = (float)eps[c], b = (float)eps[q];
        return a * b / (a + b);
    }
    DRWC_DEV bool valid(int c) const {
        const double v = eps[c];
        return v > 0.0 && isfinite(v);
    }
};

// EpsPalette: piecewise-constant structures (the walker). Each cell holds a
// material id (shared memory, 1 byte); the job's palette of permittivities
// and the table of pair conductances g(m, m') are precomputed once per job,
// so set-up and FP64 sweeps need neither divisions nor global loads.
struct EpsPalette {
    const uint8_t* mat;     // N^3 material ids (shared memory)
    const double* pal;      // P permittivities (shared memory)
    const double* palinv;   // P inverse permittivities
    const double* pair64;   // P x P conductances (shared memory)
    const float* pair32;    // P x P, FP32
    int P;
    DRWC_DEV double e64(int c) const { return pal[mat[c]]; }
    DRWC_DEV double inv64(int c) const { return palinv[mat[c]]; }
    DRWC_DEV float e32(int c) const { return (float)pal[mat[c]]; }
    DRWC_DEV double g64(int c, int q) const { return pair64[mat[c] * P + mat[q]]; }
    DRWC_DEV float g32(int c, int q) const { return pair32[mat[c] * P + mat[q]]; }
    DRWC_DEV bool valid(int c) const { return true; }  // palette checked on the host
};

// EpsPlanar: a stratified cube, whose material depends only on the z index
// (every cell of plane k holds material lm[k]); same palette tables as
// EpsPalette. cube_solve_planar solves such cubes without per-cell
// coefficient arrays.
template <int N>
struct EpsPlanar {
    const int* lm;          // N material ids, one per z index (shared memory)
    const double* pal;
    const double* palinv;
    const double* pair64;
    const float* pair32;
    int P;
    DRWC_DEV int m(int c) const { return lm[c / (N * N)]; }
    DRWC_DEV double e64(int c) const { return pal[m(c)]; }
    DRWC_DEV double inv64(int c) const { return palinv[m(c)]; }
    DRWC_DEV float e32(int c) const { return (float)pal[m(c)]; }
    DRWC_DEV double g64(int c, int q) const { return pair64[m(c) * P + m(q)]; }
    DRWC_DEV float g32(int c, int q) const { return pair32[m(c) * P + m(q)]; }
    DRWC_DEV bool valid(int) const { return true; }  // palette checked on the host
    // Plane k's permittivity, its inverse and the conductances of its x/y
    // links and of the z links up (k, k+1) and down (k-1, k), FP64 and FP32
    // (0 for a link that leaves the cube).
    DRWC_DEV void plane(int k, double& e, double& einv, double& gxy, double& gzu, double& gzd,
                        float& gxy32, float& gzu32, float& gzd32) const {
        const int mk = lm[k];
        e = pal[mk];
        einv = palinv[mk];
        gxy = pair64[mk * P + mk];
        gzu = k + 1 < N ? pair64[mk * P + lm[k + 1]] : 0.0;
        gzd = k > 0 ? pair64[lm[k - 1] * P + mk] : 0.0;
        gxy32 = pair32[mk * P + mk];
        gzu32 = k + 1 < N ? pair32[mk * P + lm[k + 1]] : 0.f;
        gzd32 = k > 0 ? pair32[lm[k - 1] * P + mk] : 0.f;
    }
};

// EpsGlobalPlanar: an FP64 permittivity array in global memory (as EpsGlobal)
// known to hold one value per z plane (planar_cube checked it); conductances
// as EpsGlobal computes them.
template <int N>
struct EpsGlobalPlanar {
    const double* __restrict__ eps;
    DRWC_DEV double e64(int c) const { return eps[c]; }
    DRWC_DEV double inv64(int c) const { return 1.0 / eps[c]; }
    DRWC_DEV float e32(int c) const { return (float)eps[c]; }
    DRWC_DEV void plane(int k, double& e, double& einv, double& gxy, double& gzu, double& gzd,
                        float& gxy32, float& gzu32, float& gzd32) const {
        constexpr int NN = N * N;
        e = eps[k * NN];
        einv = 1.0 / e;
        gxy = e * e / (e + e);
        const float f = (float)e;
        gxy32 = f * f / (f + f);
        gzu = 0.0; gzd = 0.0; gzu32 = 0.f; gzd32 = 0.f;
        if (k + 1 < N) {
            const double b = eps[(k + 1) * NN];
            const float fb = (float)b;
            gzu = e * b / (e + b);
            gzu32 = f * fb / (f + fb);
        }
        if (k > 0) {
            const double b = eps[(k - 1) * NN];
            const float fb = (float)b;
            gzd = b * e / (b + e);
            gzd32 = fb * f / (fb + f);
        }
    }
};

// Whether an FP64 permittivity array holds one valid value per z plane
// (CTA-wide; all threads get the answer).
template <int N>
DRWC_DEV bool planar_cube(const double* __restrict__ eps) {
    constexpr int NN = N * N;
    bool ok = true;
    for (int c = threadIdx.x; c < N * NN; c += blockDim.x) {
        const double v = eps[c], v0 = eps[(c / NN) * NN];
        ok &= v == v0 && v > 0.0 && isfinite(v);
    }
    return __syncthreads_and(ok) != 0;
}

// EpsUniform: permittivity 1 everywhere (the warm-start bootstrap).
struct EpsUniform {
    DRWC_DEV double e64(int) const { return 1.0; }
    DRWC_DEV double inv64(int) const { return 1.0; }
    DRWC_DEV float e32(int) const { return 1.f; }
    DRWC_DEV double g64(int, int) const { return 0.5; }
    DRWC_DEV float g32(int, int) const { return 0.5f; }
    DRWC_DEV bool valid(int) const { return true; }
};

// ------------------------------------------------------------ right-hand side
// Centre sources of ggft_solver.cpp:137-274 (unit source / centre gradient,
// h = 2/N), into smem as (cell, value) pairs. Threads 0..7 each write one
// entry (the shared sums are formed by each of them in the same order).
template <int N, class E>
DRWC_DEV void build_rhs(const E& eps, int code, const CubeSmem<N>& sm) {
    const int t = threadIdx.x;
    if (t >= kMaxRhs) return;
    const double h = 2.0 / N;
    const int c = N / 2;
    auto id = [](int i, int j, int k) { return i + j * N + k * N * N; };
    auto Ev = [&](int cell) { return eps.e64(cell); };
    int n = 0;
    if (N % 2) {
        const int zzz = id(c, c, c);
        if (code == DRWC_GFT) {
            if (t == 0) { sm.rhs_idx[0] = zzz; sm.rhs_val[0] = 1.0; }
            n = 1;
        } else {
            const int stride = code == DRWC_WVTZ ? N * N : code == DRWC_WVTX ? 1 : N;
            const int pp = zzz + stride, mm = zzz - stride;
            const double d_plus = Ev(pp) + Ev(zzz);
            const double d_minus = -(Ev(zzz) + Ev(mm));
            if (t == 0) { sm.rhs_idx[0] = pp;  sm.rhs_val[0] = Ev(pp) / d_plus / h; }
            if (t == 1) { sm.rhs_idx[1] = zzz; sm.rhs_val[1] = Ev(zzz) * (1. / d_plus + 1. / d_minus) / h; }
            if (t == 2) { sm.rhs_idx[2] = mm;  sm.rhs_val[2] = Ev(mm) / d_minus / h; }
            n = 3;
        }
    } else {
        const int zzz = id(c, c, c), zmz = id(c, c - 1, c), zzm = id(c, c, c - 1),
                  zmm = id(c, c - 1, c - 1), mzz = id(c - 1, c, c), mmz = id(c - 1, c - 1, c),
                  mzm = id(c - 1, c, c - 1), mmm = id(c - 1, c - 1, c - 1);
        const double dsum = Ev(zzz) + Ev(zmz) + Ev(zzm) + Ev(zmm) + Ev(mzz) + Ev(mmz) + Ev(mzm) + Ev(mmm);
        if (code == DRWC_GFT) {
            const int cells[8] = {zzz, mzz, zmz, zzm, mmz, mzm, zmm, mmm};
            sm.rhs_idx[t] = cells[t];
            sm.rhs_val[t] = Ev(cells[t]) / dsum;
        } else {
            int plus[4], minus[4];
            double d_minus;
            if (code == DRWC_WVTZ) {
                plus[0] = zzz; plus[1] = mzz; plus[2] = zmz; plus[3] = mmz;
                minus[0] = zzm; minus[1] = mzm; minus[2] = zmm; minus[3] = mmm;
                d_minus = -(Ev(zzm) + Ev(mzm) + Ev(zmm) + Ev(mmm));
            } else if (code == DRWC_WVTX) {
                plus[0] = zzz; plus[1] = zmz; plus[2] = zzm; plus[3] = zmm;
                minus[0] = mzz; minus[1] = mmz; minus[2] = mzm; minus[3] = mmm;
                d_minus = -(Ev(mzz) + Ev(mmz) + Ev(mzm) + Ev(mmm));
            } else {
                plus[0] = zzz; plus[1] = mzz; plus[2] = zzm; plus[3] = mzm;
                minus[0] = zmz; minus[1] = mmz; minus[2] = zmm; minus[3] = mmm;
                d_minus = -(Ev(zmz) + Ev(mmz) + Ev(zmm) + Ev(mmm));
            }
            if (t < 4) {
                sm.rhs_idx[t] = plus[t];
                sm.rhs_val[t] = Ev(plus[t]) / dsum / h * 2;
            } else {
                sm.rhs_idx[t] = minus[t - 4];
                sm.rhs_val[t] = Ev(minus[t - 4]) * (1. / dsum + 1. / d_minus) / h * 2;
            }
        }
        n = 8;
    }
    if (t == 0) sm.flags[0] = n;
}

// Permittivity the first-hop weight is scaled by (ggft_solver.cpp:649-671):
// odd N the centre cell, even N the mean of the four centre cells on the
// minus side of the gradient axis.
template <int N, class E>
DRWC_DEV double center_diel(const E& eps, int code) {
    const int c = N / 2;
    auto id = [](int i, int j, int k) { return i + j * N + k * N * N; };
    auto V = [&](int cell) { return eps.e64(cell); };
    if ((N % 2) || code == DRWC_GFT) return V(id(c, c, c));
    if (code == DRWC_WVTZ)
        return (V(id(c, c, c - 1)) + V(id(c - 1, c - 1, c - 1)) + V(id(c, c - 1, c - 1)) +
                V(id(c - 1, c, c - 1))) / 4;
    if (code == DRWC_WVTX)
        return (V(id(c - 1, c, c)) + V(id(c - 1, c - 1, c)) + V(id(c - 1, c, c - 1)) +
                V(id(c - 1, c - 1, c - 1))) / 4;
    return (V(id(c, c - 1, c)) + V(id(c - 1, c - 1, c)) + V(id(c, c - 1, c - 1)) +
            V(id(c - 1, c - 1, c - 1))) / 4;
}

#ifndef DRWC_PREGS_MAX_N
#define DRWC_PREGS_MAX_N 16
#endif
#ifndef DRWC_MIN_BLOCKS_SMALL
#define DRWC_MIN_BLOCKS_SMALL 2
#endif

template <int N>
struct CubeTraits {
    // Keep the thread's own column of p in registers too (saves three shared
    // loads per cell and iteration) when the register file allows it.
    static constexpr bool kPRegs = N <= DRWC_PREGS_MAX_N;
    // Resident CTAs per SM the register allocation is sized for (N <= 16;
    // larger cubes run one CTA per SM, bounded by shared memory).
    static constexpr int kMinBlocks = N <= 16 ? DRWC_MIN_BLOCKS_SMALL : 1;
};

// --------------------------------------------------------------- the solver
// eps:  permittivity source (EpsGlobal / EpsPalette), cell i + j*N + k*N*N.
// ys:   N^3 doubles of global scratch for the FP64 solution y of K y = e
//       (unused when Cube<N>::YSMEM: y then lives in shared memory).
// ss:   N^3 floats of global scratch (the Jacobi scale S, each thread's own
//       cells only).
// On return (all threads) cube_y<N>(ys) holds y and the stats are filled;
// shared memory p/cx/cy/cz are free for the caller.
#ifndef DRWC_SOLVE_INLINE
#define DRWC_SOLVE_INLINE 0
#endif
#if DRWC_SOLVE_INLINE
#define DRWC_SOLVE_ATTR __device__ __forceinline__
#else
#define DRWC_SOLVE_ATTR __device__ __noinline__
#endif

// The kernel's dynamic shared memory; the cube's arrays sit at its start.
// Carving them from this symbol (not from pointers handed in) lets the
// compiler address them as shared memory.
extern __shared__ __align__(128) unsigned char drwc_dyn_smem[];

// Where cube_solve leaves the solution y: shared memory for N <= the YSMEM
// bound, else the caller's global scratch.
template <int N>
DRWC_DEV const double* cube_y(const double* ys) {
    if constexpr (Cube<N>::YSMEM) return CubeSmem<N>::carve(drwc_dyn_smem).y;
    else return ys;
}

template <int N, class E>
DRWC_SOLVE_ATTR void cube_solve(const E eps, double* __restrict__ ys, float* __restrict__ ss,
                                int code, const FdmParams& prm, FdmStats* st) {
    const CubeSmem<N> sm = CubeSmem<N>::carve(drwc_dyn_smem);
    using D = Cube<N>;
    constexpr int NN = D::NN;
    constexpr int NW = D::NW;
    constexpr int KH = D::KH;
    constexpr bool PR = CubeTraits<N>::kPRegs;
    const int t = threadIdx.x;
    const bool active = t < D::SPLIT * NN;
    const int col = active ? t % NN : 0;
    const int i = col % N, j = col / N;
    const int k0 = active ? (t / NN) * KH : 0;       // first k of this thread's cells
    const int kend = active ? min(k0 + KH, N) : 0;    // one past the last k
    auto own = [&](int kk) { return k0 + kk < kend; };
    double* __restrict__ Y;
    if constexpr (D::YSMEM) Y = sm.y;
    else Y = ys;

    // ---- setup 1: validity, Jacobi scale S = diag(K)^-1/2 (FP32; into p,
    //      which is free until the CG starts, and into ss), y = the warm
    //      start (or 0), guards zeroed, right-hand side.
    const double* __restrict__ warm = prm.warm[code & 3];
    if (t == 0) sm.flags[1] = 0;
    for (int g = t; g < D::PAD; g += D::NT) {
        sm.p[-D::PAD + g] = 0.f; sm.p[D::NNN + g] = 0.f;
        sm.cx[-D::PAD + g] = 0.f; sm.cx[D::NNN + g] = 0.f;
        sm.cy[-D::PAD + g] = 0.f; sm.cy[D::NNN + g] = 0.f;
        sm.cz[-D::PAD + g] = 0.f; sm.cz[D::NNN + g] = 0.f;
    }
    build_rhs<N>(eps, code, sm);
    __syncthreads();
    {
        bool bad = false;
#pragma unroll
        for (int kk = 0; kk < KH; ++kk) {
            if (!own(kk)) continue;
            const int k = k0 + kk;
            const int c = col + k * NN;
            bad |= !eps.valid(c);
            const float ec = eps.e32(c);
            float d = 0.f;
            d += (i + 1 < N) ? eps.g32(c, c + 1) : ec;
            d += (i > 0) ? eps.g32(c, c - 1) : ec;
            d += (j + 1 < N) ? eps.g32(c, c + N) : ec;
            d += (j > 0) ? eps.g32(c, c - N) : ec;
            d += (k + 1 < N) ? eps.g32(c, c + NN) : ec;
            d += (k > 0) ? eps.g32(c, c - NN) : ec;
            const float sc = rsqrtf(d);
            sm.p[c] = sc;
            ss[c] = sc;
            Y[c] = warm ? warm[c] * eps.inv64(c) : 0.0;
        }
        if (bad) atomicOr(&sm.flags[1], 1);
    }
    __syncthreads();
    if (sm.flags[1]) {
        st->status = 2; st->iters = 0; st->sweeps = 0; st->relres = CUDART_NAN;
        st->escalated = 0;
        return;
    }
    // ||e|| (FP64) from the rhs table; which of this thread's cells carry a
    // source term (bit kk)
    double enorm2 = 0.0;
    const int nrhs = sm.flags[0];
    unsigned int rmask = 0u;
    for (int v = 0; v < nrhs; ++v) {
        const double ev = sm.rhs_val[v];
        enorm2 += ev * ev;
        const int cell = sm.rhs_idx[v];
        const int kk = cell / NN - k0;
        if (active && cell % NN == col && kk >= 0 && kk < KH) rmask |= 1u << kk;
    }
    const double enorm = sqrt(enorm2);

    float r[KH], x[KH], q[KH], pr[(PR || DRWC_CG_ONE_REDUCTION) ? KH : 1];
    // FP64 residual r64 = e - K y into the next inner rhs b = S r64 (FP32
    // registers); returns ||r64|| / ||e|| (all threads). first: the sweep
    // from the warm start, where S is still in p and (y in global scratch)
    // the neighbours' y are formed from the warm table instead of being read
    // back from scratch the other threads just wrote.
    auto residual = [&](bool first) -> double {
        auto yv = [&](int cell) -> double {
            if constexpr (!D::YSMEM) {
                if (first) return warm[cell] * eps.inv64(cell);
            }
            return Y[cell];
        };
        double rn2 = 0.0;
#pragma unroll
        for (int kk = 0; kk < KH; ++kk) {
            if (!own(kk)) { r[kk] = 0.f; continue; }
            const int k = k0 + kk;
            const int c = col + k * NN;
            const double ec = eps.e64(c);
            const double yc = Y[c];
            double diag = 0.0, off = 0.0;
            if (i + 1 < N) { const double g = eps.g64(c, c + 1); diag += g; off += g * yv(c + 1); } else diag += ec;
            if (i > 0) { const double g = eps.g64(c, c - 1); diag += g; off += g * yv(c - 1); } else diag += ec;
            if (j + 1 < N) { const double g = eps.g64(c, c + N); diag += g; off += g * yv(c + N); } else diag += ec;
            if (j > 0) { const double g = eps.g64(c, c - N); diag += g; off += g * yv(c - N); } else diag += ec;
            if (k + 1 < N) { const double g = eps.g64(c, c + NN); diag += g; off += g * yv(c + NN); } else diag += ec;
            if (k > 0) { const double g = eps.g64(c, c - NN); diag += g; off += g * yv(c - NN); } else diag += ec;
            double e_c = 0.0;
            if ((rmask >> kk) & 1u)
                for (int v = 0; v < nrhs; ++v)
                    if (sm.rhs_idx[v] == c) e_c = sm.rhs_val[v];
            const double r64 = e_c - (diag * yc - off);
            rn2 += r64 * r64;
            const float sc = first ? sm.p[c] : ss[c];
            r[kk] = (float)((double)sc * r64);
        }
        rn2 = block_sum_d<NW>(rn2, sm.red, 0);
        return sqrt(rn2) / enorm;
    };
    int sweeps = 0;
    double relres = 1.0;
    if (warm) {
        // sweep 0 from the warm start (y and S written above, visible after
        // the barrier that follows set-up 1)
        relres = residual(true);
        sweeps = 1;
    } else {
        // y = 0, so e - K y = e (non-zero only at the centre source)
#pragma unroll
        for (int kk = 0; kk < KH; ++kk) {
            r[kk] = 0.f;
            if (own(kk) && ((rmask >> kk) & 1u)) {
                const int c = col + (k0 + kk) * NN;
                for (int v = 0; v < nrhs; ++v)
                    if (sm.rhs_idx[v] == c) r[kk] = (float)((double)sm.p[c] * sm.rhs_val[v]);
            }
        }
    }
    if (relres > prm.tol) {
        // ---- setup 2 (only when the warm start is not already the solution):
        //      scaled link coefficients cx/cy/cz = g * S_p * S_q, S from p.
#pragma unroll
        for (int kk = 0; kk < KH; ++kk) {
            if (!own(kk)) continue;
            const int k = k0 + kk;
            const int c = col + k * NN;
            const float sc = sm.p[c];
            float vx = 0.f, vy = 0.f, vz = 0.f;
            if (i + 1 < N) vx = eps.g32(c, c + 1) * sc * sm.p[c + 1];
            if (j + 1 < N) vy = eps.g32(c, c + N) * sc * sm.p[c + N];
            if (k + 1 < N) vz = eps.g32(c, c + NN) * sc * sm.p[c + NN];
            sm.cx[c] = vx; sm.cy[c] = vy; sm.cz[c] = vz;
        }
        __syncthreads();  // every S read before the CG overwrites p
    }
    int total_inner = 0, outer = 0;
    int status = relres <= prm.tol ? 0 : 1;
#pragma unroll 1
    for (outer = 0; status != 0 && outer < prm.max_outer + prm.extra_outer; ++outer) {
        const int max_inner = outer < prm.max_outer ? prm.max_inner : 4 * prm.max_inner;
        // ---- FP32 CG on K~ d = b, d in x[], starting from 0. The reduction
        //      it needs is set so this sweep brings ||e - K y|| to about half
        //      the target (no deeper than inner_tol per sweep).
        float rr = 0.f;
#pragma unroll
        for (int kk = 0; kk < KH; ++kk) {
            x[kk] = 0.f;
            if (own(kk)) {
                sm.p[col + (k0 + kk) * NN] = r[kk];
                rr += r[kk] * r[kk];
            } else {
                r[kk] = 0.f;
            }
            if constexpr (PR) pr[kk] = r[kk];
        }
#if DRWC_CG_ONE_REDUCTION
        // Chronopoulos-Gear CG: one fused reduction (r.r, w.r) and two
        // barriers per iteration; p and s = K~p live only in registers and
        // the stencil runs on r, which is the vector shared through smem.
        (void)rr;
        float sv[KH], gamma_old = 1.f, alpha_old = 1.f, stop2 = 0.f;
        int it = 0;
#pragma unroll 1
        for (it = 0; it <= max_inner; ++it) {
            __syncthreads();  // r published
            float gam = 0.f, del = 0.f;
            if (active) {
                float rm = k0 > 0 ? sm.p[col + (k0 - 1) * NN] : 0.f;
                float czm = k0 > 0 ? sm.cz[col + (k0 - 1) * NN] : 0.f;
                float rc = r[0];
#pragma unroll
                for (int kk = 0; kk < KH; ++kk) {
                    const int k = k0 + kk;
                    const int c = col + k * NN;
                    float rn;
                    if (kk + 1 < KH) rn = r[(kk + 1) % KH];
                    else rn = (k + 1 < N) ? sm.p[c + NN] : 0.f;
                    if (own(kk)) {
                        const float czc = sm.cz[c];
                        const float nb = sm.cx[c - 1] * sm.p[c - 1] + sm.cx[c] * sm.p[c + 1] +
                                         sm.cy[c - N] * sm.p[c - N] + sm.cy[c] * sm.p[c + N] +
                                         czm * rm + czc * rn;
                        q[kk] = rc - nb;  // w = K~ r
                        gam += rc * rc;
                        del += q[kk] * rc;
                        czm = czc;
                    } else {
                        q[kk] = 0.f;
                    }
                    rm = rc; rc = rn;
                }
            }
            const float2 gd = block_sum_f2<NW>(gam, del, sm.red, it & 1);
            if (it == 0) {
                const float want = fmaxf(prm.inner_tol, (float)(0.5 * prm.tol / relres));
                stop2 = gd.x * want * want;
            }
            if (gd.x <= stop2 || it == max_inner) break;
            const float beta = it == 0 ? 0.f : gd.x / gamma_old;
            const float alpha = gd.x / (gd.y - beta * gd.x / alpha_old);
            gamma_old = gd.x;
            alpha_old = alpha;
#pragma unroll
            for (int kk = 0; kk < KH; ++kk) {
                if (own(kk)) {
                    pr[kk] = (it == 0 ? 0.f : beta * pr[kk]) + r[kk];
                    sv[kk] = (it == 0 ? 0.f : beta * sv[kk]) + q[kk];
                    x[kk] += alpha * pr[kk];
                    r[kk] -= alpha * sv[kk];
                    sm.p[col + (k0 + kk) * NN] = r[kk];
                }
            }
        }
#else
        rr = block_sum_f<NW>(rr, sm.red, 1);  // barrier also publishes p
        const float want = fmaxf(prm.inner_tol, (float)(0.5 * prm.tol / relres));
        const float stop2 = rr * want * want;
        int it = 0;
#pragma unroll 1
        for (it = 0; it < max_inner && rr > stop2; ++it) {
            // q = K~ p  (K~_pp = 1)
            float pq = 0.f;
            if (active) {
                // z-neighbours across the split come from shared memory
                float pm = k0 > 0 ? sm.p[col + (k0 - 1) * NN] : 0.f;
                float czm = k0 > 0 ? sm.cz[col + (k0 - 1) * NN] : 0.f;
                float pc;
                if constexpr (PR) pc = pr[0];
                else pc = sm.p[col + k0 * NN];
#pragma unroll
                for (int kk = 0; kk < KH; ++kk) {
                    const int k = k0 + kk;
                    const int c = col + k * NN;
                    float pn;
                    if constexpr (PR) {
                        if (kk + 1 < KH) pn = pr[(kk + 1) % KH];
                        else pn = (k + 1 < N) ? sm.p[c + NN] : 0.f;
                    } else {
                        pn = (k + 1 < N) ? sm.p[c + NN] : 0.f;
                    }
                    if (own(kk)) {
                        const float czc = sm.cz[c];
                        const float nb = sm.cx[c - 1] * sm.p[c - 1] + sm.cx[c] * sm.p[c + 1] +
                                         sm.cy[c - N] * sm.p[c - N] + sm.cy[c] * sm.p[c + N] +
                                         czm * pm + czc * pn;
                        q[kk] = pc - nb;
                        pq += pc * q[kk];
                        czm = czc;
                    } else {
                        q[kk] = 0.f;
                    }
                    pm = pc; pc = pn;
                }
            }
            pq = block_sum_f<NW>(pq, sm.red, 0);
            const float alpha = rr / pq;
            float rr2 = 0.f;
#pragma unroll
            for (int kk = 0; kk < KH; ++kk) {
                if (own(kk)) {
                    if constexpr (PR) x[kk] += alpha * pr[kk];
                    else x[kk] += alpha * sm.p[col + (k0 + kk) * NN];
                    r[kk] -= alpha * q[kk];
                    rr2 += r[kk] * r[kk];
                }
            }
            rr2 = block_sum_f<NW>(rr2, sm.red, 1);
            const float beta = rr2 / rr;
            rr = rr2;
#pragma unroll
            for (int kk = 0; kk < KH; ++kk) {
                if (own(kk)) {
                    const int c = col + (k0 + kk) * NN;
                    if constexpr (PR) {
                        pr[kk] = r[kk] + beta * pr[kk];
                        sm.p[c] = pr[kk];
                    } else {
                        sm.p[c] = r[kk] + beta * sm.p[c];
                    }
                }
            }
            __syncthreads();
        }
#endif
        total_inner += it;
        // ---- y += S d
#pragma unroll
        for (int kk = 0; kk < KH; ++kk) {
            if (own(kk)) {
                const int c = col + (k0 + kk) * NN;
                Y[c] += (double)ss[c] * (double)x[kk];
            }
        }
        __syncthreads();  // y of the neighbours visible
        relres = residual(false);
        ++sweeps;
        if (relres <= prm.tol) status = 0;
    }
    st->status = status;
    st->escalated = outer > prm.max_outer;
    st->iters = total_inner;
    st->sweeps = sweeps;
    st->relres = relres;
    __syncthreads();
}

// Block sum of a float through FP32 partials read back four at a time (one
// shared-memory wavefront per four warps); fixed order, all threads get it.
// Its two slots lie after red[0..NW) (block_sum_d's slot 0), so it can follow
// a block_sum_d without a barrier in between.
template <int NW>
DRWC_DEV float block_sum_f4(float v, double* red, int slot) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    float* rf = reinterpret_cast<float*>(red + NW) + slot * ((NW + 3) / 4) * 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) rf[warp] = v;
    __syncthreads();
    float s = 0.f;
    if constexpr (NW % 4 == 0) {
        const float4* r4 = reinterpret_cast<const float4*>(rf);
#pragma unroll
        for (int w = 0; w < NW / 4; ++w) {
            const float4 q = r4[w];
            s += q.x; s += q.y; s += q.z; s += q.w;
        }
    } else {
#pragma unroll
        for (int w = 0; w < NW; ++w) s += rf[w];
    }
    return s;
}

// ------------------------------------------------------------ stratified cubes
// The system K y = e of cube_solve for a cube whose material depends only on
// the z index. Every x/y link of plane k has conductance g_k = g(k,k) =
// eps_k / 2 and a cell on an x or y face adds eps_k = 2 g_k to its diagonal,
// so the x/y part of K on plane k is g_k (T (x) I + I (x) T), where T is the
// N x N matrix tridiag(-1, 2, -1) with 3 at both ends, the same for every
// plane. T's eigenvectors are the cell-centred sine modes
//   u_m(i) = s_m sin(pi (m+1) (2i+1) / (2N)),  lambda_m = 4 sin^2(pi (m+1) / (2N)),
// m = 0..N-1, s_m = sqrt(2/N) (sqrt(1/N) for m = N-1), orthonormal. In that
// basis K splits into N^2 independent tridiagonal systems along z, one per
// mode (m, n):  (zd_k + (lambda_m + lambda_n) g_k) v_k - gz_k v_{k+1}
// - gz_{k-1} v_{k-1} = rhs_k,  with gz_k = g(k,k+1) and zd_k the z part of
// the diagonal (eps_k on the top and bottom faces). So K d = r is solved
// exactly, without iterations: a 2-D sine transform of r (two passes through
// shared memory), one Thomas solve per mode (one thread each, in registers)
// and the inverse transform (two passes). This direct solve runs in FP32
// as the inner solver of cube_solve's FP64 iterative refinement: the FP64
// residual e - K y is formed from the FP64 permittivity (so the refinement
// converges to the FP64 solution whatever the x/y operator's last-bit
// agreement with g_k T), and every sweep gains about as many digits as FP32
// carries. FdmStats::iters counts the direct solves.
//
// Shared memory (the p|cx|cy|cz block of the cube layout): two transform
// buffers of N planes x N rows x TS floats, then the tables
//   T64 (3N double2): {g_k, gz_k}, {zd_k, eps_k}, {1/eps_k, 0}
//   T32 (N float4):   {g_k, gz_k, zd_k, eps_k} in FP32
//   U (N x N floats): U[m][i] = u_m(i);  L (N floats): lambda_m.
// E provides plane(k, ...) (EpsPlanar, EpsGlobalPlanar) and e64(c). On
// return cube_y<N>(ys) holds y, as after cube_solve.
template <int N, class E>
DRWC_SOLVE_ATTR void cube_solve_planar(const E eps, double* __restrict__ ys, int code,
                                       const FdmParams& prm, FdmStats* st) {
    const CubeSmem<N> sm = CubeSmem<N>::carve(drwc_dyn_smem);
    using D = Cube<N>;
    static_assert(D::SPLIT == 1, "planar solve: one thread per column");
    constexpr int NN = D::NN;
    constexpr int NW = D::NW;
    constexpr int TS = D::TS;          // transform row stride (floats)
    constexpr int TP = N * TS;         // transform plane stride
    const int t = threadIdx.x;
    const bool active = t < NN;
    const int col = active ? t : 0;
    const int i = col % N, j = col / N;
    // the other index pair of the transform passes: a = t % N (lanes), b = t / N
    const int ta = col % N, tb = col / N;
    double* __restrict__ Y;
    if constexpr (D::YSMEM) Y = sm.y;
    else Y = ys;
    float* XB = sm.p - D::PAD;               // transform buffer 1
    float* ZB = XB + D::kTBuf;               // transform buffer 2
    double2* T64 = reinterpret_cast<double2*>(ZB + D::kTBuf);
    float4* T32 = reinterpret_cast<float4*>(T64 + 3 * N);
    float* U = reinterpret_cast<float*>(T32 + N);
    float* L = U + NN;
    const double* __restrict__ warm = prm.warm[code & 3];

    // ---- set-up: plane tables, sine modes, right-hand side, y = the warm
    //      start (or 0). The warm-start values of this thread's column are
    //      requested first, so their trip to L2 overlaps the table set-up.
    double w0[N];
    if (active && warm) {
#pragma unroll
        for (int k = 0; k < N; ++k) w0[k] = warm[col + k * NN];
    }
    if (t < N) {
        const int k = t;
        double e, einv, gxy, gzu, gzd;
        float gxy32, gzu32, gzd32;
        eps.plane(k, e, einv, gxy, gzu, gzd, gxy32, gzu32, gzd32);
        const double zd = (k + 1 < N ? gzu : e) + (k > 0 ? gzd : e);
        T64[3 * k] = make_double2(gxy, gzu);
        T64[3 * k + 1] = make_double2(zd, e);
        T64[3 * k + 2] = make_double2(einv, 0.0);
        const float e32 = (float)e;
        const float zd32 = (k + 1 < N ? gzu32 : e32) + (k > 0 ? gzd32 : e32);
        T32[k] = make_float4(gxy32, gzu32, zd32, e32);
        const float sl = sinpif((float)(k + 1) / (float)(2 * N));
        L[k] = 4.f * sl * sl;
    }
    if (active) {  // U[m][i], m = tb, i = ta
        const float s = tb + 1 < N ? sqrtf(2.f / N) : sqrtf(1.f / N);
        U[tb * N + ta] = s * sinpif((float)((tb + 1) * (2 * ta + 1)) / (float)(2 * N));
    }
    build_rhs<N>(eps, code, sm);
    __syncthreads();  // tables written
    if (active) {
#pragma unroll
        for (int k = 0; k < N; ++k) Y[col + k * NN] = warm ? w0[k] * T64[3 * k + 2].x : 0.0;
    }
    __syncthreads();
    double enorm2 = 0.0;
    const int nrhs = sm.flags[0];
    unsigned int rmask = 0u;  // bit k: cell (col, k) carries a source term
    for (int v = 0; v < nrhs; ++v) {
        const double ev = sm.rhs_val[v];
        enorm2 += ev * ev;
        const int cell = sm.rhs_idx[v];
        if (active && cell % NN == col) rmask |= 1u << (cell / NN);
    }
    const double enorm = sqrt(enorm2);
    // x/y neighbour offsets clamped to the cell itself outside the cube, and
    // 0/1 weights: the residual's loads are unconditional and in bounds
    const bool xm = i > 0, xp = i + 1 < N, ym = j > 0, yp = j + 1 < N;
    const int nxy = (int)xm + (int)xp + (int)ym + (int)yp;
    const int oxm = xm ? -1 : 0, oxp = xp ? 1 : 0, oym = ym ? -N : 0, oyp = yp ? N : 0;
    const double fxm = xm, fxp = xp, fym = ym, fyp = yp;

    float r[N];
    // FP64 residual r64 = e - K y into r (FP32); returns ||r64|| / ||e||
    auto residual = [&]() -> double {
        double rn2 = 0.0, rn2b = 0.0;
        double yb = 0.0;              // y of the cell below
        double yc = Y[col];
        double gzb = 0.0;             // g(k-1,k)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int c = col + k * NN;
            const double ya = k + 1 < N ? Y[c + NN] : 0.0;
            const double2 a = T64[3 * k], b = T64[3 * k + 1];
            const double sxy = fxm * Y[c + oxm] + fxp * Y[c + oxp] + fym * Y[c + oym] +
                               fyp * Y[c + oyp];
            const double diag = (double)nxy * a.x + (double)(4 - nxy) * b.y + b.x;
            const double off = a.x * sxy + a.y * ya + gzb * yb;
            double e_c = 0.0;
            if ((rmask >> k) & 1u)
                for (int v = 0; v < nrhs; ++v)
                    if (sm.rhs_idx[v] == c) e_c = sm.rhs_val[v];
            const double r64 = e_c - (diag * yc - off);
            if (active) {
                if (k & 1) rn2b += r64 * r64;
                else rn2 += r64 * r64;
            }
            r[k] = active ? (float)r64 : 0.f;
            yb = yc;
            yc = ya;
            gzb = a.y;
        }
        rn2 = block_sum_d<NW>(rn2 + rn2b, sm.red, 0);
        return sqrt(rn2) / enorm;
    };
    // one sum of a transform pass: row[0..N) . w[0..N) (w in registers)
    // (four partial sums: short dependency chains)
    auto dot_row = [&](const float* row, const float (&w)[N]) -> float {
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
        if constexpr (N % 4 == 0) {
#pragma unroll
            for (int q = 0; q < N / 4; ++q) {
                const float4 v = reinterpret_cast<const float4*>(row)[q];
                a0 = fmaf(v.x, w[4 * q], a0);
                a1 = fmaf(v.y, w[4 * q + 1], a1);
                a2 = fmaf(v.z, w[4 * q + 2], a2);
                a3 = fmaf(v.w, w[4 * q + 3], a3);
            }
        } else {
#pragma unroll
            for (int q = 0; q < N; ++q) {
                if (q % 4 == 0) a0 = fmaf(row[q], w[q], a0);
                else if (q % 4 == 1) a1 = fmaf(row[q], w[q], a1);
                else if (q % 4 == 2) a2 = fmaf(row[q], w[q], a2);
                else a3 = fmaf(row[q], w[q], a3);
            }
        }
        return (a0 + a1) + (a2 + a3);
    };
    // FP32 direct solve K d = r (r in this thread's column): d into r
    auto direct_solve = [&]() {
        float w[N];
        // r -> buffer 1 as [k][j][i]
        if (active) {
#pragma unroll
            for (int k = 0; k < N; ++k) XB[k * TP + j * TS + i] = r[k];
        }
        __syncthreads();
        // pass 1 (thread m = ta, j = tb): P[k][m][j] = sum_i U[m][i] X[k][j][i]
        if (active) {
#pragma unroll
            for (int q = 0; q < N; ++q) w[q] = U[ta * N + q];
#pragma unroll 4
            for (int k = 0; k < N; ++k) ZB[k * TP + ta * TS + tb] = dot_row(XB + k * TP + tb * TS, w);
        }
        __syncthreads();
        // pass 2 (thread n = ta, m = tb): mode (m, n) = sum_j U[n][j] P[k][m][j],
        // then the mode's tridiagonal solve along k, all in registers
        float v[N];
        if (active) {
#pragma unroll
            for (int q = 0; q < N; ++q) w[q] = U[ta * N + q];
#pragma unroll 4
            for (int k = 0; k < N; ++k) v[k] = dot_row(ZB + k * TP + tb * TS, w);
            const float lam = L[ta] + L[tb];
            float gprev = 0.f, fprev = 0.f, gzb = 0.f;
            float g[N];
#pragma unroll
            for (int k = 0; k < N; ++k) {  // Thomas, forward
                const float4 tk = T32[k];
                // sub- and super-diagonal -gz: den_k = b_k - gz_{k-1}^2 / den_{k-1}
                const float den = fmaf(lam, tk.x, tk.z) + gzb * gprev;
                const float inv = __frcp_rn(den);
                g[k] = -tk.y * inv;
                fprev = (v[k] + gzb * fprev) * inv;
                v[k] = fprev;
                gprev = g[k];
                gzb = tk.y;
            }
#pragma unroll
            for (int k = N - 2; k >= 0; --k) v[k] -= g[k] * v[k + 1];  // back
        }
        __syncthreads();  // buffer 1 free
        // modes -> buffer 1 as [k][m][n]
        if (active) {
#pragma unroll
            for (int k = 0; k < N; ++k) XB[k * TP + tb * TS + ta] = v[k];
        }
        __syncthreads();
        // pass 3 (thread j = ta, m = tb): Q[k][j][m] = sum_n U[n][j] V[k][m][n]
        if (active) {
#pragma unroll
            for (int q = 0; q < N; ++q) w[q] = U[q * N + ta];
#pragma unroll 4
            for (int k = 0; k < N; ++k) ZB[k * TP + ta * TS + tb] = dot_row(XB + k * TP + tb * TS, w);
        }
        __syncthreads();
        // pass 4 (thread i, j): d[k] = sum_m U[m][i] Q[k][j][m]
        if (active) {
#pragma unroll
            for (int q = 0; q < N; ++q) w[q] = U[q * N + i];
#pragma unroll 4
            for (int k = 0; k < N; ++k) r[k] = dot_row(ZB + k * TP + j * TS, w);
        }
    };
    int sweeps = 0;
    double relres = 1.0;
    if (warm) {
        relres = residual();
        sweeps = 1;
    } else {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r[k] = 0.f;
            if ((rmask >> k) & 1u) {
                const int c = col + k * NN;
                for (int v = 0; v < nrhs; ++v)
                    if (sm.rhs_idx[v] == c) r[k] = (float)sm.rhs_val[v];
            }
        }
    }
    int solves = 0, outer = 0;
    int status = relres <= prm.tol ? 0 : 1;
#pragma unroll 1
    for (outer = 0; status != 0 && outer < prm.max_outer + prm.extra_outer; ++outer) {
        direct_solve();
        ++solves;
        // ---- y += d
        if (active) {
#pragma unroll
            for (int k = 0; k < N; ++k) Y[col + k * NN] += (double)r[k];
        }
        __syncthreads();  // y of the neighbours visible
        relres = residual();
        ++sweeps;
        if (relres <= prm.tol) status = 0;
    }
    st->status = status;
    st->escalated = outer > prm.max_outer;
    st->iters = solves;
    st->sweeps = sweeps;
    st->relres = relres;
    __syncthreads();
}

// Surface values gft[b] = eps_c * y_c under panel b (ggft panel order,
// ggft_solver.h:65-77). Cooperative over the CTA; writes through `put(b, v)`.
template <int N, class E, class Put>
DRWC_DEV void for_each_panel(const E& eps, const double* __restrict__ ys, Put put) {
    constexpr int NN = N * N;
    for (int b = threadIdx.x; b < 6 * NN; b += blockDim.x) {
        const int f = b / NN, tt = b % NN;
        const int a = tt % N, bb = tt / N;
        int c;
        switch (f) {
            case 0: c = a + bb * N; break;                        // z-: (i,j,0)
            case 1: c = a + bb * N + (N - 1) * NN; break;         // z+
            case 2: c = a + bb * NN; break;                       // y-: (i,0,k)
            case 3: c = a + (N - 1) * N + bb * NN; break;         // y+
            case 4: c = a * N + bb * NN; break;                   // x-: (0,j,k)
            default: c = (N - 1) + a * N + bb * NN; break;        // x+
        }
        put(b, eps.e64(c) * ys[c]);
    }
}


// The same values with panel b written by thread b / chunk (contiguous chunks
// of chunk = ceil(6N^2 / NT) panels, the chunks cta_sample<NT> reads): a
// thread can sample right after writing its own chunk, without a barrier.
template <int N, int NT, class E, class Put>
DRWC_DEV void for_each_panel_chunked(const E& eps, const double* __restrict__ ys, Put put) {
    constexpr int NN = N * N;
    constexpr int M = 6 * NN;
    constexpr int CH = (M + NT - 1) / NT;
    const int b0 = min((int)threadIdx.x * CH, M), b1 = min(b0 + CH, M);
    for (int b = b0; b < b1; ++b) {
        const int f = b / NN, tt = b % NN;
        const int a = tt % N, bb = tt / N;
        int c;
        switch (f) {
            case 0: c = a + bb * N; break;
            case 1: c = a + bb * N + (N - 1) * NN; break;
            case 2: c = a + bb * NN; break;
            case 3: c = a + (N - 1) * N + bb * NN; break;
            case 4: c = a * N + bb * NN; break;
            default: c = (N - 1) + a * N + bb * NN; break;
        }
        put(b, eps.e64(c) * ys[c]);
    }
}

}  // namespace drwc
