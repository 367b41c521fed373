// Structure geometry of the FRW transition engine, shared by the single-job
// walker (walker.cu) and the multi-job server (serve.cu): the device view of
// a structure (conductor boxes, stratified dielectric, dielectric blocks, a
// uniform grid of boxes for the nearest-conductor search, the material
// palette), the Gaussian surface, the walk start point, cube voxelisation and
// the fixed-order reduction of walk records. Host-side packing of a
// structure into one device blob is here as well.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "fdm_cube.cuh"
#include "host.cuh"
#include "sample.cuh"

namespace drwc {

FdmParams make_params(const drwc_fdm_opts* o, int N);

constexpr double kEps0FfPerUm = 8.8541878128e-3;  // vacuum permittivity, fF/um
constexpr int kBruteBoxes = 16;                  // <= this many boxes: scan all

constexpr int kMaxMaterials = 32;              // distinct permittivities per structure

struct DevGeom {
    int n_boxes, n_nets, n_layers, n_diel;
    const double* box;      // n_boxes x 6 (lo xyz, hi xyz)
    const int* net;         // n_boxes
    const double* zlo;      // n_layers
    const int* lmat;        // n_layers material ids
    const double* diel;     // n_diel x 7 (eps slot unused on the device)
    const int* dmat;        // n_diel material ids
    const double* pal;      // n_mat distinct permittivities
    const double* pair64;   // n_mat x n_mat conductances e e' / (e + e')
    const float* pair32;
    int n_mat;
    double encl_lo[3], encl_hi[3];
    // uniform grid over the enclosure (CSR cell -> boxes)
    int gdim[3];
    double gcell[3];
    double gmin_cell;
    const int* gstart;      // ncells + 1
    const int* gitems;
    // Gaussian surface made of rectangles (the union of the master's grown
    // boxes): n_grect x 9 doubles {axis, side, x, u0, u1, v0, v1, cumulative
    // sampling mass, 1 / sampling density factor}; none: the Gauss box
    const double* grect;
    int n_grect;
};

struct Gauss {
    double lo[3], hi[3], area[6], total;
};

struct WalkParams {
    int N, max_hops, master;
    double stop;
    uint64_t seed;
    FdmParams prm;
    // optional hop log: centre + half-width (4 doubles) and solver code per hop
    double* log;
    int* log_code;
    unsigned int* log_count;
    unsigned int log_cap;
};

// ------------------------------------------------------------------ geometry
DRWC_DEV double box_dist(const double* b, const double r[3]) {
    double d = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double lo = dsub(b[a], r[a]);
        const double hi = dsub(r[a], b[3 + a]);
        const double m = lo > hi ? lo : hi;
        if (m > d) d = m;
    }
    return d;
}

DRWC_DEV double encl_dist(const DevGeom& g, const double r[3]) {
    double best = CUDART_INF;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double d1 = dsub(r[a], g.encl_lo[a]);
        const double d2 = dsub(g.encl_hi[a], r[a]);
        if (d1 < best) best = d1;
        if (d2 < best) best = d2;
    }
    return best;
}

// Nearest conductor (L-infinity), called by a whole warp: the enclosure wins
// ties, then the lowest box index. Every lane gets the result.
DRWC_DEV void nearest(const DevGeom& g, const double r[3], double* d_out, int* net_out) {
    const int lane = threadIdx.x & 31;
    double best = CUDART_INF;
    int bidx = 0x7fffffff;
    if (g.n_boxes <= kBruteBoxes || g.gstart == nullptr) {
        for (int b = lane; b < g.n_boxes; b += 32) {
            const double d = box_dist(g.box + 6 * b, r);
            if (d < best || (d == best && b < bidx)) { best = d; bidx = b; }
        }
    } else {
        // rings of grid cells at Chebyshev distance `ring` from the point's
        // cell, the ring's cells spread over the lanes; the warp agrees on
        // the best box after each ring, so it stops at the same ring as a
        // scan in ring order would
        int ci[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            int v = (int)floor((r[a] - g.encl_lo[a]) / g.gcell[a]);
            ci[a] = v < 0 ? 0 : (v >= g.gdim[a] ? g.gdim[a] - 1 : v);
        }
        const double dwall = encl_dist(g, r);
        const int rmax = max(g.gdim[0], max(g.gdim[1], g.gdim[2]));
        for (int ring = 0; ring <= rmax; ++ring) {
            // boxes not met in rings < ring lie at least (ring-1) cells away
            const double reach = (double)(ring - 1) * g.gmin_cell * (1.0 - 1e-12);
            if (ring > 1 && (best < reach || dwall < reach)) break;
            const int side = 2 * ring + 1, per = 4 * (side - 1);
            const int cells = ring == 0 ? 1 : 2 * side * side + (side - 2) * per;
            for (int t = lane; t < cells; t += 32) {
                int dx, dy, dz;
                if (ring == 0) {
                    dx = dy = dz = 0;
                } else if (t < 2 * side * side) {  // the two full faces z = -ring, +ring
                    const int u = t % (side * side);
                    dz = t < side * side ? -ring : ring;
                    dx = u % side - ring;
                    dy = u / side - ring;
                } else {  // the square border of each layer in between
                    const int u = t - 2 * side * side, k = u % per, e = side - 1;
                    dz = -ring + 1 + u / per;
                    if (k < e) { dx = -ring + k; dy = -ring; }
                    else if (k < 2 * e) { dx = ring; dy = -ring + (k - e); }
                    else if (k < 3 * e) { dx = ring - (k - 2 * e); dy = ring; }
                    else { dx = -ring; dy = ring - (k - 3 * e); }
                }
                const int x = ci[0] + dx, y = ci[1] + dy, z = ci[2] + dz;
                if (x < 0 || x >= g.gdim[0] || y < 0 || y >= g.gdim[1] || z < 0 || z >= g.gdim[2])
                    continue;
                const int cell = x + g.gdim[0] * (y + g.gdim[1] * z);
                for (int it = g.gstart[cell]; it < g.gstart[cell + 1]; ++it) {
                    const int b = g.gitems[it];
                    const double d = box_dist(g.box + 6 * b, r);
                    if (d < best || (d == best && b < bidx)) { best = d; bidx = b; }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
                if (ob < best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
        if (ob < best || (ob == best && oi < bidx)) { best = ob; bidx = oi; }
    }
    const double dw = encl_dist(g, r);
    if (dw <= best) {
        *d_out = dw;
        *net_out = g.n_nets;
    } else {
        *d_out = best;
        *net_out = g.net[bidx];
    }
}

// Material id at a point: first containing dielectric block, else the last
// stratified layer with zlo <= z (layer 0 below all of them).
// Layer index of height z: the last layer l with zlo[l] <= z among the
// first layers that all satisfy it (scan in order, stop at the first layer
// above z; layer 0 below all of them). The bounds are read eight at a time,
// so a cube's layer search waits for one memory round trip per eight layers
// instead of one per layer.
DRWC_DEV int layer_index(const DevGeom& g, double z) {
    int li = 0;
    for (int l0 = 0; l0 < g.n_layers; l0 += 8) {
        double zz[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) zz[e] = l0 + e < g.n_layers ? g.zlo[l0 + e] : 0.0;
        bool stop = false;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            if (!stop && l0 + e < g.n_layers) {
                if (z >= zz[e]) li = l0 + e;
                else stop = true;
            }
        }
        if (stop) break;
    }
    return li;
}

DRWC_DEV int mat_at(const DevGeom& g, const double p[3]) {
    for (int b = 0; b < g.n_diel; ++b) {
        const double* D = g.diel + 7 * b;
        if (p[0] >= D[0] && p[0] <= D[3] && p[1] >= D[1] && p[1] <= D[4] && p[2] >= D[2] &&
            p[2] <= D[5])
            return g.dmat[b];
    }
    if (g.n_layers <= 0) return 0;
    return g.lmat[layer_index(g, p[2])];
}

// Cell-centre offsets (2i+1)/N - 1, rounded exactly as the CPU walk computes them.
template <int N>
DRWC_DEV void centre_offsets(double* tco) {
    for (int i = threadIdx.x; i < N; i += blockDim.x)
        tco[i] = dsub(ddiv(dadd(dmul(2.0, (double)i), 1.0), (double)N), 1.0);
}

template <int N>
DRWC_DEV void voxelise(const DevGeom& g, const double c[3], double a, const double* tco,
                       uint8_t* mat) {
    for (int v = threadIdx.x; v < N * N * N; v += blockDim.x) {
        const int i = v % N, j = (v / N) % N, k = v / (N * N);
        double p[3];
        p[0] = dadd(c[0], dmul(a, tco[i]));
        p[1] = dadd(c[1], dmul(a, tco[j]));
        p[2] = dadd(c[2], dmul(a, tco[k]));
        mat[v] = (uint8_t)mat_at(g, p);
    }
}

// Structures without dielectric blocks: a cell's material is the layer of
// its z index (mat_at's layer rule at that index's centre z), decided once
// per index into lm (shared, N ints).
template <int N>
DRWC_DEV void plane_layers(const DevGeom& g, const double c[3], double a, const double* tco,
                           int* lm) {
    const int t = threadIdx.x;
    if (t < N) {
        const double z = dadd(c[2], dmul(a, tco[t]));
        lm[t] = g.n_layers > 0 ? g.lmat[layer_index(g, z)] : 0;
    }
}

template <int N>
DRWC_DEV void voxelise_planes(const DevGeom& g, const double c[3], double a, const double* tco,
                              uint8_t* mat, int* lm) {
    const int t = threadIdx.x;
    plane_layers<N>(g, c, a, tco, lm);
    __syncthreads();
    for (int v = t; v < N * N * N; v += blockDim.x) mat[v] = (uint8_t)lm[v / (N * N)];
}

// Shared memory beyond the solver's: material ids, cell-centre offsets, the
// palette and its pair-conductance tables.
template <int N>
struct VoxScratch;

template <int N>
struct WalkSmem {
    __host__ __device__ static size_t base(int P) {
        return Cube<N>::kSmemBytes + ((size_t)N * N * N + 15) / 16 * 16 + 8 * N + 16 * P +
               8 * (size_t)P * P + 4 * (size_t)P * P + 16;
    }
    // vox: room for the separable voxeliser's scratch after the rest (walks
    // in structures with dielectric blocks)
    __host__ __device__ static size_t bytes(int P, bool vox = false) {
        return vox ? (base(P) + 15) / 16 * 16 + (sizeof(VoxScratch<N>) + 15) / 16 * 16 : base(P);
    }
};

// Per-entry sums of one batch of walk records in a fixed order, for a block
// of 256 threads: entry e (0..n_nets = ground; n_entries collects the lost
// walks, net -1) over all walks. out[3e..3e+2] = {sum w, sum w^2, count}.
// The order of every addition depends only on the records, never on how
// the walks were scheduled.
DRWC_DEV void reduce_entry(int e, int n_entries, long long nw, const int32_t* __restrict__ end,
                           const double* __restrict__ w, double* __restrict__ out) {
    double s = 0, s2 = 0, cnt = 0;
    for (long long i = threadIdx.x; i < nw; i += blockDim.x) {
        const int ne = end[i] < 0 ? n_entries : end[i];
        if (ne == e) {
            const double v = w[i];
            s += v; s2 += v * v; cnt += 1.0;
        }
    }
    __shared__ double r0[256], r1[256], r2[256];
    r0[threadIdx.x] = s; r1[threadIdx.x] = s2; r2[threadIdx.x] = cnt;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            r0[threadIdx.x] += r0[threadIdx.x + o];
            r1[threadIdx.x] += r1[threadIdx.x + o];
            r2[threadIdx.x] += r2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[3 * e + 0] = r0[0];
        out[3 * e + 1] = r1[0];
        out[3 * e + 2] = r2[0];
    }
}

// Start point of walk w on the Gaussian surface (Philox counter (w, 0, 0..1)):
// a face chosen by area, a uniform point on it; the outward sign of that
// face and the solver code of its normal (WVTX/Y/Z) for the first hop.
DRWC_DEV void walk_start_point(const Gauss& G, const DevGeom& g, uint64_t seed, uint64_t w,
                               double r[3], double* sgn_out, int* code) {
    const double2 u = philox_uniform2(seed, w, 0, 0);
    const double2 v = philox_uniform2(seed, w, 0, 1);
    const double target = dmul(u.x, G.total);
    if (g.n_grect > 0) {
        // the first rectangle whose cumulative area exceeds the target
        int lo = 0, hi = g.n_grect - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (g.grect[9 * mid + 7] > target) hi = mid;
            else lo = mid + 1;
        }
        const double* R = g.grect + 9 * lo;
        const int axis = (int)R[0], side = (int)R[1];
        const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
        r[t0] = dadd(R[3], dmul(u.y, dsub(R[4], R[3])));
        r[t1] = dadd(R[5], dmul(v.x, dsub(R[6], R[5])));
        r[axis] = R[2];
        // the outward sign, times the importance ratio of this rectangle
        // (first_hop_weight multiplies by G.total, the total sampling mass)
        *sgn_out = side ? R[8] : -R[8];
        *code = axis == 0 ? DRWC_WVTX : axis == 1 ? DRWC_WVTY : DRWC_WVTZ;
        return;
    }
    double run = 0.0;
    int f = 5;
    for (int q = 0; q < 6; ++q) {
        run = dadd(run, G.area[q]);
        if (run > target) { f = q; break; }
    }
    const int axis = f < 2 ? 2 : f < 4 ? 1 : 0;
    const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
    r[t0] = dadd(G.lo[t0], dmul(u.y, dsub(G.hi[t0], G.lo[t0])));
    r[t1] = dadd(G.lo[t1], dmul(v.x, dsub(G.hi[t1], G.lo[t1])));
    r[axis] = (f & 1) ? G.hi[axis] : G.lo[axis];
    *sgn_out = (f & 1) ? 1.0 : -1.0;
    *code = axis == 0 ? DRWC_WVTX : axis == 1 ? DRWC_WVTY : DRWC_WVTZ;
}

// First-hop walk weight (fF) from the drawn gradient panel value's sign, the
// summed |gradient| `tot`, the centre permittivity and the cube half-width.
DRWC_DEV double first_hop_weight(const Gauss& G, double sgn_out, double eps_w, double tot,
                                 double g_b, double a) {
    const double sg = g_b < 0.0 ? -1.0 : 1.0;
    double om = dmul(-sgn_out, G.total);
    om = dmul(om, eps_w);
    om = dmul(om, tot);
    om = dmul(om, sg);
    om = ddiv(om, a);
    return dmul(om, kEps0FfPerUm);
}

// Cell-centre points of a cube in the frame the gradient head works in: the
// gradient axis becomes z'. rot = 0: identity; rot = 1 (x gradient):
// (x, y, z) = (z', x', y'); rot = 2 (y gradient): (x, y, z) = (y', z', x').
DRWC_DEV void rotated_point(const double c[3], double a, const double* tco, int i, int j, int k,
                            int rot, double p[3]) {
    int ax, ay, az;  // original-axis offsets taken from rotated indices
    if (rot == 1) { ax = k; ay = i; az = j; }
    else if (rot == 2) { ax = j; ay = k; az = i; }
    else { ax = i; ay = j; az = k; }
    p[0] = dadd(c[0], dmul(a, tco[ax]));
    p[1] = dadd(c[1], dmul(a, tco[ay]));
    p[2] = dadd(c[2], dmul(a, tco[az]));
}

DRWC_DEV void unrotate(int rot, const double v[3], double out[3]) {
    if (rot == 1) { out[0] = v[2]; out[1] = v[0]; out[2] = v[1]; }
    else if (rot == 2) { out[0] = v[1]; out[1] = v[2]; out[2] = v[0]; }
    else { out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; }
}

DRWC_DEV int rot_of_code(int code) { return code == DRWC_WVTX ? 1 : code == DRWC_WVTY ? 2 : 0; }

// Separable voxelisation. The cell-centre coordinates c + a*t_i are monotone
// in i on every axis (explicitly rounded FP64, as the CPU walk computes
// them), so a dielectric block's inclusive bounds select a contiguous index
// range per axis, and the layer rule gives one layer per z index. Per cube:
// the 3N coordinates, the layer material of each z index and the index
// ranges of the blocks that reach the cube (in block order: the first
// containing block wins, as in mat_at); per voxel a few integer tests. The
// result is mat_at's at every cell centre.
constexpr int kVoxMaxBlocks = 64;  // blocks reaching one cube; beyond: mat_at per voxel
constexpr int kVoxMaskFrom = 4;    // more blocks than this: per-axis block masks

template <int N>
struct VoxScratch {
    double crd[3][N];
    int lm[N];
    int rel[kVoxMaxBlocks][7];  // i0, i1, j0, j1, k0, k1 (original axes), material
    uint64_t msk[3][N];         // bit q: block q's range holds this index (axis, index)
    int nrel;
    float lmax;                 // largest layer permittivity over the z indices (FP32)
};

template <int N>
DRWC_DEV void vox_prepare(const DevGeom& g, const double c[3], double a, const double* tco,
                          VoxScratch<N>& vs, const double* palsm = nullptr,
                          __nv_bfloat16* pv = nullptr) {
    const int t = threadIdx.x;
    // warp 0: the layer of each z index, from the lane's own coordinate, and
    // the largest layer permittivity; with pv set, pv[t] = the BF16 value
    // (eps / largest) of z index t, which is the cube's value at every cell
    // of that index when no block reaches the cube
    if (t < 32) {
        const double* pal = palsm ? palsm : g.pal;
        float pm = 0.f;
        int m = 0;
        if (t < N) {
            const double z = dadd(c[2], dmul(a, tco[t]));
            m = g.n_layers > 0 ? g.lmat[layer_index(g, z)] : 0;
            vs.lm[t] = m;
            pm = (float)pal[m];
        }
        for (int o = 16; o > 0; o >>= 1) pm = fmaxf(pm, __shfl_xor_sync(0xffffffffu, pm, o));
        if (t == 0) vs.lmax = pm;
        if (pv && t < N) pv[t] = __float2bfloat16((float)pal[m] * (1.f / pm));
    }
    // warp 1 (warp 0 in CTAs of one warp): the cell-centre coordinates, then
    // the blocks that reach the cube, in block order, while warp 0 decides
    // the layers
    const int scan_warp = blockDim.x >= 64 ? 1 : 0;
    if ((t >> 5) == scan_warp) {
        const int lane = t & 31;
        for (int q = lane; q < 3 * N; q += 32) vs.crd[q / N][q % N] = dadd(c[q / N], dmul(a, tco[q % N]));
        if (lane == 0) vs.nrel = 0;
        __syncwarp();
        for (int b0 = 0; b0 < g.n_diel; b0 += 32) {
            const int b = b0 + lane;
            int r[6] = {0, -1, 0, -1, 0, -1};
            bool hit = false;
            double Dv[6];
            int dm = 0;
            if (b < g.n_diel) {
                const double* D = g.diel + 7 * b;
#pragma unroll
                for (int e = 0; e < 6; ++e) Dv[e] = D[e];
                dm = g.dmat[b];
                hit = true;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    // the centres are non-decreasing along an axis, so the
                    // ones inside [lo, hi] form the range [first >= lo,
                    // last <= hi]: two binary searches
                    const double* x = vs.crd[d];
                    const double lo = Dv[d], hi = Dv[3 + d];
                    int i0 = 0, n = N;
                    while (n > 0) {  // first index with x >= lo
                        const int h = n >> 1;
                        if (x[i0 + h] < lo) { i0 += h + 1; n -= h + 1; }
                        else n = h;
                    }
                    int i1 = 0;
                    n = N;
                    while (n > 0) {  // first index with x > hi
                        const int h = n >> 1;
                        if (x[i1 + h] <= hi) { i1 += h + 1; n -= h + 1; }
                        else n = h;
                    }
                    i1 -= 1;
                    if (i0 > i1) { i0 = N; i1 = -1; }
                    r[2 * d] = i0;
                    r[2 * d + 1] = i1;
                    hit &= i0 <= i1;
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            const int base = vs.nrel;
            if (hit) {
                const int q = base + __popc(m & ((1u << lane) - 1));
                if (q < kVoxMaxBlocks) {
#pragma unroll
                    for (int e = 0; e < 6; ++e) vs.rel[q][e] = r[e];
                    vs.rel[q][6] = dm;
                }
            }
            __syncwarp();
            if (lane == 0) vs.nrel = base + __popc(m);
            __syncwarp();
        }
    }
    __syncthreads();
    // many blocks: one mask per axis index, so a voxel's first block is the
    // lowest bit of three ANDed masks (block order kept)
    const int nrel = vs.nrel;
    if (nrel > kVoxMaskFrom && nrel <= kVoxMaxBlocks) {
        if (t < 3 * N) {
            const int d = t / N, i = t % N;
            uint64_t m = 0;
            for (int q = 0; q < nrel; ++q)
                if (i >= vs.rel[q][2 * d] && i <= vs.rel[q][2 * d + 1]) m |= 1ull << q;
            vs.msk[d][i] = m;
        }
        __syncthreads();
    }
}

// Material of voxel (i, j, k) of the (possibly rotated) cube.
template <int N>
DRWC_DEV int vox_material(const DevGeom& g, const VoxScratch<N>& vs, const double c[3], double a,
                          const double* tco, int i, int j, int k, int rot) {
    int ox, oy, oz;
    if (rot == 1) { ox = k; oy = i; oz = j; }
    else if (rot == 2) { ox = j; oy = k; oz = i; }
    else { ox = i; oy = j; oz = k; }
    if (vs.nrel > kVoxMaxBlocks) {  // too many blocks reach this cube: test them all
        double p[3];
        rotated_point(c, a, tco, i, j, k, rot, p);
        return mat_at(g, p);
    }
    if (vs.nrel > kVoxMaskFrom) {
        const uint64_t m = vs.msk[0][ox] & vs.msk[1][oy] & vs.msk[2][oz];
        return m ? vs.rel[__ffsll((long long)m) - 1][6] : vs.lm[oz];
    }
    for (int q = 0; q < vs.nrel; ++q) {
        const int* r = vs.rel[q];
        if (ox >= r[0] && ox <= r[1] && oy >= r[2] && oy <= r[3] && oz >= r[4] && oz <= r[5])
            return r[6];
    }
    return vs.lm[oz];
}

// The cells of a cube whose vox_prepare has run (see voxelise_net).
template <int N>
DRWC_DEV void voxelise_cells(const DevGeom& g, const double c[3], double a, int rot,
                             const double* tco, const double* palsm, uint8_t* matsm,
                             __nv_bfloat16* X, double* eps64, float* red, VoxScratch<N>& vs) {
    constexpr int NNN = N * N * N;
    if (vs.nrel == 0) {
        // no block reaches the cube: a cell's material is its layer, one per
        // index along the original z axis, and the largest permittivity is
        // the largest of those layers'
        const float inv = 1.f / vs.lmax;
        for (int v = threadIdx.x; v < NNN; v += blockDim.x) {
            const int i = v % N, j = (v / N) % N, k = v / (N * N);
            const int m = vs.lm[rot == 1 ? j : rot == 2 ? i : k];
            matsm[v] = (uint8_t)m;
            const double e = palsm[m];
            X[v] = __float2bfloat16((float)e * inv);
            if (eps64) eps64[v] = e;
        }
        __syncthreads();
        return;
    }
    float mx = 0.f;
    for (int v = threadIdx.x; v < NNN; v += blockDim.x) {
        const int i = v % N, j = (v / N) % N, k = v / (N * N);
        const int m = vox_material<N>(g, vs, c, a, tco, i, j, k, rot);
        matsm[v] = (uint8_t)m;
        mx = fmaxf(mx, (float)palsm[m]);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    float m = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, red[w]);
    const float inv = 1.f / m;
    for (int v = threadIdx.x; v < NNN; v += blockDim.x) {
        const double e = palsm[matsm[v]];
        X[v] = __float2bfloat16((float)e * inv);
        if (eps64) eps64[v] = e;
    }
    __syncthreads();
}

// CTA-wide: voxelise one cube (rotated frame) into BF16 eps / max eps and,
// optionally, FP64 eps. vs: shared scratch (separable voxelisation).
template <int N>
DRWC_DEV void voxelise_net(const DevGeom& g, const double c[3], double a, int rot,
                           const double* tco, const double* palsm, uint8_t* matsm,
                           __nv_bfloat16* X, double* eps64, float* red, VoxScratch<N>& vs) {
    vox_prepare<N>(g, c, a, tco, vs, palsm);
    voxelise_cells<N>(g, c, a, rot, tco, palsm, matsm, X, eps64, red, vs);
}

// log-sum-exp of M FP32 values over the CTA (all threads get it).
template <int NW>
DRWC_DEV double block_lse(const float* o, int M, double* red) {
    float mx = -1e30f;
    for (int j = threadIdx.x; j < M; j += blockDim.x) mx = fmaxf(mx, o[j]);
    for (int s = 16; s > 0; s >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, s));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = (double)mx;
    __syncthreads();
    double m = red[0];
    for (int w = 1; w < NW; ++w) m = fmax(m, red[w]);
    __syncthreads();
    double se = 0.0;
    for (int j = threadIdx.x; j < M; j += blockDim.x) se += exp((double)o[j] - m);
    se = block_sum_d<NW>(se, red, 0);
    return log(se) + m;
}

struct HostGeom {
    std::vector<double> box, zlo, diel, pal, pair64, grect;
    std::vector<float> pair32;
    std::vector<int> net, gstart, gitems, lmat, dmat;
    DevGeom dev{};
    void* dbuf = nullptr;
    std::vector<unsigned char> blob;  // every device array, 256-byte aligned, in one block
    size_t o_box = 0, o_net = 0, o_zlo = 0, o_lmat = 0, o_dmat = 0, o_pal = 0, o_p64 = 0,
           o_p32 = 0, o_diel = 0, o_gs = 0, o_gi = 0, o_gr = 0;
};

inline int validate(const drwc_structure* s) {
    if (!s || s->n_boxes < 1 || s->n_nets < 1 || s->n_nets > DRWC_MAX_NETS || !s->boxes)
        return DRWC_ERR_INVALID;
    if (s->n_layers < 0 || s->n_diel < 0) return DRWC_ERR_INVALID;
    if (s->n_layers > 0 && (!s->layer_zlo || !s->layer_eps)) return DRWC_ERR_INVALID;
    if (s->n_diel > 0 && !s->diel) return DRWC_ERR_INVALID;
    for (int a = 0; a < 3; ++a)
        if (!(s->encl_hi[a] > s->encl_lo[a])) return DRWC_ERR_GEOMETRY;
    for (int b = 0; b < s->n_boxes; ++b) {
        const drwc_box& B = s->boxes[b];
        if (B.net < 0 || B.net >= s->n_nets) return DRWC_ERR_INVALID;
        for (int a = 0; a < 3; ++a)
            if (!(B.hi[a] > B.lo[a]) || B.lo[a] < s->encl_lo[a] || B.hi[a] > s->encl_hi[a])
                return DRWC_ERR_GEOMETRY;
    }
    for (int l = 0; l < s->n_layers; ++l) {
        if (!(s->layer_eps[l] > 0)) return DRWC_ERR_INVALID;
        if (l > 0 && !(s->layer_zlo[l] >= s->layer_zlo[l - 1])) return DRWC_ERR_INVALID;
    }
    for (int d = 0; d < s->n_diel; ++d)
        if (!(s->diel[d].eps > 0)) return DRWC_ERR_INVALID;
    return DRWC_OK;
}

// Host side of a structure: material palette, pair conductances, uniform
// grid, all packed into h->blob; h->dev gets the scalar fields (pointers are
// set by bind_geom once the blob has a device address).
inline int pack_geom(const drwc_structure* s, HostGeom* h) {
    const int nb = s->n_boxes;
    h->box.resize(6 * nb);
    h->net.resize(nb);
    for (int b = 0; b < nb; ++b) {
        for (int a = 0; a < 3; ++a) {
            h->box[6 * b + a] = s->boxes[b].lo[a];
            h->box[6 * b + 3 + a] = s->boxes[b].hi[a];
        }
        h->net[b] = s->boxes[b].net;
    }
    h->zlo.assign(s->layer_zlo, s->layer_zlo + s->n_layers);
    // material palette: distinct permittivities of layers and blocks
    h->pal.clear();
    auto mat_of = [&](double e) {
        for (size_t m = 0; m < h->pal.size(); ++m)
            if (h->pal[m] == e) return (int)m;
        h->pal.push_back(e);
        return (int)h->pal.size() - 1;
    };
    h->lmat.resize(s->n_layers);
    for (int l = 0; l < s->n_layers; ++l) h->lmat[l] = mat_of(s->layer_eps[l]);
    if (s->n_layers == 0) mat_of(1.0);  // vacuum when no layer is given
    h->dmat.resize(s->n_diel);
    for (int d = 0; d < s->n_diel; ++d) h->dmat[d] = mat_of(s->diel[d].eps);
    const int P = (int)h->pal.size();
    if (P > kMaxMaterials) return DRWC_ERR_GEOMETRY;
    h->pair64.resize((size_t)P * P);
    h->pair32.resize((size_t)P * P);
    for (int a = 0; a < P; ++a)
        for (int b = 0; b < P; ++b) {
            const double e1 = h->pal[a], e2 = h->pal[b];
            h->pair64[a * P + b] = e1 * e2 / (e1 + e2);
            const float f1 = (float)e1, f2 = (float)e2;
            h->pair32[a * P + b] = f1 * f2 / (f1 + f2);
        }
    h->diel.resize(7 * s->n_diel);
    for (int d = 0; d < s->n_diel; ++d) {
        for (int a = 0; a < 3; ++a) {
            h->diel[7 * d + a] = s->diel[d].lo[a];
            h->diel[7 * d + 3 + a] = s->diel[d].hi[a];
        }
        h->diel[7 * d + 6] = s->diel[d].eps;
    }
    // uniform grid: about 4 cells per box, at most 128 per axis
    double ext[3], vol = 1.0;
    for (int a = 0; a < 3; ++a) {
        ext[a] = s->encl_hi[a] - s->encl_lo[a];
        vol *= ext[a];
    }
    const double hcell = std::cbrt(vol / (4.0 * nb));
    int dim[3];
    double cell[3], minc = 1e300;
    for (int a = 0; a < 3; ++a) {
        dim[a] = (int)std::min(128.0, std::max(1.0, std::ceil(ext[a] / hcell)));
        cell[a] = ext[a] / dim[a];
        minc = std::min(minc, cell[a]);
    }
    const int ncell = dim[0] * dim[1] * dim[2];
    std::vector<std::vector<int>> lists(ncell);
    for (int b = 0; b < nb; ++b) {
        int lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = (int)std::floor((s->boxes[b].lo[a] - s->encl_lo[a]) / cell[a]) - 1;
            hi[a] = (int)std::floor((s->boxes[b].hi[a] - s->encl_lo[a]) / cell[a]) + 1;
            lo[a] = std::max(0, lo[a]);
            hi[a] = std::min(dim[a] - 1, hi[a]);
        }
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int x = lo[0]; x <= hi[0]; ++x) {
                    // keep the box in every cell its (slightly grown) extent touches
                    const double cx0 = s->encl_lo[0] + x * cell[0], cx1 = cx0 + cell[0];
                    const double cy0 = s->encl_lo[1] + y * cell[1], cy1 = cy0 + cell[1];
                    const double cz0 = s->encl_lo[2] + z * cell[2], cz1 = cz0 + cell[2];
                    const double tol = 1e-9 * minc;
                    if (s->boxes[b].lo[0] <= cx1 + tol && s->boxes[b].hi[0] >= cx0 - tol &&
                        s->boxes[b].lo[1] <= cy1 + tol && s->boxes[b].hi[1] >= cy0 - tol &&
                        s->boxes[b].lo[2] <= cz1 + tol && s->boxes[b].hi[2] >= cz0 - tol)
                        lists[x + dim[0] * (y + dim[1] * z)].push_back(b);
                }
    }
    h->gstart.assign(ncell + 1, 0);
    for (int c = 0; c < ncell; ++c) h->gstart[c + 1] = h->gstart[c] + (int)lists[c].size();
    h->gitems.clear();
    for (int c = 0; c < ncell; ++c) h->gitems.insert(h->gitems.end(), lists[c].begin(), lists[c].end());
    if (h->gitems.empty()) h->gitems.push_back(0);

    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
    h->o_box = take(h->box.size() * 8);
    h->o_net = take(h->net.size() * 4);
    h->o_zlo = take(std::max<size_t>(1, h->zlo.size()) * 8);
    h->o_lmat = take(std::max<size_t>(1, h->lmat.size()) * 4);
    h->o_dmat = take(std::max<size_t>(1, h->dmat.size()) * 4);
    h->o_pal = take(h->pal.size() * 8);
    h->o_p64 = take(h->pair64.size() * 8);
    h->o_p32 = take(h->pair32.size() * 4);
    h->o_diel = take(std::max<size_t>(1, h->diel.size()) * 8);
    h->o_gs = take(h->gstart.size() * 4);
    h->o_gi = take(h->gitems.size() * 4);
    h->o_gr = take(std::max<size_t>(1, h->grect.size()) * 8);
    std::vector<unsigned char>& hb = h->blob;
    hb.assign(off, 0);
    std::memcpy(hb.data() + h->o_box, h->box.data(), h->box.size() * 8);
    std::memcpy(hb.data() + h->o_net, h->net.data(), h->net.size() * 4);
    if (!h->zlo.empty()) std::memcpy(hb.data() + h->o_zlo, h->zlo.data(), h->zlo.size() * 8);
    if (!h->lmat.empty()) std::memcpy(hb.data() + h->o_lmat, h->lmat.data(), h->lmat.size() * 4);
    if (!h->dmat.empty()) std::memcpy(hb.data() + h->o_dmat, h->dmat.data(), h->dmat.size() * 4);
    std::memcpy(hb.data() + h->o_pal, h->pal.data(), h->pal.size() * 8);
    std::memcpy(hb.data() + h->o_p64, h->pair64.data(), h->pair64.size() * 8);
    std::memcpy(hb.data() + h->o_p32, h->pair32.data(), h->pair32.size() * 4);
    if (!h->diel.empty()) std::memcpy(hb.data() + h->o_diel, h->diel.data(), h->diel.size() * 8);
    std::memcpy(hb.data() + h->o_gs, h->gstart.data(), h->gstart.size() * 4);
    std::memcpy(hb.data() + h->o_gi, h->gitems.data(), h->gitems.size() * 4);
    if (!h->grect.empty()) std::memcpy(hb.data() + h->o_gr, h->grect.data(), h->grect.size() * 8);
    DevGeom& g = h->dev;
    g.n_grect = (int)(h->grect.size() / 9);
    g.n_boxes = nb;
    g.n_nets = s->n_nets;
    g.n_layers = s->n_layers;
    g.n_diel = s->n_diel;
    g.n_mat = (int)h->pal.size();
    for (int a = 0; a < 3; ++a) {
        g.encl_lo[a] = s->encl_lo[a];
        g.encl_hi[a] = s->encl_hi[a];
        g.gdim[a] = dim[a];
        g.gcell[a] = cell[a];
    }
    g.gmin_cell = minc;
    return DRWC_OK;
}

// Point h->dev at a device copy of h->blob.
inline void bind_geom(HostGeom* h, void* d) {
    const unsigned char* base = (const unsigned char*)d;
    DevGeom& g = h->dev;
    g.box = (const double*)(base + h->o_box);
    g.net = (const int*)(base + h->o_net);
    g.zlo = (const double*)(base + h->o_zlo);
    g.lmat = (const int*)(base + h->o_lmat);
    g.dmat = (const int*)(base + h->o_dmat);
    g.pal = (const double*)(base + h->o_pal);
    g.pair64 = (const double*)(base + h->o_p64);
    g.pair32 = (const float*)(base + h->o_p32);
    g.diel = (const double*)(base + h->o_diel);
    g.gstart = (const int*)(base + h->o_gs);
    g.gitems = (const int*)(base + h->o_gi);
    g.grect = (const double*)(base + h->o_gr);
    h->dbuf = d;
}

// Pack, copy into the context's geometry workspace and bind.
inline int upload_geom(drwc_ctx* ctx, const drwc_structure* s, HostGeom* h) {
    int rc = pack_geom(s, h);
    if (rc) return rc;
    void* d = nullptr;
    rc = ws_get(ctx, WS_AUX2, h->blob.size(), &d);
    if (rc) return rc;
    // a copy from pageable memory has read the source when it returns
    DRWC_CUDA_TRY(cudaMemcpyAsync(d, h->blob.data(), h->blob.size(), cudaMemcpyHostToDevice,
                                  ctx->stream));
    bind_geom(h, d);
    return DRWC_OK;
}

// Gaussian surface of gauss_surface = 1: the outer boundary of the union of
// the master's boxes, each grown by min(gauss_offset, half its L-infinity
// clearance to the other nets' boxes and the enclosure), as rectangles on the faces
// of the grown boxes. A face point belongs to the surface when no grown box
// covers the space just outside it, and, among the coplanar faces of the same
// orientation that contain it, to the lowest box. Each face is cut along the
// other boxes' edges that cross it, and every cell of that grid is kept or
// dropped whole (tested at its centre). Rectangles come box by box, faces in
// the Gauss box order (z-, z+, y-, y+, x-, x+), so a master of one box gives
// the six faces of the Gauss box with the same areas and running sums.
inline int gauss_union(const drwc_structure* s, const drwc_job_params* p, Gauss* G,
                       std::vector<double>* rects) {
    std::vector<std::array<double, 6>> B;
    std::vector<double> offs;
    for (int b = 0; b < s->n_boxes; ++b) {
        if (s->boxes[b].net != p->master) continue;
        // this box's clearance: walls and every other net's box (L-infinity)
        const drwc_box& M = s->boxes[b];
        double gap = INFINITY;
        for (int a = 0; a < 3; ++a)
            gap = std::min(gap, std::min(M.lo[a] - s->encl_lo[a], s->encl_hi[a] - M.hi[a]));
        for (int q = 0; q < s->n_boxes; ++q) {
            if (s->boxes[q].net == p->master) continue;
            double sep = -INFINITY;
            for (int a = 0; a < 3; ++a)
                sep = std::max(sep, std::max(s->boxes[q].lo[a] - M.hi[a], M.lo[a] - s->boxes[q].hi[a]));
            gap = std::min(gap, sep);
        }
        if (!(gap > 0)) return DRWC_ERR_GEOMETRY;
        const double off = std::min(p->gauss_offset, 0.5 * gap);
        offs.push_back(off);
        std::array<double, 6> g;
        for (int a = 0; a < 3; ++a) {
            volatile double lo = s->boxes[b].lo[a] - off;
            volatile double hi = s->boxes[b].hi[a] + off;
            g[a] = lo;
            g[3 + a] = hi;
            if (lo < s->encl_lo[a] || hi > s->encl_hi[a]) return DRWC_ERR_GEOMETRY;
        }
        B.push_back(g);
    }
    if (B.empty()) return DRWC_ERR_INVALID;
    // no grown box may reach another net's box
    for (int b = 0; b < s->n_boxes; ++b) {
        if (s->boxes[b].net == p->master) continue;
        for (const auto& g : B) {
            bool overlap = true;
            for (int a = 0; a < 3; ++a)
                overlap &= s->boxes[b].lo[a] < g[3 + a] && s->boxes[b].hi[a] > g[a];
            if (overlap) return DRWC_ERR_GEOMETRY;
        }
    }
    for (int a = 0; a < 3; ++a) {  // the Gauss box: the union's bounds
        G->lo[a] = INFINITY;
        G->hi[a] = -INFINITY;
        for (const auto& g : B) {
            G->lo[a] = std::min(G->lo[a], g[a]);
            G->hi[a] = std::max(G->hi[a], g[3 + a]);
        }
    }
    rects->clear();
    const int K = (int)B.size();
    // Importance sampling: the first-hop weight grows as 1 / (distance to the
    // master) and a start point on box k's face lies off_k from it, so face
    // area of box k is sampled with density factor off_max / off_k (1 when
    // all offsets agree) and the weight carries the inverse factor.
    const double off_max = *std::max_element(offs.begin(), offs.end());
    volatile double run = 0.0;
    for (int k = 0; k < K; ++k) {
        for (int f = 0; f < 6; ++f) {
            const int axis = f < 2 ? 2 : f < 4 ? 1 : 0, side = f & 1;
            const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
            const double x = side ? B[k][3 + axis] : B[k][axis];
            const double u0 = B[k][t0], u1 = B[k][3 + t0], v0 = B[k][t1], v1 = B[k][3 + t1];
            // the other boxes that touch the face's plane region
            std::vector<int> near;
            std::vector<double> us{u0, u1}, vs{v0, v1};
            for (int q = 0; q < K; ++q) {
                if (q == k) continue;
                if (!(B[q][axis] <= x && B[q][3 + axis] >= x)) continue;
                if (!(B[q][t0] < u1 && B[q][3 + t0] > u0 && B[q][t1] < v1 && B[q][3 + t1] > v0))
                    continue;
                near.push_back(q);
                for (double e : {B[q][t0], B[q][3 + t0]}) if (e > u0 && e < u1) us.push_back(e);
                for (double e : {B[q][t1], B[q][3 + t1]}) if (e > v0 && e < v1) vs.push_back(e);
            }
            std::sort(us.begin(), us.end());
            us.erase(std::unique(us.begin(), us.end()), us.end());
            std::sort(vs.begin(), vs.end());
            vs.erase(std::unique(vs.begin(), vs.end()), vs.end());
            for (size_t iu = 0; iu + 1 < us.size(); ++iu) {
                for (size_t iv = 0; iv + 1 < vs.size(); ++iv) {
                    const double pu = 0.5 * (us[iu] + us[iu + 1]), pv = 0.5 * (vs[iv] + vs[iv + 1]);
                    bool keep = true;
                    for (int q : near) {
                        const bool inside_t = B[q][t0] < pu && pu < B[q][3 + t0] &&
                                              B[q][t1] < pv && pv < B[q][3 + t1];
                        if (!inside_t) continue;
                        // covers the space just outside the face
                        const bool cover = side ? (B[q][axis] <= x && x < B[q][3 + axis])
                                                : (B[q][axis] < x && x <= B[q][3 + axis]);
                        // a lower coplanar face of the same orientation owns it
                        const bool owner = q < k && (side ? B[q][3 + axis] == x : B[q][axis] == x);
                        if (cover || owner) { keep = false; break; }
                    }
                    if (!keep) continue;
                    volatile double du = us[iu + 1] - us[iu], dv = vs[iv + 1] - vs[iv];
                    volatile double ar = du * dv;
                    const double fk = offs[k] == off_max ? 1.0 : off_max / offs[k];
                    volatile double mass = fk == 1.0 ? (double)ar : ar * fk;
                    run = run + mass;
                    rects->insert(rects->end(), {(double)axis, (double)side, x, us[iu], us[iu + 1],
                                                 vs[iv], vs[iv + 1], (double)run, 1.0 / fk});
                }
            }
        }
    }
    if (rects->empty()) return DRWC_ERR_GEOMETRY;
    for (int f = 0; f < 6; ++f) G->area[f] = 0.0;
    G->total = run;
    return DRWC_OK;
}

// Same arithmetic (order, no contraction) as the CPU restatement.
inline int gauss_build(const drwc_structure* s, const drwc_job_params* p, Gauss* G) {
    for (int a = 0; a < 3; ++a) {
        G->lo[a] = INFINITY;
        G->hi[a] = -INFINITY;
    }
    bool any = false;
    for (int b = 0; b < s->n_boxes; ++b) {
        if (s->boxes[b].net != p->master) continue;
        any = true;
        for (int a = 0; a < 3; ++a) {
            if (s->boxes[b].lo[a] < G->lo[a]) G->lo[a] = s->boxes[b].lo[a];
            if (s->boxes[b].hi[a] > G->hi[a]) G->hi[a] = s->boxes[b].hi[a];
        }
    }
    if (!any) return DRWC_ERR_INVALID;
    for (int a = 0; a < 3; ++a) {
        volatile double lo = G->lo[a] - p->gauss_offset;
        volatile double hi = G->hi[a] + p->gauss_offset;
        G->lo[a] = lo;
        G->hi[a] = hi;
        if (lo < s->encl_lo[a] || hi > s->encl_hi[a]) return DRWC_ERR_GEOMETRY;
    }
    // the Gaussian surface must not cut another net's box
    for (int b = 0; b < s->n_boxes; ++b) {
        if (s->boxes[b].net == p->master) continue;
        bool overlap = true;
        for (int a = 0; a < 3; ++a)
            overlap &= s->boxes[b].lo[a] < G->hi[a] && s->boxes[b].hi[a] > G->lo[a];
        if (overlap) return DRWC_ERR_GEOMETRY;
    }
    volatile double dx = G->hi[0] - G->lo[0], dy = G->hi[1] - G->lo[1], dz = G->hi[2] - G->lo[2];
    volatile double az = dx * dy, ay = dx * dz, ax = dy * dz;
    G->area[0] = az; G->area[1] = az;
    G->area[2] = ay; G->area[3] = ay;
    G->area[4] = ax; G->area[5] = ax;
    volatile double tot = 0;
    for (int f = 0; f < 6; ++f) tot = tot + G->area[f];
    G->total = tot;
    return DRWC_OK;
}

// Validate a job, build its Gaussian surface, pack its structure and fill
// the walk parameters (FDM knobs, warm-start tables of the context).
inline int prepare(drwc_ctx* ctx, const drwc_structure* s, const drwc_job_params* p,
                   HostGeom* hg, Gauss* G, WalkParams* P) {
    int rc = validate(s);
    if (rc) return rc;
    if (!p || !n_supported(p->N) || p->master < 0 || p->master >= s->n_nets ||
        !(p->gauss_offset > 0) || !(p->stop_dist > 0) || p->max_hops < 1)
        return DRWC_ERR_INVALID;
    hg->grect.clear();
    if (p->gauss_surface == 1) rc = gauss_union(s, p, G, &hg->grect);
    else if (p->gauss_surface == 0) rc = gauss_build(s, p, G);
    else rc = DRWC_ERR_INVALID;
    if (rc) return rc;
    rc = pack_geom(s, hg);  // the caller places the blob on the device
    if (rc) return rc;
    P->N = p->N;
    P->max_hops = p->max_hops;
    P->master = p->master;
    P->stop = p->stop_dist;
    P->seed = p->seed;
    P->prm = make_params(&p->fdm, p->N);
    P->log = nullptr;
    P->log_code = nullptr;
    P->log_count = nullptr;
    P->log_cap = 0;
    if (p->fdm.warm_start) {
        rc = warm_tables(ctx, p->N, P->prm.warm);
        if (rc) return rc;
    }
    return DRWC_OK;
}

}  // namespace drwc
