// Multi-job FRW server: a persistent request loop that runs many extraction
// jobs at once on one device.
//
// Device state
//   * a job table (host-written between graph replays): each running job's
//     structure (DevGeom, in the server's HBM arena), Gaussian surface, walk
//     parameters, claim limit and the two batches of walk ids whose records
//     it is collecting;
//   * per-job counters (device-written): next walk id, finished walks per
//     batch of the claim window, walks in flight, reduced flags;
//   * a pool of S walker slots (position, weight, hop count, job, walk id);
//   * per-step work lists: network rows (N = 16 jobs when a network is
//     loaded) and FDM rows bucketed by cube resolution.
//
// One step (all slots advance one hop)
//   reset lists -> prepare (warp per slot: drop walks of finished jobs,
//   claim a walk from the running jobs, nearest conductor, absorption,
//   record the finished walk, append the hop to a list) -> [voxelise ->
//   network (tensor cores) -> sample / route] -> FDM solve per bucket.
// Buckets that do not wait for the network fork right after prepare, so
// their solves overlap the network on parallel graph branches. A replay of
// the captured graph runs steps_per_graph steps and then reduces every batch
// whose walks have all finished (fixed-order sums per capacitance entry).
//
// Host loop (one thread): admit queued jobs first-in first-out while their
// footprint fits the arena and a table entry is free, replay the graph,
// read the counters and the reduced batches, fold them into each job's
// compensated sums in batch order, test convergence exactly as
// drwc_frw_run does, retire converged jobs (their walks still in flight are
// dropped on the next step, then their arena block is freed), and widen each
// job's claim window by one batch when the oldest batch has been reduced.
// Walk w of a job draws from Philox counters (w, hop, draw) of the job's
// seed, so its record does not depend on which slot or step carried it, and
// the per-batch reduction order depends only on walk ids.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <thread>

#include "geom.cuh"
#include "nn.cuh"
#include "stem.cuh"

namespace drwc {

constexpr int kSvMaxJobs = 64;
constexpr int kSvMaxSteps = 8;
// Prepare-loop passes per slot and step (claims, finished walks, table hops).
// A slot deep in a homogeneous region chains table hops; the launch ends with
// its longest chain, so a short limit shortens every step, and the rest of
// the chain continues in the next one (learned stream: 16 passes 3 % faster
// than 64, 8 and 32 between them; the walks are the same whatever the limit).
#ifndef DRWC_SV_PREP_ITERS
#define DRWC_SV_PREP_ITERS 16
#endif
constexpr int kSvPrepIters = DRWC_SV_PREP_ITERS;
constexpr int kSvWin = 8;         // record slots per job: batches of walk ids in flight
constexpr size_t kSvBsumStride = 3 * (DRWC_MAX_NETS + 2) + 8;  // doubles per (job, window slot)
// per-step row counters: 4 per bucket (below), then per bucket the FDM rows
// that continue for several hops (kept at the top of the bucket's list)
constexpr int kSvCnt = 5 * DRWC_SERVER_MAX_SIZES;

struct SvJob {
    DevGeom g;
    Gauss G;
    WalkParams W;
    int state;         // 0 free, 1 running, 2 draining
    int use_net;       // hops go through the network
    int bucket;        // index of the job's cube resolution among the served sizes
    int n_entries;     // nets + ground
    long long total;   // walk ids [0, total)
    long long batch;   // walks per batch
    long long limit;   // ids below this may be claimed
    long long bfirst[kSvWin];  // first walk id of the batch held by record slot q (-1: free)
    long long bcount[kSvWin];
    double* rec_w;     // records: slot q at q * batch
    int32_t* rec_end;
    int32_t* rec_hops;
    int32_t* out_end;  // the caller's per-walk records by walk id (nullable)
    double* out_w;
};

struct SvCtr {
    unsigned long long next;
    unsigned long long done[kSvWin];
    unsigned long long inflight;  // two's complement
    unsigned long long reduced[kSvWin];
    unsigned long long pad[7];
};

struct SvHdr {
    int n_act;
    int act[kSvMaxJobs];
};

struct SvSlots {
    double *px, *py, *pz, *omega, *sgn, *a, *epsw;
    long long* walk;
    int *hops, *mode, *code, *job, *grow;
};

enum SvStat {
    SV_HOPS = 0, SV_NET_HOPS, SV_FDM_HOPS, SV_FALLBACKS, SV_AUDITS, SV_WALKS_DONE,
    SV_WALKS_DROPPED, SV_NET_ROWS, SV_FDM_ITERS, SV_FDM_SWEEPS, SV_FDM_BYTES, SV_TABLE_HOPS,
    SV_FDM_ESCALATED, SV_FDM_FAILED, SV_NSTATS
};

struct SvArgs {
    int S;
    int n_buckets;
    const SvJob* jobs;
    SvCtr* ctr;
    const SvHdr* hdr;
    SvSlots st;
    int* blist[DRWC_SERVER_MAX_SIZES];
    int* bkind[DRWC_SERVER_MAX_SIZES];  // bit 0 audit, bit 1 continuing, bits 2.. network row
    // per bucket b: cnt[4b] network rows, [4b + 1] first-hop rows, [4b + 2] FDM
    // rows, [4b + 3] the next unclaimed FDM row
    unsigned* cnt;
    float conf_thresh, audit_frac;
    // network of bucket b (when it has one): rows, outputs, conv1 operands
    int* alist[DRWC_SERVER_MAX_SIZES];
    int* frow[DRWC_SERVER_MAX_SIZES];
    float* O[DRWC_SERVER_MAX_SIZES];
    float* Gh[DRWC_SERVER_MAX_SIZES];
    int out_row[DRWC_SERVER_MAX_SIZES];
    int grad_row[DRWC_SERVER_MAX_SIZES];
    NetStem stem[DRWC_SERVER_MAX_SIZES];  // conv1 and conv2 run inside the voxeliser
    unsigned long long* stats;
    double* audit_kl;                   // [0] sum, [1] count
    double* bsum;
    // homogeneous-cube fast path: per bucket and solver code, the panel values
    // of the uniform-permittivity Green's function and their running sums
    int table;
    int fair;                           // claim policy (drwc_server_opts.fair_share)
    int fdm_hops;                       // hops a continuing FDM-only walk takes per step
    int strag_hops;                     // a walk with this many hops continues
    const double* tval[DRWC_SERVER_MAX_SIZES][4];
    const double* tcdf[DRWC_SERVER_MAX_SIZES][4];
};

// ------------------------------------------------------------------ device
DRWC_DEV long long sv_claim(const SvArgs& A, int slot, int* job_out) {
    const int n = A.hdr->n_act;
    // act[] lists the running jobs oldest first: FIFO with backfill, or a
    // rotation per slot for an even share
    const int first = A.fair ? slot % max(n, 1) : 0;
    for (int q = 0; q < n; ++q) {
        const int j = A.hdr->act[(first + q) % n];
        const SvJob& J = A.jobs[j];
        if (J.state != 1) continue;
        // keep the counter from running far past the limit; the host clamps it
        if (*(volatile unsigned long long*)&A.ctr[j].next >= (unsigned long long)J.limit) continue;
        const unsigned long long w = atomicAdd(&A.ctr[j].next, 1ull);
        if ((long long)w < J.limit) {
            *job_out = j;
            return (long long)w;
        }
    }
    return -1;
}

DRWC_DEV void sv_start(const SvArgs& A, int slot, int j, long long w) {
    const SvJob& J = A.jobs[j];
    double r[3], sgn;
    int code;
    walk_start_point(J.G, J.g, J.W.seed, (uint64_t)w, r, &sgn, &code);
    A.st.px[slot] = r[0]; A.st.py[slot] = r[1]; A.st.pz[slot] = r[2];
    A.st.sgn[slot] = sgn;
    A.st.code[slot] = code;
    A.st.hops[slot] = 0;
    A.st.omega[slot] = 0.0;
    A.st.walk[slot] = w;
    A.st.job[slot] = j;
    A.st.mode[slot] = 1;
    atomicAdd(&A.ctr[j].inflight, 1ull);
}

// Record the walk on `net` (-1: lost) and free the slot.
DRWC_DEV void sv_finish(const SvArgs& A, int slot, int net) {
    const int j = A.st.job[slot];
    const SvJob& J = A.jobs[j];
    const long long w = A.st.walk[slot];
    // the slot holding the walk's batch (every id below the claim limit has one)
    int p = 0;
    for (int q = 1; q < kSvWin; ++q)
        if (w >= J.bfirst[q] && w < J.bfirst[q] + J.bcount[q]) p = q;
    const long long i = w - J.bfirst[p];
    if (i >= 0 && i < J.bcount[p]) {
        const long long r = (long long)p * J.batch + i;
        J.rec_end[r] = net;
        J.rec_hops[r] = A.st.hops[slot];
        J.rec_w[r] = A.st.omega[slot];
        if (J.out_end) {
            J.out_end[w] = net;
            J.out_w[w] = A.st.omega[slot];
        }
        atomicAdd(&A.ctr[j].done[p], 1ull);
    }
    atomicAdd(&A.ctr[j].inflight, ~0ull);
    atomicAdd(A.stats + SV_WALKS_DONE, 1ull);
    A.st.mode[slot] = 0;
}

// Material id of the cube when every cell centre of its N^3 grid has the same
// one, else -1 (warp-wide; all lanes get the answer). Uses the cell-centre
// coordinates the voxeliser computes for i = 0 and i = N-1, the layer rule
// and the inclusive block bounds of mat_at, so a cube reported homogeneous
// voxelises to a single material; blocks that merely touch the span of cell
// centres make it inhomogeneous (conservative).
DRWC_DEV int sv_homogeneous(const DevGeom& g, const double c[3], double a, int N) {
    const int lane = threadIdx.x & 31;
    const double t0 = dsub(ddiv(dadd(dmul(2.0, 0.0), 1.0), (double)N), 1.0);
    const double t1 = dsub(ddiv(dadd(dmul(2.0, (double)(N - 1)), 1.0), (double)N), 1.0);
    double lo[3], hi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        lo[d] = dadd(c[d], dmul(a, t0));
        hi[d] = dadd(c[d], dmul(a, t1));
    }
    int m = 0;
    if (g.n_layers > 0) {
        int l0 = 0, l1 = 0;
        for (int l = 0; l < g.n_layers; ++l) {
            if (lo[2] >= g.zlo[l]) l0 = l;
            if (hi[2] >= g.zlo[l]) l1 = l;
        }
        m = g.lmat[l0];
        for (int l = l0 + 1; l <= l1; ++l)
            if (g.lmat[l] != m) return -1;
    }
    bool clash = false;
    for (int b = lane; b < g.n_diel; b += 32) {
        if (g.dmat[b] == m) continue;
        const double* D = g.diel + 7 * b;
        clash |= D[0] <= hi[0] && D[3] >= lo[0] && D[1] <= hi[1] && D[4] >= lo[1] &&
                 D[2] <= hi[2] && D[5] >= lo[2];
    }
    return __any_sync(0xffffffffu, clash) ? -1 : m;
}

// First index i in [0, M) with cdf[i] > target, M - 1 when there is none
// (the binary search's answer; cdf is nondecreasing), warp-wide in rounds of
// 32 loads: the first of 32 strides whose last entry passes the target, then
// the same within that stride. Three dependent loads for M <= 32768 instead
// of a binary search's eleven or twelve.
DRWC_DEV int warp_cdf_search(const double* __restrict__ cdf, int M, double target) {
    const int lane = threadIdx.x & 31;
    int lo = 0, len = M;  // the answer is in [lo, lo + len); its last entry passes
    while (len > 1) {
        const int s = (len + 31) >> 5;
        const int pos = min(lo + (lane + 1) * s, lo + len) - 1;
        const unsigned b = __ballot_sync(0xffffffffu, cdf[pos] > target);
        if (b == 0u) return M - 1;  // only in the first round: nothing passes
        const int f = __ffs(b) - 1;
        const int nlo = lo + f * s;
        len = min(lo + (f + 1) * s, lo + len) - nlo;
        lo = nlo;
    }
    return lo;
}

// One hop of a homogeneous cube from the uniform-permittivity tables: the
// surface values of a single-permittivity cube do not depend on that
// permittivity, and its centre permittivity is the material's own, so the
// draw needs no solve. Same Philox draws and weight formula as the FDM hop.
// Warp-wide (the search); lane 0 writes the slot.
DRWC_DEV void sv_table_hop(const SvArgs& A, int slot, const SvJob& J, int m) {
    const int N = J.W.N, M = 6 * N * N;
    const int h = A.st.hops[slot];
    const bool first = h == 0;
    const int code = first ? A.st.code[slot] : DRWC_GFT;
    const double* cdf = A.tcdf[J.bucket][code];
    const double* val = A.tval[J.bucket][code];
    const long long w = A.st.walk[slot];
    const double2 u2 = first ? philox_uniform2(J.W.seed, (uint64_t)w, 0, 1)
                             : philox_uniform2(J.W.seed, (uint64_t)w, (uint32_t)h, 0);
    const double tot = cdf[M - 1];
    const double target = (first ? u2.y : u2.x) * tot;
    const int b = warp_cdf_search(cdf, M, target);  // first panel whose running sum passes
    if ((threadIdx.x & 31) != 0) return;
    const double a = A.st.a[slot];
    if (first) {
        const double v = J.g.pal[m];
        const double eps_w = ((N % 2) || code == DRWC_GFT) ? v : (v + v + v + v) / 4;
        A.st.omega[slot] = first_hop_weight(J.G, A.st.sgn[slot], eps_w, tot, val[b], a);
    }
    double loc[3];
    locate_f64(N, b, loc);
    A.st.px[slot] = dadd(A.st.px[slot], dmul(a, loc[0]));
    A.st.py[slot] = dadd(A.st.py[slot], dmul(a, loc[1]));
    A.st.pz[slot] = dadd(A.st.pz[slot], dmul(a, loc[2]));
    A.st.hops[slot] = h + 1;
}

__global__ void sv_reset_kernel(SvArgs A) {
    if (threadIdx.x < kSvCnt) A.cnt[threadIdx.x] = 0;
}

// One warp per slot.
__global__ void __launch_bounds__(256) sv_prepare_kernel(SvArgs A) {
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (slot >= A.S) return;
    int act = 0;
    unsigned long long table_hops = 0;
    // claims, finished walks and table hops per slot and step are bounded
    for (int it = 0; it < kSvPrepIters; ++it) {
        int mode = A.st.mode[slot];
        if (mode == 1 && A.jobs[A.st.job[slot]].state != 1) {
            // the job has finished (or was cancelled): drop its walk
            if (lane == 0) {
                atomicAdd(&A.ctr[A.st.job[slot]].inflight, ~0ull);
                atomicAdd(A.stats + SV_WALKS_DROPPED, 1ull);
                A.st.mode[slot] = 0;
            }
            mode = 0;
        }
        if (mode == 0) {
            long long w = -1;
            if (lane == 0) {
                int j = -1;
                w = sv_claim(A, slot, &j);
                if (w >= 0) sv_start(A, slot, j, w);
            }
            w = __shfl_sync(0xffffffffu, w, 0);
            if (w < 0) break;  // nothing to claim: the slot idles this step
        }
        __syncwarp();
        const SvJob& J = A.jobs[A.st.job[slot]];
        const double r[3] = {A.st.px[slot], A.st.py[slot], A.st.pz[slot]};
        double d;
        int net;
        nearest(J.g, r, &d, &net);
        if (lane == 0) {
            if (d < J.W.stop) sv_finish(A, slot, net);
            else if (A.st.hops[slot] >= J.W.max_hops) sv_finish(A, slot, -1);
            else { A.st.a[slot] = d; act = 1; }
        }
        act = __shfl_sync(0xffffffffu, act, 0);
        if (act && A.table) {
            __syncwarp();
            const int m = sv_homogeneous(J.g, r, A.st.a[slot], J.W.N);
            if (m >= 0) {
                sv_table_hop(A, slot, J, m);
                table_hops += 1;
                act = 0;
            }
        }
        __syncwarp();
        if (act) break;
    }
    if (lane == 0 && table_hops) {
        atomicAdd(A.stats + SV_TABLE_HOPS, table_hops);
        atomicAdd(A.stats + SV_HOPS, table_hops);
    }
    if (lane == 0 && act) {
        const SvJob& J = A.jobs[A.st.job[slot]];
        const int b = J.bucket;
        if (J.use_net) {
            const unsigned idx = atomicAdd(&A.cnt[4 * b], 1u);
            A.alist[b][idx] = slot;
            if (A.st.hops[slot] == 0) {
                const unsigned f = atomicAdd(&A.cnt[4 * b + 1], 1u);
                A.frow[b][f] = (int)idx;
                A.st.grow[slot] = (int)f;
            }
        } else {
            // a walk of a job without a network takes several hops per step
            // inside the FDM solve once the job's walks are all claimed (its
            // tail) or once it is long (it holds back its batch); those rows
            // fill the list from the top and are solved first, so a launch
            // does not end waiting for a chain of hops claimed last
            const bool cont = !A.table && A.fdm_hops > 1 &&
                              (A.st.hops[slot] >= A.strag_hops ||
                               *(volatile unsigned long long*)&A.ctr[A.st.job[slot]].next >=
                                   (unsigned long long)J.total);
            unsigned pos;
            if (cont) pos = (unsigned)A.S - 1u - atomicAdd(&A.cnt[4 * DRWC_SERVER_MAX_SIZES + b], 1u);
            else pos = atomicAdd(&A.cnt[4 * b + 2], 1u);
            A.blist[b][pos] = slot;
            A.bkind[b][pos] = cont ? 2 : 0;
        }
    }
}

// The slot fields a network row's cube is built from.
struct SvCubeHdr {
    int slot, job, hops, code;
    double px, py, pz, a;
};

DRWC_DEV SvCubeHdr sv_cube_hdr(const SvArgs& A, int bucket, int row) {
    SvCubeHdr h;
    h.slot = A.alist[bucket][row];
    h.job = A.st.job[h.slot];
    h.hops = A.st.hops[h.slot];
    h.code = A.st.code[h.slot];
    h.px = A.st.px[h.slot];
    h.py = A.st.py[h.slot];
    h.pz = A.st.pz[h.slot];
    h.a = A.st.a[h.slot];
    return h;
}

// Network rows in groups (two cubes at N = 16, one at 21 and 23), one group
// at a time per CTA: each cube voxelised in shared memory (eps / max eps,
// BF16; a cube that no dielectric block reaches is kept as its N per-index
// values) and the network's stem (conv1, conv2) applied to it on the tensor
// cores there, so only conv2's activations reach global memory. The next
// group's cube headers are fetched while conv2 runs.
template <int N>
__global__ void __launch_bounds__(StemDims<N>::NT, StemDims<N>::CTAS)
    sv_stem_kernel(SvArgs A, int bucket) {
    using D = StemDims<N>;
    extern __shared__ __align__(1024) unsigned char sv_stem_smem[];
    __shared__ double tco[N];
    __shared__ double pal[kMaxMaterials];
    __shared__ VoxScratch<N> vs;
    __shared__ float red[32];
    __shared__ DevGeom gs;  // the current job's geometry header: its fields are read per voxel pass
    __shared__ SvCubeHdr hdr[D::CUBES];  // the group's cubes, fetched a group ahead
    __shared__ __nv_bfloat16 pvs[N];     // per-index values of a cube no block reaches
    const int na = (int)A.cnt[4 * bucket];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(A.stats + SV_NET_ROWS, (unsigned long long)na);
    if ((int)blockIdx.x * D::CUBES >= na) return;
    const NetStem& W = A.stem[bucket];
    centre_offsets<N>(tco);
    if ((int)threadIdx.x < D::CUBES && (int)(blockIdx.x * D::CUBES + threadIdx.x) < na)
        hdr[threadIdx.x] = sv_cube_hdr(A, bucket, blockIdx.x * D::CUBES + threadIdx.x);
    Stem<N> st{sv_stem_smem};
    st.begin(W);
    int loaded = -1;
    bool ok = true;
    for (int grp = blockIdx.x; ok && grp * D::CUBES < na; grp += gridDim.x) {
        const int g0 = grp * D::CUBES, nc = min(D::CUBES, na - g0);
        int uaxis = -1;           // of the group's last cube
        int ux0 = -1, ux1 = -1;   // of its cubes 0 and 1 (two-cube groups)
        for (int cb = 0; ok && cb < nc; ++cb) {
            // the group's headers were written after the previous group's last
            // barrier; later cubes follow conv1's closing barrier, which the
            // readers of pal and gs have passed
            if (cb == 0) __syncthreads();
            const SvCubeHdr h = hdr[cb];
            const int j = h.job;  // the same in every thread: the branch below is uniform
            if (j != loaded) {
                const SvJob& J = A.jobs[j];
                for (int v = threadIdx.x; v < J.g.n_mat; v += blockDim.x) pal[v] = J.g.pal[v];
                if (threadIdx.x == 0) gs = J.g;
                loaded = j;
                __syncthreads();
            }
            const bool first = h.hops == 0;
            const int rot = first ? rot_of_code(h.code) : 0;
            const double c[3] = {h.px, h.py, h.pz};
            vox_prepare<N>(gs, c, h.a, tco, vs, pal, pvs);
            uaxis = -1;
            if (vs.nrel == 0) {
                // no block reaches the cube: its values vary along one index
                // (the original z axis in the rotated frame), pvs holds them;
                // the voxels themselves are not written
                uaxis = rot == 1 ? 1 : rot == 2 ? 0 : 2;
                if (first && threadIdx.x == 0) {
                    // the centre cells the permittivity at the centre is read from
                    constexpr int cc = N / 2;
                    for (int k = cc - 1; k <= cc; ++k)
                        for (int jj = cc - 1; jj <= cc; ++jj)
                            for (int i = cc - 1; i <= cc; ++i)
                                st.mat()[(k * N + jj) * N + i] =
                                    (uint8_t)vs.lm[rot == 1 ? jj : rot == 2 ? i : k];
                    const EpsPalette E{st.mat(), pal, nullptr, nullptr, nullptr, 0};
                    A.st.epsw[h.slot] = center_diel<N>(E, DRWC_WVTZ);
                }
            } else {
                voxelise_cells<N>(gs, c, h.a, rot, tco, pal, st.mat(), st.xs(), nullptr, red, vs);
                if (first && threadIdx.x == 0) {
                    const EpsPalette E{st.mat(), pal, nullptr, nullptr, nullptr, 0};
                    A.st.epsw[h.slot] = center_diel<N>(E, DRWC_WVTZ);
                }
            }
            ok = st.conv1(cb, W.err, uaxis, pvs);
            if (cb == 0) ux0 = uaxis;
            else ux1 = uaxis;
        }
        // the next group's cubes are fetched while conv2 runs
        const int gn = (grp + (int)gridDim.x) * D::CUBES + (int)threadIdx.x;
        const bool fetch = (int)threadIdx.x < D::CUBES && gn < na;
        SvCubeHdr nh;
        if (fetch) nh = sv_cube_hdr(A, bucket, gn);
        if constexpr (D::CUBES == 1) {
            // one cube per group: a stratified one runs on its class rows
            if (ok) ok = uaxis >= 0 ? st.conv2_uaxis(uaxis, W.a2 + (size_t)g0 * D::P3 * 32, W.err)
                                    : st.conv2(nc, W.a2 + (size_t)g0 * D::P3 * 32, W.err);
        } else {
            // two cubes per group: the pair form when either is stratified
            if (ok) ok = (ux0 >= 0 || ux1 >= 0)
                             ? st.conv2_pair(nc, W.a2 + (size_t)g0 * D::P3 * 32, W.err, ux0, ux1)
                             : st.conv2(nc, W.a2 + (size_t)g0 * D::P3 * 32, W.err);
        }
        if (fetch) hdr[threadIdx.x] = nh;  // conv2 ended with a barrier: no cube reads hdr now
    }
    st.end();
}

// Weight of panel q of a network row: the softmax numerator exp(o_q - max)
// of the Poisson head, or |g_q| (scale removed) of the gradient head.
DRWC_DEV double sv_weight(const float* r, int q, bool first, float mx) {
    return first ? fabs((double)r[q] / (double)kGradScale) : (double)__expf(r[q] - mx);
}

// One warp per network row: draw from the prediction (FP64 running sums over
// per-lane chunks of the 6N^2 panels, scanned across the warp; the lane whose
// chunk holds the target walks it), or route the hop to the FDM bucket.
template <int N>
__global__ void __launch_bounds__(256) sv_sample_kernel(SvArgs A, int bucket) {
    constexpr int M = 6 * N * N, CH = (M + 31) / 32;
    const int ldo = A.out_row[bucket], ldg = A.grad_row[bucket];
    const float* __restrict__ Ob = A.O[bucket];
    const float* __restrict__ Gb = A.Gh[bucket];
    const int lane = threadIdx.x & 31;
    const int warps = (int)(blockDim.x >> 5) * (int)gridDim.x;
    const int na = (int)A.cnt[4 * bucket];
    unsigned long long my_net = 0;
    for (int row = blockIdx.x * (int)(blockDim.x >> 5) + (threadIdx.x >> 5); row < na;
         row += warps) {
        const int slot = A.alist[bucket][row];
        const SvJob& J = A.jobs[A.st.job[slot]];
        const long long w = A.st.walk[slot];
        const int h = A.st.hops[slot];
        const bool first = h == 0;
        int route = 0;
        if (lane == 0) {
            const float conf = Ob[(size_t)row * ldo + M];
            const bool audit =
                philox_uniform2(J.W.seed, (uint64_t)w, (uint32_t)h, 2).x < (double)A.audit_frac;
            if (audit || conf > A.conf_thresh) {
                const unsigned idx = atomicAdd(&A.cnt[4 * bucket + 2], 1u);
                A.blist[bucket][idx] = slot;
                A.bkind[bucket][idx] = (audit ? 1 : 0) | (row << 2);
                route = 1;
                atomicAdd(A.stats + (audit ? SV_AUDITS : SV_FALLBACKS), 1ull);
            }
        }
        if (__shfl_sync(0xffffffffu, route, 0)) continue;
        const float* r = first ? Gb + (size_t)A.st.grow[slot] * ldg : Ob + (size_t)row * ldo;
        float mx = 0.f;
        if (!first) {
            mx = -1e30f;
            for (int q = lane; q < M; q += 32) mx = fmaxf(mx, r[q]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        const int q0 = min(lane * CH, M), q1 = min(q0 + CH, M);
        double sum = 0.0;
        int last = -1;
        for (int q = q0; q < q1; ++q) {
            const double v = sv_weight(r, q, first, mx);
            sum += v;
            if (v > 0.0) last = q;
        }
        double incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double n = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += n;
        }
        const double tot = __shfl_sync(0xffffffffu, incl, 31);
        int lastall = last;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lastall = max(lastall, __shfl_xor_sync(0xffffffffu, lastall, o));
        const double u = first ? philox_uniform2(J.W.seed, (uint64_t)w, 0, 1).y
                               : philox_uniform2(J.W.seed, (uint64_t)w, (uint32_t)h, 0).x;
        const double target = u * tot;
        int pick = 0x7fffffff;
        if (sum > 0.0 && incl > target) {
            double run = incl - sum;
            for (int q = q0; q < q1; ++q) {
                const double v = sv_weight(r, q, first, mx);
                run += v;
                if (run > target && v > 0.0) { pick = q; break; }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) pick = min(pick, __shfl_xor_sync(0xffffffffu, pick, o));
        const int bsel = pick == 0x7fffffff ? lastall : pick;
        if (lane == 0) {
            if (bsel < 0) {
                sv_finish(A, slot, -1);  // no transition possible: the walk is lost
            } else {
                const double a = A.st.a[slot];
                double loc[3], mv[3];
                locate_f64(N, bsel, loc);
                if (first) {
                    unrotate(rot_of_code(A.st.code[slot]), loc, mv);
                    A.st.omega[slot] = first_hop_weight(J.G, A.st.sgn[slot], A.st.epsw[slot], tot,
                                                        (double)r[bsel] / (double)kGradScale, a);
                } else {
                    mv[0] = loc[0]; mv[1] = loc[1]; mv[2] = loc[2];
                }
                A.st.px[slot] = dadd(A.st.px[slot], dmul(a, mv[0]));
                A.st.py[slot] = dadd(A.st.py[slot], dmul(a, mv[1]));
                A.st.pz[slot] = dadd(A.st.pz[slot], dmul(a, mv[2]));
                A.st.hops[slot] = h + 1;
            }
            my_net += 1;
        }
    }
    // per-warp counts
    if (lane == 0 && my_net) {
        atomicAdd(A.stats + SV_NET_HOPS, my_net);
        atomicAdd(A.stats + SV_HOPS, my_net);
    }
}

// FDM hops of one resolution bucket: persistent CTAs over the bucket list;
// the palette tables are reloaded when the job changes between rows. The
// arithmetic of a hop is walk_kernel's.
template <int N>
__global__ void __launch_bounds__(Cube<N>::NT, CubeTraits<N>::kMinBlocks)
sv_fdm_kernel(SvArgs A, int bucket, int maxP, double* __restrict__ scratch_y,
              float* __restrict__ scratch_s) {
    extern __shared__ __align__(128) unsigned char drwc_dyn_smem[];
    unsigned char* smem = drwc_dyn_smem;
    using D = Cube<N>;
    constexpr int M = 6 * D::NN;
    const CubeSmem<N> sm = CubeSmem<N>::carve(smem);
    unsigned char* xs = smem + D::kSmemBytes;
    uint8_t* mat = xs;
    double* tco = reinterpret_cast<double*>(xs + ((size_t)D::NNN + 15) / 16 * 16);
    double* pal = tco + N;
    double* palinv = pal + maxP;
    double* pair64 = palinv + maxP;
    float* pair32 = reinterpret_cast<float*>(pair64 + maxP * maxP);
    centre_offsets<N>(tco);
    double* ys = scratch_y + (size_t)blockIdx.x * D::NNN;
    float* ss = scratch_s + (size_t)blockIdx.x * D::NNN;
    // continuing rows (at the top of the list) first, then the others
    const unsigned n_cont = A.cnt[4 * DRWC_SERVER_MAX_SIZES + bucket];
    const unsigned count = A.cnt[4 * bucket + 2] + n_cont;
    unsigned* next_item = A.cnt + 4 * bucket + 3;
    __shared__ unsigned s_idx;
    __shared__ int s_go;
    __shared__ int lm[N];  // layer material per z index (structures without blocks)
    __shared__ DevGeom gs;  // the current job's geometry header
    VoxScratch<N>& vs =   // separable voxeliser (structures with blocks)
        *reinterpret_cast<VoxScratch<N>*>(smem + (WalkSmem<N>::base(maxP) + 15) / 16 * 16);
    int loaded = -1, P = 0;
    unsigned long long my_hops = 0, my_iters = 0, my_sweeps = 0, my_esc = 0, my_fail = 0;
    for (;;) {
        // rows are claimed one at a time: solve costs differ by cube
        if (threadIdx.x == 0) s_idx = atomicAdd(next_item, 1u);
        __syncthreads();
        const unsigned idx = s_idx;
        if (idx >= count) break;
        const unsigned pos = idx < n_cont ? (unsigned)A.S - 1u - idx : idx - n_cont;
        const int slot = A.blist[bucket][pos];
        const int kind = A.bkind[bucket][pos];
        const int j = A.st.job[slot];
        const SvJob& J = A.jobs[j];
        if (j != loaded) {
            __syncthreads();
            P = J.g.n_mat;
            for (int v = threadIdx.x; v < P; v += blockDim.x) {
                pal[v] = J.g.pal[v];
                palinv[v] = 1.0 / J.g.pal[v];
            }
            for (int v = threadIdx.x; v < P * P; v += blockDim.x) {
                pair64[v] = J.g.pair64[v];
                pair32[v] = J.g.pair32[v];
            }
            if (threadIdx.x == 0) gs = J.g;
            loaded = j;
        }
        __syncthreads();
        // A continuing row (a walk of a job without a network or uniform table,
        // once the job's walks are all claimed or once the walk is long) takes
        // up to fdm_hops hops here: otherwise each hop of such a walk waits a
        // whole step (every other slot's hop), and its batch, or the job's
        // completion, waits for the longest walks.
        for (int hh = 0;; ++hh) {
            const EpsPalette E{mat, pal, palinv, pair64, pair32, P};
            const long long w = A.st.walk[slot];
            const int h = A.st.hops[slot];
            const bool first = h == 0;
            const int code = first ? A.st.code[slot] : DRWC_GFT;
            const double c[3] = {A.st.px[slot], A.st.py[slot], A.st.pz[slot]};
            const double a = A.st.a[slot];
            // a stratified cube (no dielectric block reaches it) goes to the
            // per-plane solver
            const int* lmc = nullptr;
            if (gs.n_diel > 0) {
                vox_prepare<N>(gs, c, a, tco, vs);
                if (vs.nrel == 0) {
                    lmc = vs.lm;
                } else {
                    for (int v = threadIdx.x; v < D::NNN; v += blockDim.x)
                        mat[v] = (uint8_t)vox_material<N>(gs, vs, c, a, tco, v % N, (v / N) % N,
                                                          v / D::NN, 0);
                }
            } else {
                plane_layers<N>(gs, c, a, tco, lm);
                lmc = lm;
            }
            __syncthreads();
            FdmStats st;
            double* wv = reinterpret_cast<double*>(sm.stage());
            const EpsPlanar<N> EP{lmc, pal, palinv, pair64, pair32, P};
            if (lmc) {
                cube_solve_planar<N>(EP, ys, code, J.W.prm, &st);
                for_each_panel<N>(EP, cube_y<N>(ys), [&](int b, double v) { wv[b] = v; });
            } else {
                cube_solve<N>(E, ys, ss, code, J.W.prm, &st);
                for_each_panel<N>(E, cube_y<N>(ys), [&](int b, double v) { wv[b] = v; });
            }
            __syncthreads();
            if ((kind & 1) && !first) {
                // audit: KL(FDM || network) over the panels
                const float* o = A.O[bucket] + (size_t)(kind >> 2) * A.out_row[bucket];
                const double ls = block_lse<D::NW>(o, M, sm.red);
                __syncthreads();
                double kl = 0.0;
                for (int q = threadIdx.x; q < M; q += blockDim.x) {
                    const double gq = fmax(wv[q], 0.0);
                    if (gq > 0.0) kl += gq * (log(gq) - ((double)o[q] - ls));
                }
                kl = block_sum_d<D::NW>(kl, sm.red, 1);
                if (threadIdx.x == 0) {
                    atomicAdd(A.audit_kl + 0, kl);
                    atomicAdd(A.audit_kl + 1, 1.0);
                }
                __syncthreads();
            }
            const double2 u2 = first ? philox_uniform2(J.W.seed, (uint64_t)w, 0, 1)
                                     : philox_uniform2(J.W.seed, (uint64_t)w, (uint32_t)h, 0);
            const double ud = first ? u2.y : u2.x;
            double tot = 0.0;
            const int b = cta_sample<D::NT>(wv, M, first, ud, sm.red, &tot);
            if (threadIdx.x == 0) {
                if (b < 0 || st.status != 0) {
                    // no transition possible, or the solve stayed unconverged
                    // after escalation: the walk is lost
                    sv_finish(A, slot, -1);
                } else {
                    if (first)
                        A.st.omega[slot] = first_hop_weight(
                            J.G, A.st.sgn[slot],
                            lmc ? center_diel<N>(EP, code) : center_diel<N>(E, code), tot, wv[b], a);
                    double loc[3];
                    locate_f64(N, b, loc);
                    A.st.px[slot] = dadd(A.st.px[slot], dmul(a, loc[0]));
                    A.st.py[slot] = dadd(A.st.py[slot], dmul(a, loc[1]));
                    A.st.pz[slot] = dadd(A.st.pz[slot], dmul(a, loc[2]));
                    A.st.hops[slot] = h + 1;
                }
                my_hops += 1;
                my_iters += (unsigned long long)st.iters;
                my_sweeps += (unsigned long long)st.sweeps;
                my_esc += (unsigned long long)st.escalated;
                my_fail += st.status == 1;
            }
            __syncthreads();
            // a continuing row (bit 1, set by the prepare kernel) takes its
            // next hops here
            if (kind != 2 || hh + 1 >= A.fdm_hops) break;
            if (A.st.mode[slot] == 0) break;  // the walk finished on this hop
            // the next hop's cube: nearest conductor, absorption (the prepare
            // kernel's geometry step for this slot)
            if (threadIdx.x < 32) {
                const double r[3] = {A.st.px[slot], A.st.py[slot], A.st.pz[slot]};
                double d;
                int net;
                nearest(gs, r, &d, &net);
                if (threadIdx.x == 0) {
                    int go = 0;
                    if (d < J.W.stop) sv_finish(A, slot, net);
                    else if (A.st.hops[slot] >= J.W.max_hops) sv_finish(A, slot, -1);
                    else { A.st.a[slot] = d; go = 1; }
                    s_go = go;
                }
            }
            __syncthreads();
            if (!s_go) break;
        }
    }
    if (threadIdx.x == 0 && (my_esc || my_fail)) {
        atomicAdd(A.stats + SV_FDM_ESCALATED, my_esc);
        atomicAdd(A.stats + SV_FDM_FAILED, my_fail);
    }
    if (threadIdx.x == 0 && my_hops) {
        atomicAdd(A.stats + SV_FDM_HOPS, my_hops);
        atomicAdd(A.stats + SV_HOPS, my_hops);
        atomicAdd(A.stats + SV_FDM_ITERS, my_iters);
        atomicAdd(A.stats + SV_FDM_SWEEPS, my_sweeps);
        // streamed-PCG algorithmic bytes: 48 B/cell per FP32 iteration, 40 B/cell per
        // FP64 sweep, the permittivity in (8 B/cell) and the 6N^2 panel values out
        atomicAdd(A.stats + SV_FDM_BYTES,
                  (48ull * my_iters + 40ull * my_sweeps + 8ull * my_hops) * D::NNN +
                      48ull * D::NN * my_hops);
    }
}

// Fixed-order sums of every batch whose walks have all finished: block
// (job, window slot) x entry; entry n_entries + 1 sums the hop counts.
__global__ void __launch_bounds__(256) sv_reduce_kernel(SvArgs A) {
    const int j = blockIdx.x / kSvWin, p = blockIdx.x % kSvWin, e = blockIdx.y;
    const SvJob& J = A.jobs[j];
    if (J.state != 1 || e > J.n_entries + 1) return;
    const SvCtr& C = A.ctr[j];
    const long long n = J.bcount[p];
    if (n <= 0 || C.reduced[p] || (long long)C.done[p] < n) return;
    double* out = A.bsum + ((size_t)j * kSvWin + p) * kSvBsumStride;
    const long long base = (long long)p * J.batch;
    if (e <= J.n_entries) {
        reduce_entry(e, J.n_entries, n, J.rec_end + base, J.rec_w + base, out);
        return;
    }
    unsigned long long s = 0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) s += (unsigned long long)J.rec_hops[base + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ unsigned long long ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += ws[q];
        out[3 * (J.n_entries + 1)] = (double)t;
    }
}

__global__ void sv_mark_kernel(SvArgs A) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kSvWin * kSvMaxJobs) return;
    const int j = t / kSvWin, p = t % kSvWin;
    const SvJob& J = A.jobs[j];
    if (J.state != 1) return;
    SvCtr& C = A.ctr[j];
    if (J.bcount[p] > 0 && !C.reduced[p] && (long long)C.done[p] >= J.bcount[p]) C.reduced[p] = 1;
}

// ------------------------------------------------------------------- host
// First-fit allocator over the job arena (offsets, 256-byte granules).
struct Arena {
    size_t size = 0, used = 0, peak = 0;
    std::map<size_t, size_t> free_;  // offset -> bytes
    void init(size_t bytes) { size = bytes; free_.clear(); free_[0] = bytes; used = peak = 0; }
    bool alloc(size_t bytes, size_t* off) {
        bytes = (bytes + 255) / 256 * 256;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t roff = it->first + bytes;
            free_.erase(it);
            if (rest) free_[roff] = rest;
            used += bytes;
            peak = std::max(peak, used);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = (bytes + 255) / 256 * 256;
        used -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct SvHostJob {
    int64_t id = 0;
    std::vector<drwc_box> boxes;
    std::vector<double> zlo, leps;
    std::vector<drwc_diel_box> diel;
    drwc_structure s{};
    drwc_job_params p{};
    HostGeom hg;
    Gauss G{};
    WalkParams W{};
    int state = DRWC_JOB_QUEUED;
    int error = DRWC_OK;
    int table = -1;
    size_t arena_off = 0, arena_bytes = 0, blob_bytes = 0;
    bool draining = false;
    std::vector<double> S, Sc, S2, S2c;
    int32_t* out_end = nullptr;                     // caller's per-walk records (device)
    double* out_w = nullptr;
    long long walks = 0, lost = 0, next_batch = 0;  // next_batch: next to fold
    long long next_assign = 0;                       // next batch to get a record slot
    std::map<long long, std::vector<double>> pending; // reduced, not yet folded
    unsigned long long hops = 0;
    drwc_job_result result{};
    std::chrono::steady_clock::time_point t_submit, t_admit, t_done;
};

}  // namespace drwc

using namespace drwc;

struct drwc_server {
    drwc_ctx* ctx = nullptr;
    drwc_net* bnet[DRWC_SERVER_MAX_SIZES] = {};  // network of each bucket, if any
    bool any_net = false;
    drwc_server_opts o{};
    int bucket_of_N[DRWC_N_MAX + 1];
    // device
    void* dblock = nullptr;
    void* arena_dev = nullptr;
    SvJob* d_jobs = nullptr;
    SvCtr* d_ctr = nullptr;
    SvHdr* d_hdr = nullptr;
    double* d_bsum = nullptr;
    unsigned long long* d_stats = nullptr;
    double* d_akl = nullptr;
    SvArgs A{};
    int fdm_grid[DRWC_SERVER_MAX_SIZES] = {};
    int stem_grid[DRWC_SERVER_MAX_SIZES] = {};
    size_t fdm_smem[DRWC_SERVER_MAX_SIZES] = {};
    double* fdm_sy[DRWC_SERVER_MAX_SIZES] = {};
    float* fdm_ss[DRWC_SERVER_MAX_SIZES] = {};
    // pinned mirrors
    void* hblock = nullptr;
    SvJob* h_jobs = nullptr;
    SvCtr* h_ctr = nullptr;
    SvHdr* h_hdr = nullptr;
    double* h_bsum = nullptr;
    unsigned long long* h_stats = nullptr;
    double* h_akl = nullptr;
    // graph
    cudaStream_t side[DRWC_SERVER_MAX_SIZES] = {};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[DRWC_SERVER_MAX_SIZES] = {};
    cudaEvent_t ev_round0 = nullptr, ev_round1 = nullptr;
    cudaEvent_t ev_t[kSvMaxSteps][2 + 2 * DRWC_SERVER_MAX_SIZES] = {};
    bool timing = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t kernels_per_graph = 0;
    // host state
    std::mutex mu;
    std::condition_variable cv;
    std::thread thr;
    bool stop = false;
    int thread_error = DRWC_OK;
    std::deque<SvHostJob*> queue;
    std::map<int64_t, std::unique_ptr<SvHostJob>> jobs;
    SvHostJob* table[kSvMaxJobs] = {};
    int64_t next_id = 1;
    Arena arena;
    drwc_server_stats st{};
};

namespace drwc {

template <int N>
static int sv_fdm_setup(drwc_server* v, int b) {
    using D = Cube<N>;
    const size_t smem = WalkSmem<N>::bytes(v->o.max_materials, true);
    DRWC_CUDA_TRY(cudaFuncSetAttribute(sv_fdm_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    int per_sm = 0;
    DRWC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sv_fdm_kernel<N>, D::NT, smem));
    if (per_sm < 1) return DRWC_ERR_INVALID;
    v->fdm_grid[b] = per_sm * v->ctx->sm_count;
    v->fdm_smem[b] = smem;
    return DRWC_OK;
}

// The stem kernel's shared memory and a persistent grid of its resident CTAs.
template <int N>
static int sv_stem_setup(drwc_server* v, int b) {
    using D = StemDims<N>;
    DRWC_CUDA_TRY(cudaFuncSetAttribute(sv_stem_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       D::BYTES));
    // all of the unified L1 as shared memory, or the SM holds one CTA fewer
    DRWC_CUDA_TRY(cudaFuncSetAttribute(sv_stem_kernel<N>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       100));
    int per_sm = 0;
    DRWC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sv_stem_kernel<N>, D::NT,
                                                                D::BYTES));
    if (per_sm < 1) return DRWC_ERR_INVALID;
    // at least the CTAs per SM the kernel is built for (the grid loops over
    // groups, so an estimate on the low side costs nothing)
    v->stem_grid[b] = std::max(per_sm, D::CTAS) * v->ctx->sm_count;
    return DRWC_OK;
}

static int sv_fdm_launch(drwc_server* v, int b, cudaStream_t s) {
    const int N = v->o.sizes[b];
    return dispatch_N(N, [&](auto nc) -> int {
        constexpr int NC = decltype(nc)::value;
        sv_fdm_kernel<NC><<<v->fdm_grid[b], Cube<NC>::NT, v->fdm_smem[b], s>>>(
            v->A, b, v->o.max_materials, v->fdm_sy[b], v->fdm_ss[b]);
        return launch_check(v->ctx);
    });
}

// Tables of the homogeneous-cube fast path: panel values of the uniform
// solutions (the warm-start tables, permittivity 1) in ggft panel order and
// their running sums (|value| for the gradient codes, max(value, 0) for the
// Green's function, the weights the FDM hop draws with).
static int sv_tables(drwc_server* v) {
    drwc_ctx* ctx = v->ctx;
    for (int b = 0; b < v->o.n_sizes; ++b) {
        const int N = v->o.sizes[b], NN = N * N, M = 6 * NN;
        const double* w[4];
        int rc = warm_tables(ctx, N, w);
        if (rc) return rc;
        std::vector<double> x((size_t)N * NN), hv(2 * (size_t)M);
        for (int code = 0; code < 4; ++code) {
            DRWC_CUDA_TRY(cudaMemcpy(x.data(), w[code], x.size() * 8, cudaMemcpyDeviceToHost));
            double run = 0.0;
            for (int q = 0; q < M; ++q) {
                const int f = q / NN, tt = q % NN, a = tt % N, bb = tt / N;
                int c;
                switch (f) {
                    case 0: c = a + bb * N; break;
                    case 1: c = a + bb * N + (N - 1) * NN; break;
                    case 2: c = a + bb * NN; break;
                    case 3: c = a + (N - 1) * N + bb * NN; break;
                    case 4: c = a * N + bb * NN; break;
                    default: c = (N - 1) + a * N + bb * NN; break;
                }
                const double val = x[c];
                run += code == DRWC_GFT ? std::max(val, 0.0) : std::fabs(val);
                hv[q] = val;
                hv[M + q] = run;
            }
            DRWC_CUDA_TRY(cudaMemcpy(const_cast<double*>(v->A.tval[b][code]), hv.data(),
                                     2 * (size_t)M * 8, cudaMemcpyHostToDevice));
        }
    }
    return DRWC_OK;
}

// Event nodes when captured (plain records otherwise): stage timing.
static int sv_mark(drwc_server* v, cudaEvent_t e, cudaStream_t s) {
    if (!v->timing) return DRWC_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    DRWC_CUDA_TRY(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusActive)
        DRWC_CUDA_TRY(cudaEventRecordWithFlags(e, s, cudaEventRecordExternal));
    else
        DRWC_CUDA_TRY(cudaEventRecord(e, s));
    return DRWC_OK;
}

// One step on the context stream (captured into the graph).
// One step on the context stream (captured into the graph). FDM buckets
// without a network fork onto their own branches right after prepare; the
// network stages run on the main stream, bucket after bucket, and each such
// bucket's FDM hops (fallbacks and audits) fork once its sampler has routed.
static int sv_step(drwc_server* v, int k) {
    drwc_ctx* ctx = v->ctx;
    cudaStream_t s = ctx->stream;
    const SvArgs& A = v->A;
    int rc;
    sv_reset_kernel<<<1, kSvCnt, 0, s>>>(A);
    if ((rc = launch_check(ctx))) return rc;
    sv_prepare_kernel<<<(A.S * 32 + 255) / 256, 256, 0, s>>>(A);
    if ((rc = launch_check(ctx))) return rc;
    auto fork_fdm = [&](int b) -> int {
        DRWC_CUDA_TRY(cudaEventRecord(v->ev_fork, s));
        DRWC_CUDA_TRY(cudaStreamWaitEvent(v->side[b], v->ev_fork, 0));
        int r = sv_mark(v, v->ev_t[k][2 + 2 * b], v->side[b]);
        if (!r) r = sv_fdm_launch(v, b, v->side[b]);
        if (!r) r = sv_mark(v, v->ev_t[k][3 + 2 * b], v->side[b]);
        if (r) return r;
        DRWC_CUDA_TRY(cudaEventRecord(v->ev_join[b], v->side[b]));
        return DRWC_OK;
    };
    for (int b = 0; b < v->o.n_sizes; ++b)
        if (!v->bnet[b] && (rc = fork_fdm(b))) return rc;
    if (v->any_net && (rc = sv_mark(v, v->ev_t[k][0], s))) return rc;
    // network stages largest cubes first: each bucket's FDM rows (audits,
    // fallbacks) fork once its sampler has run, so the longest solves overlap
    // the other buckets' network stages instead of ending the step
    int order[DRWC_SERVER_MAX_SIZES];
    for (int b = 0; b < v->o.n_sizes; ++b) order[b] = b;
    std::sort(order, order + v->o.n_sizes,
              [&](int a, int c) { return v->o.sizes[a] > v->o.sizes[c]; });
    for (int i = 0; i < v->o.n_sizes; ++i) {
        const int b = order[i];
        if (!v->bnet[b]) continue;
        const int g2 = std::min(A.S, ctx->sm_count * 16);
        rc = dispatch_N(v->o.sizes[b], [&](auto nc) -> int {
            constexpr int NC = decltype(nc)::value;
            if constexpr (NC == 16 || NC == 21 || NC == 23) {
                sv_stem_kernel<NC><<<v->stem_grid[b], StemDims<NC>::NT, StemDims<NC>::BYTES, s>>>(A, b);
                int r = launch_check(ctx);
                if (r) return r;
                r = net_forward_dyn(v->bnet[b], A.S, A.cnt + 4 * b, nullptr, A.O[b], A.Gh[b],
                                    A.frow[b], A.cnt + 4 * b + 1);
                if (r) return r;
                sv_sample_kernel<NC><<<g2, 256, 0, s>>>(A, b);
                return launch_check(ctx);
            } else {
                return DRWC_ERR_INVALID;
            }
        });
        if (rc) return rc;
        if ((rc = fork_fdm(b))) return rc;
    }
    if (v->any_net && (rc = sv_mark(v, v->ev_t[k][1], s))) return rc;
    for (int b = 0; b < v->o.n_sizes; ++b)
        DRWC_CUDA_TRY(cudaStreamWaitEvent(s, v->ev_join[b], 0));
    return DRWC_OK;
}

static int sv_round_body(drwc_server* v) {
    for (int k = 0; k < v->o.steps_per_graph; ++k) {
        const int rc = sv_step(v, k);
        if (rc) return rc;
    }
    cudaStream_t s = v->ctx->stream;
    sv_reduce_kernel<<<dim3(kSvWin * kSvMaxJobs, v->o.max_nets + 3), 256, 0, s>>>(v->A);
    int rc = launch_check(v->ctx);
    if (rc) return rc;
    sv_mark_kernel<<<1, kSvWin * kSvMaxJobs, 0, s>>>(v->A);
    return launch_check(v->ctx);
}

static int sv_capture(drwc_server* v) {
    drwc_ctx* ctx = v->ctx;
    // one uncaptured pass with no job running sets every kernel attribute
    int rc = sv_round_body(v);
    if (rc) return rc;
    DRWC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    const int64_t before = ctx->launches.load();
    DRWC_CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    rc = sv_round_body(v);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (e != cudaSuccess)
            std::fprintf(stderr, "drwc: server graph capture failed: %s\n", cudaGetErrorString(e));
        return rc ? rc : DRWC_ERR_CUDA;
    }
    v->kernels_per_graph = ctx->launches.load() - before;
    ctx->launches.fetch_sub(v->kernels_per_graph);
    v->graph = g;
    DRWC_CUDA_TRY(cudaGraphInstantiate(&v->exec, g, 0));
    return DRWC_OK;
}

static double sv_secs(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

// Footprint of a job in the arena: its structure blob and the records of
// the batches its claim window spans (16 B per walk).
static size_t sv_footprint(const SvHostJob* J, size_t* blob_bytes) {
    const size_t blob = (J->hg.blob.size() + 255) / 256 * 256;
    *blob_bytes = blob;
    const size_t b = (size_t)std::min<long long>(J->p.batch_walks, J->p.max_walks);
    const size_t nb = (size_t)std::min<long long>(kSvWin, (J->p.max_walks + b - 1) / b);
    return blob + nb * b * 16 + 256;
}

// Admit queued jobs in arrival order (caller holds v->mu and the context lock).
static int sv_admit(drwc_server* v) {
    while (!v->queue.empty()) {
        SvHostJob* J = v->queue.front();
        int t = -1;
        for (int q = 0; q < v->o.max_jobs; ++q)
            if (!v->table[q]) { t = q; break; }
        if (t < 0) break;
        size_t blob = 0;
        const size_t need = sv_footprint(J, &blob);
        size_t off = 0;
        if (!v->arena.alloc(need, &off)) {
            if (need > v->arena.size) {  // can never fit
                v->queue.pop_front();
                J->state = DRWC_JOB_FAILED;
                J->error = DRWC_ERR_NOMEM;
                v->st.failed += 1;
                v->cv.notify_all();
                continue;
            }
            break;  // wait for memory to free up
        }
        v->queue.pop_front();
        unsigned char* base = (unsigned char*)v->arena_dev + off;
        // a copy from pageable memory has read the source when it returns
        DRWC_CUDA_TRY(cudaMemcpyAsync(base, J->hg.blob.data(), J->hg.blob.size(),
                                      cudaMemcpyHostToDevice, v->ctx->stream));
        bind_geom(&J->hg, base);
        const long long total = J->p.max_walks;
        const long long batch = std::min<long long>(J->p.batch_walks, total);
        const long long nb = std::min<long long>(kSvWin, (total + batch - 1) / batch);
        SvJob& T = v->h_jobs[t];
        std::memset(&T, 0, sizeof T);
        T.g = J->hg.dev;
        T.G = J->G;
        T.W = J->W;
        T.state = 1;
        T.use_net = v->bnet[v->bucket_of_N[J->p.N]] != nullptr;
        T.bucket = v->bucket_of_N[J->p.N];
        T.n_entries = J->s.n_nets + 1;
        T.total = total;
        T.batch = batch;
        T.limit = std::min(kSvWin * batch, total);
        for (int q = 0; q < kSvWin; ++q) {
            const bool in = q * batch < total;
            T.bfirst[q] = in ? q * batch : -1;
            T.bcount[q] = in ? std::min(batch, total - q * batch) : 0;
        }
        J->next_assign = nb;
        // records: weights, end nets, hop counts for nb window slots
        T.rec_w = (double*)(base + blob);
        T.rec_end = (int32_t*)(base + blob + nb * batch * 8);
        T.rec_hops = T.rec_end + nb * batch;
        T.out_end = J->out_end;
        T.out_w = J->out_w;
        std::memset(&v->h_ctr[t], 0, sizeof(SvCtr));
        J->table = t;
        J->arena_off = off;
        J->arena_bytes = need;
        J->blob_bytes = blob;
        J->state = DRWC_JOB_RUNNING;
        J->t_admit = std::chrono::steady_clock::now();
        const int ne = J->s.n_nets + 1;
        J->S.assign(ne + 1, 0.0); J->Sc.assign(ne + 1, 0.0);
        J->S2.assign(ne + 1, 0.0); J->S2c.assign(ne + 1, 0.0);
        v->table[t] = J;
        v->st.admitted += 1;
    }
    // active list
    SvHdr& H = *v->h_hdr;
    H.n_act = 0;
    for (int q = 0; q < kSvMaxJobs; ++q)
        if (v->table[q] && !v->table[q]->draining) H.act[H.n_act++] = q;
    std::sort(H.act, H.act + H.n_act, [&](int a, int b) { return v->table[a]->id < v->table[b]->id; });
    v->st.max_running = std::max<int64_t>(v->st.max_running, H.n_act);
    return DRWC_OK;
}

// Fold the reduced batches of a running job in batch order; retire it when
// it converges or runs out of walks (same test, same order as drwc_frw_run).
static void sv_fold(drwc_server* v, int t) {
    SvHostJob* J = v->table[t];
    SvJob& T = v->h_jobs[t];
    SvCtr& C = v->h_ctr[t];
    // ids past the limit were never handed out
    if ((long long)C.next > T.limit) C.next = (unsigned long long)T.limit;
    const drwc_job_params& p = J->p;
    const int ne = J->s.n_nets + 1;
    auto kadd = [](double& s, double& c, double x) {
        const double u = s + x;
        if (std::fabs(s) >= std::fabs(x)) c += (s - u) + x;
        else c += (x - u) + s;
        s = u;
    };
    // every reduced batch: keep its sums, free its record slot for the next
    // unassigned batch (a long walk holds back only its own slot)
    for (int q = 0; q < kSvWin; ++q) {
        if (T.bcount[q] <= 0 || !C.reduced[q]) continue;
        const long long kq = T.bfirst[q] / T.batch;
        const double* sums = v->h_bsum + ((size_t)t * kSvWin + q) * kSvBsumStride;
        std::vector<double>& keep = J->pending[kq];
        keep.assign(sums, sums + 3 * (ne + 1) + 1);
        keep.push_back((double)T.bcount[q]);
        const long long kn = J->next_assign;
        if (kn * T.batch < T.total) {
            T.bfirst[q] = kn * T.batch;
            T.bcount[q] = std::min(T.batch, T.total - kn * T.batch);
            J->next_assign = kn + 1;
        } else {
            T.bfirst[q] = -1;
            T.bcount[q] = 0;
        }
        C.done[q] = 0;
        C.reduced[q] = 0;
    }
    T.limit = std::min(J->next_assign * T.batch, T.total);
    // fold in batch order, exactly as drwc_frw_run does
    for (;;) {
        auto it = J->pending.find(J->next_batch);
        if (it == J->pending.end()) break;
        const std::vector<double> sums = std::move(it->second);
        J->pending.erase(it);
        const long long k = J->next_batch;
        for (int e = 0; e <= ne; ++e) {
            kadd(J->S[e], J->Sc[e], sums[3 * e]);
            kadd(J->S2[e], J->S2c[e], sums[3 * e + 1]);
        }
        J->lost += (long long)sums[3 * ne + 2];
        J->hops += (unsigned long long)sums[3 * (ne + 1)];
        J->walks += (long long)sums[3 * (ne + 1) + 1];
        J->next_batch = k + 1;
        bool finished = J->walks >= p.max_walks;
        int converged = 0;
        if (J->walks >= p.min_walks) {
            const double n = (double)J->walks;
            auto mean = [&](int e) { return (J->S[e] + J->Sc[e]) / n; };
            auto sem = [&](int e) {
                const double m = mean(e);
                const double var = std::max(0.0, (J->S2[e] + J->S2c[e]) / n - m * m);
                return std::sqrt(var / n);
            };
            const double cs = mean(p.master);
            bool ok = cs != 0.0 && sem(p.master) <= p.p_tol * std::fabs(cs);
            std::vector<std::pair<double, int>> cpl;
            double ctot = 0.0;
            for (int e = 0; e < ne; ++e) {
                if (e == p.master) continue;
                cpl.push_back({std::fabs(mean(e)), e});
                ctot += std::fabs(mean(e));
            }
            std::sort(cpl.begin(), cpl.end(), [](auto& a, auto& b) { return a.first > b.first; });
            double acc = 0.0;
            for (auto& ce : cpl) {
                if (acc >= p.c_ratio * ctot) break;
                acc += ce.first;
                if (!(ce.first > 0.0) || sem(ce.second) > p.c_tol * ce.first) { ok = false; break; }
            }
            if (ok) { converged = 1; finished = true; }
        }
        if (finished) {
            const double n = (double)std::max(1LL, J->walks);
            drwc_job_result& R = J->result;
            std::memset(&R, 0, sizeof R);
            R.n_entries = ne;
            R.converged = converged;
            R.walks = J->walks;
            R.hops = (int64_t)J->hops;
            R.lost = J->lost;
            for (int e = 0; e < ne; ++e) {
                const double m = (J->S[e] + J->Sc[e]) / n;
                R.cap[e] = m;
                const double var = std::max(0.0, (J->S2[e] + J->S2c[e]) / n - m * m);
                R.stderr_[e] = std::sqrt(var / n);
            }
            J->t_done = std::chrono::steady_clock::now();
            R.seconds = sv_secs(J->t_submit, J->t_done);
            J->state = DRWC_JOB_DONE;
            J->draining = true;
            T.state = 2;
            v->st.completed += 1;
            v->cv.notify_all();
            return;
        }
    }
}

static void sv_release(drwc_server* v, int t) {
    SvHostJob* J = v->table[t];
    v->arena.release(J->arena_off, J->arena_bytes);
    std::memset(&v->h_jobs[t], 0, sizeof(SvJob));
    std::memset(&v->h_ctr[t], 0, sizeof(SvCtr));
    J->table = -1;
    J->hg.blob.clear();
    J->hg.blob.shrink_to_fit();
    v->table[t] = nullptr;
}

// One graph replay and the reads after it (context lock held).
static int sv_round(drwc_server* v) {
    drwc_ctx* ctx = v->ctx;
    cudaStream_t s = ctx->stream;
    DRWC_CUDA_TRY(cudaMemcpyAsync(v->d_jobs, v->h_jobs, sizeof(SvJob) * kSvMaxJobs,
                                  cudaMemcpyHostToDevice, s));
    DRWC_CUDA_TRY(cudaMemcpyAsync(v->d_ctr, v->h_ctr, sizeof(SvCtr) * kSvMaxJobs,
                                  cudaMemcpyHostToDevice, s));
    DRWC_CUDA_TRY(cudaMemcpyAsync(v->d_hdr, v->h_hdr, sizeof(SvHdr), cudaMemcpyHostToDevice, s));
    DRWC_CUDA_TRY(cudaEventRecord(v->ev_round0, s));
    DRWC_CUDA_TRY(cudaGraphLaunch(v->exec, s));
    DRWC_CUDA_TRY(cudaEventRecord(v->ev_round1, s));
    ctx->launches.fetch_add(v->kernels_per_graph);
    DRWC_CUDA_TRY(cudaMemcpyAsync(v->h_ctr, v->d_ctr, sizeof(SvCtr) * kSvMaxJobs,
                                  cudaMemcpyDeviceToHost, s));
    DRWC_CUDA_TRY(cudaMemcpyAsync(v->h_bsum, v->d_bsum, sizeof(double) * kSvBsumStride * kSvWin * kSvMaxJobs,
                                  cudaMemcpyDeviceToHost, s));
    DRWC_CUDA_TRY(cudaMemcpyAsync(v->h_stats, v->d_stats, sizeof(unsigned long long) * SV_NSTATS,
                                  cudaMemcpyDeviceToHost, s));
    DRWC_CUDA_TRY(cudaMemcpyAsync(v->h_akl, v->d_akl, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    DRWC_CUDA_TRY(cudaStreamSynchronize(s));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, v->ev_round0, v->ev_round1) == cudaSuccess)
        v->st.busy_seconds += ms * 1e-3;
    if (v->timing) {
        for (int k = 0; k < v->o.steps_per_graph; ++k) {
            if (v->any_net && cudaEventElapsedTime(&ms, v->ev_t[k][0], v->ev_t[k][1]) == cudaSuccess)
                v->st.net_seconds += ms * 1e-3;
            for (int b = 0; b < v->o.n_sizes; ++b)
                if (cudaEventElapsedTime(&ms, v->ev_t[k][2 + 2 * b], v->ev_t[k][3 + 2 * b]) ==
                    cudaSuccess)
                    v->st.fdm_seconds += ms * 1e-3;
        }
        cudaGetLastError();
    }
    v->st.graph_launches += 1;
    v->st.kernels_launched += v->kernels_per_graph;
    return DRWC_OK;
}

static void sv_thread(drwc_server* v) {
    std::unique_lock<std::mutex> lk(v->mu);
    for (;;) {
        if (v->stop) break;
        bool any = false;
        for (int q = 0; q < kSvMaxJobs; ++q) any |= v->table[q] != nullptr;
        if (!any && v->queue.empty()) {
            v->cv.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        int rc;
        {
            std::lock_guard<std::mutex> clk(v->ctx->mu);
            cudaSetDevice(v->ctx->device);
            rc = sv_admit(v);
            bool running = false;
            for (int q = 0; q < kSvMaxJobs; ++q) running |= v->table[q] != nullptr;
            if (!rc && running) {
                lk.unlock();  // submissions and polls proceed during the replay
                rc = sv_round(v);
                lk.lock();
            }
        }
        if (rc) {
            v->thread_error = rc;
            break;
        }
        std::this_thread::yield();  // let other users of the context in between replays
        for (int q = 0; q < kSvMaxJobs; ++q) {
            if (!v->table[q]) continue;
            if (!v->table[q]->draining) sv_fold(v, q);
            else if ((long long)v->h_ctr[q].inflight == 0) sv_release(v, q);
        }
        const unsigned long long* h = v->h_stats;
        v->st.hops = (int64_t)h[SV_HOPS];
        v->st.net_hops = (int64_t)h[SV_NET_HOPS];
        v->st.fdm_hops = (int64_t)h[SV_FDM_HOPS];
        v->st.fallbacks = (int64_t)h[SV_FALLBACKS];
        v->st.audits = (int64_t)h[SV_AUDITS];
        v->st.walks_finished = (int64_t)h[SV_WALKS_DONE];
        v->st.walks_dropped = (int64_t)h[SV_WALKS_DROPPED];
        v->st.net_rows = (double)h[SV_NET_ROWS];
        v->st.fdm_iters = (int64_t)h[SV_FDM_ITERS];
        v->st.fdm_sweeps = (int64_t)h[SV_FDM_SWEEPS];
        v->st.fdm_bytes = (double)h[SV_FDM_BYTES];
        v->st.table_hops = (int64_t)h[SV_TABLE_HOPS];
        v->st.fdm_escalated = (int64_t)h[SV_FDM_ESCALATED];
        v->st.fdm_failed = (int64_t)h[SV_FDM_FAILED];
        v->st.audit_kl_mean = v->h_akl[1] > 0 ? v->h_akl[0] / v->h_akl[1] : 0.0;
    }
    // stopped (destroy or an error): every job not done ends as failed
    const int why = v->thread_error ? v->thread_error : DRWC_ERR_SHUTDOWN;
    for (auto& kv : v->jobs) {
        SvHostJob* J = kv.second.get();
        if (J->state == DRWC_JOB_QUEUED || J->state == DRWC_JOB_RUNNING) {
            J->state = DRWC_JOB_FAILED;
            J->error = why;
            v->st.failed += 1;
        }
    }
    v->queue.clear();
    v->stop = true;
    v->cv.notify_all();
}

static int sv_alloc(drwc_server* v) {
    const int S = v->o.slots;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t r = off; off += (bytes + 255) / 256 * 256; return r; };
    const size_t o_jobs = take(sizeof(SvJob) * kSvMaxJobs), o_ctr = take(sizeof(SvCtr) * kSvMaxJobs),
                 o_hdr = take(sizeof(SvHdr)), o_bsum = take(8 * kSvBsumStride * kSvWin * kSvMaxJobs),
                 o_stats = take(8 * SV_NSTATS), o_akl = take(16), o_cnt = take(4 * kSvCnt),
                 o_dbl = take(8 * (size_t)S * 7), o_walk = take(8 * (size_t)S),
                 o_int = take(4 * (size_t)S * 5),
                 o_b = take(4 * (size_t)S * 2 * DRWC_SERVER_MAX_SIZES);
    size_t o_O[DRWC_SERVER_MAX_SIZES] = {}, o_G[DRWC_SERVER_MAX_SIZES] = {},
           o_al[DRWC_SERVER_MAX_SIZES] = {};
    for (int b = 0; b < v->o.n_sizes; ++b) {
        if (!v->bnet[b]) continue;
        int32_t orow = 0, grow = 0;
        drwc_net_dims(v->bnet[b], nullptr, nullptr, &orow, &grow, nullptr);
        v->A.out_row[b] = orow;
        v->A.grad_row[b] = grow;
        o_O[b] = take(4 * (size_t)S * orow);
        o_G[b] = take(4 * (size_t)S * grow);
        o_al[b] = take(4 * (size_t)S * 2);
    }
    size_t o_sy[DRWC_SERVER_MAX_SIZES], o_ss[DRWC_SERVER_MAX_SIZES], o_tab[DRWC_SERVER_MAX_SIZES];
    for (int b = 0; b < v->o.n_sizes; ++b) {
        const size_t nnn = (size_t)v->o.sizes[b] * v->o.sizes[b] * v->o.sizes[b];
        o_sy[b] = take(8 * (size_t)v->fdm_grid[b] * nnn);
        o_ss[b] = take(4 * (size_t)v->fdm_grid[b] * nnn);
        o_tab[b] = take(8 * 4 * 2 * 6 * (size_t)v->o.sizes[b] * v->o.sizes[b]);
    }
    if (cudaMalloc(&v->dblock, off) != cudaSuccess) { cudaGetLastError(); return DRWC_ERR_NOMEM; }
    DRWC_CUDA_TRY(cudaMemset(v->dblock, 0, off));
    if (cudaMalloc(&v->arena_dev, (size_t)v->o.hbm_budget) != cudaSuccess) {
        cudaGetLastError();
        return DRWC_ERR_NOMEM;
    }
    v->arena.init((size_t)v->o.hbm_budget);
    unsigned char* B = (unsigned char*)v->dblock;
    v->d_jobs = (SvJob*)(B + o_jobs);
    v->d_ctr = (SvCtr*)(B + o_ctr);
    v->d_hdr = (SvHdr*)(B + o_hdr);
    v->d_bsum = (double*)(B + o_bsum);
    v->d_stats = (unsigned long long*)(B + o_stats);
    v->d_akl = (double*)(B + o_akl);
    SvArgs& A = v->A;
    A.S = S;
    A.n_buckets = v->o.n_sizes;
    A.jobs = v->d_jobs;
    A.ctr = v->d_ctr;
    A.hdr = v->d_hdr;
    A.bsum = v->d_bsum;
    A.stats = v->d_stats;
    A.audit_kl = v->d_akl;
    A.cnt = (unsigned*)(B + o_cnt);
    double* dd = (double*)(B + o_dbl);
    A.st.px = dd; A.st.py = dd + S; A.st.pz = dd + 2 * S; A.st.omega = dd + 3 * S;
    A.st.sgn = dd + 4 * S; A.st.a = dd + 5 * S; A.st.epsw = dd + 6 * S;
    A.st.walk = (long long*)(B + o_walk);
    int* ii = (int*)(B + o_int);
    A.st.hops = ii; A.st.mode = ii + S; A.st.code = ii + 2 * S; A.st.job = ii + 3 * S;
    A.st.grow = ii + 4 * S;
    int* bl = (int*)(B + o_b);
    for (int b = 0; b < DRWC_SERVER_MAX_SIZES; ++b) {
        A.blist[b] = bl + (size_t)2 * b * S;
        A.bkind[b] = bl + (size_t)(2 * b + 1) * S;
    }
    A.conf_thresh = v->o.conf_threshold;
    A.audit_frac = v->o.audit_frac;
    for (int b = 0; b < v->o.n_sizes; ++b) {
        if (!v->bnet[b]) continue;
        A.O[b] = (float*)(B + o_O[b]);
        A.Gh[b] = (float*)(B + o_G[b]);
        A.alist[b] = (int*)(B + o_al[b]);
        A.frow[b] = A.alist[b] + S;
    }
    A.table = v->o.uniform_table;
    A.fair = v->o.fair_share;
    A.fdm_hops = v->o.fdm_hops;
    A.strag_hops = v->o.straggler_hops;
    for (int b = 0; b < v->o.n_sizes; ++b) {
        v->fdm_sy[b] = (double*)(B + o_sy[b]);
        v->fdm_ss[b] = (float*)(B + o_ss[b]);
        const size_t M = 6 * (size_t)v->o.sizes[b] * v->o.sizes[b];
        for (int code = 0; code < 4; ++code) {
            double* t = (double*)(B + o_tab[b]) + (size_t)code * 2 * M;
            A.tval[b][code] = t;
            A.tcdf[b][code] = t + M;
        }
    }
    // pinned mirrors
    size_t hoff = 0;
    auto htake = [&](size_t bytes) { size_t r = hoff; hoff += (bytes + 255) / 256 * 256; return r; };
    const size_t h_jobs = htake(sizeof(SvJob) * kSvMaxJobs), h_ctr = htake(sizeof(SvCtr) * kSvMaxJobs),
                 h_hdr = htake(sizeof(SvHdr)), h_bsum = htake(8 * kSvBsumStride * kSvWin * kSvMaxJobs),
                 h_stats = htake(8 * SV_NSTATS), h_akl = htake(16);
    if (cudaMallocHost(&v->hblock, hoff) != cudaSuccess) { cudaGetLastError(); return DRWC_ERR_NOMEM; }
    std::memset(v->hblock, 0, hoff);
    unsigned char* H = (unsigned char*)v->hblock;
    v->h_jobs = (SvJob*)(H + h_jobs);
    v->h_ctr = (SvCtr*)(H + h_ctr);
    v->h_hdr = (SvHdr*)(H + h_hdr);
    v->h_bsum = (double*)(H + h_bsum);
    v->h_stats = (unsigned long long*)(H + h_stats);
    v->h_akl = (double*)(H + h_akl);
    return DRWC_OK;
}

static void sv_free(drwc_server* v) {
    if (v->exec) cudaGraphExecDestroy(v->exec);
    if (v->graph) cudaGraphDestroy(v->graph);
    for (int b = 0; b < DRWC_SERVER_MAX_SIZES; ++b) {
        if (v->side[b]) cudaStreamDestroy(v->side[b]);
        if (v->ev_join[b]) cudaEventDestroy(v->ev_join[b]);
    }
    for (cudaEvent_t e : {v->ev_fork, v->ev_round0, v->ev_round1})
        if (e) cudaEventDestroy(e);
    for (int k = 0; k < kSvMaxSteps; ++k)
        for (int q = 0; q < 2 + 2 * DRWC_SERVER_MAX_SIZES; ++q)
            if (v->ev_t[k][q]) cudaEventDestroy(v->ev_t[k][q]);
    if (v->dblock) cudaFree(v->dblock);
    if (v->arena_dev) cudaFree(v->arena_dev);
    if (v->hblock) cudaFreeHost(v->hblock);
}

}  // namespace drwc

extern "C" {

DRWC_API void drwc_server_opts_default(drwc_server_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->slots = 0;
    o->max_jobs = 32;
    o->hbm_budget = 1LL << 30;
    o->n_sizes = 3;
    o->sizes[0] = 16;
    o->sizes[1] = 21;
    o->sizes[2] = 23;
    o->steps_per_graph = 2;
    o->max_materials = 16;
    o->max_nets = 64;
    o->conf_threshold = -1.5f;
    o->audit_frac = 0.01f;
    o->timing = 0;
    o->uniform_table = 0;
    o->fair_share = 0;
    o->fdm_hops = 0;
    o->straggler_hops = 0;
}

static_assert(sizeof(drwc_server_opts) == 80, "the option layout the bindings mirror");

DRWC_API int drwc_server_create(drwc_ctx* ctx, const drwc_server_opts* opts,
                                drwc_net* const* nets, int32_t n_nets, drwc_server** out) {
    if (!ctx || !out) return DRWC_ERR_INVALID;
    *out = nullptr;
    drwc_server_opts o;
    drwc_server_opts_default(&o);
    if (opts) o = *opts;
    if (o.slots < 0 || o.slots > (1 << 22) || o.max_jobs < 1 || o.max_jobs > kSvMaxJobs ||
        o.hbm_budget < 4096 || o.n_sizes < 1 || o.n_sizes > DRWC_SERVER_MAX_SIZES ||
        o.steps_per_graph < 1 || o.steps_per_graph > kSvMaxSteps || o.max_materials < 1 ||
        o.max_materials > kMaxMaterials || o.max_nets < 1 || o.max_nets > DRWC_MAX_NETS ||
        !(o.audit_frac >= 0.f && o.audit_frac <= 1.f) || o.uniform_table < 0 || o.uniform_table > 1 ||
        o.fair_share < 0 || o.fair_share > 1 || o.fdm_hops < 0 || o.fdm_hops > 64 ||
        o.straggler_hops < 0)
        return DRWC_ERR_INVALID;
    if (n_nets < 0 || n_nets > DRWC_SERVER_MAX_SIZES || (n_nets > 0 && !nets))
        return DRWC_ERR_INVALID;
    std::unique_ptr<drwc_server> v(new drwc_server());
    v->ctx = ctx;
    v->o = o;
    v->timing = o.timing != 0;
    for (int n = 0; n <= DRWC_N_MAX; ++n) v->bucket_of_N[n] = -1;
    for (int b = 0; b < o.n_sizes; ++b) {
        const int N = o.sizes[b];
        if (!n_supported(N) || v->bucket_of_N[N] >= 0) return DRWC_ERR_INVALID;
        v->bucket_of_N[N] = b;
    }
    // each network serves the jobs of its own resolution
    for (int q = 0; q < n_nets; ++q) {
        drwc_net* net = nets[q];
        if (!net || net_context(net) != ctx) return DRWC_ERR_INVALID;
        const int N = net_size(net);
        const int b = N <= DRWC_N_MAX ? v->bucket_of_N[N] : -1;
        if (b < 0 || v->bnet[b]) return DRWC_ERR_INVALID;
        v->bnet[b] = net;
        v->any_net = true;
    }
    if (v->o.slots == 0) v->o.slots = 65536;
    if (v->o.fdm_hops == 0) v->o.fdm_hops = 64;
    if (v->o.straggler_hops == 0) v->o.straggler_hops = 32;
    o = v->o;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        DRWC_CUDA_TRY(cudaSetDevice(ctx->device));
        int rc = DRWC_OK;
        for (int b = 0; !rc && b < o.n_sizes; ++b) {
            rc = dispatch_N(o.sizes[b], [&](auto nc) -> int {
                return sv_fdm_setup<decltype(nc)::value>(v.get(), b);
            });
            const double* w[4];
            if (!rc) rc = warm_tables(ctx, o.sizes[b], w);
        }
        for (int b = 0; !rc && b < o.n_sizes; ++b) {
            if (!v->bnet[b]) continue;
            rc = dispatch_N(o.sizes[b], [&](auto nc) -> int {
                constexpr int NC = decltype(nc)::value;
                if constexpr (NC == 16 || NC == 21 || NC == 23) {
                    return sv_stem_setup<NC>(v.get(), b);
                } else {
                    return DRWC_ERR_INVALID;
                }
            });
            if (!rc) rc = net_reserve_rows(v->bnet[b], o.slots);
            if (!rc) v->A.stem[b] = net_stem_operands(v->bnet[b]);  // a2 as reserved for `slots` rows
        }
        if (!rc) rc = sv_alloc(v.get());
        if (!rc) rc = sv_tables(v.get());
        for (int b = 0; !rc && b < o.n_sizes; ++b) {
            if (cudaStreamCreateWithFlags(&v->side[b], cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&v->ev_join[b], cudaEventDisableTiming) != cudaSuccess)
                rc = DRWC_ERR_CUDA;
        }
        if (!rc && (cudaEventCreateWithFlags(&v->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
                    cudaEventCreate(&v->ev_round0) != cudaSuccess ||
                    cudaEventCreate(&v->ev_round1) != cudaSuccess))
            rc = DRWC_ERR_CUDA;
        for (int k = 0; !rc && v->timing && k < o.steps_per_graph; ++k)
            for (int q = 0; q < 2 + 2 * o.n_sizes; ++q)
                if (cudaEventCreate(&v->ev_t[k][q]) != cudaSuccess) rc = DRWC_ERR_CUDA;
        if (!rc) rc = sv_capture(v.get());
        for (int b = 0; !rc && b < o.n_sizes; ++b)
            if (v->bnet[b]) net_hold(v->bnet[b], 1);
        if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = DRWC_ERR_CUDA;
        if (rc) {
            cudaGetLastError();
            cudaStreamSynchronize(ctx->stream);
            sv_free(v.get());
            return rc;
        }
    }
    v->st.arena_bytes = o.hbm_budget;
    drwc_server* raw = v.release();
    raw->thr = std::thread(sv_thread, raw);
    *out = raw;
    return DRWC_OK;
}

DRWC_API int drwc_server_destroy(drwc_server* v) {
    if (!v) return DRWC_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(v->mu);
        v->stop = true;
        v->cv.notify_all();
    }
    if (v->thr.joinable()) v->thr.join();
    {
        std::lock_guard<std::mutex> lock(v->ctx->mu);
        cudaSetDevice(v->ctx->device);
        cudaStreamSynchronize(v->ctx->stream);
        for (int b = 0; b < DRWC_SERVER_MAX_SIZES; ++b)
            if (v->bnet[b]) net_hold(v->bnet[b], -1);
        sv_free(v);
    }
    delete v;
    return DRWC_OK;
}

DRWC_API int drwc_server_submit(drwc_server* v, const drwc_structure* s, const drwc_job_params* p,
                                int64_t* job_id) {
    return drwc_server_submit_records(v, s, p, nullptr, nullptr, job_id);
}

DRWC_API int drwc_server_submit_records(drwc_server* v, const drwc_structure* s,
                                        const drwc_job_params* p, int32_t* end_net,
                                        double* weight, int64_t* job_id) {
    if (!v || !s || !p || !job_id || (!end_net) != (!weight)) return DRWC_ERR_INVALID;
    *job_id = 0;
    if (!n_supported(p->N) || v->bucket_of_N[p->N] < 0 || p->batch_walks < 1 ||
        p->max_walks < 1 || p->min_walks < 0 || s->n_nets > v->o.max_nets || s->n_boxes < 0 ||
        (s->n_boxes > 0 && !s->boxes))
        return DRWC_ERR_INVALID;
    std::unique_ptr<SvHostJob> J(new SvHostJob());
    J->boxes.assign(s->boxes, s->boxes + s->n_boxes);
    if (s->n_layers > 0 && s->layer_zlo && s->layer_eps) {
        J->zlo.assign(s->layer_zlo, s->layer_zlo + s->n_layers);
        J->leps.assign(s->layer_eps, s->layer_eps + s->n_layers);
    }
    if (s->n_diel > 0 && s->diel) J->diel.assign(s->diel, s->diel + s->n_diel);
    J->s = *s;
    J->s.boxes = J->boxes.data();
    J->s.layer_zlo = J->zlo.empty() ? nullptr : J->zlo.data();
    J->s.layer_eps = J->leps.empty() ? nullptr : J->leps.data();
    J->s.diel = J->diel.empty() ? nullptr : J->diel.data();
    J->p = *p;
    J->out_end = end_net;
    J->out_w = weight;
    // validation, Gaussian surface and packing run on the host; the
    // warm-start tables of the served sizes were made at creation, so this
    // needs neither the device nor the context lock
    const int rc = prepare(v->ctx, &J->s, &J->p, &J->hg, &J->G, &J->W);
    if (rc) return rc;
    if (J->hg.dev.n_mat > v->o.max_materials) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(v->mu);
    if (v->stop) return DRWC_ERR_SHUTDOWN;
    J->id = v->next_id++;
    J->t_submit = std::chrono::steady_clock::now();
    *job_id = J->id;
    v->queue.push_back(J.get());
    v->jobs[J->id] = std::move(J);
    v->st.submitted += 1;
    v->cv.notify_all();
    return DRWC_OK;
}

DRWC_API int drwc_server_poll(drwc_server* v, int64_t id, int32_t* state, drwc_job_result* out) {
    if (!v || !state) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(v->mu);
    auto it = v->jobs.find(id);
    if (it == v->jobs.end()) return DRWC_ERR_INVALID;
    const SvHostJob* J = it->second.get();
    *state = J->state;
    if (out && J->state == DRWC_JOB_DONE) *out = J->result;
    return J->state == DRWC_JOB_FAILED ? J->error : DRWC_OK;
}

DRWC_API int drwc_server_wait(drwc_server* v, int64_t id, double timeout_s, drwc_job_result* out) {
    if (!v) return DRWC_ERR_INVALID;
    std::unique_lock<std::mutex> lk(v->mu);
    auto it = v->jobs.find(id);
    if (it == v->jobs.end()) return DRWC_ERR_INVALID;
    const SvHostJob* J = it->second.get();
    const auto deadline = std::chrono::steady_clock::now() +
                          std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                              std::chrono::duration<double>(std::max(0.0, timeout_s)));
    while (J->state != DRWC_JOB_DONE && J->state != DRWC_JOB_FAILED) {
        if (v->cv.wait_until(lk, deadline) == std::cv_status::timeout &&
            J->state != DRWC_JOB_DONE && J->state != DRWC_JOB_FAILED)
            return DRWC_ERR_TIMEOUT;
    }
    if (J->state == DRWC_JOB_FAILED) return J->error ? J->error : DRWC_ERR_SHUTDOWN;
    if (out) *out = J->result;
    return DRWC_OK;
}

DRWC_API int drwc_server_job_times(drwc_server* v, int64_t id, double* queued_s, double* latency_s) {
    if (!v) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(v->mu);
    auto it = v->jobs.find(id);
    if (it == v->jobs.end()) return DRWC_ERR_INVALID;
    const SvHostJob* J = it->second.get();
    if (J->state != DRWC_JOB_DONE) return DRWC_ERR_INVALID;
    if (queued_s) *queued_s = sv_secs(J->t_submit, J->t_admit);
    if (latency_s) *latency_s = sv_secs(J->t_submit, J->t_done);
    return DRWC_OK;
}

DRWC_API int drwc_server_stats_get(drwc_server* v, drwc_server_stats* out) {
    if (!v || !out) return DRWC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(v->mu);
    drwc_server_stats s = v->st;
    s.queued = (int64_t)v->queue.size();
    s.running = 0;
    for (int q = 0; q < kSvMaxJobs; ++q) s.running += v->table[q] && !v->table[q]->draining;
    s.arena_bytes = (int64_t)v->arena.size;
    s.arena_used = (int64_t)v->arena.used;
    s.arena_peak = (int64_t)v->arena.peak;
    *out = s;
    return v->thread_error;
}

}  // extern "C"
