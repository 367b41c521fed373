/* TEST INFRASTRUCTURE ONLY — CPU restatement of the floating-random-walk
 * capacitance walk, used as the parity checker for the device walker and as
 * the timed CPU baseline. The product library never links or calls it.
 *
 * The reference walker is closed (executable/librwcapall.so ships compiled
 * only), so the walk is written from the published FRW method and from what
 * the reference's open interfaces fix:
 *   - transition cubes are the largest conductor-free cubes centred at the
 *     walker (L-infinity distance to the nearest conductor or enclosure wall);
 *   - the cube's permittivity is sampled at cell centres (2i+1)/N-1
 *     (cuda_kernels.cu:41-44; dielectric_generator.h:109-127);
 *   - every hop's transition probabilities are the FDM surface Green's
 *     function of that cube (ggft GFT solve), the first hop uses the
 *     centre-gradient surface values along the Gaussian-surface normal
 *     (WVTX/Y/Z) and carries weight sum|g| * sign(g_b) * centre permittivity
 *     (dnn_solver_gradient.cpp:143-162), scaled by the Gaussian surface area
 *     and the cube half-width;
 *   - panel b moves the walker to the panel centre (locate_index_simple,
 *     cuda_kernels.cu:219-264) scaled by the cube half-width.
 * Walk w draws from Philox4x32-10 keyed by the job seed with counter
 * (w, hop, draw, 0), so every walk is independent of how walks are batched.
 *
 * Geometry arithmetic is plain FP64 without contraction (the Makefile builds
 * with -ffp-contract=off) so that the device walker, which uses explicitly
 * rounded operations, visits the same points.
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "philox.h"

#define EPS0_FF_PER_UM 8.8541878128e-3 /* vacuum permittivity, fF per um */

double orc_distance(const drwc_structure* s, const double r[3], int32_t* net) {
    double best = INFINITY;
    int32_t bn = s->n_nets; /* ground */
    for (int a = 0; a < 3; ++a) {
        double d1 = r[a] - s->encl_lo[a];
        double d2 = s->encl_hi[a] - r[a];
        if (d1 < best) best = d1;
        if (d2 < best) best = d2;
    }
    for (int b = 0; b < s->n_boxes; ++b) {
        const drwc_box* B = &s->boxes[b];
        double d = 0;
        for (int a = 0; a < 3; ++a) {
            double lo = B->lo[a] - r[a];
            double hi = r[a] - B->hi[a];
            double m = lo > hi ? lo : hi;
            if (m > d) d = m;
        }
        if (d < best) {
            best = d;
            bn = B->net;
        }
    }
    if (net) *net = bn;
    return best;
}

double orc_eps_at(const drwc_structure* s, const double r[3]) {
    for (int b = 0; b < s->n_diel; ++b) {
        const drwc_diel_box* D = &s->diel[b];
        if (r[0] >= D->lo[0] && r[0] <= D->hi[0] && r[1] >= D->lo[1] && r[1] <= D->hi[1] &&
            r[2] >= D->lo[2] && r[2] <= D->hi[2])
            return D->eps;
    }
    if (s->n_layers <= 0) return 1.0;
    int li = 0;
    for (int l = 0; l < s->n_layers; ++l) {
        if (r[2] >= s->layer_zlo[l]) li = l;
        else break;
    }
    return s->layer_eps[li];
}

static void voxelise(const drwc_structure* s, int N, const double c[3], double a, double* eps) {
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                double p[3];
                p[0] = c[0] + a * ((2.0 * i + 1.0) / N - 1.0);
                p[1] = c[1] + a * ((2.0 * j + 1.0) / N - 1.0);
                p[2] = c[2] + a * ((2.0 * k + 1.0) / N - 1.0);
                eps[i + j * N + k * N * N] = orc_eps_at(s, p);
            }
}

typedef struct {
    double lo[3], hi[3];
    double area[6];
    double total;
} gauss_surface;

static void gauss_build(const drwc_structure* s, const drwc_job_params* p, gauss_surface* G) {
    for (int a = 0; a < 3; ++a) {
        G->lo[a] = INFINITY;
        G->hi[a] = -INFINITY;
    }
    for (int b = 0; b < s->n_boxes; ++b) {
        if (s->boxes[b].net != p->master) continue;
        for (int a = 0; a < 3; ++a) {
            if (s->boxes[b].lo[a] < G->lo[a]) G->lo[a] = s->boxes[b].lo[a];
            if (s->boxes[b].hi[a] > G->hi[a]) G->hi[a] = s->boxes[b].hi[a];
        }
    }
    for (int a = 0; a < 3; ++a) {
        G->lo[a] = G->lo[a] - p->gauss_offset;
        G->hi[a] = G->hi[a] + p->gauss_offset;
    }
    double dx = G->hi[0] - G->lo[0], dy = G->hi[1] - G->lo[1], dz = G->hi[2] - G->lo[2];
    double az = dx * dy, ay = dx * dz, ax = dy * dz;
    G->area[0] = az; G->area[1] = az;
    G->area[2] = ay; G->area[3] = ay;
    G->area[4] = ax; G->area[5] = ax;
    G->total = 0;
    for (int f = 0; f < 6; ++f) G->total += G->area[f];
}

static void walk_one(const drwc_structure* s, const drwc_job_params* p, const gauss_surface* G,
                     orc_fdm_fn fdm, double tol, int64_t w, double* eps, double* g,
                     int32_t* end_out, int32_t* hops_out, double* omega_out) {
    const int N = p->N, M = 6 * N * N;
    double u[2], v[2];
    orc_philox_uniform2(p->seed, (uint64_t)w, 0, 0, &u[0], &u[1]);
    orc_philox_uniform2(p->seed, (uint64_t)w, 0, 1, &v[0], &v[1]);
    /* start point: face by area, then uniform on the face */
    double target = u[0] * G->total, run = 0;
    int f = 5;
    for (int t = 0; t < 6; ++t) {
        run += G->area[t];
        if (run > target) { f = t; break; }
    }
    double r[3];
    int axis = f < 2 ? 2 : f < 4 ? 1 : 0;
    int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2; /* tangential axes */
    r[t0] = G->lo[t0] + u[1] * (G->hi[t0] - G->lo[t0]);
    r[t1] = G->lo[t1] + v[0] * (G->hi[t1] - G->lo[t1]);
    r[axis] = (f & 1) ? G->hi[axis] : G->lo[axis];
    const double sgn_out = (f & 1) ? 1.0 : -1.0;
    const int code = axis == 0 ? DRWC_WVTX : axis == 1 ? DRWC_WVTY : DRWC_WVTZ;

    int32_t net;
    double a = orc_distance(s, r, &net);
    if (a < p->stop_dist) { /* degenerate start: no transition possible */
        *end_out = net; *hops_out = 0; *omega_out = 0.0;
        return;
    }
    voxelise(s, N, r, a, eps);
    fdm(N, eps, code, tol, g);
    int b = orc_sample_index(M, g, 1, v[1]);
    double W = 0;
    for (int i = 0; i < M; ++i) W += fabs(g[i]);
    double sg = g[b] < 0 ? -1.0 : 1.0;
    double eps_w = orc_center_diel(N, eps, code);
    double omega = -sgn_out * G->total * eps_w * W * sg / a * EPS0_FF_PER_UM;
    double loc[3];
    orc_locate_f64(N, b, loc);
    for (int d = 0; d < 3; ++d) r[d] = r[d] + a * loc[d];
    int32_t hops = 1;
    for (;;) {
        a = orc_distance(s, r, &net);
        if (a < p->stop_dist) break;
        if (hops >= p->max_hops) { net = -1; break; }
        voxelise(s, N, r, a, eps);
        fdm(N, eps, DRWC_GFT, tol, g);
        orc_philox_uniform2(p->seed, (uint64_t)w, (uint32_t)hops, 0, &u[0], &u[1]);
        b = orc_sample_index(M, g, 0, u[0]);
        orc_locate_f64(N, b, loc);
        for (int d = 0; d < 3; ++d) r[d] = r[d] + a * loc[d];
        ++hops;
    }
    *end_out = net;
    *hops_out = hops;
    *omega_out = omega;
}

int orc_frw_walks(const drwc_structure* s, const drwc_job_params* p, int64_t walk0,
                  int64_t nwalks, orc_fdm_fn fdm, double fdm_tol, int nthreads,
                  int32_t* end_net, int32_t* hops, double* weight, double* seconds) {
    gauss_surface G;
    gauss_build(s, p, &G);
    if (!fdm) fdm = orc_fdm_solve_cb;
    if (nthreads < 1) nthreads = 1;
    const int N = p->N;
    double t0 = omp_get_wtime();
#pragma omp parallel num_threads(nthreads)
    {
        double* eps = (double*)malloc(sizeof(double) * N * N * N);
        double* g = (double*)malloc(sizeof(double) * 6 * N * N);
#pragma omp for schedule(dynamic, 1)
        for (int64_t i = 0; i < nwalks; ++i)
            walk_one(s, p, &G, fdm, fdm_tol, walk0 + i, eps, g, &end_net[i], &hops[i], &weight[i]);
        free(eps);
        free(g);
    }
    if (seconds) *seconds = omp_get_wtime() - t0;
    return 0;
}
