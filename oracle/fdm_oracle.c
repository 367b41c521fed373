/* TEST INFRASTRUCTURE ONLY — CPU restatement (FP64) of the reference's FDM
 * surface Green's function and of the dnnsolver data path. Used by tests/,
 * the smoke check and bench.py's CPU baseline as the checker; never by the
 * product library.
 *
 * FDM operator. ggft assembles, per cube, A = A21*A12 + 6I and then rewrites
 * it cell by cell (dielectric_opt, ggft/src/ggft_solver.cpp:447-518, driven
 * by update_matrix :276-290). Written out, row p of that matrix is
 *     A_pp = 6 - sum_q eps_p/(eps_p+eps_q),   A_pq = -eps_p/(eps_p+eps_q)
 * over the face neighbours q inside the cube. This equals K * diag(1/eps)
 * with K symmetric positive definite:
 *     K_pq = -g_pq,  g_pq = eps_p*eps_q/(eps_p+eps_q),
 *     K_pp = sum_q g_pq + eps_p * (number of cube faces cell p touches).
 * So ggft's `inner` = A^{-1} e is eps .* y with K y = e, and gft = A13*inner
 * (ggft_solver.cpp:594-596; A13 picks the cell under each boundary panel,
 * laplace() :292-326) is eps_c * y_c for the cell c under each panel. This
 * file solves K y = e with Jacobi-preconditioned CG in FP64 instead of
 * ggft's BiCGSTAB/SparseLU (:552-589); the two agree to the solvers'
 * tolerances (checked against the reference build in tests/).
 *
 * Right-hand sides restate update_ek (ggft_solver.cpp:137-274): a unit source
 * at the centre cell for odd N, split over the 8 centre cells in proportion
 * to eps for even N, and the centre-gradient (h = 2/N) sources WVTX/Y/Z.
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "philox.h"

static inline int cidx(int N, int i, int j, int k) { return i + j * N + k * N * N; }

/* ggft_solver.cpp:137-274 */
void orc_rhs(int N, const double* eps, int code, double* e) {
    const int nnn = N * N * N;
    memset(e, 0, sizeof(double) * nnn);
    const double h = 2.0 / N;
    const int c = N / 2;
    if (N % 2) {
        const int zzz = cidx(N, c, c, c);
        if (code == DRWC_GFT) {
            e[zzz] = 1.0;
            return;
        }
        int stride = (code == DRWC_WVTZ) ? N * N : (code == DRWC_WVTX) ? 1 : N;
        const int pp = zzz + stride, mm = zzz - stride;
        double d_plus = eps[pp] + eps[zzz];
        double d_minus = -(eps[zzz] + eps[mm]);
        e[pp] = eps[pp] / d_plus / h;
        e[zzz] = eps[zzz] * (1. / d_plus + 1. / d_minus) / h;
        e[mm] = eps[mm] / d_minus / h;
        return;
    }
    const int zzz = cidx(N, c, c, c), zmz = cidx(N, c, c - 1, c), zzm = cidx(N, c, c, c - 1),
              zmm = cidx(N, c, c - 1, c - 1), mzz = cidx(N, c - 1, c, c),
              mmz = cidx(N, c - 1, c - 1, c), mzm = cidx(N, c - 1, c, c - 1),
              mmm = cidx(N, c - 1, c - 1, c - 1);
    /* summation order of ggft_solver.cpp:181-185 */
    double dsum = eps[zzz] + eps[zmz] + eps[zzm] + eps[zmm] + eps[mzz] + eps[mmz] + eps[mzm] +
                  eps[mmm];
    if (code == DRWC_GFT) {
        const int cells[8] = {zzz, mzz, zmz, zzm, mmz, mzm, zmm, mmm};
        for (int t = 0; t < 8; ++t) e[cells[t]] = eps[cells[t]] / dsum;
        return;
    }
    int plus[4], minus[4];
    double d_minus;
    if (code == DRWC_WVTZ) {
        int pl[4] = {zzz, mzz, zmz, mmz}, mi[4] = {zzm, mzm, zmm, mmm};
        memcpy(plus, pl, sizeof pl); memcpy(minus, mi, sizeof mi);
        d_minus = -(eps[zzm] + eps[mzm] + eps[zmm] + eps[mmm]);
    } else if (code == DRWC_WVTX) {
        int pl[4] = {zzz, zmz, zzm, zmm}, mi[4] = {mzz, mmz, mzm, mmm};
        memcpy(plus, pl, sizeof pl); memcpy(minus, mi, sizeof mi);
        d_minus = -(eps[mzz] + eps[mmz] + eps[mzm] + eps[mmm]);
    } else {
        int pl[4] = {zzz, mzz, zzm, mzm}, mi[4] = {zmz, mmz, zmm, mmm};
        memcpy(plus, pl, sizeof pl); memcpy(minus, mi, sizeof mi);
        d_minus = -(eps[zmz] + eps[mmz] + eps[zmm] + eps[mmm]);
    }
    for (int t = 0; t < 4; ++t) e[plus[t]] = eps[plus[t]] / dsum / h * 2;
    for (int t = 0; t < 4; ++t) e[minus[t]] = eps[minus[t]] * (1. / dsum + 1. / d_minus) / h * 2;
}

/* Permittivity the gradient output is scaled by: the centre cell for odd N,
 * the mean of the four centre cells on the minus side of the gradient axis
 * for even N (ggft_solver.cpp:649-671). */
double orc_center_diel(int N, const double* eps, int code) {
    const int c = N / 2;
    if (N % 2 || code == DRWC_GFT) return eps[cidx(N, c, c, c)];
    const int zzm = cidx(N, c, c, c - 1), mmm = cidx(N, c - 1, c - 1, c - 1),
              zmm = cidx(N, c, c - 1, c - 1), mzm = cidx(N, c - 1, c, c - 1),
              mzz = cidx(N, c - 1, c, c), mmz = cidx(N, c - 1, c - 1, c),
              zmz = cidx(N, c, c - 1, c);
    if (code == DRWC_WVTZ) return (eps[zzm] + eps[mmm] + eps[zmm] + eps[mzm]) / 4;
    if (code == DRWC_WVTX) return (eps[mzz] + eps[mmz] + eps[mzm] + eps[mmm]) / 4;
    return (eps[zmz] + eps[mmz] + eps[zmm] + eps[mmm]) / 4;
}

typedef struct {
    int N;
    double* gx; /* conductance between c and c+x (0 on the last plane) */
    double* gy;
    double* gz;
    double* diag;
} korc;

static void k_build(korc* K, int N, const double* eps) {
    const int nnn = N * N * N;
    K->N = N;
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                int p = cidx(N, i, j, k);
                double ep = eps[p];
                K->gx[p] = (i + 1 < N) ? ep * eps[p + 1] / (ep + eps[p + 1]) : 0.0;
                K->gy[p] = (j + 1 < N) ? ep * eps[p + N] / (ep + eps[p + N]) : 0.0;
                K->gz[p] = (k + 1 < N) ? ep * eps[p + N * N] / (ep + eps[p + N * N]) : 0.0;
            }
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                int p = cidx(N, i, j, k);
                double d = 0;
                d += (i + 1 < N) ? K->gx[p] : eps[p];
                d += (i > 0) ? K->gx[p - 1] : eps[p];
                d += (j + 1 < N) ? K->gy[p] : eps[p];
                d += (j > 0) ? K->gy[p - N] : eps[p];
                d += (k + 1 < N) ? K->gz[p] : eps[p];
                d += (k > 0) ? K->gz[p - N * N] : eps[p];
                K->diag[p] = d;
            }
    (void)nnn;
}

static void k_apply(const korc* K, const double* y, double* out) {
    const int N = K->N;
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                int p = cidx(N, i, j, k);
                double s = K->diag[p] * y[p];
                if (i + 1 < N) s -= K->gx[p] * y[p + 1];
                if (i > 0) s -= K->gx[p - 1] * y[p - 1];
                if (j + 1 < N) s -= K->gy[p] * y[p + N];
                if (j > 0) s -= K->gy[p - N] * y[p - N];
                if (k + 1 < N) s -= K->gz[p] * y[p + N * N];
                if (k > 0) s -= K->gz[p - N * N] * y[p - N * N];
                out[p] = s;
            }
}

static double dot(int n, const double* a, const double* b) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* Surface values from the cell solution y: gft[b] = eps_c * y_c for the cell
 * c under panel b (A13 of ggft_solver.cpp:292-326, order ggft_solver.h:65-77). */
static void extract_surface(int N, const double* eps, const double* y, double* out) {
    const int NN = N * N;
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
            int lo = cidx(N, i, j, 0), hi = cidx(N, i, j, N - 1);
            out[i + j * N] = eps[lo] * y[lo];
            out[NN + i + j * N] = eps[hi] * y[hi];
        }
    for (int k = 0; k < N; ++k)
        for (int i = 0; i < N; ++i) {
            int lo = cidx(N, i, 0, k), hi = cidx(N, i, N - 1, k);
            out[2 * NN + i + k * N] = eps[lo] * y[lo];
            out[3 * NN + i + k * N] = eps[hi] * y[hi];
        }
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j) {
            int lo = cidx(N, 0, j, k), hi = cidx(N, N - 1, j, k);
            out[4 * NN + j + k * N] = eps[lo] * y[lo];
            out[5 * NN + j + k * N] = eps[hi] * y[hi];
        }
}

/* Returns 0 on convergence, 1 if maxit was reached, 2 for invalid eps. */
int orc_fdm_solve(int N, const double* eps, int code, double tol, int maxit, double* out,
                  int* iters, double* relres) {
    const int nnn = N * N * N;
    for (int p = 0; p < nnn; ++p)
        if (!(eps[p] > 0) || !isfinite(eps[p])) {
            memset(out, 0, sizeof(double) * 6 * N * N);
            if (iters) *iters = 0;
            if (relres) *relres = NAN;
            return 2;
        }
    double* buf = (double*)malloc(sizeof(double) * nnn * 10);
    korc K = {N, buf, buf + nnn, buf + 2 * nnn, buf + 3 * nnn};
    double *e = buf + 4 * nnn, *y = buf + 5 * nnn, *r = buf + 6 * nnn, *z = buf + 7 * nnn,
           *pp = buf + 8 * nnn, *q = buf + 9 * nnn;
    k_build(&K, N, eps);
    orc_rhs(N, eps, code, e);
    if (maxit <= 0) maxit = 20 * N * N;
    const double enorm = sqrt(dot(nnn, e, e));
    memset(y, 0, sizeof(double) * nnn);
    memcpy(r, e, sizeof(double) * nnn);
    for (int p = 0; p < nnn; ++p) z[p] = r[p] / K.diag[p];
    memcpy(pp, z, sizeof(double) * nnn);
    double rz = dot(nnn, r, z);
    int it = 0, rc = 1;
    for (it = 1; it <= maxit; ++it) {
        k_apply(&K, pp, q);
        double alpha = rz / dot(nnn, pp, q);
        for (int p = 0; p < nnn; ++p) {
            y[p] += alpha * pp[p];
            r[p] -= alpha * q[p];
        }
        if (sqrt(dot(nnn, r, r)) <= tol * enorm) {
            /* confirm with the true residual */
            k_apply(&K, y, q);
            for (int p = 0; p < nnn; ++p) r[p] = e[p] - q[p];
            if (sqrt(dot(nnn, r, r)) <= tol * enorm) { rc = 0; break; }
        }
        for (int p = 0; p < nnn; ++p) z[p] = r[p] / K.diag[p];
        double rz2 = dot(nnn, r, z);
        double beta = rz2 / rz;
        rz = rz2;
        for (int p = 0; p < nnn; ++p) pp[p] = z[p] + beta * pp[p];
    }
    k_apply(&K, y, q);
    for (int p = 0; p < nnn; ++p) r[p] = e[p] - q[p];
    if (relres) *relres = sqrt(dot(nnn, r, r)) / enorm;
    if (iters) *iters = it > maxit ? maxit : it;
    extract_surface(N, eps, y, out);
    free(buf);
    return rc;
}

int orc_fdm_solve_cb(int N, const double* eps, int code, double tol, double* out) {
    return orc_fdm_solve(N, eps, code, tol, 0, out, NULL, NULL);
}

int orc_fdm_solve_batch(int ncubes, int N, const double* eps, const int32_t* code, double tol,
                        double* out, int32_t* ok, int nthreads, double* seconds) {
    const size_t nnn = (size_t)N * N * N, n3 = (size_t)6 * N * N;
    int failed = 0;
    if (nthreads < 1) nthreads = 1;
    double t0 = omp_get_wtime();
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1) reduction(+ : failed)
    for (int c = 0; c < ncubes; ++c) {
        int rc = orc_fdm_solve(N, eps + c * nnn, code ? code[c] : DRWC_GFT, tol, 0, out + c * n3,
                               NULL, NULL);
        if (ok) ok[c] = (rc == 0);
        failed += (rc != 0);
    }
    if (seconds) *seconds = omp_get_wtime() - t0;
    return failed;
}

/* ---- dnnsolver data path ------------------------------------------------- */

/* dnn_solver.cpp:274-285 (normalisation) + cuda_kernels.cu:21-84 (fill),
 * float32 arithmetic as in the reference kernel. */
void orc_structure_construction(int n, int N, const float* layers, const float* cuboids,
                                int normalise, float* eps_out, float* max_out) {
    const int L = DRWC_MAX_LAYERS, C = DRWC_MAX_CUBOIDS;
    float lay[2 * DRWC_MAX_LAYERS], cub[7 * DRWC_MAX_CUBOIDS];
    for (int b = 0; b < n; ++b) {
        memcpy(lay, layers + (size_t)b * 2 * L, sizeof lay);
        memcpy(cub, cuboids + (size_t)b * 7 * C, sizeof cub);
        float m = lay[1];
        for (int l = 0; l < L; ++l) m = fmaxf(m, lay[2 * l + 1]);
        for (int c = 0; c < C; ++c) m = fmaxf(m, cub[7 * c + 6]);
        if (max_out) max_out[b] = m;
        if (normalise) {
            for (int l = 0; l < L; ++l) lay[2 * l + 1] /= m;
            for (int c = 0; c < C; ++c) cub[7 * c + 6] /= m;
        }
        float* out = eps_out + (size_t)b * N * N * N;
        for (int z = 0; z < N; ++z)
            for (int y = 0; y < N; ++y)
                for (int x = 0; x < N; ++x) {
                    const float xc = (2.0f * (float)x + 1.0f) / (float)N - 1.0f;
                    const float yc = (2.0f * (float)y + 1.0f) / (float)N - 1.0f;
                    const float zc = (2.0f * (float)z + 1.0f) / (float)N - 1.0f;
                    int li = 0;
                    for (int l = 0; l < L; ++l) {
                        float mz = lay[2 * l];
                        if (mz == DRWC_PADDING) break;
                        if (zc >= mz) li = l;
                        else break;
                    }
                    float val = lay[2 * li + 1];
                    for (int c = 0; c < C; ++c) {
                        const float* q = cub + 7 * c;
                        if (q[0] == DRWC_PADDING) break;
                        if (xc >= q[0] && xc <= q[3] && yc >= q[1] && yc <= q[4] && zc >= q[2] &&
                            zc <= q[5]) {
                            val = q[6];
                            break;
                        }
                    }
                    out[x + y * N + z * N * N] = val;
                }
    }
}

/* locate_index_simple_kernel (cuda_kernels.cu:219-264): panel -> point on the
 * surface of [-1,1]^3. Face vectors {(x,y,-z),(x,y,+z),(x,-1,y'),(x,+1,y'),
 * (-1,x',y'),(+1,x',y')} applied to ((2a+1)/N-1, (2b+1)/N-1, 1). */
void orc_locate(int N, int panel, float out[3]) {
    static const int fv[6][3] = {{1, 2, -3}, {1, 2, 3}, {1, -3, 2}, {1, 3, 2}, {-3, 1, 2}, {3, 1, 2}};
    const int NN = N * N;
    int f = panel / NN, t = panel % NN;
    int a = t % N, b = t / N;
    float tmp[3] = {(2.0f * a + 1.0f) / N - 1.0f, (2.0f * b + 1.0f) / N - 1.0f, 1.0f};
    for (int j = 0; j < 3; ++j) {
        int v = fv[f][j];
        out[j] = tmp[abs(v) - 1] * (v < 0 ? -1.0f : 1.0f);
    }
}

void orc_locate_f64(int N, int panel, double out[3]) {
    static const int fv[6][3] = {{1, 2, -3}, {1, 2, 3}, {1, -3, 2}, {1, 3, 2}, {-3, 1, 2}, {3, 1, 2}};
    const int NN = N * N;
    int f = panel / NN, t = panel % NN;
    int a = t % N, b = t / N;
    double tmp[3] = {(2.0 * a + 1.0) / N - 1.0, (2.0 * b + 1.0) / N - 1.0, 1.0};
    for (int j = 0; j < 3; ++j) {
        int v = fv[f][j];
        out[j] = tmp[abs(v) - 1] * (v < 0 ? -1.0 : 1.0);
    }
}

/* Inverse-CDF draw over M weights (|w| when use_abs): the first index whose
 * running sum exceeds u * total; when rounding leaves none, the last index
 * with non-zero weight. Replaces the two-stage face/tile torch::multinomial
 * (dnn_solver_poisson.cpp:92,107), which draws from the same distribution. */
int orc_sample_index(int M, const double* w, int use_abs, double u) {
    double tot = 0;
    for (int i = 0; i < M; ++i) tot += use_abs ? fabs(w[i]) : fmax(w[i], 0.0);
    double target = u * tot, run = 0;
    int last = -1;
    for (int i = 0; i < M; ++i) {
        double wi = use_abs ? fabs(w[i]) : fmax(w[i], 0.0);
        if (wi > 0) last = i;
        run += wi;
        if (run > target && wi > 0) return i;
    }
    return last;
}

void orc_philox_uniform2_c(uint64_t seed, uint64_t stream, uint32_t c2, uint32_t c3, double* u) {
    orc_philox_uniform2(seed, stream, c2, c3, &u[0], &u[1]);
}

int orc_transition(int N, const double* eps, double tol, uint64_t seed, uint64_t stream,
                   float out[3], int32_t* panel) {
    double* g = (double*)malloc(sizeof(double) * 6 * N * N);
    int rc = orc_fdm_solve(N, eps, DRWC_GFT, tol, 0, g, NULL, NULL);
    double u[2];
    orc_philox_uniform2(seed, stream, 0, 0, &u[0], &u[1]);
    int b = orc_sample_index(6 * N * N, g, 0, u[0]);
    if (panel) *panel = b;
    orc_locate(N, b < 0 ? 0 : b, out);
    free(g);
    return rc;
}

/* dnn_solver_gradient.cpp:143-162 with the FDM in place of the networks:
 * [panel centre (3), sum|g| * sign(g_b), centre eps * eps_scale]. */
int orc_first_hop(int N, const double* eps, int axis, double tol, uint64_t seed,
                  uint64_t stream, double eps_scale, float out[5], int32_t* panel) {
    const int code = axis == 0 ? DRWC_WVTX : axis == 1 ? DRWC_WVTY : DRWC_WVTZ;
    const int M = 6 * N * N;
    double* g = (double*)malloc(sizeof(double) * M);
    int rc = orc_fdm_solve(N, eps, code, tol, 0, g, NULL, NULL);
    double u[2];
    orc_philox_uniform2(seed, stream, 0, 0, &u[0], &u[1]);
    int b = orc_sample_index(M, g, 1, u[0]);
    if (panel) *panel = b;
    double W = 0;
    for (int i = 0; i < M; ++i) W += fabs(g[i]);
    orc_locate(N, b < 0 ? 0 : b, out);
    double sg = (b >= 0 && g[b] < 0) ? -1.0 : 1.0;
    out[3] = (float)(W * sg);
    out[4] = (float)(orc_center_diel(N, eps, code) * eps_scale);
    free(g);
    return rc;
}
