/* TEST INFRASTRUCTURE ONLY — CPU restatement of the reference algorithms on
 * the FRW transition path, used by tests/, the smoke check and the CPU
 * baseline leg of bench.py as the checker. The product library never links,
 * loads or calls anything here.
 *
 * Parity pins: orc_fdm_* is checked against the reference ggft solver built
 * from its own sources (oracle/_ref, ggft_ref_harness.cpp) and against the
 * committed golden vectors in tests/golden/, which that build produced.
 */
#ifndef ORC_ORACLE_H
#define ORC_ORACLE_H
#include <stdint.h>

#include "../include/drwc.h"

#ifdef __cplusplus
extern "C" {
#endif

/* FDM surface Green's function (ggft_solver.cpp:137-326, 447-636). */
void orc_rhs(int N, const double* eps, int code, double* e);
double orc_center_diel(int N, const double* eps, int code);
int orc_fdm_solve(int N, const double* eps, int code, double tol, int maxit, double* out,
                  int* iters, double* relres);
int orc_fdm_solve_batch(int ncubes, int N, const double* eps, const int32_t* code, double tol,
                        double* out, int32_t* ok, int nthreads, double* seconds);

/* dnnsolver data path (cuda_kernels.cu, dnn_solver*.cpp). */
void orc_structure_construction(int n, int N, const float* layers, const float* cuboids,
                                int normalise, float* eps_out, float* max_out);
void orc_locate(int N, int panel, float out[3]);
void orc_locate_f64(int N, int panel, double out[3]);
int orc_sample_index(int M, const double* w, int use_abs, double u);
void orc_philox_uniform2_c(uint64_t seed, uint64_t stream, uint32_t c2, uint32_t c3, double* u);
int orc_transition(int N, const double* eps, double tol, uint64_t seed, uint64_t stream,
                   float out[3], int32_t* panel);
int orc_first_hop(int N, const double* eps, int axis, double tol, uint64_t seed,
                  uint64_t stream, double eps_scale, float out[5], int32_t* panel);

/* FRW walker restated (frw_oracle.c). The per-hop FDM solve is a callback so
 * the same walk loop runs over this file's FP64 PCG or the reference ggft. */
typedef int (*orc_fdm_fn)(int N, const double* eps, int code, double tol, double* out);
int orc_fdm_solve_cb(int N, const double* eps, int code, double tol, double* out);
int orc_frw_walks(const drwc_structure* s, const drwc_job_params* p, int64_t walk0,
                  int64_t nwalks, orc_fdm_fn fdm, double fdm_tol, int nthreads,
                  int32_t* end_net, int32_t* hops, double* weight, double* seconds);
double orc_distance(const drwc_structure* s, const double r[3], int32_t* net);
double orc_eps_at(const drwc_structure* s, const double r[3]);

#ifdef __cplusplus
}
#endif
#endif
