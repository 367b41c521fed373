// TEST INFRASTRUCTURE ONLY — never linked into the product library.
//
// C-callable harness around the reference ggft FDM Green's-function solver
// (ggft/src/ggft_solver.{h,cpp}), compiled from the reference's own sources by
// oracle/Makefile, one shared object per cube resolution N (N is a
// compile-time constant in ggft/src/ggft_solver.h:33, so the recipe patches it
// in a private copy of the two source files and builds each N separately).
//
// What the harness does, per cube, mirrors ggft/src/main.cpp:41-50: one
// ggft_solver per OpenMP thread, DIEL filled with the cube's permittivity
// (x fastest, ggft_solver.h:48), set_tolerance(tol) (ggft_solver.h:193-198),
// solve(code) (ggft_solver.cpp:521-636) and the public `gft` vector
// (6*N*N panel values, order ggft_solver.h:65-77) copied out.
//
// write_to="/dev/null" keeps the constructor's prepare_file
// (ggft_solver.cpp:32-49) from creating a dated data directory.
#include <omp.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "ggft_solver.h"

extern "C" {

int ggft_ref_N() { return deeprwcap::index::N; }

// eps: ncubes x N^3 doubles; out: ncubes x 6N^2 doubles; ok: ncubes ints
// (1 = ggft's solve() returned true). Returns the number of failed cubes.
// *seconds receives the wall time of the solve loop alone (solver
// construction, i.e. matrix build + uniform bootstrap solves, excluded).
int ggft_ref_solve_batch(int ncubes, const double* eps, int code, double tol,
                         double* out, int* ok, int nthreads, double* seconds) {
    using deeprwcap::ggft_solver;
    using deeprwcap::index;
    if (nthreads < 1) nthreads = 1;
    const int nnn = index::NNN;
    const int n3 = index::N3;
    int failed = 0;
    double t_solve = 0.0;
    std::vector<std::unique_ptr<ggft_solver>> solvers(nthreads);
#pragma omp parallel num_threads(nthreads) reduction(+ : failed)
    {
        const int tid = omp_get_thread_num();
        solvers[tid].reset(new ggft_solver("/dev/null"));
        solvers[tid]->set_tolerance(tol);
#pragma omp barrier
        double t0 = omp_get_wtime();
#pragma omp for schedule(dynamic, 1)
        for (int c = 0; c < ncubes; ++c) {
            ggft_solver& s = *solvers[tid];
            std::memcpy(s.DIEL.data(), eps + (size_t)c * nnn, sizeof(double) * nnn);
            bool good = s.solve(static_cast<ggft_solver::solver_code>(code));
            if (ok) ok[c] = good ? 1 : 0;
            if (!good) {
                ++failed;
                std::memset(out + (size_t)c * n3, 0, sizeof(double) * n3);
            } else {
                std::memcpy(out + (size_t)c * n3, s.gft.data(), sizeof(double) * n3);
            }
        }
        double t1 = omp_get_wtime();
#pragma omp critical
        { if (t1 - t0 > t_solve) t_solve = t1 - t0; }
    }
    if (seconds) *seconds = t_solve;
    return failed;
}

}  // extern "C"

// One cube on the calling thread's own solver (constructed on first use), in
// the oracle's per-hop callback form: returns 0 when ggft's solve() returned
// true. N must equal the compiled N.
extern "C" int ggft_ref_solve_one(int N, const double* eps, int code, double tol, double* out) {
    using deeprwcap::ggft_solver;
    using deeprwcap::index;
    if (N != index::N) return 3;
    static thread_local std::unique_ptr<ggft_solver> solver;
    if (!solver) solver.reset(new ggft_solver("/dev/null"));
    solver->set_tolerance(tol);
    std::memcpy(solver->DIEL.data(), eps, sizeof(double) * index::NNN);
    bool good = solver->solve(static_cast<ggft_solver::solver_code>(code));
    std::memcpy(out, solver->gft.data(), sizeof(double) * index::N3);
    return good ? 0 : 1;
}
