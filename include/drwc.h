/*
 * drwc.h — C ABI of the B200 floating-random-walk (FRW) transition engine.
 *
 * Plain C: pointers, sizes and status codes; no C++ or torch types cross the
 * boundary and no exception leaves the library. Every entry point returns a
 * drwc_status (0 = success). Entry points taking HOST buffers are synchronous;
 * the *_device variants take device pointers and run asynchronously on the
 * context's stream.
 *
 * The entry points replace two plug points of the reference (DeepRWCap):
 *   - ggft's FDM Green's-function generator
 *     (ggft/src/ggft_solver.h:112-198: DIEL, solve(solver_code), gft,
 *     set_tolerance), and
 *   - the walker's calls into the dnnsolver library
 *     (inference_cpp/src/dnn_solver.h:43-201: DNNSolverPoisson::sample,
 *     DNNSolverGrad::sample, DNNSolver::structureConstruction,
 *     ParallelSampler::submit),
 * plus the walker itself (the reference ships it closed, executable/), as a
 * device-resident job API.
 *
 * Conventions shared by every entry point:
 *   - Cube permittivity is N^3 values, cell (i,j,k) at i + j*N + k*N*N
 *     (x fastest), the order of ggft_solver.h:48 and of the dnnsolver's
 *     [z][y][x] tensors (cuda_kernels.cu:36-39, 82).
 *   - Surface values are 6*N*N panels in ggft order (ggft_solver.h:65-77):
 *     face 0 z- (i + j*N), 1 z+, 2 y- (i + k*N), 3 y+, 4 x- (j + k*N), 5 x+.
 *   - Solver codes follow ggft_solver::solver_code (ggft_solver.h:119).
 */
#ifndef DRWC_H
#define DRWC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define DRWC_API __declspec(dllexport)
#else
#define DRWC_API __attribute__((visibility("default")))
#endif

/* ---- status codes --------------------------------------------------------- */
typedef enum drwc_status {
    DRWC_OK = 0,
    DRWC_ERR_INVALID = 1,       /* bad argument (null pointer, size, N, code) */
    DRWC_ERR_CUDA = 2,          /* a CUDA runtime call failed */
    DRWC_ERR_NOMEM = 3,         /* device or host allocation failed */
    DRWC_ERR_NOT_CONVERGED = 4, /* at least one cube missed its tolerance */
    DRWC_ERR_NO_DEVICE = 5,     /* no CUDA device / wrong architecture */
    DRWC_ERR_TIMEOUT = 6,       /* a bounded wait ran out */
    DRWC_ERR_SHUTDOWN = 7,      /* object is shutting down */
    DRWC_ERR_GEOMETRY = 8       /* structure rejected (overlaps, empty, ...) */
} drwc_status;

/* ---- solver codes (ggft_solver.h:119) -------------------------------------- */
enum { DRWC_GFT = 0, DRWC_WVTZ = 1, DRWC_WVTX = 2, DRWC_WVTY = 3 };

/* ---- limits ----------------------------------------------------------------- */
#define DRWC_N_MIN 4             /* smallest cube resolution */
#define DRWC_N_MAX 23            /* largest cube resolution (the CTA-resident solve holds 18 B per cell on chip) */
#define DRWC_MAX_LAYERS 15       /* dnn_solver.h:29 */
#define DRWC_MAX_CUBOIDS 15      /* dnn_solver.h:28 */
#define DRWC_LAYER_STRIDE (2 * DRWC_MAX_LAYERS)    /* floats per query (30) */
#define DRWC_CUBOID_STRIDE (7 * DRWC_MAX_CUBOIDS)  /* floats per query (105) */
#define DRWC_PADDING (-9999.0f)  /* dnn_solver.h:30 */
#define DRWC_MAX_NETS 256        /* conductor nets per structure (+1 ground) */

/* ---- library / context ------------------------------------------------------ */
typedef struct drwc_ctx drwc_ctx;

DRWC_API const char* drwc_version(void);
DRWC_API const char* drwc_status_string(int status);
/* Create a context on `device`: a non-blocking stream and lazily grown device
 * workspaces, as DNNSolver's constructor (dnn_solver.cpp:13-38). Fails with
 * DRWC_ERR_NO_DEVICE when the device is not sm_100. */
DRWC_API int drwc_ctx_create(int device, drwc_ctx** out);
DRWC_API int drwc_ctx_destroy(drwc_ctx* ctx);
/* The context's stream (a cudaStream_t) for callers that enqueue around it. */
DRWC_API int drwc_ctx_stream(drwc_ctx* ctx, void** stream_out);
DRWC_API int drwc_ctx_synchronize(drwc_ctx* ctx);
/* Number of kernels this context has launched so far. */
DRWC_API int drwc_ctx_launch_count(drwc_ctx* ctx, int64_t* count_out);

/* ---- FDM surface Green's function (ggft replacement) ------------------------ */
/* Solver knobs. tol is the FP64 relative residual ||e - K y|| / ||e|| the
 * refinement loop stops at; inner_tol is the relative reduction each FP32 PCG
 * sweep aims for. */
typedef struct drwc_fdm_opts {
    double tol;         /* default 1e-10 */
    double inner_tol;   /* default 1e-5 */
    int32_t max_outer;  /* FP64 refinement sweeps, default 8 */
    int32_t max_inner;  /* FP32 PCG iterations per sweep, default 4 * N * N */
    int32_t warm_start; /* start from the uniform-permittivity solution, as ggft's
                           solveWithGuess (ggft_solver.cpp:554-560); default 1 */
    int32_t extra_outer; /* escalation: a cube still above tol after max_outer
                           sweeps gets up to this many more, each with 4 *
                           max_inner iterations, before it is reported not
                           converged (ggft falls back to a direct solve,
                           ggft_solver.cpp:565-589); default 8, 0 = none.
                           Walks drop a hop whose cube stays unconverged:
                           the walk ends lost and is counted. */
} drwc_fdm_opts;
DRWC_API void drwc_fdm_opts_default(drwc_fdm_opts* opts);

/* Drop-in for ggft_solver::solve(code) followed by reading ggft_solver::gft
 * (ggft/src/ggft_solver.cpp:521-636): one cube, host buffers.
 * eps: N^3 doubles (ggft's DIEL), gft_out: 6*N^2 doubles. tol has the meaning
 * of ggft_solver::set_tolerance (ggft_solver.h:193-198) applied to the
 * relative residual. iters_out (nullable) receives the FP32 CG iterations
 * of all refinement sweeps. Returns DRWC_ERR_NOT_CONVERGED where ggft's solve() would
 * return false. */
DRWC_API int drwc_ggft_solve(drwc_ctx* ctx, int N, const double* eps, int code,
                             double tol, double* gft_out, int32_t* iters_out);

/* Batched solve of ncubes cubes of mixed resolution, device buffers, async on
 * the context stream. Cube c has resolution N[c], permittivity at
 * eps + eps_off[c] (N^3 doubles), solver code code[c] (NULL: all GFT), and
 * writes 6*N^2 doubles at out + out_off[c]. N, eps_off, code and out_off are
 * HOST arrays (the library groups cubes by N). iters (FP32 CG iterations),
 * sweeps (FP64 residual evaluations), relres and status are per-cube DEVICE
 * outputs (nullable): status 0 = converged, 1 = not converged, 2 = invalid
 * permittivity (non-positive or non-finite). */
DRWC_API int drwc_fdm_solve_batch_device(drwc_ctx* ctx, int ncubes, const int32_t* N,
                                         const int64_t* eps_off, const double* eps,
                                         const int32_t* code, const drwc_fdm_opts* opts,
                                         const int64_t* out_off, double* out,
                                         int32_t* iters, int32_t* sweeps, double* relres,
                                         int32_t* status);

/* Same, host buffers (eps/out/iters/relres/status on the host); synchronous. */
DRWC_API int drwc_fdm_solve_batch(drwc_ctx* ctx, int ncubes, const int32_t* N,
                                  const int64_t* eps_off, const double* eps,
                                  const int32_t* code, const drwc_fdm_opts* opts,
                                  const int64_t* out_off, double* out,
                                  int32_t* iters, double* relres, int32_t* status);

/* Same-N batch with no device allocation. No counterpart in the reference:
 * it exists for callers that cannot allocate device memory when they call in
 * (an application that owns all GPU memory through its own pool and forbids
 * later driver allocations, or a latency-critical loop where a cudaMalloc and
 * its implicit synchronisation are not allowed). Cube c reads N^3 doubles at
 * eps + c*N^3 and writes 6*N^2 doubles at out + c*6*N^2; code (nullable: all
 * GFT), iters and status (nullable) are DEVICE arrays of ncubes entries, as
 * in drwc_fdm_solve_batch_device; a cube whose code is not a solver code
 * gets status 2 and zero rows. opts->warm_start is honoured as in the other
 * entry points. Runs async on the context stream. Solver scratch comes from a
 * fixed 16 MiB static device array in the library (12 bytes per cell per
 * resident CTA) and the warm starts from a 2.4 MB static array of
 * uniform-permittivity solutions (every N and code); every GPU that loads the
 * library holds both until exit. drwc_ctx_create loads their module, looks up
 * their device addresses, sets the kernel attributes and solves the warm
 * tables, once per device, so this call itself allocates and loads nothing:
 * create the context before giving the GPU's memory to your own pool. N
 * outside [DRWC_N_MIN, DRWC_N_MAX] is rejected with DRWC_ERR_INVALID. Calls
 * share the scratch array: calls that overlap on the GPU race, so issue them
 * on one stream. */
DRWC_API int drwc_fdm_solve_noalloc(drwc_ctx* ctx, int N, int ncubes, const double* eps,
                                    const int32_t* code, const drwc_fdm_opts* opts, double* out,
                                    int32_t* iters, int32_t* status);

/* ---- dnnsolver replacements ------------------------------------------------- */
/* Drop-in for DNNSolver::structureConstruction (dnn_solver.cpp:252-300) with
 * fill_structure_kernel (cuda_kernels.cu:21-84): n queries of 30 layer floats
 * (15 x (min_z, eps)) and 105 cuboid floats (15 x (x0,y0,z0,x1,y1,z1,eps)),
 * cube-normalised [-1,1] coordinates, padding -9999. Writes n x N^3 floats
 * (eps / max eps per query when normalise != 0) and n max values. Host
 * buffers. */
DRWC_API int drwc_structure_construction(drwc_ctx* ctx, int n, int N, const float* layers,
                                         const float* cuboids, int normalise,
                                         float* eps_out, float* max_out);

/* Drop-in for DNNSolverPoisson::sample (dnn_solver_poisson.cpp:35-63): for
 * each of n queries voxelise the cube, solve its surface Green's function
 * (FDM, GFT), sample one panel with probability G[b] and write the panel
 * centre on the surface of [-1,1]^3 (3 floats, locate_index_simple_kernel,
 * cuda_kernels.cu:219-264). Randomness: Philox4x32-10 keyed by `seed`,
 * counter (stream + query index, 0, 0, 0). Host buffers. */
DRWC_API int drwc_transition_batch(drwc_ctx* ctx, int n, int N, const float* layers,
                                   const float* cuboids, uint64_t seed, uint64_t stream,
                                   float* out_pos);

/* Drop-in for DNNSolverGrad::sample (dnn_solver_gradient.cpp:49-73,
 * 111-163): per query solve the centre-gradient surface values along axis
 * (0 = x, 1 = y, 2 = z; WVTX/WVTY/WVTZ), sample a panel with probability
 * |g_b| / sum|g| and write 5 floats: panel centre (3), sum|g| * sign(g_b),
 * centre permittivity in the query's own units. axis may be NULL only to get
 * the reference's error (DRWC_ERR_INVALID, dnn_solver_gradient.cpp:40-47).
 * Host buffers. */
DRWC_API int drwc_first_hop_batch(drwc_ctx* ctx, int n, int N, const float* layers,
                                  const float* cuboids, const int32_t* axis, uint64_t seed,
                                  uint64_t stream, float* out);

/* ---- tensor-core GEMM (the learned transition kernels' building block) ----- */
/* C[M,N] (FP32, row-major, ldc) = act(A[M,K] * B[N,K]^T + bias[N]) with A, B
 * BF16 row-major (lda, ldb >= K), FP32 accumulation in tensor memory
 * (tcgen05.mma, sm_100a). act: 0 none, 1 ReLU. bias and err_flag (an int the
 * kernel sets to 1 if a bounded wait ran out) are nullable. Device pointers;
 * async on the context stream. */
DRWC_API int drwc_gemm_bf16(drwc_ctx* ctx, int M, int N, int K, const void* A, int64_t lda,
                            const void* B, int64_t ldb, float* C, int64_t ldc, const float* bias,
                            int act, int* err_flag);

/* ---- learned transition kernels (N = 16) ----------------------------------- */
/* A 3-D convolutional network on the cube's normalised permittivity (eps /
 * max eps, BF16 [B, 16^3], cell order as above): encoder 1 -> 16 -> 32 -> 64
 * channels (3^3 kernels, stride 2, pad 1, ReLU), Poisson head (1536 logits,
 * softmax over the 6N^2 panels, plus a confidence output = predicted log10 KL
 * divergence to the FDM Green's function) and gradient head (1536 WVTZ
 * values, scaled). BF16 operands, FP32 accumulation on tcgen05 tensor cores,
 * FP32 master weights. Architecture family of training_pytorch/src/
 * architecture.py; trained here on FDM data the engine generates. */
typedef struct drwc_net drwc_net;
#define DRWC_NET_N 16          /* the learned walker's resolution */
#define DRWC_NET_OUT 1552      /* N = 16: Poisson logits (1536) + confidence + padding */
#define DRWC_NET_PANELS 1536   /* N = 16: 6 N^2 */
/* N: 16, 21 or 23 (the cube resolution the network reads and predicts). */
DRWC_API int drwc_net_create(drwc_ctx* ctx, int N, uint64_t seed, drwc_net** out);
DRWC_API int drwc_net_destroy(drwc_net* net);
/* Sizes (host, each nullable): N, panels = 6 N^2, out_row = floats per row of
 * O (panels + confidence, padded to 16), grad_row = floats per row of G
 * (panels padded to 16), features = encoder outputs per cube. */
DRWC_API int drwc_net_dims(drwc_net* net, int32_t* N, int32_t* panels, int32_t* out_row,
                           int32_t* grad_row, int32_t* features);
DRWC_API int drwc_net_param_count(drwc_net* net, int64_t* count);
DRWC_API int drwc_net_get_params(drwc_net* net, float* host);
DRWC_API int drwc_net_set_params(drwc_net* net, const float* host);
DRWC_API int drwc_net_gradients(drwc_net* net, float* host);
/* Device buffers: X [B, N^3] BF16 -> O [B, out_row] FP32, G [B, grad_row]
 * FP32 (nullable). Async on the context stream. */
DRWC_API int drwc_net_forward(drwc_net* net, int B, const void* X, float* O, float* G);
/* One optimisation step (device buffers X [B, N^3], T = target Green's
 * functions [B, panels] rows summing to 1, TG = scaled gradient targets
 * [B, panels] or NULL); apply = 0 computes losses and gradients without
 * updating.
 * loss_out (host, 3): cross entropy, confidence MSE, gradient MSE. */
DRWC_API int drwc_net_train_step(drwc_net* net, int B, const void* X, const float* T,
                                 const float* TG, float lr, float weight_decay, float clip,
                                 float w_conf, float w_grad, int apply, float* loss_out);

/* ---- structures and the FRW walk (the closed walker's role) --------------- */
typedef struct drwc_box {
    double lo[3];
    double hi[3];
    int32_t net;   /* conductor net id in [0, n_nets) */
    int32_t pad_;
} drwc_box;

typedef struct drwc_diel_box {
    double lo[3];
    double hi[3];
    double eps;    /* relative permittivity, overrides the layers inside */
} drwc_diel_box;

typedef struct drwc_structure {
    int32_t n_boxes;          /* conductor boxes */
    int32_t n_nets;           /* nets; ground (the enclosure) is net n_nets */
    const drwc_box* boxes;
    int32_t n_layers;         /* stratified dielectric, sorted by zlo */
    int32_t n_diel;           /* dielectric blocks (first containing wins) */
    const double* layer_zlo;  /* layer l covers [zlo[l], zlo[l+1]) */
    const double* layer_eps;
    const drwc_diel_box* diel;
    double encl_lo[3];        /* grounded enclosure */
    double encl_hi[3];
} drwc_structure;

typedef struct drwc_job_params {
    int32_t master;           /* master net */
    int32_t N;                /* cube resolution of every hop */
    double gauss_offset;      /* Gaussian surface offset from the master (um) */
    double stop_dist;         /* absorption distance (um) */
    double p_tol;             /* self-capacitance relative 1-sigma target (-p) */
    double c_tol;             /* coupling relative 1-sigma target (-c) */
    double c_ratio;           /* the largest couplings (ground included) that make up
                                 this fraction of the summed coupling magnitude must
                                 each meet c_tol (--c-ratio) */
    int64_t min_walks;        /* walks before the first convergence check */
    int64_t max_walks;        /* hard cap */
    int64_t batch_walks;      /* walks per device batch between checks */
    int32_t max_hops;         /* per walk; a walk reaching it is "lost" */
    int32_t gauss_surface;    /* 0: the master's bounding box grown by gauss_offset;
                                 1: the outer boundary of the union of the master's boxes,
                                 each grown by min(gauss_offset, half its clearance to
                                 the other nets and the enclosure) (masters whose
                                 bounding box reaches another net) */
    uint64_t seed;
    drwc_fdm_opts fdm;        /* per-hop solve knobs */
} drwc_job_params;
DRWC_API void drwc_job_params_default(drwc_job_params* p);

typedef struct drwc_job_result {
    int32_t n_entries;        /* n_nets + 1 (last = ground) */
    int32_t converged;        /* 1 when -p/-c/--c-ratio were met */
    int64_t walks;
    int64_t hops;
    int64_t lost;             /* walks cut at max_hops or ended by a failed solve */
    int64_t solves_escalated; /* cube solves that needed escalation sweeps */
    int64_t solves_failed;    /* cube solves unconverged after escalation (walk lost) */
    double seconds;           /* job wall time on the device */
    double cap[DRWC_MAX_NETS + 1];     /* fF, row of the master */
    double stderr_[DRWC_MAX_NETS + 1]; /* 1-sigma standard error, fF */
} drwc_job_result;

/* A prepared job: the structure validated and uploaded once (conductor boxes,
 * dielectric layers and blocks, a uniform grid of conductor boxes for the
 * nearest-conductor search), the Gaussian surface of the master built. */
typedef struct drwc_job drwc_job;
DRWC_API int drwc_job_create(drwc_ctx* ctx, const drwc_structure* s, const drwc_job_params* p,
                             drwc_job** out);
DRWC_API int drwc_job_destroy(drwc_job* job);
/* Launch walks [walk0, walk0 + nwalks) on the context stream (async). Per-walk
 * records go to DEVICE arrays end_net / hops / weight (fF); solver_stats
 * (DEVICE, nullable, 5 int64) receives total hops, FP32 CG iterations, FP64
 * residual sweeps, solves that needed escalation sweeps and solves that did
 * not converge even then (their walks end lost) of the launch. */
DRWC_API int drwc_job_walks_device(drwc_job* job, int64_t walk0, int64_t nwalks,
                                   int32_t* end_net, int32_t* hops, double* weight,
                                   int64_t* solver_stats);
/* Bytes of structure data the job uploaded to the device. */
DRWC_API int drwc_job_h2d_bytes(drwc_job* job, int64_t* bytes);

/* Training data from the walks themselves: run walks [walk0, walk0+nwalks)
 * of a job and log every hop's transition cube (centre xyz, half-width: 4
 * doubles) and solver code into DEVICE arrays rec / code (up to cap hops);
 * *count (host) receives the number logged. */
DRWC_API int drwc_frw_harvest(drwc_ctx* ctx, const drwc_structure* s, const drwc_job_params* p,
                              int64_t walk0, int64_t nwalks, int32_t cap, double* rec,
                              int32_t* code, int32_t* count);
/* Logged cubes -> network inputs X (BF16 [n, N^3], eps / max eps) and FP64
 * permittivity (nullable) at resolution N (16, 21, 23). First-hop cubes are
 * voxelised in the frame where their gradient axis is z, so their gradient
 * target is WVTZ. */
DRWC_API int drwc_records_voxelise(drwc_ctx* ctx, const drwc_structure* s, int N, int n,
                                   const double* rec, const int32_t* code, void* X,
                                   double* eps64);
/* Random transition cubes (1-4 layers along a random axis, 0-2 boxes, eps in
 * [2, 8], noise_frac of them with voxel noise) at resolution N (16, 21, 23):
 * X BF16 [n, N^3] and FP64. */
DRWC_API int drwc_cubes_random(drwc_ctx* ctx, int N, int n, uint64_t seed, float noise_frac,
                               void* X, double* eps64);

typedef struct drwc_learned_opts {
    int32_t slots;          /* walks in flight (default 65536) */
    float conf_threshold;   /* route a hop to FDM when the predicted log10 KL exceeds it */
    float audit_frac;       /* fraction of hops also solved by FDM (default 0.01) */
    int32_t use_graph;      /* reserved (steps size their launches to the active slots) */
    int32_t max_steps;
} drwc_learned_opts;
DRWC_API void drwc_learned_opts_default(drwc_learned_opts* o);
/* Walks with the learned transition kernels (N = 16): per step, every slot's
 * cube goes through the network on the tensor cores; low-confidence hops and
 * audits go through the FDM solve. Records as drwc_frw_walks (host arrays).
 * stats (host, 8 doubles, nullable): network hops, FDM hops, fallbacks,
 * audits, mean audited KL(FDM || network), steps, seconds, walks finished. */
DRWC_API int drwc_frw_walks_learned(drwc_ctx* ctx, const drwc_structure* s,
                                    const drwc_job_params* p, drwc_net* net,
                                    const drwc_learned_opts* opts, int64_t walk0, int64_t nwalks,
                                    int32_t* end_net, int32_t* hops, double* weight,
                                    double* stats);

/* ---- serving: a persistent multi-job extraction engine -------------------
 * No counterpart in the reference (its walker runs one job per process and
 * batches single-walker network queries through ParallelSampler,
 * inference_cpp/src/parallel_sampler.cpp:12-211). A server owns a pool of
 * walker slots on the device and a request thread: submitted jobs queue,
 * are admitted first-in first-out when their device footprint (structure +
 * two batches of walk records) fits the HBM arena and a job-table entry is
 * free, and their walks then share the slots with every other running job.
 * Each replay of a captured CUDA graph advances every slot by
 * steps_per_graph hops: the geometry step of all slots, then one batched
 * network pass per resolution that has a network over the cubes of all its
 * jobs, and the FDM solves bucketed by cube resolution, buckets on parallel
 * graph branches. A job's walks are reduced batch by batch in walk-id order, so its
 * result is bit-identical to drwc_frw_run (plain form) whatever else runs. */
typedef struct drwc_server drwc_server;
#define DRWC_SERVER_MAX_SIZES 4
typedef struct drwc_server_opts {
    int32_t slots;            /* walks in flight over all jobs; 0 (default) = 65536 */
    int32_t max_jobs;         /* job-table entries, <= 64 (default 32) */
    int64_t hbm_budget;       /* bytes of the job arena (default 1 GiB) */
    int32_t n_sizes;          /* cube resolutions served (default 3) */
    int32_t sizes[DRWC_SERVER_MAX_SIZES];  /* default {16, 21, 23} */
    int32_t steps_per_graph;  /* hops per slot per graph replay (default 2, <= 8) */
    int32_t max_materials;    /* distinct permittivities per structure (default 16) */
    int32_t max_nets;         /* conductor nets per structure (default 64) */
    float conf_threshold;     /* network hops: route to FDM above this predicted log10 KL */
    float audit_frac;         /* network hops: fraction also solved by FDM */
    int32_t timing;           /* 1: time the FDM and network stages with graph event nodes */
    int32_t uniform_table;    /* 1: a hop whose cube voxelises to one permittivity draws from
                                 the precomputed uniform-permittivity Green's function (exact
                                 for such cubes: their surface values do not depend on the
                                 permittivity) instead of the network or the FDM solve */
    int32_t fair_share;       /* 0: free slots go to the oldest running job first (first in,
                                 first out, later jobs fill what it leaves); 1: slots rotate
                                 over the running jobs (an even share) */
    int32_t fdm_hops;         /* once all walks of a job without a network have been
                                 claimed (uniform_table = 0), each of its remaining walks
                                 takes up to this many hops per step inside the FDM solve,
                                 1..64; 0 (default) = 64. Otherwise each hop of such a
                                 tail walk waits a whole step, and the job's completion
                                 waits for its longest walks */
    int32_t straggler_hops;   /* a walk of such a job (no network, uniform_table = 0) that
                                 has taken this many hops also takes up to fdm_hops hops per
                                 step, so a batch does not wait many steps for its longest
                                 walks (a job holds at most 8 batches of walk ids in flight);
                                 0 (default) = 32; a value above max_hops turns it off */
} drwc_server_opts;
DRWC_API void drwc_server_opts_default(drwc_server_opts* o);
/* nets (n_nets of them, each of a different served resolution; none: every
 * hop is an FDM solve): the hops of a job whose N has a network go through it
 * (confidence routing + audits as drwc_frw_walks_learned), the others through
 * the FDM solve. The server uses the context's stream and lock and holds the
 * networks (destroy it before them). */
DRWC_API int drwc_server_create(drwc_ctx* ctx, const drwc_server_opts* opts,
                                drwc_net* const* nets, int32_t n_nets, drwc_server** out);
/* Stops the request thread; queued and running jobs end as failed
 * (DRWC_ERR_SHUTDOWN). */
DRWC_API int drwc_server_destroy(drwc_server* srv);
/* Queue a job (structure and parameters are copied). Rejected at once when
 * invalid, when its N is not served or its structure exceeds max_nets /
 * max_materials. */
DRWC_API int drwc_server_submit(drwc_server* srv, const drwc_structure* s,
                                const drwc_job_params* p, int64_t* job_id);
/* As drwc_server_submit, and every walk that finishes also writes its end net
 * (-1: lost) and weight (fF) at its walk id into the caller's DEVICE arrays
 * end_net / weight (p->max_walks entries each; ids a converged job never ran
 * keep what the caller put there). Walk w of a job is walk w of
 * drwc_frw_walks with the same parameters, so the records can be compared
 * walk by walk with another form of the same job. The arrays must stay
 * valid until the job is done. */
DRWC_API int drwc_server_submit_records(drwc_server* srv, const drwc_structure* s,
                                        const drwc_job_params* p, int32_t* end_net,
                                        double* weight, int64_t* job_id);
enum { DRWC_JOB_QUEUED = 0, DRWC_JOB_RUNNING = 1, DRWC_JOB_DONE = 2, DRWC_JOB_FAILED = 3 };
/* state (host): queued / running / done / failed; out (nullable) gets the
 * result once done, with seconds = submission to completion. Returns the
 * job's error code when it failed. */
DRWC_API int drwc_server_poll(drwc_server* srv, int64_t job_id, int32_t* state,
                              drwc_job_result* out);
/* Block until the job is done or failed (DRWC_ERR_TIMEOUT after timeout_s). */
DRWC_API int drwc_server_wait(drwc_server* srv, int64_t job_id, double timeout_s,
                              drwc_job_result* out);
/* Seconds from submission to admission and to completion of a finished job. */
DRWC_API int drwc_server_job_times(drwc_server* srv, int64_t job_id, double* queued_s,
                                   double* latency_s);
typedef struct drwc_server_stats {
    int64_t submitted, admitted, completed, failed;
    int64_t queued, running;          /* now */
    int64_t max_running;              /* most jobs resident at once */
    int64_t hops;                     /* hops executed (all jobs, dropped walks included) */
    int64_t net_hops, fdm_hops, fallbacks, audits;
    int64_t walks_finished, walks_dropped;
    int64_t graph_launches, kernels_launched;
    int64_t arena_bytes, arena_used, arena_peak;
    double busy_seconds;              /* device time of the graph replays */
    double fdm_seconds, net_seconds;  /* summed stage times (timing = 1), else 0 */
    double net_rows;                  /* network rows evaluated */
    double audit_kl_mean;             /* mean KL(FDM || network) over audited hops */
    int64_t fdm_iters, fdm_sweeps;    /* FP32 CG iterations and FP64 sweeps of the FDM hops */
    double fdm_bytes;                 /* streamed-PCG algorithmic bytes of the FDM hops */
    int64_t table_hops;               /* hops drawn from the uniform-permittivity tables */
    int64_t fdm_escalated;            /* FDM solves that needed escalation sweeps */
    int64_t fdm_failed;               /* FDM solves unconverged after escalation (walk lost) */
} drwc_server_stats;
/* Returns the request thread's error code, if it stopped on one. */
DRWC_API int drwc_server_stats_get(drwc_server* srv, drwc_server_stats* out);

/* Run one extraction job (master row of the capacitance matrix) to
 * convergence on the device. Host structure in, host result out. */
DRWC_API int drwc_frw_run(drwc_ctx* ctx, const drwc_structure* s, const drwc_job_params* p,
                          drwc_job_result* out);

/* Run walks [walk0, walk0 + nwalks) of a job and return the per-walk records
 * (end net, hop count, weight in fF) to host arrays. Same walk ids give the
 * same records whatever the batch; this is what the parity tests compare.
 * solver_stats (nullable, 6 int64): total hops, FP32 CG iterations, FP64
 * residual sweeps, cube cells solved (sum of N^3 over hops), escalated
 * solves and failed solves (walk lost). */
DRWC_API int drwc_frw_walks(drwc_ctx* ctx, const drwc_structure* s, const drwc_job_params* p,
                            int64_t walk0, int64_t nwalks, int32_t* end_net, int32_t* hops,
                            double* weight, int64_t* solver_stats);

#ifdef __cplusplus
}
#endif
#endif /* DRWC_H */
