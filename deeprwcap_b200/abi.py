"""ctypes mirrors of the structs in ``include/drwc.h`` and the loader of the
CUDA library ``deeprwcap_b200/libdrwc.so``.

The library is the product: every compute entry point of this package goes
through it. There is no CPU fallback — when the library or a CUDA device is
missing the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("DRWC_LIBRARY", str(PKG / "libdrwc.so")))

MAX_NETS = 256
MAX_LAYERS = 15
MAX_CUBOIDS = 15
LAYER_STRIDE = 2 * MAX_LAYERS
CUBOID_STRIDE = 7 * MAX_CUBOIDS
PADDING = -9999.0
N_MIN, N_MAX = 4, 23

GFT, WVTZ, WVTX, WVTY = 0, 1, 2, 3

STATUS = {
    0: "DRWC_OK", 1: "DRWC_ERR_INVALID", 2: "DRWC_ERR_CUDA", 3: "DRWC_ERR_NOMEM",
    4: "DRWC_ERR_NOT_CONVERGED", 5: "DRWC_ERR_NO_DEVICE", 6: "DRWC_ERR_TIMEOUT",
    7: "DRWC_ERR_SHUTDOWN", 8: "DRWC_ERR_GEOMETRY",
}

# Every symbol include/drwc.h declares (checked by the CPU tests).
EXPORTS = [
    "drwc_version", "drwc_status_string", "drwc_ctx_create", "drwc_ctx_destroy",
    "drwc_ctx_stream", "drwc_ctx_synchronize", "drwc_ctx_launch_count",
    "drwc_fdm_opts_default", "drwc_ggft_solve", "drwc_fdm_solve_batch_device",
    "drwc_fdm_solve_batch", "drwc_structure_construction", "drwc_transition_batch",
    "drwc_first_hop_batch", "drwc_job_params_default", "drwc_frw_run", "drwc_frw_walks",
    "drwc_job_create", "drwc_job_destroy", "drwc_job_walks_device", "drwc_job_h2d_bytes",
    "drwc_fdm_solve_noalloc", "drwc_gemm_bf16",
    "drwc_net_create", "drwc_net_destroy", "drwc_net_dims", "drwc_net_param_count",
    "drwc_net_get_params",
    "drwc_net_set_params", "drwc_net_gradients", "drwc_net_forward", "drwc_net_train_step",
    "drwc_frw_harvest", "drwc_records_voxelise", "drwc_cubes_random", "drwc_learned_opts_default",
    "drwc_frw_walks_learned",
    "drwc_server_opts_default", "drwc_server_create", "drwc_server_destroy", "drwc_server_submit",
    "drwc_server_poll", "drwc_server_wait", "drwc_server_job_times", "drwc_server_stats_get",
    "drwc_server_submit_records",
]


class DrwcError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where}: {STATUS.get(status, status)}")
        self.status = status


class FdmOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("inner_tol", C.c_double),
                ("max_outer", C.c_int32), ("max_inner", C.c_int32),
                ("warm_start", C.c_int32), ("extra_outer", C.c_int32)]

    def __init__(self, tol=1e-10, inner_tol=1e-5, max_outer=8, max_inner=0, warm_start=1,
                 extra_outer=8):
        super().__init__(tol, inner_tol, max_outer, max_inner, warm_start, extra_outer)


class Box(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3), ("net", C.c_int32),
                ("pad_", C.c_int32)]


class DielBox(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3), ("eps", C.c_double)]


class Structure(C.Structure):
    _fields_ = [("n_boxes", C.c_int32), ("n_nets", C.c_int32), ("boxes", C.POINTER(Box)),
                ("n_layers", C.c_int32), ("n_diel", C.c_int32),
                ("layer_zlo", C.POINTER(C.c_double)), ("layer_eps", C.POINTER(C.c_double)),
                ("diel", C.POINTER(DielBox)), ("encl_lo", C.c_double * 3),
                ("encl_hi", C.c_double * 3)]


class JobParams(C.Structure):
    _fields_ = [("master", C.c_int32), ("N", C.c_int32), ("gauss_offset", C.c_double),
                ("stop_dist", C.c_double), ("p_tol", C.c_double), ("c_tol", C.c_double),
                ("c_ratio", C.c_double), ("min_walks", C.c_int64), ("max_walks", C.c_int64),
                ("batch_walks", C.c_int64), ("max_hops", C.c_int32), ("gauss_surface", C.c_int32),
                ("seed", C.c_uint64), ("fdm", FdmOpts)]


class LearnedOpts(C.Structure):
    _fields_ = [("slots", C.c_int32), ("conf_threshold", C.c_float), ("audit_frac", C.c_float),
                ("use_graph", C.c_int32), ("max_steps", C.c_int32)]


SERVER_MAX_SIZES = 4
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


class ServerOpts(C.Structure):
    _fields_ = [("slots", C.c_int32), ("max_jobs", C.c_int32), ("hbm_budget", C.c_int64),
                ("n_sizes", C.c_int32), ("sizes", C.c_int32 * SERVER_MAX_SIZES),
                ("steps_per_graph", C.c_int32), ("max_materials", C.c_int32),
                ("max_nets", C.c_int32), ("conf_threshold", C.c_float), ("audit_frac", C.c_float),
                ("timing", C.c_int32), ("uniform_table", C.c_int32), ("fair_share", C.c_int32),
                ("fdm_hops", C.c_int32), ("straggler_hops", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "submitted", "admitted", "completed", "failed", "queued", "running", "max_running",
        "hops", "net_hops", "fdm_hops", "fallbacks", "audits", "walks_finished", "walks_dropped",
        "graph_launches", "kernels_launched", "arena_bytes", "arena_used", "arena_peak")] + \
        [(n, C.c_double) for n in ("busy_seconds", "fdm_seconds", "net_seconds", "net_rows",
                                   "audit_kl_mean")] + \
        [("fdm_iters", C.c_int64), ("fdm_sweeps", C.c_int64), ("fdm_bytes", C.c_double),
         ("table_hops", C.c_int64), ("fdm_escalated", C.c_int64), ("fdm_failed", C.c_int64)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class JobResult(C.Structure):
    _fields_ = [("n_entries", C.c_int32), ("converged", C.c_int32), ("walks", C.c_int64),
                ("hops", C.c_int64), ("lost", C.c_int64), ("solves_escalated", C.c_int64),
                ("solves_failed", C.c_int64), ("seconds", C.c_double),
                ("cap", C.c_double * (MAX_NETS + 1)), ("stderr_", C.c_double * (MAX_NETS + 1))]


_lib = None


def load():
    """Load libdrwc.so (built by ``deeprwcap_b200.build``). Raises when it is
    missing: there is no fallback path."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(
            f"{LIB_PATH} is missing: build it with `python -m deeprwcap_b200.build` "
            "(the FRW engine has no CPU fallback)")
    L = C.CDLL(str(LIB_PATH))
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    L.drwc_version.restype = C.c_char_p
    L.drwc_status_string.restype = C.c_char_p
    L.drwc_status_string.argtypes = [C.c_int]
    L.drwc_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.drwc_ctx_destroy.argtypes = [vp]
    L.drwc_ctx_stream.argtypes = [vp, C.POINTER(vp)]
    L.drwc_ctx_synchronize.argtypes = [vp]
    L.drwc_ctx_launch_count.argtypes = [vp, C.POINTER(i64)]
    L.drwc_fdm_opts_default.argtypes = [C.POINTER(FdmOpts)]
    L.drwc_fdm_opts_default.restype = None
    L.drwc_ggft_solve.argtypes = [vp, C.c_int, vp, C.c_int, dbl, vp, C.POINTER(i32)]
    L.drwc_fdm_solve_batch_device.argtypes = [vp, C.c_int, vp, vp, vp, vp,
                                              C.POINTER(FdmOpts), vp, vp, vp, vp, vp, vp]
    L.drwc_fdm_solve_batch.argtypes = [vp, C.c_int, vp, vp, vp, vp, C.POINTER(FdmOpts), vp,
                                       vp, vp, vp, vp]
    L.drwc_structure_construction.argtypes = [vp, C.c_int, C.c_int, vp, vp, C.c_int, vp, vp]
    L.drwc_transition_batch.argtypes = [vp, C.c_int, C.c_int, vp, vp, C.c_uint64, C.c_uint64,
                                        vp]
    L.drwc_first_hop_batch.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, C.c_uint64,
                                       C.c_uint64, vp]
    L.drwc_job_params_default.argtypes = [C.POINTER(JobParams)]
    L.drwc_job_params_default.restype = None
    L.drwc_frw_run.argtypes = [vp, C.POINTER(Structure), C.POINTER(JobParams),
                               C.POINTER(JobResult)]
    L.drwc_frw_walks.argtypes = [vp, C.POINTER(Structure), C.POINTER(JobParams), i64, i64, vp,
                                 vp, vp, vp]
    L.drwc_job_create.argtypes = [vp, C.POINTER(Structure), C.POINTER(JobParams), C.POINTER(vp)]
    L.drwc_job_destroy.argtypes = [vp]
    L.drwc_job_walks_device.argtypes = [vp, i64, i64, vp, vp, vp, vp]
    L.drwc_job_h2d_bytes.argtypes = [vp, C.POINTER(i64)]
    L.drwc_fdm_solve_noalloc.argtypes = [vp, C.c_int, C.c_int, vp, vp, C.POINTER(FdmOpts), vp,
                                         vp, vp]
    L.drwc_gemm_bf16.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, i64, vp, i64, vp, i64, vp,
                                 C.c_int, vp]
    L.drwc_net_create.argtypes = [vp, C.c_int, C.c_uint64, C.POINTER(vp)]
    L.drwc_net_destroy.argtypes = [vp]
    L.drwc_net_param_count.argtypes = [vp, C.POINTER(i64)]
    L.drwc_net_get_params.argtypes = [vp, vp]
    L.drwc_net_set_params.argtypes = [vp, vp]
    L.drwc_net_gradients.argtypes = [vp, vp]
    L.drwc_net_forward.argtypes = [vp, C.c_int, vp, vp, vp]
    L.drwc_net_train_step.argtypes = [vp, C.c_int, vp, vp, vp, C.c_float, C.c_float, C.c_float,
                                      C.c_float, C.c_float, C.c_int, vp]
    L.drwc_frw_harvest.argtypes = [vp, C.POINTER(Structure), C.POINTER(JobParams), i64, i64,
                                   i32, vp, vp, C.POINTER(i32)]
    L.drwc_records_voxelise.argtypes = [vp, C.POINTER(Structure), C.c_int, C.c_int, vp, vp, vp, vp]
    L.drwc_cubes_random.argtypes = [vp, C.c_int, C.c_int, C.c_uint64, C.c_float, vp, vp]
    L.drwc_net_dims.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32),
                                C.POINTER(i32), C.POINTER(i32)]
    L.drwc_learned_opts_default.argtypes = [C.POINTER(LearnedOpts)]
    L.drwc_learned_opts_default.restype = None
    L.drwc_frw_walks_learned.argtypes = [vp, C.POINTER(Structure), C.POINTER(JobParams), vp,
                                         C.POINTER(LearnedOpts), i64, i64, vp, vp, vp, vp]
    L.drwc_server_opts_default.argtypes = [C.POINTER(ServerOpts)]
    L.drwc_server_opts_default.restype = None
    L.drwc_server_create.argtypes = [vp, C.POINTER(ServerOpts), C.POINTER(vp), i32, C.POINTER(vp)]
    L.drwc_server_destroy.argtypes = [vp]
    L.drwc_server_submit.argtypes = [vp, C.POINTER(Structure), C.POINTER(JobParams),
                                     C.POINTER(i64)]
    L.drwc_server_submit_records.argtypes = [vp, C.POINTER(Structure), C.POINTER(JobParams),
                                             vp, vp, C.POINTER(i64)]
    L.drwc_server_poll.argtypes = [vp, i64, C.POINTER(i32), C.POINTER(JobResult)]
    L.drwc_server_wait.argtypes = [vp, i64, dbl, C.POINTER(JobResult)]
    L.drwc_server_job_times.argtypes = [vp, i64, C.POINTER(dbl), C.POINTER(dbl)]
    L.drwc_server_stats_get.argtypes = [vp, C.POINTER(ServerStats)]
    _lib = L
    return L


def check(status: int, where: str) -> None:
    if status != 0:
        raise DrwcError(status, where)


def ptr(a) -> int:
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def default_fdm_opts() -> FdmOpts:
    o = FdmOpts()
    load().drwc_fdm_opts_default(C.byref(o))
    return o


def default_job_params() -> JobParams:
    p = JobParams()
    load().drwc_job_params_default(C.byref(p))
    return p
