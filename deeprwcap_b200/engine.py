"""Python mirror of the reference's interfaces for the FRW transition path,
over the C ABI of ``libdrwc.so`` (``include/drwc.h``).

* ``GgftSolver`` mirrors ``deeprwcap::ggft_solver`` (ggft/src/ggft_solver.h:112-198):
  public ``DIEL``, ``gft``, ``solve(code) -> bool``, ``set_tolerance(tol)``.
* ``DNNSolverPoisson`` / ``DNNSolverGrad`` mirror the dnnsolver classes
  (inference_cpp/src/dnn_solver.h:98-149): ``loadModels()``,
  ``sample(layers, cuboids[, axis]) -> list[float]``.
* ``ParallelSampler`` mirrors inference_cpp/src/parallel_sampler.cpp: many
  producer threads ``submit`` single queries and get futures; one worker
  thread batches them (<= batch_size) into one library call.
* ``extract`` runs an FRW capacitance job on the device.

Every compute call goes through the CUDA library; nothing here computes on
the CPU.
"""
from __future__ import annotations

import ctypes as C
import queue
import threading
import warnings
from concurrent.futures import Future

import numpy as np

from . import abi
from .abi import GFT, WVTX, WVTY, WVTZ, check, load, ptr


def torch_ready() -> None:
    """Order the library after the torch work queued so far: the library runs
    on its context's own (non-blocking) stream, torch plumbing on torch's
    current stream. Call before handing torch-produced device buffers to the
    library; library outputs are ordered back by Context.synchronize()."""
    import sys
    torch = sys.modules.get("torch")
    if torch is not None and torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.current_stream().synchronize()


class Context:
    """One device context (stream + workspaces), as DNNSolver's constructor
    (dnn_solver.cpp:13-38)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.drwc_ctx_create(int(device), C.byref(h)), "drwc_ctx_create")
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            self.lib.drwc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(self.lib.drwc_ctx_stream(self.h, C.byref(s)), "drwc_ctx_stream")
        return s.value or 0

    def synchronize(self):
        check(self.lib.drwc_ctx_synchronize(self.h), "drwc_ctx_synchronize")

    @property
    def launches(self) -> int:
        n = C.c_int64()
        check(self.lib.drwc_ctx_launch_count(self.h, C.byref(n)), "drwc_ctx_launch_count")
        return n.value


_default_ctx = {}


def default_context(device: int = 0) -> Context:
    if device not in _default_ctx:
        _default_ctx[device] = Context(device)
    return _default_ctx[device]


# ---------------------------------------------------------------------- ggft
class GgftSolver:
    """Drop-in for ``deeprwcap::ggft_solver`` on the device."""
    GFT, WVTZ, WVTX, WVTY = GFT, WVTZ, WVTX, WVTY

    def __init__(self, N: int, ctx: Context | None = None):
        if not (abi.N_MIN <= N <= abi.N_MAX):
            raise ValueError(f"N={N} outside [{abi.N_MIN}, {abi.N_MAX}]")
        self.N = N
        self.ctx = ctx or default_context()
        self.DIEL = np.ones(N ** 3)           # ggft_solver.h:152 (DIEL = 1)
        self.gft = np.zeros(6 * N * N)
        self.tolerance = 1e-8                  # ggft_solver.h:155
        self.iterations = 0

    def set_tolerance(self, tol: float) -> None:
        self.tolerance = float(tol)

    def solve(self, code: int) -> bool:
        eps = np.ascontiguousarray(self.DIEL, dtype=np.float64).reshape(-1)
        if eps.size != self.N ** 3:
            raise ValueError("DIEL must hold N^3 values")
        out = np.zeros(6 * self.N * self.N)
        it = C.c_int32(0)
        rc = self.ctx.lib.drwc_ggft_solve(self.ctx.h, self.N, eps.ctypes.data, int(code),
                                          self.tolerance, out.ctypes.data, C.byref(it))
        self.iterations = it.value
        if rc not in (0, 4):
            check(rc, "drwc_ggft_solve")
        self.gft = out
        return rc == 0


def fdm_solve_batch(eps_list_or_batch, code=None, tol: float = 1e-10, inner_tol: float = 1e-5,
                    ctx: Context | None = None, max_outer: int = 8, max_inner: int = 0,
                    warm_start: bool = True):
    """Solve many cubes (host arrays). Accepts a list of [N,N,N] arrays or a
    ``workloads.MixedBatch``. Returns (list of 6N^2 arrays, iters, relres,
    status)."""
    ctx = ctx or default_context()
    if hasattr(eps_list_or_batch, "eps_off"):
        b = eps_list_or_batch
        Ns, eoff, ooff, eps = b.N, b.eps_off, b.out_off, b.eps
        out = np.zeros(b.out_size)
    else:
        cubes = [np.ascontiguousarray(e, dtype=np.float64) for e in eps_list_or_batch]
        Ns = np.array([c.shape[-1] for c in cubes], dtype=np.int32)
        sizes = Ns.astype(np.int64) ** 3
        eoff = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        ooff = np.concatenate([[0], np.cumsum(6 * Ns.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
        eps = np.concatenate([c.reshape(-1) for c in cubes]) if cubes else np.zeros(1)
        out = np.zeros(int(ooff[-1] + 6 * Ns[-1] ** 2) if len(cubes) else 1)
    n = len(Ns)
    Ns = np.ascontiguousarray(Ns, dtype=np.int32)
    codes = None
    if code is not None:
        codes = np.ascontiguousarray(np.broadcast_to(np.asarray(code, dtype=np.int32), (n,)))
    opts = abi.FdmOpts(tol, inner_tol, max_outer, max_inner, 1 if warm_start else 0)
    iters = np.zeros(n, dtype=np.int32)
    relres = np.zeros(n)
    status = np.zeros(n, dtype=np.int32)
    rc = ctx.lib.drwc_fdm_solve_batch(ctx.h, n, Ns.ctypes.data, eoff.ctypes.data, eps.ctypes.data,
                                      None if codes is None else codes.ctypes.data,
                                      C.byref(opts), ooff.ctypes.data, out.ctypes.data,
                                      iters.ctypes.data, relres.ctypes.data, status.ctypes.data)
    if rc not in (0, 4):
        check(rc, "drwc_fdm_solve_batch")
    res = [out[ooff[c]:ooff[c] + 6 * int(Ns[c]) ** 2] for c in range(n)]
    return res, iters, relres, status


# ------------------------------------------------------------------ dnnsolver
class _DNNSolver:
    """Common part of the dnnsolver drop-ins (dnn_solver.h:43-95)."""

    def __init__(self, device_idx: int = 0, N: int = 23, seed: int = 0x5EED):
        self.ctx = default_context(device_idx)
        self.N = N
        self.seed = seed
        self._stream = 0           # Philox stream position, advanced per query

    def loadModels(self, verbose: bool = False) -> None:
        """The FDM transition kernels need no model files."""
        if verbose:
            print("\tFDM transition kernels: no models to load")

    def structureConstruction(self, layers, cuboids, normalise: bool = True):
        L = np.ascontiguousarray(layers, dtype=np.float32).reshape(-1)
        Cb = np.ascontiguousarray(cuboids, dtype=np.float32).reshape(-1)
        n = L.size // abi.LAYER_STRIDE
        eps = np.zeros((n, self.N, self.N, self.N), dtype=np.float32)
        mx = np.zeros(n, dtype=np.float32)
        check(self.ctx.lib.drwc_structure_construction(self.ctx.h, n, self.N, L.ctypes.data,
                                                       Cb.ctypes.data, 1 if normalise else 0,
                                                       eps.ctypes.data, mx.ctypes.data),
              "drwc_structure_construction")
        return eps, mx

    def _take_stream(self, n: int) -> int:
        s = self._stream
        self._stream += n
        return s


class DNNSolverPoisson(_DNNSolver):
    """Drop-in for DNNSolverPoisson::sample (dnn_solver_poisson.cpp:35-84)."""

    def sample(self, layers, cuboids, axis=None) -> list:
        if axis is not None and not getattr(self, "_warned", False):
            warnings.warn("Axis parameter provided to Green's function solver but will be "
                          "ignored (shown once)")
            self._warned = True
        L = np.ascontiguousarray(layers, dtype=np.float32).reshape(-1)
        Cb = np.ascontiguousarray(cuboids, dtype=np.float32).reshape(-1)
        n = L.size // abi.LAYER_STRIDE
        if Cb.size != n * abi.CUBOID_STRIDE:
            raise ValueError("cuboids must hold 105 floats per query")
        out = np.zeros(3 * n, dtype=np.float32)
        rc = self.ctx.lib.drwc_transition_batch(self.ctx.h, n, self.N, L.ctypes.data,
                                                Cb.ctypes.data, self.seed, self._take_stream(n),
                                                out.ctypes.data)
        check(rc, "drwc_transition_batch")
        return out.tolist()


class DNNSolverGrad(_DNNSolver):
    """Drop-in for DNNSolverGrad::sample (dnn_solver_gradient.cpp:40-73)."""

    def sample(self, layers, cuboids, axis=None) -> list:
        if axis is None:
            raise RuntimeError("Gradient solver requires axis parameter")
        L = np.ascontiguousarray(layers, dtype=np.float32).reshape(-1)
        Cb = np.ascontiguousarray(cuboids, dtype=np.float32).reshape(-1)
        n = L.size // abi.LAYER_STRIDE
        ax = np.ascontiguousarray(axis, dtype=np.int32).reshape(-1)
        if ax.size != n:
            raise ValueError("one axis per query")
        out = np.zeros(5 * n, dtype=np.float32)
        rc = self.ctx.lib.drwc_first_hop_batch(self.ctx.h, n, self.N, L.ctypes.data,
                                               Cb.ctypes.data, ax.ctypes.data, self.seed,
                                               self._take_stream(n), out.ctypes.data)
        check(rc, "drwc_first_hop_batch")
        return out.tolist()


class ParallelSampler:
    """Cross-thread batching of single queries (parallel_sampler.cpp:12-211):
    ``submit`` enqueues and returns a Future; one worker thread drains up to
    ``batch_size`` queries per library call and splits the result evenly.
    A solver exception is forwarded to every future of its batch."""

    def __init__(self, solver: _DNNSolver, sample_size: int, batch_size: int):
        if solver is None:
            raise ValueError("Solver pointer cannot be null")
        self.solver = solver
        self.sample_size = sample_size
        self.batch_size = max(1, min(int(batch_size), 2048))
        self._q: queue.Queue = queue.Queue()
        self._shutdown = False
        self._t = threading.Thread(target=self._loop, daemon=True)
        self._t.start()

    def submit(self, layer, cuboid, axis: int | None = None) -> Future:
        f: Future = Future()
        self._q.put((np.asarray(layer, dtype=np.float32), np.asarray(cuboid, dtype=np.float32),
                     axis, f))
        return f

    def _loop(self):
        while True:
            try:
                first = self._q.get(timeout=0.05)
            except queue.Empty:
                if self._shutdown:
                    return
                continue
            batch = [first]
            while len(batch) < self.batch_size:
                try:
                    batch.append(self._q.get_nowait())
                except queue.Empty:
                    break
            self._process(batch)

    def _process(self, batch):
        try:
            L = np.concatenate([b[0] for b in batch])
            Cb = np.concatenate([b[1] for b in batch])
            has_axis = any(b[2] is not None for b in batch)
            if has_axis:
                res = self.solver.sample(L, Cb, [b[2] if b[2] is not None else 0 for b in batch])
            else:
                res = self.solver.sample(L, Cb)
            if len(res) % len(batch):
                raise RuntimeError("Result size doesn't match expected batch output size")
            w = len(res) // len(batch)
            for i, b in enumerate(batch):
                b[3].set_result(res[i * w:(i + 1) * w])
        except Exception as e:  # forwarded to every task of the batch
            for b in batch:
                if not b[3].done():
                    b[3].set_exception(e)

    def close(self):
        self._shutdown = True
        self._t.join()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------ FRW
class JobResult:
    def __init__(self, r: abi.JobResult):
        n = r.n_entries
        self.n_entries = n
        self.converged = bool(r.converged)
        self.walks = r.walks
        self.hops = r.hops
        self.lost = r.lost
        self.solves_escalated = r.solves_escalated
        self.solves_failed = r.solves_failed
        self.seconds = r.seconds
        self.cap = np.array(r.cap[:n])
        self.stderr = np.array(r.stderr_[:n])

    @property
    def hops_per_s(self) -> float:
        return self.hops / self.seconds if self.seconds > 0 else 0.0

    def __repr__(self):
        return (f"JobResult(walks={self.walks}, hops={self.hops}, converged={self.converged}, "
                f"seconds={self.seconds:.3f}, cap={np.array2string(self.cap, precision=5)})")


def extract(structure, params, ctx: Context | None = None) -> JobResult:
    """Run one FRW job (master row of the capacitance matrix, fF)."""
    ctx = ctx or default_context()
    s = structure.to_c() if hasattr(structure, "to_c") else structure
    r = abi.JobResult()
    check(ctx.lib.drwc_frw_run(ctx.h, C.byref(s), C.byref(params), C.byref(r)), "drwc_frw_run")
    return JobResult(r)


def frw_walks(structure, params, walk0: int, nwalks: int, ctx: Context | None = None,
              stats: bool = False):
    """Per-walk records (end net, hops, weight in fF) for walks
    [walk0, walk0+nwalks); with stats=True also the solver counters
    (hops, FP32 iterations, FP64 sweeps, cells solved, escalated solves,
    failed solves)."""
    ctx = ctx or default_context()
    s = structure.to_c() if hasattr(structure, "to_c") else structure
    end = np.zeros(nwalks, dtype=np.int32)
    hops = np.zeros(nwalks, dtype=np.int32)
    w = np.zeros(nwalks)
    st = np.zeros(6, dtype=np.int64)
    check(ctx.lib.drwc_frw_walks(ctx.h, C.byref(s), C.byref(params), int(walk0), int(nwalks),
                                 end.ctypes.data, hops.ctypes.data, w.ctypes.data,
                                 st.ctypes.data),
          "drwc_frw_walks")
    if stats:
        return end, hops, w, st
    return end, hops, w


class Job:
    """A prepared FRW job (structure uploaded once). ``walks_device`` launches
    walks asynchronously on the context stream into device arrays (torch
    tensors or raw pointers)."""

    def __init__(self, structure, params, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self._s = structure.to_c() if hasattr(structure, "to_c") else structure
        self.params = params
        h = C.c_void_p()
        check(self.ctx.lib.drwc_job_create(self.ctx.h, C.byref(self._s), C.byref(params),
                                           C.byref(h)), "drwc_job_create")
        self.h = h

    def walks_device(self, walk0: int, nwalks: int, end, hops, weight, stats=None) -> None:
        """Async on the context stream; order torch work before it with
        torch_ready() and read the outputs after Context.synchronize()."""
        check(self.ctx.lib.drwc_job_walks_device(self.h, int(walk0), int(nwalks), ptr(end),
                                                 ptr(hops), ptr(weight), ptr(stats)),
              "drwc_job_walks_device")

    @property
    def h2d_bytes(self) -> int:
        b = C.c_int64()
        check(self.ctx.lib.drwc_job_h2d_bytes(self.h, C.byref(b)), "drwc_job_h2d_bytes")
        return b.value

    def close(self):
        if self.h:
            self.ctx.lib.drwc_job_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ learned
NET_OUT = 1552
NET_PANELS = 1536


def net_dims(N: int) -> dict:
    """Layer sizes of the network for cube resolution N (mirrors NetDims in nn.cu)."""
    d = [N]
    for _ in range(3):
        d.append((d[-1] - 1) // 2 + 1)
    np_ = 6 * N * N
    return {"N": N, "D": d, "panels": np_, "out_row": (np_ + 1 + 15) // 16 * 16,
            "grad_row": (np_ + 15) // 16 * 16, "features": 64 * d[3] ** 3}


def _param_layout(N: int = 16):
    """Offsets of the flat FP32 parameter vector (mirrors ParamLayout in nn.cu)."""
    dm = net_dims(N)
    names = [("w1", 16 * 27), ("b1", 16), ("w2", 32 * 432), ("b2", 32), ("w3", 64 * 864),
             ("b3", 64), ("wd", dm["out_row"] * dm["features"]), ("bd", dm["out_row"]),
             ("wg", dm["panels"] * dm["features"]), ("bg", dm["panels"])]
    off, lay = 0, {}
    for name, n in names:
        lay[name] = (off, n)
        off += (n + 63) // 64 * 64
    return lay, off


class Net:
    """The learned transition network (device-resident; see include/drwc.h)."""

    def __init__(self, seed: int = 0, ctx: Context | None = None, N: int = 16):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(self.ctx.lib.drwc_net_create(self.ctx.h, int(N), seed, C.byref(h)), "drwc_net_create")
        self.h = h
        v = [C.c_int32() for _ in range(5)]
        check(self.ctx.lib.drwc_net_dims(h, *[C.byref(x) for x in v]), "drwc_net_dims")
        self.N, self.panels, self.out_row, self.grad_row, self.features = (x.value for x in v)
        n = C.c_int64()
        check(self.ctx.lib.drwc_net_param_count(h, C.byref(n)), "drwc_net_param_count")
        self.nparams = n.value

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.nparams, dtype=np.float32)
        check(self.ctx.lib.drwc_net_get_params(self.h, out.ctypes.data), "drwc_net_get_params")
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        check(self.ctx.lib.drwc_net_set_params(self.h, p.ctypes.data), "drwc_net_set_params")

    def gradients(self) -> np.ndarray:
        out = np.zeros(self.nparams, dtype=np.float32)
        check(self.ctx.lib.drwc_net_gradients(self.h, out.ctypes.data), "drwc_net_gradients")
        return out

    def forward(self, X, O, G=None) -> None:
        """X: [B, N^3] bfloat16 device tensor; O: [B, out_row] float32; G: [B, grad_row]."""
        torch_ready()
        check(self.ctx.lib.drwc_net_forward(self.h, int(X.shape[0]), ptr(X), ptr(O), ptr(G)),
              "drwc_net_forward")
        self.ctx.synchronize()

    def train_step(self, X, T, TG=None, lr=1e-3, weight_decay=1e-10, clip=1.0, w_conf=0.1,
                   w_grad=1.0, apply=True):
        loss = (C.c_float * 3)()
        torch_ready()
        check(self.ctx.lib.drwc_net_train_step(self.h, int(X.shape[0]), ptr(X), ptr(T), ptr(TG),
                                               lr, weight_decay, clip, w_conf, w_grad,
                                               1 if apply else 0, loss), "drwc_net_train_step")
        return list(loss)

    def close(self):
        if self.h:
            self.ctx.lib.drwc_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def learned_opts(**kw) -> "abi.LearnedOpts":
    o = abi.LearnedOpts()
    load().drwc_learned_opts_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def frw_walks_learned(structure, params, net: Net, walk0: int, nwalks: int, opts=None,
                      ctx: Context | None = None):
    """Walks with the learned transition kernels. Returns (end, hops, weight,
    stats dict)."""
    ctx = ctx or net.ctx
    s = structure.to_c() if hasattr(structure, "to_c") else structure
    end = np.zeros(nwalks, dtype=np.int32)
    hops = np.zeros(nwalks, dtype=np.int32)
    w = np.zeros(nwalks)
    st = np.zeros(8)
    o = opts or learned_opts()
    rc = ctx.lib.drwc_frw_walks_learned(ctx.h, C.byref(s), C.byref(params), net.h, C.byref(o),
                                        int(walk0), int(nwalks), end.ctypes.data,
                                        hops.ctypes.data, w.ctypes.data, st.ctypes.data)
    check(rc, "drwc_frw_walks_learned")
    keys = ["net_hops", "fdm_hops", "fallbacks", "audits", "audit_kl", "steps", "seconds",
            "walks"]
    return end, hops, w, dict(zip(keys, st.tolist()))


def harvest(structure, params, walk0: int, nwalks: int, cap: int, ctx: Context | None = None):
    """Log the transition cubes of real walks: device tensors rec [n, 4] (centre,
    half-width) and code [n] (solver code), n <= cap."""
    import torch
    ctx = ctx or default_context()
    s = structure.to_c() if hasattr(structure, "to_c") else structure
    dev = torch.device("cuda", ctx.device)
    rec = torch.empty(cap, 4, dtype=torch.float64, device=dev)
    code = torch.empty(cap, dtype=torch.int32, device=dev)
    cnt = C.c_int32(0)
    torch_ready()
    check(ctx.lib.drwc_frw_harvest(ctx.h, C.byref(s), C.byref(params), int(walk0), int(nwalks),
                                   int(cap), ptr(rec), ptr(code), C.byref(cnt)),
          "drwc_frw_harvest")
    return rec[:cnt.value], code[:cnt.value]


def records_voxelise(structure, rec, code, X, eps64=None, ctx: Context | None = None, N: int = 16):
    """Logged cubes -> network inputs X [n, N^3] (BF16) and FP64 permittivity."""
    ctx = ctx or default_context()
    s = structure.to_c() if hasattr(structure, "to_c") else structure
    torch_ready()
    check(ctx.lib.drwc_records_voxelise(ctx.h, C.byref(s), int(N), int(rec.shape[0]), ptr(rec),
                                        ptr(code), ptr(X), ptr(eps64)), "drwc_records_voxelise")


def cubes_random(n: int, seed: int, X, eps64, noise_frac: float = 0.1,
                 ctx: Context | None = None, N: int = 16):
    """Random transition cubes at resolution N: X [n, N^3] BF16, eps64 FP64."""
    ctx = ctx or default_context()
    torch_ready()
    check(ctx.lib.drwc_cubes_random(ctx.h, int(N), int(n), seed, noise_frac, ptr(X), ptr(eps64)),
          "drwc_cubes_random")
    ctx.synchronize()


def fdm_solve_device(ctx: Context, eps64, N: int, code, out, tol: float = 1e-8):
    """Packed same-N device batch through the regular batched entry point:
    eps64 [n, N^3] float64, code int or [n] int32 host array, out [n, 6N^2]."""
    n = int(eps64.shape[0])
    Ns = np.full(n, N, dtype=np.int32)
    eoff = np.arange(n, dtype=np.int64) * N ** 3
    ooff = np.arange(n, dtype=np.int64) * 6 * N * N
    codes = np.ascontiguousarray(np.broadcast_to(np.asarray(code, dtype=np.int32), (n,)))
    opts = abi.FdmOpts(tol, 1e-5, 8, 0, 1)
    torch_ready()
    check(ctx.lib.drwc_fdm_solve_batch_device(ctx.h, n, Ns.ctypes.data, eoff.ctypes.data,
                                              ptr(eps64), codes.ctypes.data, C.byref(opts),
                                              ooff.ctypes.data, ptr(out), None, None, None, None),
          "drwc_fdm_solve_batch_device")
    ctx.synchronize()


# ------------------------------------------------------------------ serving
def server_opts(**kw) -> "abi.ServerOpts":
    o = abi.ServerOpts()
    load().drwc_server_opts_default(C.byref(o))
    for k, v in kw.items():
        if k == "sizes":
            o.n_sizes = len(v)
            for i, n in enumerate(v):
                o.sizes[i] = int(n)
        else:
            setattr(o, k, v)
    return o


class Server:
    """The persistent multi-job extraction server (drwc_server_* in
    include/drwc.h): jobs are submitted from the host, admitted by device
    footprint and run concurrently on the device; results come back per job.
    ``net``: a Net or a list of Nets of different resolutions; the hops of a
    job whose N has a network go through it."""

    def __init__(self, ctx: Context | None = None, net=None, **opts):
        nets = [] if net is None else (list(net) if isinstance(net, (list, tuple)) else [net])
        self.ctx = ctx or (nets[0].ctx if nets else default_context())
        self.opts = server_opts(**opts)
        h = C.c_void_p()
        arr = (C.c_void_p * max(1, len(nets)))(*[n.h for n in nets])
        torch_ready()
        check(self.ctx.lib.drwc_server_create(self.ctx.h, C.byref(self.opts), arr, len(nets),
                                              C.byref(h)), "drwc_server_create")
        self.h = h
        self.nets = nets  # the server holds them

    def submit(self, structure, params, records=None) -> int:
        """Queue a job. records = (end_net, weight) device tensors of
        params.max_walks entries: every finished walk writes its end net and
        weight there at its walk id (drwc_server_submit_records)."""
        s = structure.to_c() if hasattr(structure, "to_c") else structure
        jid = C.c_int64()
        if records is None:
            check(self.ctx.lib.drwc_server_submit(self.h, C.byref(s), C.byref(params),
                                                  C.byref(jid)), "drwc_server_submit")
        else:
            end, w = records
            torch_ready()
            check(self.ctx.lib.drwc_server_submit_records(self.h, C.byref(s), C.byref(params),
                                                          ptr(end), ptr(w), C.byref(jid)),
                  "drwc_server_submit_records")
        return jid.value

    def poll(self, jid: int):
        """(state, JobResult or None); state is one of abi.JOB_*."""
        st = C.c_int32()
        r = abi.JobResult()
        check(self.ctx.lib.drwc_server_poll(self.h, int(jid), C.byref(st), C.byref(r)),
              "drwc_server_poll")
        return st.value, (JobResult(r) if st.value == abi.JOB_DONE else None)

    def wait(self, jid: int, timeout: float = 600.0) -> JobResult:
        r = abi.JobResult()
        check(self.ctx.lib.drwc_server_wait(self.h, int(jid), float(timeout), C.byref(r)),
              "drwc_server_wait")
        return JobResult(r)

    def times(self, jid: int):
        """(seconds queued before admission, seconds from submission to result)."""
        q, l = C.c_double(), C.c_double()
        check(self.ctx.lib.drwc_server_job_times(self.h, int(jid), C.byref(q), C.byref(l)),
              "drwc_server_job_times")
        return q.value, l.value

    def stats(self) -> dict:
        st = abi.ServerStats()
        check(self.ctx.lib.drwc_server_stats_get(self.h, C.byref(st)), "drwc_server_stats_get")
        return st.as_dict()

    def close(self):
        if self.h:
            self.ctx.lib.drwc_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
