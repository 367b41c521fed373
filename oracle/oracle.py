"""TEST INFRASTRUCTURE ONLY — ctypes front end of the CPU checkers.

Loads ``oracle/liboracle.so`` (the C restatement, ``fdm_oracle.c`` and
``frw_oracle.c``) and, when present, ``oracle/_ref/libggft_ref_N<N>.so`` (the
reference ggft solver compiled from its own sources by ``oracle/Makefile``).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GFT, WVTZ, WVTX, WVTY = 0, 1, 2, 3

_lib = None
_ref = {}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def reference_dir() -> Path:
    """Where the reference tree is mounted: $DRWC_REFERENCE_DIR, else a
    directory named ``reference`` beside this repository's folder."""
    env = os.environ.get("DRWC_REFERENCE_DIR")
    return Path(env) if env else HERE.parents[1] / "reference"


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and the reference objects when the reference
    tree is present) with oracle/Makefile."""
    import subprocess
    subprocess.run(["make", "-C", str(HERE), "-j8", f"REF={reference_dir()}"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def lib():
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        L.orc_rhs.argtypes = [C.c_int, _dp, C.c_int, _dp]
        L.orc_center_diel.argtypes = [C.c_int, _dp, C.c_int]
        L.orc_center_diel.restype = C.c_double
        L.orc_fdm_solve.argtypes = [C.c_int, _dp, C.c_int, C.c_double, C.c_int, _dp,
                                    C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_fdm_solve_batch.argtypes = [C.c_int, C.c_int, _dp, C.c_void_p, C.c_double, _dp,
                                          C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        L.orc_structure_construction.argtypes = [C.c_int, C.c_int, _fp, _fp, C.c_int, _fp, _fp]
        L.orc_locate.argtypes = [C.c_int, C.c_int, _fp]
        L.orc_sample_index.argtypes = [C.c_int, _dp, C.c_int, C.c_double]
        L.orc_sample_index.restype = C.c_int
        L.orc_philox_uniform2_c.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, _dp]
        L.orc_transition.argtypes = [C.c_int, _dp, C.c_double, C.c_uint64, C.c_uint64, _fp,
                                     C.POINTER(C.c_int32)]
        L.orc_first_hop.argtypes = [C.c_int, _dp, C.c_int, C.c_double, C.c_uint64, C.c_uint64,
                                    C.c_double, _fp, C.POINTER(C.c_int32)]
        L.orc_frw_walks.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                    C.c_double, C.c_int, _ip, _ip, _dp, C.POINTER(C.c_double)]
        L.orc_distance.argtypes = [C.c_void_p, _dp, C.POINTER(C.c_int32)]
        L.orc_distance.restype = C.c_double
        L.orc_eps_at.argtypes = [C.c_void_p, _dp]
        L.orc_eps_at.restype = C.c_double
        _lib = L
    return _lib


def ref_available(N: int) -> bool:
    return (HERE / "_ref" / f"libggft_ref_N{N}.so").exists()


def ref_lib(N: int):
    if N not in _ref:
        path = HERE / "_ref" / f"libggft_ref_N{N}.so"
        if not path.exists():
            raise FileNotFoundError(f"reference ggft for N={N} not built ({path})")
        L = C.CDLL(str(path))
        L.ggft_ref_N.restype = C.c_int
        L.ggft_ref_solve_batch.argtypes = [C.c_int, _dp, C.c_int, C.c_double, _dp, C.c_void_p,
                                           C.c_int, C.POINTER(C.c_double)]
        L.ggft_ref_solve_one.argtypes = [C.c_int, _dp, C.c_int, C.c_double, _dp]
        assert L.ggft_ref_N() == N
        _ref[N] = L
    return _ref[N]


def ggft_ref(eps: np.ndarray, code: int = GFT, tol: float = 1e-12, nthreads: int = 1):
    """Reference ggft (compiled from the reference sources) on a batch of
    cubes ``eps[c, k, j, i]``. Returns (gft[c, 6N^2], ok[c], seconds)."""
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    n, N = eps.shape[0], eps.shape[-1]
    out = np.zeros((n, 6 * N * N))
    ok = np.zeros(n, dtype=np.int32)
    sec = C.c_double(0)
    ref_lib(N).ggft_ref_solve_batch(n, eps.reshape(-1), int(code), float(tol), out.reshape(-1),
                                    ok.ctypes.data, int(nthreads), C.byref(sec))
    return out, ok, sec.value


def fdm_solve(eps: np.ndarray, code: int = GFT, tol: float = 1e-13, maxit: int = 0):
    """FP64 Jacobi-PCG restatement, one cube. Returns (gft, rc, iters, relres)."""
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    N = eps.shape[-1]
    out = np.zeros(6 * N * N)
    it, rr = C.c_int(0), C.c_double(0)
    rc = lib().orc_fdm_solve(N, eps.reshape(-1), int(code), float(tol), int(maxit), out,
                             C.byref(it), C.byref(rr))
    return out, rc, it.value, rr.value


def fdm_solve_batch(eps: np.ndarray, code=GFT, tol: float = 1e-13, nthreads: int = 8):
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    n, N = eps.shape[0], eps.shape[-1]
    codes = np.ascontiguousarray(np.broadcast_to(np.asarray(code, dtype=np.int32), (n,)))
    out = np.zeros((n, 6 * N * N))
    ok = np.zeros(n, dtype=np.int32)
    sec = C.c_double(0)
    lib().orc_fdm_solve_batch(n, N, eps.reshape(-1), codes.ctypes.data, float(tol),
                              out.reshape(-1), ok.ctypes.data, int(nthreads), C.byref(sec))
    return out, ok, sec.value


def rhs(eps: np.ndarray, code: int) -> np.ndarray:
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    e = np.zeros(eps.size)
    lib().orc_rhs(eps.shape[-1], eps.reshape(-1), int(code), e)
    return e


def center_diel(eps: np.ndarray, code: int) -> float:
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    return lib().orc_center_diel(eps.shape[-1], eps.reshape(-1), int(code))


def structure_construction(layers: np.ndarray, cuboids: np.ndarray, N: int, normalise=True):
    layers = np.ascontiguousarray(layers, dtype=np.float32).reshape(-1, 30)
    cuboids = np.ascontiguousarray(cuboids, dtype=np.float32).reshape(-1, 105)
    n = layers.shape[0]
    eps = np.zeros((n, N, N, N), dtype=np.float32)
    mx = np.zeros(n, dtype=np.float32)
    lib().orc_structure_construction(n, N, layers.reshape(-1), cuboids.reshape(-1),
                                     1 if normalise else 0, eps.reshape(-1), mx)
    return eps, mx


def locate(N: int, panel: int) -> np.ndarray:
    out = np.zeros(3, dtype=np.float32)
    lib().orc_locate(N, int(panel), out)
    return out


def sample_index(w: np.ndarray, u: float, use_abs: bool = False) -> int:
    w = np.ascontiguousarray(w, dtype=np.float64)
    return lib().orc_sample_index(w.size, w, 1 if use_abs else 0, float(u))


def philox_uniform2(seed: int, stream: int, c2: int, c3: int):
    u = np.zeros(2)
    lib().orc_philox_uniform2_c(seed, stream, c2, c3, u)
    return u


def transition(eps: np.ndarray, seed: int, stream: int, tol: float = 1e-13):
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    out = np.zeros(3, dtype=np.float32)
    panel = C.c_int32(0)
    lib().orc_transition(eps.shape[-1], eps.reshape(-1), tol, seed, stream, out,
                         C.byref(panel))
    return out, panel.value


def first_hop(eps: np.ndarray, axis: int, seed: int, stream: int, eps_scale: float = 1.0,
              tol: float = 1e-13):
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    out = np.zeros(5, dtype=np.float32)
    panel = C.c_int32(0)
    lib().orc_first_hop(eps.shape[-1], eps.reshape(-1), int(axis), tol, seed, stream,
                        float(eps_scale), out, C.byref(panel))
    return out, panel.value


def frw_walks(structure, params, walk0: int, nwalks: int, fdm: str = "oracle",
              fdm_tol: float = 1e-10, nthreads: int = 8):
    """Run walks [walk0, walk0+nwalks) on the CPU. ``structure``/``params``
    are the ctypes mirrors from deeprwcap_b200.abi (drwc_structure,
    drwc_job_params). fdm = "oracle" (FP64 PCG restatement) or "ggft" (the
    reference solver for params.N). Returns (end, hops, weight, seconds)."""
    end = np.zeros(nwalks, dtype=np.int32)
    hops = np.zeros(nwalks, dtype=np.int32)
    w = np.zeros(nwalks)
    sec = C.c_double(0)
    fn = None
    if fdm == "ggft":
        fn = C.cast(ref_lib(int(params.N)).ggft_ref_solve_one, C.c_void_p).value
    lib().orc_frw_walks(C.addressof(structure), C.addressof(params), int(walk0), int(nwalks), fn,
                        float(fdm_tol), int(nthreads), end, hops, w, C.byref(sec))
    return end, hops, w, sec.value
