"""GPU parity of the FDM surface Green's function (the ggft replacement)
against the reference ggft golden vectors and the FP64 oracle.

Tolerance: 1e-6 relative (normwise per cube, and elementwise relative to the
cube's largest value), the parity bar for the FDM kernel."""
import numpy as np
import pytest

from conftest import golden
from deeprwcap_b200 import abi, engine
from deeprwcap_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-6


def rel_err(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b), np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("N", (5, 8, 16, 21, 23))
def test_golden_ggft(ctx, N):
    g = golden(N)
    eps, ref, codes = g["eps"], g["gft"], g["codes"]
    for ci, code in enumerate(codes):
        out, iters, relres, status = engine.fdm_solve_batch(list(eps), code=int(code), ctx=ctx)
        assert (status == 0).all()
        assert (relres <= 1e-10).all()
        for c in range(len(eps)):
            nw, el = rel_err(out[c], ref[ci, c])
            assert nw < TOL and el < TOL, (N, code, c, nw, el)


def test_ggft_solver_dropin(ctx):
    """GgftSolver mirrors ggft_solver: DIEL in, solve(code) -> bool, gft out."""
    g = golden(16)
    s = engine.GgftSolver(16, ctx)
    s.set_tolerance(1e-10)
    for c in range(3):
        s.DIEL = g["eps"][c].reshape(-1)
        for ci, code in enumerate(g["codes"]):
            assert s.solve(int(code)) is True
            nw, el = rel_err(s.gft, g["gft"][ci, c])
            assert nw < TOL and el < TOL


def test_invariants_and_oracle_mixed_batch(ctx, oracle):
    b = W.mixed_fdm_batch(96, seed=7)
    codes = np.arange(96, dtype=np.int32) % 4
    out, iters, relres, status = engine.fdm_solve_batch(b, code=codes, ctx=ctx)
    assert (status == 0).all()
    for c in range(b.ncubes):
        e = b.cube(c)
        ref, rc, _, _ = oracle.fdm_solve(e, int(codes[c]), tol=1e-13)
        nw, el = rel_err(out[c], ref)
        assert nw < TOL and el < TOL, (c, int(b.N[c]), int(codes[c]), nw, el)
        if codes[c] == 0:
            assert abs(out[c].sum() - 1) < 1e-8
            assert out[c].min() > -1e-12


@pytest.mark.parametrize("N", tuple(range(4, 24)))
def test_every_resolution(ctx, oracle, N):
    eps, _ = W.fdm_cubes(2, N, seed=300 + N, noise_frac=0.5)
    for code in (0, 1 + N % 3):
        out, _, relres, status = engine.fdm_solve_batch(list(eps), code=code, ctx=ctx)
        assert (status == 0).all()
        for c in range(2):
            ref, *_ = oracle.fdm_solve(eps[c], code, tol=1e-13)
            nw, el = rel_err(out[c], ref)
            assert nw < TOL and el < TOL, (N, code, nw, el)


def test_high_contrast_and_noise(ctx, oracle):
    rng = np.random.default_rng(3)
    N = 16
    cubes = [np.exp(rng.uniform(np.log(1), np.log(12), (N, N, N))) for _ in range(3)]
    cubes.append(np.where(rng.uniform(size=(N, N, N)) < 0.5, 1.0, 80.0))
    out, _, relres, status = engine.fdm_solve_batch(cubes, ctx=ctx)
    assert (status == 0).all()
    for c, e in enumerate(cubes):
        ref, *_ = oracle.fdm_solve(e, 0, tol=1e-13)
        nw, el = rel_err(out[c], ref)
        assert nw < TOL and el < TOL


def test_scale_invariance(ctx):
    eps, _ = W.fdm_cubes(1, 12, seed=1)
    a, *_ = engine.fdm_solve_batch([eps[0]], ctx=ctx)
    b, *_ = engine.fdm_solve_batch([eps[0] * 1e-11], ctx=ctx)
    assert np.max(np.abs(a[0] - b[0])) < 1e-9


def test_invalid_permittivity_status(ctx):
    N = 8
    good, _ = W.fdm_cubes(2, N, seed=2)
    bad = good[1].copy()
    bad[3, 3, 3] = -1.0
    nan = good[1].copy()
    nan[0, 0, 0] = np.nan
    out, iters, relres, status = engine.fdm_solve_batch([good[0], bad, nan], ctx=ctx)
    assert list(status) == [0, 2, 2]
    assert np.all(out[1] == 0) and np.all(out[2] == 0)
    s = engine.GgftSolver(N, ctx)
    s.DIEL = bad.reshape(-1)
    assert s.solve(0) is False


def test_empty_and_invalid_arguments(ctx):
    import ctypes as C
    L = ctx.lib
    assert L.drwc_fdm_solve_batch(ctx.h, 0, None, None, None, None, None, None, None, None,
                                  None, None) == 0
    eps = np.ones(27 ** 3)
    out = np.zeros(6 * 27 * 27)
    assert L.drwc_ggft_solve(ctx.h, 27, eps.ctypes.data, 0, 1e-8, out.ctypes.data, None) == 1
    assert L.drwc_ggft_solve(ctx.h, 8, eps.ctypes.data, 7, 1e-8, out.ctypes.data, None) == 1


def test_not_converged_is_reported(ctx):
    eps, _ = W.fdm_cubes(1, 16, seed=4)
    out, iters, relres, status = engine.fdm_solve_batch([eps[0]], ctx=ctx, max_outer=1,
                                                        max_inner=3)
    assert status[0] == 1 and relres[0] > 1e-10
