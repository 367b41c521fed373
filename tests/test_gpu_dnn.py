"""GPU parity of the dnnsolver drop-ins (structure construction, transition
and first-hop sampling) against the CPU oracle on the same seeded inputs.

Voxelisation is compared bit for bit; sampled panels must be the same
panel; first-hop weights within 1e-6 relative."""
import numpy as np
import pytest

from deeprwcap_b200 import abi, engine
from deeprwcap_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", (8, 16, 23))
def test_structure_construction_bitexact(ctx, oracle, N):
    L, Cb = W.query_batch(40, seed=N)
    s = engine.DNNSolverPoisson(0, N=N)
    for norm in (True, False):
        eps, mx = s.structureConstruction(L, Cb, normalise=norm)
        ref, rmx = oracle.structure_construction(L, Cb, N, normalise=norm)
        assert np.array_equal(mx, rmx)
        assert np.array_equal(eps, ref)


@pytest.mark.parametrize("N", (8, 16, 23))
def test_transition_matches_oracle(ctx, oracle, N):
    n = 24
    L, Cb = W.query_batch(n, seed=100 + N)
    s = engine.DNNSolverPoisson(0, N=N, seed=1234)
    out = np.array(s.sample(L, Cb)).reshape(n, 3)
    eps, _ = oracle.structure_construction(L, Cb, N, normalise=True)
    for q in range(n):
        ref, panel = oracle.transition(eps[q].astype(np.float64), 1234, q)
        assert np.array_equal(out[q], ref), (q, out[q], ref)
        assert np.max(np.abs(out[q])) == 1.0   # on the cube surface


@pytest.mark.parametrize("N", (8, 16, 23))
def test_first_hop_matches_oracle(ctx, oracle, N):
    n = 24
    L, Cb = W.query_batch(n, seed=200 + N)
    axis = (np.arange(n) % 3).astype(np.int32)
    s = engine.DNNSolverGrad(0, N=N, seed=99)
    out = np.array(s.sample(L, Cb, axis)).reshape(n, 5)
    eps, mx = oracle.structure_construction(L, Cb, N, normalise=True)
    for q in range(n):
        ref, panel = oracle.first_hop(eps[q].astype(np.float64), int(axis[q]), 99, q,
                                      eps_scale=float(mx[q]))
        assert np.array_equal(out[q, :3], ref[:3]), (q, out[q], ref)
        assert abs(out[q, 3] - ref[3]) <= 1e-6 * abs(ref[3])
        assert abs(out[q, 4] - ref[4]) <= 1e-6 * abs(ref[4])


def test_grad_requires_axis(ctx):
    L, Cb = W.query_batch(2, seed=1)
    s = engine.DNNSolverGrad(0, N=8)
    with pytest.raises(RuntimeError):
        s.sample(L, Cb)
    rc = ctx.lib.drwc_first_hop_batch(ctx.h, 2, 8, L.ctypes.data, Cb.ctypes.data, None, 1, 0,
                                      np.zeros(10, dtype=np.float32).ctypes.data)
    assert rc == 1


def test_transition_distribution_chi2(ctx, oracle):
    """Repeated draws on one cube follow the FDM Green's function."""
    N, n = 6, 6000
    L, Cb = W.query_batch(1, seed=77)
    Lr, Cr = np.repeat(L, n, axis=0), np.repeat(Cb, n, axis=0)
    s = engine.DNNSolverPoisson(0, N=N, seed=5)
    pts = np.array(s.sample(Lr, Cr)).reshape(n, 3)
    eps, _ = oracle.structure_construction(L, Cb, N, normalise=True)
    g, *_ = oracle.fdm_solve(eps[0].astype(np.float64), 0, tol=1e-13)
    # map points back to faces and compare face frequencies
    face = np.where(pts[:, 2] == -1, 0, np.where(pts[:, 2] == 1, 1, np.where(
        pts[:, 1] == -1, 2, np.where(pts[:, 1] == 1, 3, np.where(pts[:, 0] == -1, 4, 5)))))
    obs = np.bincount(face, minlength=6)
    exp = g.reshape(6, -1).sum(1) * n
    chi2 = ((obs - exp) ** 2 / exp).sum()
    assert chi2 < 25.0, (obs, exp, chi2)  # 5 dof, p ~ 1e-4


def test_parallel_sampler_batches_and_forwards_errors(ctx):
    L, Cb = W.query_batch(64, seed=9)
    s = engine.DNNSolverPoisson(0, N=8)
    ps = engine.ParallelSampler(s, 3, 16)
    futs = [ps.submit(L[q], Cb[q]) for q in range(64)]
    res = [f.result(timeout=60) for f in futs]
    assert all(len(r) == 3 for r in res)
    g = engine.DNNSolverGrad(0, N=8)
    pg = engine.ParallelSampler(g, 5, 8)
    f = pg.submit(L[0], Cb[0], 5)  # invalid axis -> error reaches the future
    with pytest.raises(Exception):
        f.result(timeout=60)
    ps.close(); pg.close()
