"""GPU parity of the device walker against the restated CPU walker (same
Philox streams, FP64 FDM per hop): per-walk records must match, and the
capacitance estimate behaves as the estimator should."""
import numpy as np
import pytest

from deeprwcap_b200 import engine
from deeprwcap_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _params(N, **kw):
    p = W.job_params_plain(N=N, seed=21, **kw)
    return p


@pytest.mark.parametrize("N", (6, 8, 16))
def test_walk_records_match_cpu(ctx, oracle, N):
    s = W.two_layer_crossing()
    sc = s.to_c()
    p = _params(N)
    nw = 48 if N == 16 else 160
    e, h, w = engine.frw_walks(s, p, 0, nw, ctx=ctx)
    e0, h0, w0, _ = oracle.frw_walks(sc, p, 0, nw, fdm_tol=1e-13, nthreads=8)
    same = (e == e0) & (h == h0)
    assert same.mean() >= 0.97, (same.mean(), np.nonzero(~same))
    assert np.allclose(w[same], w0[same], rtol=1e-7, atol=0)


def test_walk_records_dense_structure_grid(ctx, oracle):
    """24 conductors + dielectric blocks: the uniform-grid nearest-conductor
    search and the block permittivity lookup."""
    s = W.dense_stack(seed=2)
    p = _params(6)
    e, h, w = engine.frw_walks(s, p, 0, 96, ctx=ctx)
    e0, h0, w0, _ = oracle.frw_walks(s.to_c(), p, 0, 96, fdm_tol=1e-13, nthreads=8)
    same = (e == e0) & (h == h0)
    assert same.mean() >= 0.97
    assert np.allclose(w[same], w0[same], rtol=1e-7)


def test_batch_independence(ctx):
    s = W.two_layer_crossing()
    p = _params(8)
    e1, h1, w1 = engine.frw_walks(s, p, 0, 300, ctx=ctx)
    e2, h2, w2 = engine.frw_walks(s, p, 100, 200, ctx=ctx)
    assert np.array_equal(e1[100:], e2) and np.array_equal(h1[100:], h2)
    assert np.array_equal(w1[100:], w2)


def test_extract_capacitance_row(ctx):
    s = W.two_layer_crossing()
    p = _params(8, min_walks=20000, max_walks=20000, batch_walks=10000)
    r = engine.extract(s, p, ctx=ctx)
    assert r.walks == 20000 and r.lost == 0
    assert r.cap[0] > 0 and r.cap[1] < 0 and r.cap[8] < 0
    # charge neutrality of the full row (ground included)
    assert abs(r.cap.sum()) < 4 * np.sqrt((r.stderr ** 2).sum())
    # deterministic: same job, same numbers
    r2 = engine.extract(s, p, ctx=ctx)
    assert np.array_equal(r.cap, r2.cap)
