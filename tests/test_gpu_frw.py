"""GPU parity of the device walker against the restated CPU walker (same
Philox streams, FP64 FDM per hop): per-walk records must match, and the
capacitance estimate behaves as the estimator should."""
import os

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
    nw = 1024 if N == 16 else 2048
    e, h, w = engine.frw_walks(s, p, 0, nw, ctx=ctx)
    e0, h0, w0, _ = oracle.frw_walks(sc, p, 0, nw, fdm_tol=1e-13,
                                     nthreads=os.cpu_count() or 8)
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


def test_converged_row_matches_fp64_oracle_walk(ctx, oracle):
    """A converged row at N = 6 against the FP64-FDM CPU walker on independent
    walks (other walk ids): every significant entry within 3 combined sigma."""
    s = W.two_layer_crossing()
    p = _params(6, min_walks=1 << 17, max_walks=1 << 17, batch_walks=1 << 16)
    r = engine.extract(s, p, ctx=ctx)
    nw = 30000
    e0, h0, w0, _ = oracle.frw_walks(s.to_c(), p, 5_000_000, nw, fdm_tol=1e-13,
                                     nthreads=os.cpu_count() or 8)
    assert (e0 >= 0).all()
    for ent in range(s.n_nets + 1):
        x = np.where(e0 == ent, w0, 0.0)
        c0, se0 = x.mean(), x.std() / np.sqrt(nw)
        if abs(c0) < 3 * se0:
            continue  # not resolved by the CPU sample
        z = abs(r.cap[ent] - c0) / np.hypot(r.stderr[ent], se0)
        assert z < 3.0, (ent, r.cap[ent], c0, r.stderr[ent], se0)


def test_unconverged_solves_escalate(ctx):
    """A per-sweep budget far too small for the cube solves: the escalation
    sweeps finish them, and the walks match those of the default budget."""
    s = W.two_layer_crossing()
    nw = 512
    e0, h0, w0, st0 = engine.frw_walks(s, _params(16), 0, nw, ctx=ctx, stats=True)
    p = _params(16, max_outer=1, max_inner=8, extra_outer=16)
    e1, h1, w1, st1 = engine.frw_walks(s, p, 0, nw, ctx=ctx, stats=True)
    assert st0[4] == 0 and st0[5] == 0
    assert st1[4] > 0 and st1[5] == 0, st1
    same = (e0 == e1) & (h0 == h1)
    assert same.mean() >= 0.97
    assert np.allclose(w0[same], w1[same], rtol=1e-6)


def test_failed_solves_end_walks_lost(ctx):
    """With escalation off and a budget the solves cannot meet, hops whose
    cube stays unconverged end their walk as lost and are counted; nothing
    is sampled from an unconverged Green's function."""
    s = W.two_layer_crossing()
    p = _params(16, max_outer=1, max_inner=4, extra_outer=0)
    e, h, w, st = engine.frw_walks(s, p, 0, 256, ctx=ctx, stats=True)
    assert st[5] > 0
    assert (e == -1).sum() == st[5]  # each failed solve ended exactly one walk
    pj = _params(16, max_outer=1, max_inner=4, extra_outer=0, min_walks=4096, max_walks=4096,
                 batch_walks=4096)
    r = engine.extract(s, pj, ctx=ctx)
    assert r.solves_failed > 0 and r.lost >= r.solves_failed


def test_union_gauss_surface_of_one_box_is_the_box(ctx):
    """gauss_surface = 1 (the outer boundary of the master's grown boxes)
    for a master of one box is the Gauss box itself, face by face with the
    same areas: the walks are identical."""
    s = W.two_layer_crossing()
    # an offset below half the master's clearance (0.05 um), so the per-box
    # offset of gauss_surface = 1 is gauss_offset itself
    e0, h0, w0 = engine.frw_walks(s, _params(8, gauss_offset=0.04), 0, 2000, ctx=ctx)
    e1, h1, w1 = engine.frw_walks(s, _params(8, gauss_offset=0.04, gauss_surface=1), 0, 2000,
                                  ctx=ctx)
    assert np.array_equal(e0, e1) and np.array_equal(h0, h1) and np.array_equal(w0, w1)
