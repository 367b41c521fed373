"""The multi-job server (drwc_server_*): continuous batching of extraction jobs
on one device.

Checks: (1) a job served alone gives exactly drwc_frw_run's result (same
walks, same fixed-order batch sums, same compensated accumulation); (2) jobs
of different structures and cube resolutions submitted one after another,
with an arena that holds only two at a time, overlap on the device, wait for
memory when it is full, and each still gives exactly its stand-alone result;
(3) with the learned network, each job's result in the mix equals its result
served alone; (4) requests the server cannot take fail cleanly."""
import time

import numpy as np
import pytest

from deeprwcap_b200 import abi, engine, train
from deeprwcap_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _params(N, seed, walks, batch):
    return W.job_params_plain(N=N, seed=seed, min_walks=walks, max_walks=walks,
                              batch_walks=batch)


def _same(a, b):
    assert (a.walks, a.hops, a.lost, a.converged) == (b.walks, b.hops, b.lost, b.converged)
    np.testing.assert_array_equal(a.cap, b.cap)
    np.testing.assert_array_equal(a.stderr, b.stderr)


def _jobs():
    return [
        (W.two_layer_crossing(), _params(16, 11, 40000, 8192)),
        (W.wire_stack(3, 6, diel_eps=[3.0, 4.0, 2.5, 3.6, 4.4], n_diel_blocks=6, seed=2),
         _params(21, 12, 30000, 8192)),
        (W.wire_stack(2, 8, seed=3), _params(23, 13, 26000, 8192)),
        (W.wire_stack(4, 4, diel_eps=[3.9, 2.7, 4.2], seed=4), _params(16, 14, 35000, 8192)),
        (W.dense_stack(seed=5), _params(21, 15, 27000, 8192)),
    ]


def test_served_job_equals_frw_run(ctx):
    s = W.two_layer_crossing()
    p = _params(16, 7, 3 * 16384 + 1000, 16384)
    ref = engine.extract(s, p, ctx)
    with engine.Server(ctx, slots=8192, hbm_budget=64 << 20) as srv:
        r = srv.wait(srv.submit(s, p), timeout=300)
        st = srv.stats()
    _same(r, ref)
    assert st["completed"] == 1 and st["fdm_hops"] >= r.hops


@pytest.mark.parametrize("fdm_hops,straggler_hops", [(1, 0), (64, 2), (5, 1)])
def test_continuing_walks_give_the_same_rows(ctx, fdm_hops, straggler_hops):
    """Walks that take several hops per step inside the FDM bucket (every
    walk past its first hops, or past its second; at most 5 or 64 per step;
    or none with fdm_hops = 1) give exactly drwc_frw_run's rows, alone and
    beside a second job: a hop's draws depend only on (walk, hop)."""
    jobs = [(W.two_layer_crossing(), _params(16, 21, 2 * 16384 + 777, 16384)),
            (W.wire_stack(3, 5, diel_eps=[3.0, 4.0, 2.5], n_diel_blocks=4, seed=6),
             _params(21, 22, 20000, 8192))]
    alone = [engine.extract(s, p, ctx) for s, p in jobs]
    with engine.Server(ctx, slots=4096, fdm_hops=fdm_hops, straggler_hops=straggler_hops) as srv:
        ids = [srv.submit(s, p) for s, p in jobs]
        res = [srv.wait(i, timeout=600) for i in ids]
    for r, a in zip(res, alone):
        _same(r, a)


def test_mix_equals_alone_with_admission_by_footprint(ctx):
    jobs = _jobs()
    alone = [engine.extract(s, p, ctx) for s, p in jobs]
    # each job needs its structure + 16 B of records per walk of the batches it
    # can hold at once (4-5 batches of 8192 here): two fit, three do not
    budget = 1400 * 1024
    with engine.Server(ctx, slots=16384, max_jobs=8, hbm_budget=budget) as srv:
        ids = []
        for s, p in jobs:
            ids.append(srv.submit(s, p))
            time.sleep(0.005)
        res = [srv.wait(i, timeout=600) for i in ids]
        st = srv.stats()
        queued = [srv.times(i)[0] for i in ids]
    for r, a in zip(res, alone):
        _same(r, a)
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert st["max_running"] == 2           # the arena held two jobs at a time
    assert st["arena_peak"] <= budget
    assert max(queued) > 0.0                # later jobs waited for memory
    assert st["walks_dropped"] >= 0 and st["hops"] >= sum(r.hops for r in res)


@pytest.fixture(scope="module")
def small_net(ctx):
    X, T, TG = train.build_dataset(ctx, 1 << 16, seed=8, log=lambda *a: None)
    net = engine.Net(seed=3, ctx=ctx)
    train.train(net, X, T, TG, epochs=2, batch=512, lr=1e-3, log=lambda *a: None)
    return net


def test_learned_mix_equals_alone(ctx, small_net):
    """Networks for N = 16 and 21 (the 21 one untrained: the equality does not
    depend on the weights) and an N = 23 job on the FDM path, alone and mixed."""
    net21 = engine.Net(seed=11, ctx=ctx, N=21)
    nets = [small_net, net21]
    jobs = [
        (W.two_layer_crossing(), _params(16, 21, 20000, 8192)),
        (W.wire_stack(3, 5, seed=6), _params(16, 22, 15000, 8192)),
        (W.wire_stack(2, 6, seed=7), _params(21, 23, 10000, 8192)),
        (W.wire_stack(2, 4, seed=8), _params(23, 24, 8000, 8192)),
    ]
    opts = dict(slots=8192, audit_frac=0.05, conf_threshold=-1.0)
    alone = []
    for s, p in jobs:
        with engine.Server(ctx, net=nets, **opts) as srv:
            alone.append(srv.wait(srv.submit(s, p), timeout=600))
    with engine.Server(ctx, net=nets, **opts) as srv:
        ids = [srv.submit(s, p) for s, p in jobs]
        res = [srv.wait(i, timeout=600) for i in ids]
        st = srv.stats()
    for r, a in zip(res, alone):
        _same(r, a)
    assert st["net_hops"] > 0 and st["audits"] > 0 and st["fdm_hops"] > 0
    assert st["audit_kl_mean"] > 0.0
    # the untrained N = 21 network cannot be in the same place as a trained one,
    # but its walks finish and are counted
    assert res[2].walks == 10000


def test_rejected_requests(ctx):
    s = W.two_layer_crossing()
    with engine.Server(ctx, slots=1024, hbm_budget=1 << 20, sizes=(16,)) as srv:
        with pytest.raises(abi.DrwcError):
            srv.submit(s, _params(21, 1, 1000, 1000))         # N not served
        jid = srv.submit(s, _params(16, 1, 1 << 20, 1 << 20))  # records exceed the arena
        with pytest.raises(abi.DrwcError) as e:
            srv.wait(jid, timeout=60)
        assert e.value.status == 3                              # DRWC_ERR_NOMEM
        ok = srv.wait(srv.submit(s, _params(16, 2, 2000, 1000)), timeout=120)
        assert ok.walks == 2000


def test_uniform_table_hops_follow_the_fdm_walk(ctx):
    """Cubes of a single permittivity take their hop from the precomputed
    uniform-permittivity Green's function. Their surface values equal the FDM
    solution (it does not depend on the permittivity), and the hop uses the
    same Philox draws, so the walks follow the FDM walks: the capacitance row
    agrees far inside the statistical error."""
    s = W.two_layer_crossing()
    p = _params(16, 17, 1 << 16, 1 << 14)
    ref = engine.extract(s, p, ctx)
    with engine.Server(ctx, slots=8192, uniform_table=1) as srv:
        r = srv.wait(srv.submit(s, p), timeout=300)
        st = srv.stats()
    assert st["table_hops"] > 0.2 * r.hops, st
    assert st["fdm_hops"] + st["table_hops"] == st["hops"]
    assert r.walks == ref.walks and abs(r.hops - ref.hops) <= 1e-4 * ref.hops
    np.testing.assert_allclose(r.cap, ref.cap, rtol=1e-6, atol=1e-9 * abs(ref.cap[0]))


def test_learned_server_agrees_with_learned_walker(ctx, small_net):
    """The server runs conv1 and conv2 on the tensor cores inside its
    voxeliser; the learned walker voxelises to global memory first. Same BF16
    operands, same walks, same network: the capacitance rows agree well
    inside the statistical error."""
    s = W.two_layer_crossing()
    nw = 40000
    p = _params(16, 31, nw, 8192)
    o = engine.learned_opts(slots=8192, conf_threshold=1e9, audit_frac=0.0)
    e1, h1, w1, st1 = engine.frw_walks_learned(s, p, small_net, 0, nw, o)
    c1 = np.array([w1[e1 == j].sum() / nw for j in range(s.n_nets + 1)])
    with engine.Server(ctx, net=small_net, slots=8192, conf_threshold=1e9, audit_frac=0.0) as srv:
        r = srv.wait(srv.submit(s, p), timeout=600)
        st = srv.stats()
    assert st["net_hops"] == st["hops"] and r.walks == nw
    assert abs(r.hops - int(h1.sum())) <= 0.01 * h1.sum()
    assert np.all(np.abs(r.cap - c1) <= 1.0 * r.stderr + 1e-12), (r.cap, c1, r.stderr)


@pytest.mark.parametrize("N", [21, 23])
def test_learned_server_at_larger_resolutions(ctx, N):
    """A network trained here at N = 21 / 23 (2^16 engine-generated samples,
    3 epochs) drives the hops of a job at that resolution: the walks finish,
    nearly every hop goes through the network, and the self-capacitance
    lands near the FDM walk's. The bar is loose: a network trained this
    briefly lands anywhere within a few percent (training order is not
    deterministic; repeated trainings here have landed 3 % below to 10 %
    above); the benchmark measures the accuracy of the full-size training
    walk by walk."""
    X, T, TG = train.build_dataset(ctx, 1 << 16, seed=3, log=lambda *a: None, N=N)
    net = engine.Net(seed=4, ctx=ctx, N=N)
    train.train(net, X, T, TG, epochs=3, batch=512, lr=1e-3, log=lambda *a: None)
    s = W.two_layer_crossing()
    p = _params(N, 51, 60000, 16384)
    ref = engine.extract(s, p, ctx)
    with engine.Server(ctx, net=net, slots=16384, audit_frac=0.01, conf_threshold=1e9) as srv:
        r = srv.wait(srv.submit(s, p), timeout=900)
        st = srv.stats()
    assert r.walks == 60000 and st["net_hops"] >= 0.95 * st["hops"]
    assert abs(r.cap[0] - ref.cap[0]) <= 0.15 * abs(ref.cap[0]), (r.cap[0], ref.cap[0])

