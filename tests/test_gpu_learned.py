"""The learned transition path: a network trained here on engine-generated
FDM data drives the walk; low-confidence hops and audits take the FDM solve.

Checks: (1) with every hop routed to the FDM solve (confidence threshold
below anything the network predicts) the learned walker reproduces the FDM
walker's records walk for walk (same Philox draws, same solve); (2) a trained
network's capacitance row matches the FDM walk on the same walks within 1%
(self) and 2% (significant couplings), with the network taking >= 95% of the
hops and a small audited KL; (3) it reports its gain in hops/s over the FDM
walk on the same walks."""
import numpy as np
import pytest

from deeprwcap_b200 import engine, train
from deeprwcap_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained(ctx):
    X, T, TG = train.build_dataset(ctx, 1 << 19, seed=5, log=lambda *a: None)
    Xt, Tt, TGt, Xv, Tv, TGv = train.split(X, T, TG, seed=5)
    net = engine.Net(seed=9, ctx=ctx)
    train.train(net, Xt, Tt, TGt, epochs=6, batch=512, lr=1e-3, log=lambda *a: None)
    ev = train.evaluate(net, Xv, Tv, TGv)
    return net, ev


def _cap(e, w, n_entries):
    n = len(w)
    return np.array([w[e == j].sum() / n for j in range(n_entries)])


def test_all_hops_routed_to_fdm_reproduce_fdm_walk(ctx):
    s = W.two_layer_crossing()
    p = W.job_params_plain(N=16, seed=41, tol=1e-8)
    net = engine.Net(seed=1, ctx=ctx)
    o = engine.learned_opts(slots=4096, conf_threshold=-1e9, audit_frac=0.0)
    e1, h1, w1, st = engine.frw_walks_learned(s, p, net, 0, 3000, o)
    e0, h0, w0 = engine.frw_walks(s, p, 0, 3000, ctx=ctx)
    assert st["net_hops"] == 0 and st["fallbacks"] == st["fdm_hops"] == h1.sum()
    same = (e1 == e0) & (h1 == h0)
    assert same.mean() >= 0.99
    assert np.allclose(w1[same], w0[same], rtol=1e-9, atol=0)


def test_trained_network_matches_fdm_walk(ctx, trained):
    net, ev = trained
    assert ev["kl_mean"] < 0.02, ev
    for s in (W.two_layer_crossing(), W.dense_stack(seed=3)):
        p = W.job_params_plain(N=16, seed=77, tol=1e-8)
        nw = 300000
        o = engine.learned_opts(slots=65536, conf_threshold=-1.5, audit_frac=0.01)
        e1, h1, w1, st = engine.frw_walks_learned(s, p, net, 0, nw, o)
        e0, h0, w0 = engine.frw_walks(s, p, 0, nw, ctx=ctx)
        c1, c0 = _cap(e1, w1, s.n_nets + 1), _cap(e0, w0, s.n_nets + 1)

        def paired_sem(j):  # standard error of the walk-by-walk difference
            d = np.where(e1 == j, w1, 0.0) - np.where(e0 == j, w0, 0.0)
            return d.std() / np.sqrt(len(d))
        assert abs(c1[0] - c0[0]) <= 0.01 * abs(c0[0]) + 3 * paired_sem(0), (c1[0], c0[0])
        cpl = np.argsort(-np.abs(c0[1:]))[:3] + 1  # the significant couplings
        for j in cpl:
            assert abs(c1[j] - c0[j]) <= 0.02 * abs(c0[j]) + 3 * paired_sem(j), (j, c1[j], c0[j])
        assert st["net_hops"] >= 0.90 * (st["net_hops"] + st["fdm_hops"])
        assert st["audit_kl"] < 0.01
        assert st["audits"] > 0


def test_learned_gain_over_fdm(ctx, trained):
    import time
    net, _ = trained
    s = W.dense_stack(seed=3)
    p = W.job_params_plain(N=16, seed=99, tol=1e-8)
    nw = 400000
    o = engine.learned_opts(slots=65536, conf_threshold=-1.5, audit_frac=0.01)
    engine.frw_walks_learned(s, p, net, 10_000_000, 20000, o)  # warm-up
    e1, h1, w1, st = engine.frw_walks_learned(s, p, net, 0, nw, o)
    t0 = time.perf_counter()
    e0, h0, w0 = engine.frw_walks(s, p, 0, nw, ctx=ctx)
    t_fdm = time.perf_counter() - t0
    gain = (h1.sum() / st["seconds"]) / (h0.sum() / t_fdm)
    print(f"learned {h1.sum() / st['seconds']:.3e} hops/s, FDM {h0.sum() / t_fdm:.3e} hops/s, "
          f"gain {gain:.2f}x")
    assert gain > 1.0


def _eps_cpu(s, pts):
    """The fill rule at points [n, 3]: first containing dielectric block, else
    the last layer with zlo <= z (layer 0 below all)."""
    eps = s.layer_eps[np.clip(np.searchsorted(s.layer_zlo, pts[:, 2], side="right") - 1, 0, None)]
    done = np.zeros(len(pts), dtype=bool)
    for d in s.diel:
        inside = np.all((pts >= d[:3]) & (pts <= d[3:6]), axis=1) & ~done
        eps = np.where(inside, d[6], eps)
        done |= inside
    return eps


@pytest.mark.parametrize("N", [16, 23])
def test_separable_voxelisation_matches_fill_rule(ctx, N):
    """Network inputs of logged walk cubes (dense stack: 5 layers, 10 blocks;
    first-hop cubes in their rotated frames) equal the fill rule evaluated at
    every cell centre, bit for bit, at N = 16 and 23."""
    import torch
    s = W.dense_stack(seed=3)
    p = W.job_params_plain(N=16, seed=77)
    rec, code = engine.harvest(s, p, 0, 256, 6000, ctx=ctx)
    n = int(rec.shape[0])
    dev = rec.device
    X = torch.empty(n, N ** 3, dtype=torch.bfloat16, device=dev)
    eps = torch.empty(n, N ** 3, dtype=torch.float64, device=dev)
    engine.records_voxelise(s, rec, code, X, eps, ctx=ctx, N=N)
    torch.cuda.synchronize()
    rec, code, eps = rec.cpu().numpy(), code.cpu().numpy(), eps.cpu().numpy()
    t = np.array([(2.0 * i + 1.0) / N - 1.0 for i in range(N)])
    k, j, i = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    blocks_hit = 0
    for r in range(n):
        c, a = rec[r, :3], rec[r, 3]
        rot = {2: 1, 3: 2}.get(int(code[r]), 0)  # WVTX -> x is z', WVTY -> y is z'
        ox, oy, oz = (k, i, j) if rot == 1 else (j, k, i) if rot == 2 else (i, j, k)
        pts = np.stack([c[0] + a * t[ox], c[1] + a * t[oy], c[2] + a * t[oz]], axis=1)
        ref = _eps_cpu(s, pts)
        assert np.array_equal(eps[r], ref), r
        blocks_hit += int(np.any(~np.isin(ref, s.layer_eps)))
    assert n > 1000 and blocks_hit > 0
