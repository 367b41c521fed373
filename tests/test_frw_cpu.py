"""CPU checks of the restated walker (the device walker's checker) and of the
structure generators."""
import numpy as np
import pytest

from deeprwcap_b200 import workloads as W


def _params(N=6, **kw):
    return W.job_params_plain(N=N, seed=11, **kw)


def test_structure_generators():
    s = W.two_layer_crossing()
    assert len(s.boxes) == 8 and s.n_nets == 8
    assert np.allclose(s.layer_eps, [3.9, 2.7, 4.2])
    assert np.allclose(s.layer_zlo[1:], [0.05, 0.35])
    assert np.allclose(s.encl_lo, [-1, -1, -1]) and np.allclose(s.encl_hi, [3, 3, 1.4])
    d = W.dense_stack(seed=3)
    assert len(d.boxes) == 24 and len(d.diel) == 10 and len(d.layer_eps) == 5
    for b in d.diel:  # blocks keep clear of conductors
        for c in d.boxes:
            assert not (np.all(b[:3] < c[3:]) and np.all(b[3:6] > c[:3]))


def test_cpu_walks_deterministic_and_batch_independent(oracle):
    s = W.two_layer_crossing().to_c()
    p = _params()
    e1, h1, w1, _ = oracle.frw_walks(s, p, 0, 40, nthreads=4)
    e2, h2, w2, _ = oracle.frw_walks(s, p, 20, 20, nthreads=2)
    assert np.array_equal(e1[20:], e2) and np.array_equal(h1[20:], h2)
    assert np.array_equal(w1[20:], w2)
    assert (h1 >= 1).all() and (e1 >= 0).all() and (e1 <= 8).all()


def test_cpu_walker_ggft_vs_restatement(oracle):
    """The same walks with the reference ggft (tol 1e-12) per hop and with the
    FP64 restatement end on the same nets with the same weights."""
    if not oracle.ref_available(6):
        pytest.skip("reference ggft not built here")
    s = W.two_layer_crossing().to_c()
    p = _params(6)
    e1, h1, w1, _ = oracle.frw_walks(s, p, 0, 30, fdm="oracle", fdm_tol=1e-12, nthreads=4)
    e2, h2, w2, _ = oracle.frw_walks(s, p, 0, 30, fdm="ggft", fdm_tol=1e-12, nthreads=4)
    same = (e1 == e2) & (h1 == h2)
    assert same.mean() >= 0.9
    assert np.allclose(w1[same], w2[same], rtol=1e-8)


def test_weight_signs_and_charge_neutrality(oracle):
    """Self term positive, couplings negative; the row (with ground) sums to
    zero within the statistics."""
    s = W.two_layer_crossing().to_c()
    p = _params(6)
    end, hops, w, _ = oracle.frw_walks(s, p, 0, 600, nthreads=8)
    n = len(w)
    cap = np.array([w[end == j].sum() / n for j in range(9)])
    sem = np.array([np.sqrt(max(0.0, (np.where(end == j, w, 0) ** 2).mean() - cap[j] ** 2) / n)
                    for j in range(9)])
    assert cap[0] > 0
    # the adjacent wire and the grounded enclosure: clearly negative couplings
    assert cap[1] < -3 * sem[1] and cap[8] < -3 * sem[8]
    # no coupling is significantly positive
    assert np.all(cap[1:] < 4 * sem[1:])
    tot = w.mean()
    sem = w.std() / np.sqrt(n)
    assert abs(tot) < 4 * sem
