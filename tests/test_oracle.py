"""CPU checks of the oracle (test infrastructure): pinned against the golden
vectors produced by the reference ggft build, against that build itself when
it is present, and on its own invariants."""
import numpy as np
import pytest

from conftest import golden
from deeprwcap_b200 import workloads as W

GOLDEN_NS = (5, 8, 16, 21, 23)


@pytest.mark.parametrize("N", GOLDEN_NS)
def test_oracle_matches_golden(oracle, N):
    g = golden(N)
    eps, ref, codes = g["eps"], g["gft"], g["codes"]
    for ci, code in enumerate(codes):
        mine, ok, _ = oracle.fdm_solve_batch(eps, int(code), tol=1e-13)
        assert ok.all()
        err = np.linalg.norm(mine - ref[ci], axis=1) / np.linalg.norm(ref[ci], axis=1)
        assert err.max() < 1e-8, (N, code, err.max())


@pytest.mark.parametrize("N", (4, 5, 6, 8))
def test_oracle_vs_reference_build(oracle, N):
    if not oracle.ref_available(N):
        pytest.skip("reference ggft not built here")
    eps, _ = W.fdm_cubes(4, N, seed=900 + N)
    for code in range(4):
        ref, ok, _ = oracle.ggft_ref(eps, code, tol=1e-12)
        mine, ok2, _ = oracle.fdm_solve_batch(eps, code, tol=1e-13)
        assert ok.all() and ok2.all()
        err = np.linalg.norm(mine - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert err.max() < 1e-8


@pytest.mark.parametrize("N", (5, 8, 16))
def test_gf_is_a_distribution(oracle, N):
    """ggft's own invariants (ggft_solver.cpp:598-626): sum G = 1, G >= 0;
    gradient sources sum to zero so the WVT surface values do too."""
    eps, _ = W.fdm_cubes(3, N, seed=N, noise_frac=0.5)
    for e in eps:
        g, rc, it, rr = oracle.fdm_solve(e, 0, tol=1e-13)
        assert rc == 0 and rr < 1e-13
        assert abs(g.sum() - 1) < 1e-11
        assert g.min() >= 0
        for code in (1, 2, 3):
            w, rc, _, _ = oracle.fdm_solve(e, code, tol=1e-13)
            assert abs(w.sum()) < 1e-9 * np.abs(w).sum()


def test_rotation_equivariance(oracle):
    """Rotating the permittivity about z by 90 degrees permutes the faces."""
    N = 7
    eps, _ = W.fdm_cubes(1, N, seed=5, noise_frac=1.0)
    e = eps[0]
    g, *_ = oracle.fdm_solve(e, 0, tol=1e-13)
    # eps[k, j, i] -> eps'[k, j', i'] with (i', j') = (N-1-j, i): x' = -y, y' = x
    e2 = np.empty_like(e)
    for j in range(N):
        for i in range(N):
            e2[:, i, N - 1 - j] = e[:, j, i]
    g2, *_ = oracle.fdm_solve(e2, 0, tol=1e-13)
    NN = N * N
    f = lambda g, face: g[face * NN:(face + 1) * NN].reshape(N, N)  # [row, col]
    # z faces: index i + j*N -> [j, i]; rotated: g2_z[j', i'] = g_z[j, i] with i' = N-1-j, j' = i
    gz, g2z = f(g, 0), f(g2, 0)
    for j in range(N):
        for i in range(N):
            assert abs(g2z[i, N - 1 - j] - gz[j, i]) < 1e-12
    # y- face of the rotated cube (y'=0 <=> x=0) is the x- face of the original
    assert abs(f(g2, 2).sum() - f(g, 4).sum()) < 1e-12


def test_even_n_rhs_split(oracle):
    N = 6
    eps, _ = W.fdm_cubes(1, N, seed=3, noise_frac=1.0)
    e = oracle.rhs(eps[0], 0)
    assert abs(e.sum() - 1) < 1e-15 and np.count_nonzero(e) == 8
    for code in (1, 2, 3):
        e = oracle.rhs(eps[0], code)
        assert abs(e.sum()) < 1e-12 and np.count_nonzero(e) == 8
    N = 7
    eps, _ = W.fdm_cubes(1, N, seed=3, noise_frac=1.0)
    assert np.count_nonzero(oracle.rhs(eps[0], 0)) == 1
    assert np.count_nonzero(oracle.rhs(eps[0], 1)) == 3


def test_philox_known_answers(oracle):
    """Philox4x32-10 known-answer vectors of the Random123 distribution."""
    def py_philox(c, k):
        c = list(c); k = list(k)
        for _ in range(10):
            p0 = 0xD2511F53 * c[0]
            p1 = 0xCD9E8D57 * c[2]
            c = [((p1 >> 32) ^ c[1] ^ k[0]) & 0xFFFFFFFF, p1 & 0xFFFFFFFF,
                 ((p0 >> 32) ^ c[3] ^ k[1]) & 0xFFFFFFFF, p0 & 0xFFFFFFFF]
            k = [(k[0] + 0x9E3779B9) & 0xFFFFFFFF, (k[1] + 0xBB67AE85) & 0xFFFFFFFF]
        return c

    assert py_philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert py_philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e,
                                                             0xa20bc7c6, 0x6d5451fd]
    assert py_philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                     [0xa4093822, 0x299f31d0]) == [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]
    # the C oracle's doubles are built from the same words
    for seed, stream, c2, c3 in [(0, 0, 0, 0), (7, 123456789012, 5, 1), (2**63 + 5, 2**40, 9, 0)]:
        w = py_philox([stream & 0xFFFFFFFF, stream >> 32, c2, c3],
                      [seed & 0xFFFFFFFF, seed >> 32])
        u0 = ((w[0] >> 5) * 2**26 + (w[1] >> 6)) / 2**53
        u1 = ((w[2] >> 5) * 2**26 + (w[3] >> 6)) / 2**53
        got = oracle.philox_uniform2(seed, stream, c2, c3)
        assert got[0] == u0 and got[1] == u1


def test_sample_index_semantics(oracle):
    w = np.array([0.0, 0.25, 0.0, 0.5, 0.25])
    assert oracle.sample_index(w, 0.0) == 1
    assert oracle.sample_index(w, 0.2499) == 1
    assert oracle.sample_index(w, 0.25) == 3
    assert oracle.sample_index(w, 0.7499) == 3
    assert oracle.sample_index(w, 0.75) == 4
    assert oracle.sample_index(w, 0.999999) == 4
    assert oracle.sample_index(-w, 0.3, use_abs=True) == 3
    assert oracle.sample_index(np.zeros(4), 0.5) == -1


def test_locate_matches_reference_table(oracle):
    """locate_index_simple_kernel's face table (cuda_kernels.cu:229-263)."""
    N = 23
    for f, expect in enumerate([(0, 0, -1), (0, 0, 1), (0, -1, 0), (0, 1, 0), (-1, 0, 0),
                                (1, 0, 0)]):
        centre = (N // 2) + (N // 2) * N
        p = oracle.locate(N, f * N * N + centre)
        assert np.allclose(p, expect, atol=1e-6)
    p = oracle.locate(N, 2 * N * N + 3 + 5 * N)  # y- face: (x_3, -1, z_5)
    assert np.allclose(p, [(2 * 3 + 1) / N - 1, -1, (2 * 5 + 1) / N - 1], atol=1e-7)


def test_structure_construction_rules(oracle):
    """fill_structure_kernel: last layer with min_z <= z, first cuboid wins,
    padding ends the lists; normalisation by the max permittivity."""
    N = 4
    lay = np.full((15, 2), -9999.0, dtype=np.float32)
    cub = np.full((15, 7), -9999.0, dtype=np.float32)
    lay[0] = (-1.0, 2.0); lay[1] = (0.0, 4.0)
    cub[0] = (-1, -1, -1, -0.5, 1, 1, 8.0)     # x <= -0.5
    cub[1] = (-1, -1, -1, 1, 1, 1, 1.0)        # everything else would be 1 ...
    eps, mx = oracle.structure_construction(lay, cub, N, normalise=False)
    assert mx[0] == 8.0
    e = eps[0]
    assert np.all(e[:, :, 0] == 8.0)           # first cuboid wins at x = -0.75
    assert np.all(e[:, :, 1:] == 1.0)          # ... and the second covers the rest
    cub[1, 0] = -9999.0                        # padding ends the cuboid list
    eps, _ = oracle.structure_construction(lay, cub, N, normalise=True)
    e = eps[0]
    assert np.allclose(e[:, :, 0], 1.0)
    assert np.allclose(e[:2, :, 1:], 2.0 / 8.0) and np.allclose(e[2:, :, 1:], 4.0 / 8.0)
