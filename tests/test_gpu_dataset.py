"""ggft training-data files on the device: the engine's batched FDM solve
reproduces the targets the reference generator stored, the device generator
writes files the reference layout reads back, and training arrays built from
them are well formed."""
from pathlib import Path

import numpy as np
import pytest

from deeprwcap_b200 import engine
from deeprwcap_b200 import ggft_dataset as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("kind,code", [("poisson", 0), ("gradient", 1)])
def test_engine_reproduces_reference_targets(ctx, kind, code):
    """Targets stored by ggft at tolerance 1e-6: the engine's solve to 1e-10
    agrees within 5e-5 of each row's largest magnitude."""
    diel, _, gft, _ = G.read_bin(GOLD / f"ggft_bin_N8_{kind}.bin", 8)
    res, _, _, status = engine.fdm_solve_batch(list(diel.reshape(-1, 8, 8, 8)), code=code,
                                               tol=1e-10, ctx=ctx)
    got = np.stack(res)
    assert (status == 0).all()
    err = np.abs(got - gft).max(1) / np.abs(gft).max(1)
    assert err.max() <= 5e-5, err


def test_generated_files_read_back(ctx, tmp_path):
    N, n = 16, 96
    info = {k: G.generate(ctx, tmp_path / f"{k}.bin", n, N, k, seed=4, chunk=40, log=lambda *a: None)
            for k in ("poisson", "gradient")}
    dp, sp, gp, _ = G.read_bin(tmp_path / "poisson.bin", N)
    dg, sg, gg, _ = G.read_bin(tmp_path / "gradient.bin", N)
    assert info["poisson"]["samples"] == n and dp.shape == (n, N ** 3)
    np.testing.assert_array_equal(dp, dg)                    # same seed, same cubes
    np.testing.assert_array_equal(G.voxelise_structures(sp, N), dp)
    assert np.allclose(gp.sum(1), 1.0, atol=1e-6) and gp.min() > -1e-9
    assert (gg < 0).any()
    ref, ok, _ = O.fdm_solve_batch(dp[:3].reshape(3, N, N, N), O.GFT)
    assert ok.all() and np.abs(ref - gp[:3]).max() <= 2e-5 * np.abs(ref).max()
    X, T, TG = G.training_arrays(ctx, [tmp_path / "poisson.bin", tmp_path / "gradient.bin"], N)
    assert X.shape == (2 * n, N ** 3) and T.shape == (2 * n, 6 * N * N)
    assert float(X.float().max(dim=1).values.min()) == 1.0
    np.testing.assert_allclose(T.sum(dim=1).cpu().numpy(), 1.0, atol=1e-4)
    # the poisson file's gradient targets were solved here, the gradient file's stored ones
    np.testing.assert_allclose(TG[n:].cpu().numpy(), (gg * 64.0).astype(np.float32), rtol=0, atol=1e-6)
    np.testing.assert_allclose(T[:n].cpu().numpy(), gp.astype(np.float32), rtol=0, atol=1e-7)
