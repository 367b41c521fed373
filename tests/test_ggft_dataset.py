"""The ggft training-data file (.bin): reader, writer and preprocessing
against files written by the reference's own generator (ggft/src/main.cpp,
built from its sources) and tensors produced by the reference's own reader
(training_pytorch/src/dataset.py), both stored in tests/golden by
make_ggft_bin_fixtures.py."""
from pathlib import Path

import numpy as np
import pytest

from deeprwcap_b200 import ggft_dataset as G
from oracle import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"
N = 8
FILES = {k: GOLD / f"ggft_bin_N{N}_{k}.bin" for k in ("poisson", "gradient")}


@pytest.mark.parametrize("kind", ["poisson", "gradient"])
def test_reader_layout(kind):
    diel, st, gft, bw = G.read_bin(FILES[kind], N)
    assert bw == 1 and diel.shape == (6, N ** 3) and st.shape == (6, 7 * 16)
    assert gft.shape == (6, 6 * N * N)
    # the background block closes every block list (dielectric_generator.h:79)
    bg = st.reshape(6, 16, 7)[:, -1]
    np.testing.assert_array_equal(bg[:, :6], np.tile([0, 0, 0, 2, 2, 2], (6, 1)))
    if kind == "poisson":
        assert np.all(gft >= 0) and np.allclose(gft.sum(1), 1.0, atol=1e-5)
    else:
        assert (gft < 0).any() and (gft > 0).any()


@pytest.mark.parametrize("kind", ["poisson", "gradient"])
def test_legacy_record_length_inference(kind):
    """Without a structure count the reader takes the smallest sample count
    whose record leaves a structure part divisible by 7 (dataset.py:87-96):
    for these files that is one record holding everything, which is why the
    reference reader gained its n_structures argument."""
    diel, st, gft, _ = G.read_bin(FILES[kind], N, n_structures=None)
    assert diel.shape[0] == 1 and st.shape[1] == 6 * 1008 - N ** 3 - 6 * N * N
    a = G.read_bin(FILES[kind], N)
    np.testing.assert_array_equal(diel[0], a[0][0])
    np.testing.assert_array_equal(gft[0], a[2][-1])


@pytest.mark.parametrize("kind", ["poisson", "gradient"])
def test_block_lists_voxelise_to_the_stored_permittivity(kind):
    diel, st, _, _ = G.read_bin(FILES[kind], N)
    np.testing.assert_array_equal(G.voxelise_structures(st, N), diel)


@pytest.mark.parametrize("kind", ["poisson", "gradient"])
def test_writer_reproduces_the_reference_file(kind, tmp_path):
    diel, st, gft, bw = G.read_bin(FILES[kind], N)
    out = tmp_path / f"{kind}.bin"
    assert G.write_bin(out, N, diel, st, gft, bw) == 6
    assert out.read_bytes() == FILES[kind].read_bytes()


def test_preprocessing_matches_the_reference_reader():
    ref = np.load(GOLD / f"ggft_bin_N{N}_reader.npz")
    _, _, g, _ = G.read_bin(FILES["poisson"], N)
    gt, fd = G.prep_greens_function(g, N)
    np.testing.assert_array_equal(gt, ref["greens_tensor"])
    np.testing.assert_array_equal(fd, ref["face_distribution"])
    _, _, g, _ = G.read_bin(FILES["gradient"], N)
    ng, fw = G.prep_gradient(g, N)
    np.testing.assert_array_equal(ng, ref["normalised_gradient"])
    np.testing.assert_array_equal(fw, ref["face_grad_weights"])


@pytest.mark.parametrize("kind,code", [("poisson", O.GFT), ("gradient", O.WVTZ)])
def test_stored_targets_match_the_oracle_solve(kind, code):
    """The file's targets come from ggft at tolerance 1e-6 (main.cpp:43); the
    FP64 oracle solved to 1e-13 agrees within 5e-5 of each row's largest
    magnitude."""
    diel, _, gft, _ = G.read_bin(FILES[kind], N)
    ref, ok, _ = O.fdm_solve_batch(diel.reshape(-1, N, N, N), code)
    assert ok.all()
    err = np.abs(ref - gft).max(1) / np.abs(ref).max(1)
    assert err.max() <= 5e-5, err


def test_bad_files_are_rejected(tmp_path):
    with pytest.raises(ValueError):
        G.read_bin(FILES["poisson"], 16)                       # header names N = 8
    cut = tmp_path / "cut.bin"
    cut.write_bytes(FILES["poisson"].read_bytes()[:-8])
    with pytest.raises(ValueError):
        G.read_bin(cut, N)
    with pytest.raises(ValueError):
        G.write_bin(tmp_path / "x.bin", N, np.zeros((2, 10)), None, np.zeros((2, 6 * N * N)))


def test_random_structures_follow_the_generator_laws():
    st = G.random_structures(400, seed=5).reshape(400, 16, 7)
    bg = st[:, -1]
    np.testing.assert_array_equal(bg[:, :6], np.tile([0, 0, 0, 2, 2, 2], (400, 1)))
    used = st[:, :-1][st[:, :-1, 6] > 0]
    assert used.shape[0] >= 5 * 400
    assert np.all(np.abs(used[:, :3]) <= 2) and np.all(used[:, 6] >= 2) and np.all(used[:, 6] <= 80)
    assert 0.1 < np.mean(used[:, 6] > 10) < 0.35             # high-k share about 0.2
    diel = G.voxelise_structures(st[:8].reshape(8, -1), 16)
    assert diel.shape == (8, 16 ** 3) and np.all(diel >= 2)
    np.testing.assert_array_equal(G.random_structures(3, seed=9), G.random_structures(3, seed=9))


def test_block_width_expansion():
    d = np.arange(8, dtype=np.float64).reshape(1, 8)  # 2^3 blocks, x fastest
    e = G.cell_eps(d, 4, block_width=2).reshape(4, 4, 4)  # [k][j][i]
    assert e[0, 0, 0] == 0 and e[0, 0, 3] == 1 and e[0, 3, 0] == 2 and e[3, 0, 0] == 4
    assert e[3, 3, 3] == 7
