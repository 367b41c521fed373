"""Regenerate the ggft training-data fixtures in this folder with the
reference's own generator and reader.

    python tests/golden/make_ggft_bin_fixtures.py

1. Builds the reference generator (ggft/src/main.cpp + dielectric_generator.h
   against the per-N solver copy) as oracle/_ref/ggft_gen_N8 with
   oracle/Makefile and runs it single-threaded for 6 cubes of each kind:
   ``ggft_gen_N8 1 6 <dir> poisson`` / ``gradient``. Its generator is seeded
   with the thread id (main.cpp:43), so the files are the same on every run.
   They are copied here as ggft_bin_N8_poisson.bin / ggft_bin_N8_gradient.bin.
2. Reads both files with the reference's training reader
   (training_pytorch/src/dataset.py, ``GreenDataset``; FP64, 16 structures
   per sample as the generator writes them) and stores its tensors in
   ggft_bin_N8_reader.npz: greens_tensor, face_distribution (poisson) and
   normalised_gradient, face_grad_weights (gradient).

Needs the reference tree ($DRWC_REFERENCE_DIR, else ``reference`` beside
this repository's folder), so it runs only where that tree is mounted; the
committed files are what the tests read.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
N, COUNT = 8, 6


def main() -> None:
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import reference_dir
    REF = reference_dir()
    subprocess.run(["make", "-C", str(ROOT / "oracle"), f"REF={REF}", f"_ref/ggft_gen_N{N}"],
                   check=True)
    gen = ROOT / "oracle" / "_ref" / f"ggft_gen_N{N}"
    out = {}
    sys.path.insert(0, str(REF / "training_pytorch" / "src"))
    from dataset import GreenDataset  # the reference reader

    with tempfile.TemporaryDirectory() as tmp:
        for kind, dtype_name in (("poisson", "greens_function"), ("gradient", "gradient")):
            subprocess.run([str(gen), "1", str(COUNT), tmp, kind], check=True,
                           stdout=subprocess.DEVNULL)
            dst = HERE / f"ggft_bin_N{N}_{kind}.bin"
            shutil.copyfile(Path(tmp) / f"{kind}.bin", dst)
            ds = GreenDataset(files=[str(dst)], dataset_type=dtype_name, N=N, dtype=np.float64,
                              n_structures=16)
            if kind == "poisson":
                out["greens_tensor"] = ds.greens_tensor
                out["face_distribution"] = ds.face_distribution
            else:
                out["normalised_gradient"] = ds.normalised_grad
                out["face_grad_weights"] = ds.face_grad_weights
    np.savez(HERE / f"ggft_bin_N{N}_reader.npz", **out)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()
