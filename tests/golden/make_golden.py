"""Regenerate the golden vectors in this folder from the reference ggft
solver compiled from the reference's own sources (oracle/_ref, built by
oracle/Makefile from ggft/src/ggft_solver.{h,cpp}).

    python tests/golden/make_golden.py

Inputs are seeded transition cubes (deeprwcap_b200.workloads.fdm_cubes: 1-4
horizontal layers with eps ~ U[2,8] and 0-2 dielectric boxes with
eps ~ U[2,8]); outputs are ggft's `gft` after set_tolerance(1e-12) and
solve(code) for the solver codes listed per case. Needs the reference tree,
so it only runs where that tree is mounted; the committed .npz files are what
the tests read.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from deeprwcap_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = [  # (N, ncubes, codes, seed)
    (5, 6, (0, 1, 2, 3), 105),
    (8, 6, (0, 1, 2, 3), 108),
    (16, 12, (0, 1, 2, 3), 116),
    (21, 2, (0, 1), 121),
    (23, 2, (0, 2), 123),
]
TOL = 1e-12


def main() -> None:
    O.build()
    for N, n, codes, seed in CASES:
        eps, structs = W.fdm_cubes(n, N, seed=seed)
        gft = np.zeros((len(codes), n, 6 * N * N))
        for ci, code in enumerate(codes):
            out, ok, _ = O.ggft_ref(eps, code, tol=TOL, nthreads=8)
            assert ok.all(), f"ggft failed for N={N} code={code}"
            gft[ci] = out
        path = HERE / f"ggft_N{N}.npz"
        np.savez_compressed(path, N=N, seed=seed, tol=TOL, codes=np.array(codes, dtype=np.int32),
                            eps=eps, gft=gft)
        print(path, path.stat().st_size)


if __name__ == "__main__":
    main()
