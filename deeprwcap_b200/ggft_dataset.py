"""The ggft training-data file (``<kind>.bin``): reader, writer, the
reference reader's preprocessing, and a device generator that writes it.

File layout (writer ``ggft/src/main.cpp:59-78`` with the per-sample record of
``ggft_solver::dump_matrix``, ``ggft/src/ggft_solver.h:180-191``; reader
``training_pytorch/src/dataset.py:57-85``). Every value is a little-endian
FP64 (``ggft_solver::real`` is double, ``ggft_solver.h:114``):

    header     N, block_width
    per sample DIEL       (N / block_width)^3 permittivities, x fastest
                          (i + j*bN + k*bN^2, ``ggft_solver.h:48``)
               STRUCTURE  7 values per dielectric block: centre x, y, z,
                          half-widths x, y, z, permittivity; the reference
                          generator writes 15 blocks (unused ones all zero)
                          and then the background block
               gft        6N^2 surface values in ggft panel order: the
                          Green's function (``poisson`` files, code GFT) or
                          the centre-gradient weights along z (``gradient``
                          files, code WVTZ)

The same cube order and panel order are what the engine uses, so a file's
DIEL rows are network inputs after max normalisation and its gft rows are
training targets as they stand.

    python -m deeprwcap_b200.ggft_dataset <nthreads> <total_count> <output_folder> \\
        <poisson|gradient> [--N 23] [--seed 0] [--tol 1e-6]

mirrors the reference generator's command line (``ggft/src/main.cpp:10-25``)
and writes ``<output_folder>/<kind>.bin``; the cubes are solved in batches on
the GPU (``drwc_fdm_solve_batch_device``), ``nthreads`` is accepted and
ignored.
"""
from __future__ import annotations

import argparse
import math
import time
from pathlib import Path

import numpy as np

STRUCT_VALUES = 7           # dielectric_generator.h:100-106
GEN_BLOCKS = 15             # dielectric_generator::MAX_BLOCK_COUNT
GEN_STRUCTURES = GEN_BLOCKS + 1
KINDS = {"poisson": 0, "gradient": 1}   # solver codes GFT, WVTZ (ggft_solver.h:119)


# ---------------------------------------------------------------- file format
def read_bin(path, N: int, n_structures: int | None = GEN_STRUCTURES, dtype=np.float64):
    """(diel [S, bN^3], structure [S, 7 * ns], gft [S, 6N^2], block_width).

    Follows ``GreenDataset._load_single_file`` (dataset.py:57-85): the header
    must name N; with ``n_structures`` given the record length is fixed and
    the body must hold whole records, with None the record length is the
    first divisor split that leaves a structure part divisible by 7
    (``_factor_file``, dataset.py:87-96)."""
    vec = np.fromfile(path, dtype=dtype)
    if vec.size < 2:
        raise ValueError(f"{path}: shorter than its header")
    n, bw = int(vec[0]), int(vec[1])
    if n != N:
        raise ValueError(f"{path}: header N={n}, expected {N}")
    if bw < 1 or n % bw:
        raise ValueError(f"{path}: block width {bw} does not divide N={n}")
    bn = n // bw
    diel_len, gf_len = bn ** 3, 6 * n * n
    body = vec[2:]
    if n_structures is not None:
        struct_len = STRUCT_VALUES * n_structures
        rec = diel_len + struct_len + gf_len
        if body.size % rec:
            raise ValueError(f"{path}: file length not compatible with {n_structures} "
                             f"structures per sample")
        count = body.size // rec
    else:
        count, struct_len = _factor_records(body.size, diel_len, gf_len)
        rec = diel_len + struct_len + gf_len
    data = body.reshape(count, rec)
    return (data[:, :diel_len].copy(), data[:, diel_len:diel_len + struct_len].copy(),
            data[:, rec - gf_len:].copy(), bw)


def _factor_records(total: int, diel_len: int, gf_len: int):
    small, large = [], []
    for i in range(1, math.isqrt(total) + 1):
        if total % i == 0:
            small.append(i)
            if i * i != total:
                large.append(total // i)
    for count in small + large[::-1]:
        struct_len = total // count - diel_len - gf_len
        if struct_len >= 0 and struct_len % STRUCT_VALUES == 0:
            return count, struct_len
    raise ValueError("could not determine the per-sample structure length")


def write_bin(path, N: int, diel, structure, gft, block_width: int = 1) -> int:
    """Write a file the reference reader accepts; returns the sample count.
    ``structure`` may have zero columns (records without block lists)."""
    diel = np.ascontiguousarray(diel, dtype="<f8")
    gft = np.ascontiguousarray(gft, dtype="<f8")
    S = diel.shape[0]
    structure = np.ascontiguousarray(
        np.zeros((S, 0)) if structure is None else structure, dtype="<f8").reshape(S, -1)
    bn = N // block_width
    if N % block_width or diel.shape != (S, bn ** 3) or gft.shape != (S, 6 * N * N):
        raise ValueError("diel [S, (N/bw)^3] and gft [S, 6N^2] expected")
    if structure.shape[1] % STRUCT_VALUES:
        raise ValueError("structure rows hold 7 values per block")
    with open(path, "wb") as f:
        np.array([N, block_width], dtype="<f8").tofile(f)
        np.concatenate([diel, structure, gft], axis=1).tofile(f)
    return S


def cell_eps(diel, N: int, block_width: int = 1):
    """Per-cell permittivity [S, N^3] (cell (i, j, k) takes block (i/bw, j/bw,
    k/bw), ggft_solver.h:90-96)."""
    diel = np.asarray(diel, dtype=np.float64)
    if block_width == 1:
        return diel.reshape(-1, N ** 3)
    bn = N // block_width
    d = diel.reshape(-1, bn, bn, bn)  # [k][j][i]
    d = np.repeat(np.repeat(np.repeat(d, block_width, 1), block_width, 2), block_width, 3)
    return d.reshape(-1, N ** 3)


# ------------------------------------------------- reference preprocessing
def prep_greens_function(gft, N: int):
    """(greens_tensor [S, 6, 1, N, N], face_distribution [S, 6]) in FP32, as
    ``GreenDataset._prep_greens_function`` (dataset.py:110-114): each face
    normalised by its own sum (zero sums left as they are), and the face
    sums."""
    g = np.asarray(gft, dtype=np.float32).reshape(-1, 6, 1, N, N)
    face_sum = g.sum(axis=(2, 3, 4))
    grid_sum = g.sum(axis=(3, 4), keepdims=True)
    grid_sum[grid_sum == 0] = 1
    return (g / grid_sum).astype(np.float32), face_sum.astype(np.float32)


def prep_gradient(gft, N: int):
    """(normalised_gradient [S, 6, 1, N, N], face_grad_weights [S, 7]) in
    FP32, as ``GreenDataset._prep_gradient`` (dataset.py:116-122): signed
    values over each face's absolute sum; per-face shares of the total
    absolute weight, then the total."""
    g = np.asarray(gft, dtype=np.float32).reshape(-1, 6, 1, N, N)
    signs, mags = np.sign(g), np.abs(g)
    face_tot = mags.sum(axis=(3, 4), keepdims=True)
    norm = (mags / face_tot * signs).astype(np.float32)
    w = face_tot.reshape(face_tot.shape[0], 6)
    share = (w / w.sum(axis=1, keepdims=True)).astype(np.float32)
    return norm, np.concatenate((share, w.sum(axis=1, keepdims=True)), axis=1).astype(np.float32)


# ------------------------------------------------------- cube generator
def random_structures(count: int, seed: int = 0, block_count: int = 5) -> np.ndarray:
    """[count, 7 * 16] block lists drawn like ``random_blocks_practical``
    (dielectric_generator.h:47-82): ``block_count`` boxes with centres
    U(-2, 2)^3, half-widths U(0, 2)^3 and permittivity U(2, 10) with
    probability 0.8 else U(10, 80); after each box, while U(0, 1) <= 0.2, a
    copy grown by 0.1 x its largest half-width with a new permittivity;
    truncated (or zero-padded) to 15 boxes, then the background box (centre 0,
    half-width 2, new permittivity). numpy's generator stands in for the
    reference's mt19937, so the draws follow the same laws, not the same
    sequence."""
    rng = np.random.default_rng(seed)
    out = np.zeros((count, STRUCT_VALUES * GEN_STRUCTURES))

    def eps():
        return rng.uniform(2, 10) if rng.uniform() <= 0.8 else rng.uniform(10, 80)

    for s in range(count):
        blocks = []
        for _ in range(block_count):
            c = rng.uniform(-2, 2, 3)
            r = rng.uniform(0, 2, 3)
            b = [*c, *r, eps()]
            blocks.append(b)
            while rng.uniform() <= 0.2:
                dr = 0.1 * max(b[3:6])
                blocks.append([*b[:3], b[3] + dr, b[4] + dr, b[5] + dr, eps()])
        blocks = blocks[:GEN_BLOCKS] + [[0.0] * STRUCT_VALUES] * max(0, GEN_BLOCKS - len(blocks))
        blocks.append([0.0, 0.0, 0.0, 2.0, 2.0, 2.0, eps()])
        out[s] = np.asarray(blocks).reshape(-1)
    return out


def voxelise_structures(structure, bn: int) -> np.ndarray:
    """DIEL [S, bn^3] of block lists by the generator's rule
    (dielectric_generator.h:109-127): cell centres (2i + 1) / bn - 1 on each
    axis, the first block that strictly contains the centre gives the
    permittivity (|x - cx| < rx on all three axes); a centre no block holds
    keeps 1 (``DIEL`` starts at 1, ggft_solver.h:152)."""
    st = np.asarray(structure, dtype=np.float64).reshape(len(structure), -1, STRUCT_VALUES)
    t = (2.0 * np.arange(bn) + 1.0) / bn - 1.0
    S, nb = st.shape[:2]
    out = np.ones((S, bn, bn, bn))  # [k][j][i]
    for s in range(S):
        filled = np.zeros((bn, bn, bn), dtype=bool)
        for b in range(nb):
            cx, cy, cz, rx, ry, rz, v = st[s, b]
            ix = np.abs(t - cx) < rx
            iy = np.abs(t - cy) < ry
            iz = np.abs(t - cz) < rz
            m = iz[:, None, None] & iy[None, :, None] & ix[None, None, :] & ~filled
            out[s][m] = v
            filled |= m
    return out.reshape(S, -1)


def generate(ctx, out_path, count: int, N: int, kind: str, seed: int = 0, tol: float = 1e-6,
             chunk: int = 16384, log=print) -> dict:
    """Write ``count`` random cubes of resolution N and their ``kind``
    solutions to ``out_path``, solving ``chunk`` cubes per device batch. The
    cube sequence depends only on ``seed``, so a poisson file and a gradient
    file made with the same seed hold the same cubes."""
    import torch

    from . import engine
    if kind not in KINDS:
        raise ValueError(f"kind must be one of {tuple(KINDS)}")
    dev = torch.device("cuda", ctx.device)
    t0 = time.time()
    structure = random_structures(count, seed)
    diel = voxelise_structures(structure, N)
    t_gen = time.time() - t0
    gft = np.empty((count, 6 * N * N))
    t1 = time.time()
    for lo in range(0, count, chunk):
        hi = min(count, lo + chunk)
        e = torch.from_numpy(diel[lo:hi]).to(dev)
        o = torch.empty(hi - lo, 6 * N * N, dtype=torch.float64, device=dev)
        engine.fdm_solve_device(ctx, e, N, KINDS[kind], o, tol=tol)
        gft[lo:hi] = o.cpu().numpy()
    t_solve = time.time() - t1
    write_bin(out_path, N, diel, structure, gft)
    info = {"samples": count, "N": N, "kind": kind, "generate_s": t_gen, "solve_s": t_solve,
            "solves_per_s": count / max(t_solve, 1e-9), "path": str(out_path)}
    log(f"ggft dataset: {info}")
    return info


def training_arrays(ctx, paths, N: int, n_structures: int | None = GEN_STRUCTURES,
                    tol: float = 1e-8, chunk: int = 16384):
    """X [S, N^3] BF16, T [S, 6N^2] FP32, TG [S, 6N^2] FP32 (device) from
    ggft files: X = DIEL / its maximum, T = the Green's function, TG = the z
    gradient weights times the gradient-head scale. A file supplies the
    target of its kind (named by the file, ``poisson.bin`` / ``gradient.bin``
    as the reference generator writes them, else by sign: only gradient
    weights go negative); the engine's batched FDM solve supplies the
    other."""
    import torch

    from . import engine
    from .train import GRAD_SCALE
    dev = torch.device("cuda", ctx.device)
    parts = []
    for p in paths:
        diel, _, gft, bw = read_bin(p, N, n_structures)
        stem = Path(p).stem
        kind = stem if stem in KINDS else ("gradient" if (gft < 0).any() else "poisson")
        parts.append((cell_eps(diel, N, bw), gft, kind))
    S = sum(e.shape[0] for e, _, _ in parts)
    X = torch.empty(S, N ** 3, dtype=torch.bfloat16, device=dev)
    T = torch.empty(S, 6 * N * N, dtype=torch.float32, device=dev)
    TG = torch.empty(S, 6 * N * N, dtype=torch.float32, device=dev)
    pos = 0
    for eps, gft, kind in parts:
        for lo in range(0, eps.shape[0], chunk):
            hi = min(eps.shape[0], lo + chunk)
            e = torch.from_numpy(eps[lo:hi]).to(dev)
            g = torch.from_numpy(gft[lo:hi]).to(dev)
            n = hi - lo
            X[pos:pos + n] = (e / e.max(dim=1, keepdim=True).values).to(torch.bfloat16)
            other = torch.empty(n, 6 * N * N, dtype=torch.float64, device=dev)
            engine.fdm_solve_device(ctx, e, N, 1 if kind == "poisson" else 0, other, tol=tol)
            if kind == "poisson":
                T[pos:pos + n] = g.float()
                TG[pos:pos + n] = (other * GRAD_SCALE).float()
            else:
                T[pos:pos + n] = other.float()
                TG[pos:pos + n] = (g * GRAD_SCALE).float()
            pos += n
    return X, T, TG


def main() -> None:
    ap = argparse.ArgumentParser(description="write a ggft training-data file")
    ap.add_argument("nthreads", type=int, help="accepted for command-line compatibility; unused")
    ap.add_argument("total_count", type=int)
    ap.add_argument("output_folder")
    ap.add_argument("kind", choices=sorted(KINDS))
    ap.add_argument("--N", type=int, default=23)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--tol", type=float, default=1e-6)  # main.cpp:43
    a = ap.parse_args()
    from . import engine
    ctx = engine.default_context(0)
    out = Path(a.output_folder)
    out.mkdir(parents=True, exist_ok=True)
    generate(ctx, out / f"{a.kind}.bin", a.total_count, a.N, a.kind, seed=a.seed, tol=a.tol)


if __name__ == "__main__":
    main()
