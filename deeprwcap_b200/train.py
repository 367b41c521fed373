"""Train the learned transition network on FDM data the engine generates.

    python -m deeprwcap_b200.train [--N 16|21|23] [--samples 1048576] [--epochs 3] [--out PATH]
        [--data poisson.bin gradient.bin]

With --data the training cubes come from ggft training-data files (the
reference generator's, or ones deeprwcap_b200.ggft_dataset wrote); the target
a file does not hold is solved by the engine. Otherwise:

Training data (all on the device):
  * transition cubes logged from real walks (drwc_frw_harvest) on the
    8-conductor two-layer crossing and the 24-conductor dense stack, first-hop
    cubes voxelised in the frame of their gradient axis, and
  * random transition cubes of the batched-FDM generator (drwc_cubes_random);
targets are the engine's own FDM solves (drwc_fdm_solve_batch_device, FP32 CG
+ FP64 refinement to 1e-8): the surface Green's function (GFT) for the
Poisson head and the centre-gradient surface values (WVTZ) for the gradient
head. Optimiser and loss follow DeepRWCap's training setup
(training_pytorch/src/train.py:36-38, 69-120: AdamW lr 1e-3, weight decay
1e-10, gradient clipping 1.0, KL loss on the normalised Poisson kernel) with
a cosine learning-rate decay. The forward and backward passes are the
library's own tensor-core kernels (drwc_net_train_step); this script only
orders the batches.
"""
from __future__ import annotations

import argparse
import math
import time
from pathlib import Path

import numpy as np

from . import engine
from . import workloads as W

GRAD_SCALE = 64.0  # gradient-head target scale (kGradScale in csrc/nn.cuh)
DEFAULT_CKPT = Path(__file__).resolve().parent / "models" / "net_n16.npz"


def build_dataset(ctx, n_total: int, walk_frac: float = 0.5, seed: int = 0, chunk: int = 32768,
                  log=print, N: int = 16):
    """X [n, N^3] bf16, T [n, 6N^2] f32, TG [n, 6N^2] f32 (device tensors)."""
    import torch
    dev = torch.device("cuda", ctx.device)
    n_walk = int(n_total * walk_frac)
    n_rand = n_total - n_walk
    X = torch.empty(n_total, N ** 3, dtype=torch.bfloat16, device=dev)
    T = torch.empty(n_total, 6 * N * N, dtype=torch.float32, device=dev)
    TG = torch.empty(n_total, 6 * N * N, dtype=torch.float32, device=dev)
    eps = torch.empty(chunk, N ** 3, dtype=torch.float64, device=dev)
    out = torch.empty(chunk, 6 * N * N, dtype=torch.float64, device=dev)
    t0 = time.time()
    pos = 0

    def solve_chunk(lo, hi):
        n = hi - lo
        engine.fdm_solve_device(ctx, eps[:n], N, 0, out[:n])
        T[lo:hi] = out[:n].float()
        engine.fdm_solve_device(ctx, eps[:n], N, 1, out[:n])  # WVTZ
        TG[lo:hi] = (out[:n] * GRAD_SCALE).float()

    # cubes of real walks, half on each structure
    structs = [W.two_layer_crossing(), W.dense_stack(seed=3)]
    per = n_walk // len(structs)
    for si, s in enumerate(structs):
        want = per if si < len(structs) - 1 else n_walk - per * (len(structs) - 1)
        p = W.job_params_plain(N=N, seed=1000 + seed * 10 + si, tol=1e-8)
        got, walk0 = 0, 0
        while got < want:
            cap = min(chunk, want - got)
            rec, code = engine.harvest(s, p, walk0, max(64, cap // 6), cap, ctx=ctx)
            walk0 += max(64, cap // 6)
            n = int(rec.shape[0])
            if n == 0:
                continue
            engine.records_voxelise(s, rec, code, X[pos:pos + n], eps[:n], ctx=ctx, N=N)
            solve_chunk(pos, pos + n)
            pos += n
            got += n
    # random cubes
    done = 0
    while done < n_rand:
        n = min(chunk, n_rand - done)
        engine.cubes_random(n, seed * 7919 + done, X[pos:pos + n], eps[:n], ctx=ctx, N=N)
        solve_chunk(pos, pos + n)
        pos += n
        done += n
    torch.cuda.synchronize()
    log(f"dataset: {pos} cubes ({n_walk} from walks, {n_rand} random) in {time.time() - t0:.1f} s")
    return X[:pos], T[:pos], TG[:pos]


def evaluate(net, X, T, TG, batch: int = 4096):
    """Mean / p95 KL(T || softmax), relative L1 error of the gradient head."""
    import torch
    dev = X.device
    kls, g_err = [], []
    P = net.panels
    O = torch.empty(batch, net.out_row, device=dev)
    G = torch.empty(batch, net.grad_row, device=dev)
    for lo in range(0, X.shape[0], batch):
        hi = min(X.shape[0], lo + batch)
        n = hi - lo
        net.forward(X[lo:hi], O[:n], G[:n])
        torch.cuda.synchronize()
        logp = torch.log_softmax(O[:n, :P], dim=1)
        t = T[lo:hi]
        kl = (t * (torch.log(t.clamp_min(1e-30)) - logp)).sum(1)
        kls.append(kl)
        ge = (G[:n, :P] - TG[lo:hi]).abs().sum(1) / TG[lo:hi].abs().sum(1).clamp_min(1e-12)
        g_err.append(ge)
    kl = torch.cat(kls)
    ge = torch.cat(g_err)
    return {"kl_mean": kl.mean().item(), "kl_p95": kl.quantile(0.95).item(),
            "grad_rel_l1": ge.mean().item()}


def train(net, X, T, TG, epochs: int = 3, batch: int = 512, lr: float = 1e-3, seed: int = 0,
          log=print):
    import torch
    n = X.shape[0]
    steps_per = n // batch
    total = epochs * steps_per
    g = torch.Generator(device=X.device).manual_seed(seed)
    step = 0
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(n, device=X.device, generator=g)
        acc = np.zeros(3)
        for k in range(steps_per):
            idx = perm[k * batch:(k + 1) * batch]
            cur = lr * 0.5 * (1 + math.cos(math.pi * step / total))
            loss = net.train_step(X[idx], T[idx], TG[idx], lr=cur, weight_decay=1e-10, clip=1.0,
                                  w_conf=0.1, w_grad=1.0)
            acc += loss
            step += 1
        log(f"epoch {ep}: CE {acc[0] / steps_per:.5f}  conf {acc[1] / steps_per:.4f}  "
            f"grad {acc[2] / steps_per:.5f}  ({time.time() - t0:.1f} s)")
    return time.time() - t0


def split(X, T, TG, seed: int = 0, nval: int = 16384):
    """Random held-out split (the dataset is ordered by source)."""
    import torch
    n = X.shape[0]
    nval = min(nval, n // 10)
    g = torch.Generator(device=X.device).manual_seed(seed + 12345)
    perm = torch.randperm(n, device=X.device, generator=g)
    v, t = perm[:nval], perm[nval:]
    return X[t], T[t], TG[t], X[v], T[v], TG[v]


def save(net, path: Path, meta: dict):
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, params=net.get_params(), **{k: np.asarray(v) for k, v in meta.items()})


def load(path: Path = DEFAULT_CKPT, ctx=None) -> "engine.Net":
    d = np.load(path)
    N = int(d["N"]) if "N" in d else 16
    net = engine.Net(seed=0, ctx=ctx, N=N)
    net.set_params(d["params"])
    return net


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=1 << 20)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", type=str, default=str(DEFAULT_CKPT))
    ap.add_argument("--N", type=int, default=16, choices=[16, 21, 23])
    ap.add_argument("--data", nargs="*", default=None,
                    help="ggft .bin files (poisson.bin / gradient.bin) instead of engine-generated cubes")
    a = ap.parse_args()
    import torch
    ctx = engine.default_context(0)
    if a.data:
        from . import ggft_dataset
        X, T, TG = ggft_dataset.training_arrays(ctx, a.data, a.N)
    else:
        X, T, TG = build_dataset(ctx, a.samples, seed=a.seed, N=a.N)
    Xt, Tt, TGt, Xv, Tv, TGv = split(X, T, TG, seed=a.seed)
    net = engine.Net(seed=a.seed + 1, ctx=ctx, N=a.N)
    before = evaluate(net, Xv, Tv, TGv)
    print("before:", before)
    secs = train(net, Xt, Tt, TGt, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed)
    after = evaluate(net, Xv, Tv, TGv)
    print("after:", after)
    save(net, Path(a.out), {"N": a.N, "samples": X.shape[0], "epochs": a.epochs, "train_seconds": secs,
                            "val_kl_mean": after["kl_mean"], "val_kl_p95": after["kl_p95"],
                            "val_grad_rel_l1": after["grad_rel_l1"]})
    print("saved", a.out)


if __name__ == "__main__":
    main()
