"""GPU checks of the learned transition network: forward and hand-written
backward (tcgen05 tensor-core GEMMs) against a PyTorch CPU FP32 reference of
the same architecture on the same BF16-rounded weights and inputs.

Tolerances: forward 2e-2 of the largest |output| (BF16 activations between
layers are rounded the same way in the reference); gradients 5e-2 relative
(normwise per tensor: the device backward uses BF16 operands)."""
import numpy as np
import pytest

from deeprwcap_b200 import engine
from deeprwcap_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _bf(t):
    import torch
    return t.to(torch.bfloat16).float()


def _unpack(p, N=16):
    import torch
    lay, _ = engine._param_layout(N)
    P = {k: torch.from_numpy(p[o:o + n].copy()) for k, (o, n) in lay.items()}
    return P


def ref_forward(P, X, round_act=True):
    """X [B, N, N, N] (z, y, x) float; returns O [B, out_row], G [B, panels]."""
    import torch
    import torch.nn.functional as F
    B, N = X.shape[0], X.shape[1]
    dm = engine.net_dims(N)
    w1 = _bf(P["w1"]).view(16, 1, 3, 3, 3)
    w2 = _bf(P["w2"]).view(32, 27, 16).permute(0, 2, 1).reshape(32, 16, 3, 3, 3)
    w3 = _bf(P["w3"]).view(64, 27, 32).permute(0, 2, 1).reshape(64, 32, 3, 3, 3)
    rb = _bf if round_act else (lambda t: t)
    h = rb(F.relu(F.conv3d(X[:, None], w1, P["b1"], stride=2, padding=1)))
    h = rb(F.relu(F.conv3d(h, w2, P["b2"], stride=2, padding=1)))
    h = rb(F.relu(F.conv3d(h, w3, P["b3"], stride=2, padding=1)))
    F_ = dm["features"]
    feat = h.permute(0, 2, 3, 4, 1).reshape(B, F_)
    O = feat @ _bf(P["wd"]).view(dm["out_row"], F_).T + P["bd"]
    G = feat @ _bf(P["wg"]).view(dm["panels"], F_).T + P["bg"]
    return O, G


def _inputs(B, seed, N=16):
    import torch
    eps, _ = W.fdm_cubes(B, N, seed=seed, noise_frac=0.3)
    x = eps / eps.reshape(B, -1).max(axis=1)[:, None, None, None]
    return torch.from_numpy(x.astype(np.float32)).to(torch.bfloat16)


@pytest.mark.parametrize("N,B", [(16, 37), (16, 701), (21, 37), (23, 37), (23, 203)])
def test_forward_matches_reference(ctx, N, B):
    """Inference runs conv1 and conv2 fused per group of cubes (two cubes per
    CTA pass at N = 16, one at 21 / 23; odd B leaves a half group, the larger
    B give CTAs several groups), conv3 and the heads as tile GEMMs."""
    import torch
    net = engine.Net(seed=3, ctx=ctx, N=N)
    assert (net.N, net.panels, net.out_row, net.grad_row, net.features) == tuple(
        engine.net_dims(N)[k] for k in ("N", "panels", "out_row", "grad_row", "features"))
    X = _inputs(B, 1, N)
    dev = torch.device("cuda", 0)
    O = torch.zeros(B, net.out_row, device=dev)
    G = torch.zeros(B, net.grad_row, device=dev)
    net.forward(X.view(B, -1).to(dev), O, G)
    ctx.synchronize()
    P = _unpack(net.get_params(), N)
    Or, Gr = ref_forward(P, X.float())
    for got, ref in ((O.cpu(), Or), (G.cpu()[:, :net.panels], Gr)):
        scale = ref.abs().max().item()
        assert (got - ref).abs().max().item() <= 2e-2 * scale


@pytest.mark.parametrize("B,N", [(64, 16), (512, 16), (96, 21), (96, 23)])
def test_backward_matches_autograd(ctx, B, N):
    import torch
    net = engine.Net(seed=5, ctx=ctx, N=N)
    NP = net.panels
    X = _inputs(B, 2, N)
    g = torch.Generator().manual_seed(0)
    T = torch.rand(B, NP, generator=g) ** 4
    T = T / T.sum(1, keepdim=True)
    TG = torch.randn(B, NP, generator=g) * 0.1
    dev = torch.device("cuda", 0)
    loss = net.train_step(X.view(B, -1).to(dev), T.to(dev), TG.to(dev), lr=0.0, apply=False,
                          w_conf=0.1, w_grad=1.0)
    grads = net.gradients()
    P = _unpack(net.get_params(), N)
    Pt = {k: v.clone().requires_grad_(True) for k, v in P.items()}
    O, G = ref_forward(Pt, X.float(), round_act=False)
    logs = torch.log_softmax(O[:, :NP], dim=1)
    ce = -(T * logs).sum(1).mean()
    kl = (T * (torch.log(T.clamp_min(1e-30)) - logs)).sum(1)
    cstar = torch.log10(kl.detach().clamp_min(0) + 1e-8)
    conf = ((O[:, NP] - cstar) ** 2).mean()
    gm = ((G - TG) ** 2).mean()
    total = ce + 0.1 * conf + 1.0 * gm
    total.backward()
    assert abs(loss[0] - ce.item()) <= 1e-2 * abs(ce.item())
    lay, _ = engine._param_layout(N)
    for k in ("w1", "b1", "w2", "b2", "w3", "b3", "wd", "bd", "wg", "bg"):
        o, n = lay[k]
        gd = torch.from_numpy(grads[o:o + n])
        gr = Pt[k].grad.reshape(-1)
        if k in ("wd", "bd"):  # rows past the confidence output carry no gradient
            m = (NP + 1) * (net.features if k == "wd" else 1)
            gd, gr = gd[:m], gr[:m]
        rel = (gd - gr).norm().item() / max(gr.norm().item(), 1e-12)
        assert rel < 5e-2, (k, rel)


def test_training_reduces_loss(ctx):
    import torch
    from oracle import oracle as O  # the FDM oracle provides the targets
    net = engine.Net(seed=7, ctx=ctx)
    B = 128
    eps, _ = W.fdm_cubes(B, 16, seed=11)
    T, _, _ = O.fdm_solve_batch(eps, 0, tol=1e-10)
    x = eps / eps.reshape(B, -1).max(axis=1)[:, None, None, None]
    dev = torch.device("cuda", 0)
    X = torch.from_numpy(x.astype(np.float32)).to(torch.bfloat16).view(B, -1).to(dev)
    Tt = torch.from_numpy(T.astype(np.float32)).to(dev)
    ent = float(-(T * np.log(np.clip(T, 1e-30, None))).sum(1).mean())
    first = net.train_step(X, Tt, None, lr=1e-3)[0] - ent   # KL = CE - H(T)
    for _ in range(150):
        last = net.train_step(X, Tt, None, lr=1e-3)[0] - ent
    assert last < 0.5 * first, (first, last)
