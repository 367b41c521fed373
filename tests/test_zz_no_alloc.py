"""The no-allocation FDM entry point (drwc_fdm_solve_noalloc), for callers
that cannot allocate device memory when they call the library (an
application whose own pool holds all GPU memory, or a loop that must not
meet cudaMalloc's implicit synchronisation). Checked through the C ABI
against the regular batched entry point on the same cubes, on two calls in a
row per case (the second call reuses the static scratch the first one left
behind), with and without warm starts, with more cubes than resident CTAs
(each CTA then solves several cubes in one call), and with the device's free
memory unchanged across a call. Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

from deeprwcap_b200 import abi, engine
from deeprwcap_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-6  # same bar as the other FDM parity tests


def _regular(ctx, eps_dev, N, n, codes_host, opts, out_dev):
    Ns = np.full(n, N, dtype=np.int32)
    eoff = (np.arange(n, dtype=np.int64) * N ** 3)
    ooff = (np.arange(n, dtype=np.int64) * 6 * N * N)
    rc = ctx.lib.drwc_fdm_solve_batch_device(ctx.h, n, Ns.ctypes.data, eoff.ctypes.data,
                                             eps_dev.data_ptr(), codes_host.ctypes.data,
                                             C.byref(opts), ooff.ctypes.data, out_dev.data_ptr(),
                                             None, None, None, None)
    assert rc == 0
    ctx.synchronize()


# (N, cubes, warm start): 300 cubes at N = 23 is more than the 114 CTAs the
# static scratch holds at that size
CASES = [(16, 37, 1), (23, 300, 1), (5, 37, 1), (16, 37, 0)]


@pytest.mark.parametrize("N,n,warm", CASES)
def test_noalloc_matches_regular_entry_point(N, n, warm):
    import torch
    ctx = engine.default_context(0)
    eps, _ = W.fdm_cubes(n, N, seed=4000 + N, noise_frac=0.2)
    codes = (np.arange(n) % 4).astype(np.int32)
    dev = torch.device("cuda", 0)
    eps_dev = torch.from_numpy(eps.reshape(-1).copy()).to(dev)
    code_dev = torch.from_numpy(codes).to(dev)
    opts = abi.FdmOpts(1e-10, 1e-5, 8, 0, warm)
    ref = torch.zeros(n * 6 * N * N, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    _regular(ctx, eps_dev, N, n, codes, opts, ref)
    ref = ref.cpu().numpy().reshape(n, -1)
    outs = [torch.full((n * 6 * N * N,), float("nan"), dtype=torch.float64, device=dev)
            for _ in range(2)]
    iters = [torch.full((n,), -1, dtype=torch.int32, device=dev) for _ in range(2)]
    status = [torch.full((n,), -1, dtype=torch.int32, device=dev) for _ in range(2)]
    torch.cuda.synchronize()  # buffers filled before the library's stream uses them
    for call in range(2):
        free0 = torch.cuda.mem_get_info(0)[0]
        rc = ctx.lib.drwc_fdm_solve_noalloc(ctx.h, N, n, eps_dev.data_ptr(), code_dev.data_ptr(),
                                            C.byref(opts), outs[call].data_ptr(),
                                            iters[call].data_ptr(), status[call].data_ptr())
        assert rc == 0, (call, rc)
        ctx.synchronize()
        free1 = torch.cuda.mem_get_info(0)[0]
        assert free1 == free0, (call, free0, free1)  # nothing allocated by the call
        assert (status[call].cpu().numpy() == 0).all()
        it = iters[call].cpu().numpy()
        assert (it >= 0).all()
        got = outs[call].cpu().numpy().reshape(n, -1)
        for c in range(n):
            err = np.linalg.norm(got[c] - ref[c]) / np.linalg.norm(ref[c])
            assert err < TOL, (N, call, c, err)
    # both calls did the same work
    assert np.array_equal(iters[0].cpu().numpy(), iters[1].cpu().numpy())
    if not warm:
        assert (iters[0].cpu().numpy() > 0).all()


def test_noalloc_rejects_unsupported_size():
    ctx = engine.default_context(0)
    rc = ctx.lib.drwc_fdm_solve_noalloc(ctx.h, abi.N_MAX + 1, 1, None, None, None, None, None,
                                        None)
    assert rc == 1


def test_noalloc_flags_unknown_solver_code():
    import torch
    ctx = engine.default_context(0)
    N, n = 8, 3
    eps, _ = W.fdm_cubes(n, N, seed=11)
    dev = torch.device("cuda", 0)
    eps_dev = torch.from_numpy(eps.reshape(-1).copy()).to(dev)
    code_dev = torch.tensor([0, 7, -1], dtype=torch.int32, device=dev)
    out = torch.full((n * 6 * N * N,), float("nan"), dtype=torch.float64, device=dev)
    status = torch.full((n,), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    rc = ctx.lib.drwc_fdm_solve_noalloc(ctx.h, N, n, eps_dev.data_ptr(), code_dev.data_ptr(),
                                        None, out.data_ptr(), None, status.data_ptr())
    assert rc == 0
    ctx.synchronize()
    assert status.cpu().tolist() == [0, 2, 2]
    got = out.cpu().numpy().reshape(n, -1)
    assert np.isfinite(got[0]).all() and abs(got[0].sum() - 1.0) < 1e-8
    assert (got[1:] == 0).all()
