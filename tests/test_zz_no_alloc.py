"""The no-allocation FDM entry point (drwc_fdm_solve_noalloc), for callers
that cannot allocate device memory when they call the library: checked
through the C ABI against the regular batched entry point on the same cubes,
on two calls in a row per resolution (the second call reuses the static
scratch the first one left behind). Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

from deeprwcap_b200 import abi, engine
from deeprwcap_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-6  # same bar as the other FDM parity tests


def _regular(ctx, eps_dev, N, n, codes_host, out_dev, torch):
    Ns = np.full(n, N, dtype=np.int32)
    eoff = (np.arange(n, dtype=np.int64) * N ** 3)
    ooff = (np.arange(n, dtype=np.int64) * 6 * N * N)
    opts = abi.FdmOpts(1e-10, 1e-5, 8, 0)
    rc = ctx.lib.drwc_fdm_solve_batch_device(ctx.h, n, Ns.ctypes.data, eoff.ctypes.data,
                                             eps_dev.data_ptr(), codes_host.ctypes.data,
                                             C.byref(opts), ooff.ctypes.data, out_dev.data_ptr(),
                                             None, None, None, None)
    assert rc == 0
    ctx.synchronize()


@pytest.mark.parametrize("N", (16, 23, 5))
def test_noalloc_matches_regular_entry_point(N):
    import torch
    ctx = engine.default_context(0)
    n = 37
    eps, _ = W.fdm_cubes(n, N, seed=4000 + N, noise_frac=0.2)
    codes = (np.arange(n) % 4).astype(np.int32)
    dev = torch.device("cuda", 0)
    eps_dev = torch.from_numpy(eps.reshape(-1).copy()).to(dev)
    code_dev = torch.from_numpy(codes).to(dev)
    ref = torch.zeros(n * 6 * N * N, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    _regular(ctx, eps_dev, N, n, codes, ref, torch)
    ref = ref.cpu().numpy().reshape(n, -1)
    opts = abi.FdmOpts(1e-10, 1e-5, 8, 0)
    for call in range(2):
        out = torch.full((n * 6 * N * N,), float("nan"), dtype=torch.float64, device=dev)
        iters = torch.full((n,), -1, dtype=torch.int32, device=dev)
        status = torch.full((n,), -1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()  # buffers filled before the library's stream uses them
        rc = ctx.lib.drwc_fdm_solve_noalloc(ctx.h, N, n, eps_dev.data_ptr(), code_dev.data_ptr(),
                                            C.byref(opts), out.data_ptr(), iters.data_ptr(),
                                            status.data_ptr())
        assert rc == 0, (call, rc)
        ctx.synchronize()
        assert (status.cpu().numpy() == 0).all()
        assert (iters.cpu().numpy() > 0).all()
        got = out.cpu().numpy().reshape(n, -1)
        for c in range(n):
            err = np.linalg.norm(got[c] - ref[c]) / np.linalg.norm(ref[c])
            assert err < TOL, (N, call, c, err)


def test_noalloc_rejects_unsupported_size():
    ctx = engine.default_context(0)
    rc = ctx.lib.drwc_fdm_solve_noalloc(ctx.h, abi.N_MAX + 1, 1, None, None, None, None, None,
                                        None)
    assert rc == 1
