"""GPU checks of the tcgen05 BF16 GEMM (tensor memory accumulator) against an
FP32 reference of the same op on the same BF16 inputs.
Tolerance: 1e-3 relative to the largest |C| (FP32 accumulation; inputs are
exactly representable BF16)."""
import numpy as np
import pytest

from deeprwcap_b200 import engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (1, 16, 16), (200, 48, 27), (300, 130, 200),
                                   (513, 256, 512), (64, 1664, 512), (4096, 32, 432)])
@pytest.mark.parametrize("act", [0, 1])
def test_gemm_bf16_matches_fp32_reference(ctx, M, N, K, act):
    import torch
    dev = torch.device("cuda", 0)
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    bias = torch.randn(N, generator=g)
    ref = A.float() @ B.float().T + bias
    if act:
        ref = ref.clamp_min(0)
    Ad, Bd, bd = A.to(dev), B.to(dev), bias.to(dev)
    C = torch.full((M, N), float("nan"), device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()  # buffers ready before the library's stream runs
    rc = ctx.lib.drwc_gemm_bf16(ctx.h, M, N, K, Ad.data_ptr(), K, Bd.data_ptr(), K, C.data_ptr(),
                                N, bd.data_ptr(), act, err.data_ptr())
    assert rc == 0
    ctx.synchronize()
    assert err.item() == 0
    got = C.cpu()
    scale = ref.abs().max().item()
    assert torch.isfinite(got).all()
    assert (got - ref).abs().max().item() <= 1e-3 * scale
