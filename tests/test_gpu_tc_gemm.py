"""The surrogate's tensor-core GEMM (tcgen05, BF16 operands, FP32 in tensor
memory) against a torch FP32 matmul of the same BF16-rounded operands.

Tolerance: max |C - C_ref| <= 1e-3 * max |C_ref| + 1e-5 (FP32 accumulation in
a different order; operands are exactly representable).
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(200, 32, 32), (128, 256, 32), (300, 256, 256), (1000, 32, 256), (257, 64, 1408),
          (130, 1408, 32), (4096, 256, 256)]


@pytest.mark.parametrize("M,N,K", SHAPES)
@pytest.mark.parametrize("act", [0, 1])
def test_tc_gemm_matches_fp32(M, N, K, act):
    import torch
    from peridem_b200 import api
    L = api.lib()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = (torch.randn(N, K, device="cuda", generator=g) / K ** 0.5).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    Cf = torch.full((M, N), float("nan"), device="cuda")
    Cb = torch.empty((M, N), device="cuda", dtype=torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.pdgpu_tc_gemm(A.data_ptr(), K, B.data_ptr(), K, M, N, K, bias.data_ptr(), act,
                         Cf.data_ptr(), Cb.data_ptr(), N, err.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0, "tensor-core wait timed out"
    ref = A.float() @ B.float().t() + bias
    if act == 1:
        ref = torch.tanh(ref)
    scale = float(ref.abs().max())
    e = float((Cf - ref).abs().max())
    print(f"M={M} N={N} K={K} act={act}: max err {e:.3e} (scale {scale:.3e})")
    assert e <= 1e-3 * scale + 1e-5
    eb = float((Cb.float() - ref).abs().max())
    assert eb <= 1e-2 * scale + 1e-3
