"""The surrogate's tensor-core kernels: the tcgen05 GEMM against an FP32
matrix product of the same BF16 inputs, and its epilogues."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (256, 16, 64), (512, 128, 256), (256, 64, 4096),
                                   (128, 48, 128), (384, 256, 256)])
def test_umma_gemm_matches_fp32_product(M, N, K):
    import torch
    from dense_b200.surrogate import Kernels
    k = Kernels()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    D = torch.full((M, N), float("nan"), device="cuda")
    k.gemm(A, B, D)
    k.check()
    ref = A.float() @ B.float().T
    err = (D - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-5, err


def test_umma_gemm_bias_gelu_epilogue():
    import torch
    from dense_b200.surrogate import EPI_BIAS, EPI_BIAS_GELU, Kernels
    k = Kernels()
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(256, 128, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(96, 128, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(96, device="cuda", generator=g)
    Z = torch.empty(256, 96, device="cuda")
    H = torch.empty(256, 96, device="cuda", dtype=torch.bfloat16)
    k.gemm(A, B, Z, EPI_BIAS_GELU, bias, H)
    Y = torch.empty(256, 96, device="cuda")
    k.gemm(A, B, Y, EPI_BIAS, bias)
    k.check()
    ref = A.float() @ B.float().T + bias
    assert (Z - ref).abs().max().item() < 1e-3
    assert (Y - ref).abs().max().item() < 1e-3
    gelu = torch.nn.functional.gelu(ref)
    assert (H.float() - gelu).abs().max().item() < 2e-2 * max(1.0, gelu.abs().max().item())
