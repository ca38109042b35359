"""tcgen05 BF16 GEMM (umma_gemm.cu) against an FP32 reference on the same
BF16-rounded operands: |C - C_ref| <= 2e-3 (|A| |B|^T)_max (FP32 accumulation
order only), plus the epilogue (bias, beta accumulation, GELU, BF16 output)."""
from __future__ import annotations

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def run(fd, A, B, bias=None, act=0, alpha=1.0, beta=0.0, C32=None, want16=False, Z=False):
    M, K = A.shape
    N = B.shape[0]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    C32 = C32 if C32 is not None else torch.zeros(M, N, dtype=torch.float32, device="cuda")
    C16 = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda") if want16 else None
    Z32 = torch.zeros(M, N, dtype=torch.float32, device="cuda") if Z else None
    fd.call("fdtd_gemm_bf16", A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K,
            bias.data_ptr() if bias is not None else None, act, alpha, beta, C32.data_ptr(), C32.stride(0),
            C16.data_ptr() if C16 is not None else None, N, Z32.data_ptr() if Z32 is not None else None, N,
            err.data_ptr(), None)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return C32, C16, Z32


def rand_bf16(*shape, seed=0):
    g = torch.Generator().manual_seed(seed)
    return torch.randn(*shape, generator=g).to(torch.bfloat16)


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K", [(128, 32, 32), (128, 256, 64), (200, 22, 256), (4096, 256, 32),
                                   (256, 256, 4096), (300, 100, 40), (77, 130, 24)])
def test_gemm_matches_fp32_reference(fd, gpu, M, N, K):
    A, B = rand_bf16(M, K, seed=M + K), rand_bf16(N, K, seed=N + 7 * K)
    ref = A.float() @ B.float().T
    C32, _, _ = run(fd, A.cuda(), B.cuda())
    scale = (A.float().abs() @ B.float().abs().T).max().item()
    assert (C32.cpu() - ref).abs().max().item() <= 2e-3 * scale


@pytest.mark.gpu
def test_gemm_epilogue(fd, gpu):
    M, N, K = 260, 48, 64
    A, B = rand_bf16(M, K, seed=1), rand_bf16(N, K, seed=2)
    bias = torch.randn(N, generator=torch.Generator().manual_seed(3))
    C0 = torch.randn(M, N, generator=torch.Generator().manual_seed(4))
    C32, C16, Z = run(fd, A.cuda(), B.cuda(), bias.cuda(), act=1, alpha=0.5, beta=2.0, C32=C0.clone().cuda(),
                      want16=True, Z=True)
    pre = 0.5 * (A.float() @ B.float().T) + 2.0 * C0 + bias
    post = 0.5 * pre * (1 + torch.erf(pre / math.sqrt(2)))
    scale = (A.float().abs() @ B.float().abs().T).max().item()
    assert (Z.cpu() - pre).abs().max().item() <= 2e-3 * scale
    assert (C32.cpu() - post).abs().max().item() <= 2e-3 * scale
    assert (C16.float().cpu() - post).abs().max().item() <= 1e-2 * post.abs().max().item()


def test_gemm_rejects_unaligned_k(fd):
    r = fd.lib.fdtd_gemm_bf16(None, 10, None, 10, 4, 4, 10, None, 0, 1.0, 0.0, None, 4, None, 4, None, 4, None, None)
    assert r in (fd.FDTD_ERR_ARG, fd.FDTD_ERR_NO_DEVICE)
    fd.lib.fdtd_clear_error()
