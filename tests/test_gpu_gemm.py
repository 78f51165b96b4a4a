"""The tcgen05 BF16 GEMM against a plain PyTorch fp32 reference of the same op (the
operands are exactly representable in bf16, so only the fp32 summation order differs)."""
import numpy as np
import pytest

import rfdem

pytestmark = pytest.mark.gpu


def _bf16(torch, shape, seed, scale=1.0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(*shape, generator=g) * scale).to(torch.bfloat16).cuda()


def _call(torch, A, B, M, N, K, mode, bias=None, mask=None, out_h=None, out_ht=None, out_f=None, ncols_f=0,
          scale=1.0, splits=1):
    p = lambda t: None if t is None else t.data_ptr()
    st = rfdem.lib.rf_gemm_bf16(p(A), A.stride(0), p(B), B.stride(0), M, N, K, mode, p(bias), p(mask),
                                mask.stride(0) if mask is not None else 0, p(out_h),
                                out_h.stride(0) if out_h is not None else 0, p(out_ht),
                                out_ht.stride(0) if out_ht is not None else 0, p(out_f),
                                out_f.stride(0) if out_f is not None else 0, ncols_f, scale, splits, None)
    rfdem.check(st, "rf_gemm_bf16")
    torch.cuda.synchronize()
    rfdem.check(rfdem.lib.rf_gemm_status(None), "rf_gemm_status")


def _tol(A, B):
    return 1e-5 * (A.float().abs() @ B.float().abs().t()) + 1e-6


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (300, 128, 64), (1000, 256, 200), (77, 48, 16), (4096, 128, 128)])
def test_gemm_linear_f32(cuda, M, N, K):
    torch = cuda
    A = _bf16(torch, (M, K), M + K)
    B = _bf16(torch, (N, K), N + 3 * K)
    bias = torch.randn(N, generator=torch.Generator().manual_seed(5)).cuda()
    out = torch.zeros(M, N, device="cuda")
    _call(torch, A, B, M, N, K, rfdem.RF_EPI_LINEAR_F32, bias=bias, out_f=out, ncols_f=N)
    ref = A.float() @ B.float().t() + bias
    assert torch.all((out - ref).abs() <= _tol(A, B)), (out - ref).abs().max().item()


def test_gemm_relu_transpose_and_mask(cuda):
    torch = cuda
    M, N, K = 513, 128, 64
    A = _bf16(torch, (M, K), 1)
    B = _bf16(torch, (N, K), 2)
    bias = torch.randn(N, generator=torch.Generator().manual_seed(3)).cuda()
    h = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    ht = torch.zeros(N, 520, dtype=torch.bfloat16, device="cuda")
    _call(torch, A, B, M, N, K, rfdem.RF_EPI_RELU_BF16, bias=bias, out_h=h, out_ht=ht)
    ref = torch.relu(A.float() @ B.float().t() + bias)
    assert torch.allclose(h.float(), ref, rtol=1e-2, atol=1e-2)
    assert torch.equal(ht[:, :M].t(), h)
    # ReLU backward: keep acc where the mask is positive
    dz = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    _call(torch, A, B, M, N, K, rfdem.RF_EPI_MASK_BF16, mask=h, out_h=dz)
    refm = (A.float() @ B.float().t()) * (h.float() > 0)
    assert torch.allclose(dz.float(), refm, rtol=1e-2, atol=1e-2)


def test_gemm_splitk_atomic(cuda):
    torch = cuda
    M, N, K = 128, 128, 4096            # a weight-gradient shape: K runs over particles
    A = _bf16(torch, (M, K), 11)
    B = _bf16(torch, (N, K), 12)
    out = torch.zeros(M, N, device="cuda")
    _call(torch, A, B, M, N, K, rfdem.RF_EPI_ATOMIC_F32, out_f=out, ncols_f=N, scale=0.5, splits=16)
    ref = 0.5 * (A.float() @ B.float().t())
    assert torch.all((out - ref).abs() <= 0.5 * _tol(A, B) + 1e-4), (out - ref).abs().max().item()
