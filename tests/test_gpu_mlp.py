"""The learned warm start's building block: the tcgen05 BF16 GEMM (TMEM accumulator), through
the C ABI, against torch's FP32 product of the same BF16 operands.

Tolerance: the BF16 products are exact in FP32; only the FP32 summation order differs, so the
results agree to ~K x 2^-24 relative; 1e-4 relative to the output scale is used.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bpf():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import blockpowerflow_b200 as bpf

    return bpf


def _gemm(bpf, A, B, D=None, accumulate=False, splits=0):
    import torch

    M, K = A.shape
    N = B.shape[0]
    if D is None:
        D = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    lib = bpf._lib.load()
    ctx = bpf._lib.context(0)
    bpf._lib.check(lib.bpf_tc_gemm_bf16(ctx, M, N, K, A.data_ptr(), A.stride(0), B.data_ptr(),
                                        B.stride(0), D.data_ptr(), D.stride(0), int(accumulate),
                                        splits), ctx)
    torch.cuda.synchronize()
    return D


@pytest.mark.parametrize("M,N,K,splits", [(128, 128, 64, 1), (256, 384, 512, 1), (300, 200, 640, 1),
                                          (128, 128, 4096, 8), (512, 128, 8192, 0), (130, 8, 128, 0)])
def test_tc_gemm_matches_fp32_product(bpf, M, N, K, splits):
    import torch

    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    A = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    D = _gemm(bpf, A, B, splits=splits)
    ref = A.float() @ B.float().t()
    err = (D - ref).abs().max().item() / ref.abs().max().item()
    assert err <= 1e-4, err


def test_tc_gemm_accumulates(bpf):
    import torch

    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn((256, 256), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((128, 256), generator=g, device="cuda").to(torch.bfloat16)
    D0 = torch.randn((256, 128), generator=g, device="cuda")
    D = _gemm(bpf, A, B, D=D0.clone(), accumulate=True)
    ref = D0 + A.float() @ B.float().t()
    assert (D - ref).abs().max().item() <= 1e-4 * ref.abs().max().item()


def test_tc_gemm_rejects_unaligned_k(bpf):
    import torch

    A = torch.zeros((128, 96), dtype=torch.bfloat16, device="cuda")
    B = torch.zeros((128, 96), dtype=torch.bfloat16, device="cuda")
    D = torch.zeros((128, 128), dtype=torch.float32, device="cuda")
    lib = bpf._lib.load()
    ctx = bpf._lib.context(0)
    st = lib.bpf_tc_gemm_bf16(ctx, 128, 128, 96, A.data_ptr(), 96, B.data_ptr(), 96, D.data_ptr(), 128, 0, 1)
    assert st == bpf._lib.BPF_ERR_INVALID_VALUE
