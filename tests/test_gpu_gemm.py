"""The tcgen05 BF16 GEMM (bpx_gemm_bf16_dev) against a PyTorch FP32 product of the same BF16 operands.

Every operand orientation the network uses (K-major and MN-major A and B), tile widths 32..256,
and edges the tiles do not cover (M not a multiple of 128, K not a multiple of 64, N past the last
full tile).  Tolerance: FP32 accumulation of exact BF16 products differs from PyTorch's FP32 sum
only in summation order, so |C - C_ref| <= 1e-5 * sum_k |a_mk b_nk| + 1e-6.
"""
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


CASES = [
    # M, N, K, a_mn, b_mn
    (128, 256, 64, 0, 0),
    (300, 256, 288, 0, 0),
    (257, 32, 256, 0, 0),
    (4096, 256, 32, 0, 1),
    (256, 288, 1000, 1, 1),
    (32, 256, 777, 1, 1),
    (200, 96, 136, 1, 0),
    (136, 48, 72, 0, 1),
]


@pytest.mark.parametrize("M,N,K,a_mn,b_mn", CASES)
def test_gemm_matches_fp32_product(torch, M, N, K, a_mn, b_mn):
    from fdt_b200 import lib

    g = torch.Generator(device="cpu").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn((M, K), generator=g).to(torch.bfloat16)
    B = torch.randn((N, K), generator=g).to(torch.bfloat16)
    a = (A.t().contiguous() if a_mn else A).cuda()
    b = (B.t().contiguous() if b_mn else B).cuda()
    c = lib.gemm_bf16(a, b, M, N, K, a_mn=bool(a_mn), b_mn=bool(b_mn))
    torch.cuda.synchronize()
    assert lib.poll_error() == 0
    Af, Bf = A.float(), B.float()
    ref = Af @ Bf.t()
    bound = 1e-5 * (Af.abs() @ Bf.abs().t()) + 1e-6
    err = (c.cpu() - ref).abs()
    assert bool((err <= bound).all()), f"max err {err.max().item()} (bound {bound.max().item()})"
