"""The tensor-core building block (tcgen05 MMA, TMEM accumulator, K-major BF16
operands in shared memory) against torch FP32 matmul (GPU tests)."""
import pytest
import torch

from pbf_b200._lib import check, lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,k", [(16, 16), (64, 16), (16, 64), (64, 64), (80, 128), (32, 128), (256, 256)])
def test_tc_gemm_matches_fp32_matmul(n, k):
    g = torch.Generator(device="cuda").manual_seed(n * 1000 + k)
    a = (torch.rand(128, k, device="cuda", generator=g) * 2 - 1).to(torch.bfloat16)
    b = (torch.rand(n, k, device="cuda", generator=g) * 2 - 1).to(torch.bfloat16)
    d = torch.empty(128, n, device="cuda", dtype=torch.float32)
    check(lib().pbf_tc_gemm_bf16(a.data_ptr(), b.data_ptr(), d.data_ptr(), n, k, None))
    want = a.float() @ b.float().T
    err = (d - want).abs().max().item()
    assert err <= 1e-4 * k, err
