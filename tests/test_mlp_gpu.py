"""GPU tests of the tcgen05 BF16 GEMM (cib_mlp_gemm) against torch on the same bf16 inputs.

Tolerance: fp32 accumulation of exact bf16 products; compared with torch's fp32 matmul of
the same bf16 values at rtol 2e-5 of the largest |C| (bf16 outputs: one bf16 ulp, 2^-8).
"""

from __future__ import annotations

import pytest
import torch

from concrete_impact_b200 import mlp

pytestmark = pytest.mark.gpu

# the last two run the K pipeline through many slot reuses (65 and 128 chunks of 64)
SHAPES = [(1, 16, 16), (100, 16, 32), (128, 128, 128), (512, 128, 32), (1000, 32, 128), (300, 128, 256), (257, 64, 80),
          (129, 48, 4112), (256, 128, 8192)]


def _rand(m: int, k: int, seed: int) -> torch.Tensor:
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn((m, k), generator=g, device="cuda").to(torch.bfloat16)


def _err() -> torch.Tensor:
    return torch.zeros(1, dtype=torch.int32, device="cuda")


def _ref(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    return a.double() @ b.double().T


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_gemm_f32_and_bias(m: int, n: int, k: int) -> None:
    a, b = _rand(m, k, 1), _rand(n, k, 2)
    bias = torch.randn(n, device="cuda")
    err = _err()
    c = torch.full((m, n), float("nan"), device="cuda")
    mlp.gemm(mlp.EPI_F32, a, b, c=c, err=err)
    ref = _ref(a, b)
    scale = ref.abs().max().item()
    torch.testing.assert_close(c.double(), ref, rtol=0, atol=2e-5 * scale)
    mlp.gemm(mlp.EPI_BIAS_F32, a, b, c=c, bias=bias, err=err)
    torch.testing.assert_close(c.double(), ref + bias.double(), rtol=0, atol=2e-5 * scale)
    assert err.item() == 0


@pytest.mark.parametrize("m,n,k", [(512, 128, 32), (300, 128, 128), (129, 16, 128)])
def test_gemm_gelu_forward_and_backward_epilogues(m: int, n: int, k: int) -> None:
    a, b = _rand(m, k, 3), _rand(n, k, 4)
    bias = torch.randn(n, device="cuda")
    err = _err()
    z = torch.empty((m, n), device="cuda")
    h = torch.empty((m, n), dtype=torch.bfloat16, device="cuda")
    ht = torch.zeros((n, m + 5), dtype=torch.bfloat16, device="cuda")
    mlp.gemm(mlp.EPI_BIAS_GELU, a, b, bias=bias, z=z, h=h, ht=ht, row_offset=5, err=err)
    zref = _ref(a, b) + bias.double()
    scale = zref.abs().max().item()
    torch.testing.assert_close(z.double(), zref, rtol=0, atol=2e-5 * scale)
    href = torch.nn.functional.gelu(z).to(torch.bfloat16)
    assert torch.equal(h, href)
    assert torch.equal(ht[:, 5:], h.T)
    # backward epilogue: H = acc * gelu'(Z)
    dz = torch.empty((m, n), dtype=torch.bfloat16, device="cuda")
    mlp.gemm(mlp.EPI_GELU_BWD, a, b, z=z, h=dz, err=err)
    zz = z.clone().requires_grad_(True)
    grad = torch.autograd.grad(torch.nn.functional.gelu(zz).sum(), zz)[0]
    ref = (_ref(a, b).float() * grad).to(torch.bfloat16)
    torch.testing.assert_close(dz.float(), ref.float(), rtol=2 ** -7, atol=2e-5 * _ref(a, b).abs().max().item())
    assert err.item() == 0


@pytest.mark.parametrize("k,splits", [(2048, 8), (25600, 5)])
def test_gemm_split_k_partials_reduce_to_the_product(k: int, splits: int) -> None:
    m, n = 128, 128
    a, b = _rand(m, k, 5), _rand(n, k, 6)
    err = _err()
    partial = torch.empty((splits, m, n), device="cuda")
    mlp.gemm(mlp.EPI_PARTIAL, a, b, c=partial.view(splits * m, n), splits=splits, err=err)
    out = torch.empty((m, n), device="cuda")
    mlp.splitk_reduce(partial, splits, m, n, out)
    ref = _ref(a, b)
    torch.testing.assert_close(out.double(), ref, rtol=0, atol=2e-5 * ref.abs().max().item())
    assert err.item() == 0
