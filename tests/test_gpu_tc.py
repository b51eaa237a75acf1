"""Tensor-core building block of the mixed-precision form (tcgen05, sm_100a).

``afr_tc_check`` runs one CTA through the shared-memory layout, descriptors and
waits the mixed-precision kernels use; the products are checked against exact
float64 products of the same BF16 inputs, and the three-term hi+lo split
(hi*hi + hi*lo + lo*hi, written as one GEMM over a tripled K) against FP64
products of the unsplit FP32 inputs.
"""

import ctypes

import pytest
import torch

from autoflowcfd_b200 import _lib

pytestmark = pytest.mark.gpu


def _tc(a_bf16, b_bf16):
    n, k = b_bf16.shape
    d = torch.empty(128, n, dtype=torch.float32, device=a_bf16.device)
    _lib.check(_lib.LIB.afr_tc_check(n, k, ctypes.c_void_p(a_bf16.data_ptr()), ctypes.c_void_p(b_bf16.data_ptr()),
                                     ctypes.c_void_p(d.data_ptr()),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return d


@pytest.mark.parametrize("n,k", [(16, 16), (32, 64), (48, 32), (64, 192), (96, 96), (256, 256)])
def test_tc_bf16_gemm_exact_inputs(n, k):
    g = torch.Generator(device="cuda").manual_seed(1000 * n + k)
    a = torch.randn(128, k, device="cuda", generator=g).to(torch.bfloat16).contiguous()
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16).contiguous()
    d = _tc(a, b).double()
    ref = a.double() @ b.double().T
    scale = a.double().abs() @ b.double().abs().T
    # FP32 accumulation of k exact BF16 products: k * 2^-24 relative to sum |a||b|
    assert ((d - ref).abs() <= k * 6e-8 * scale + 1e-30).all(), float(((d - ref).abs() / scale).max())


def test_tc_hi_lo_split_product():
    g = torch.Generator(device="cuda").manual_seed(7)
    k = 64
    a = torch.randn(128, k, device="cuda", generator=g, dtype=torch.float64) * 1e3
    b = torch.randn(32, k, device="cuda", generator=g, dtype=torch.float64)
    a32, b32 = a.float(), b.float()
    ah = a32.to(torch.bfloat16)
    al = (a32 - ah.float()).to(torch.bfloat16)
    bh = b32.to(torch.bfloat16)
    bl = (b32 - bh.float()).to(torch.bfloat16)
    acat = torch.cat([ah, ah, al], dim=1).contiguous()
    bcat = torch.cat([bh, bl, bh], dim=1).contiguous()
    d = _tc(acat, bcat).double()
    ref = a32.double() @ b32.double().T
    scale = a32.double().abs() @ b32.double().abs().T
    rel = ((d - ref).abs() / scale).max().item()
    # each split factor carries 16 significant bits: about 3 * 2^-17 per product
    assert rel < 3e-5, rel
    # the single-term BF16 product is two orders worse, so the split is doing its job
    d1 = _tc(ah.contiguous(), bh.contiguous()).double()
    assert ((d1 - ref).abs() / scale).max().item() > 30 * rel
