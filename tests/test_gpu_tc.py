"""Operator products on the tensor pipe (zb_operator_mm_tf32x3, tcgen05 MMAs
with TF32x3 split products) against FP64 products of the same FP32 inputs.

The shapes are the reference's own operator products (src/elements.cpp:
1337-1501): extrapolation, differentiation and divergence operators of
triangles P4 and hexahedra P3 applied to n = elements x variables columns,
with n not a multiple of the 128 columns a CTA takes, padded leading
dimensions, and beta = 1 accumulation.  TF32x3 keeps about 21 bits of each
operand, so the bound is 2e-6 of the largest |A| |B| column sum.
"""
import ctypes

import numpy as np
import pytest

from zefr_b200 import _lib

pytestmark = pytest.mark.gpu

_FP = ctypes.POINTER(ctypes.c_float)


def _mm(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    st = _lib.lib().zb_operator_mm_tf32x3(m, n, k, alpha, ctypes.cast(A.data_ptr(), _FP), lda,
                                          ctypes.cast(B.data_ptr(), _FP), ldb, beta,
                                          ctypes.cast(C.data_ptr(), _FP), ldc, None)
    assert st == 0, _lib.lib().zb_last_error().decode()
    import torch
    torch.cuda.synchronize()


@pytest.mark.parametrize("m,k,n", [(15, 15, 4 * 1000 + 3),     # triangle P4 oppE
                                   (30, 15, 4 * 777),          # triangle P4 oppD (2 dims stacked)
                                   (15, 30, 4 * 513),          # triangle P4 oppDiv
                                   (96, 64, 5 * 301),          # hexahedron P3 oppE
                                   (192, 64, 5 * 64),          # hexahedron P3 oppD
                                   (64, 192, 5 * 130),         # hexahedron P3 oppDiv
                                   (16, 16, 128),              # one CTA pass exactly
                                   (1, 1, 7)])                 # smallest
def test_operator_product_matches_fp64(m, k, n):
    import torch
    g = torch.Generator().manual_seed(m * 1000 + k)
    A = torch.randn(m, k, generator=g, dtype=torch.float64)
    B = torch.randn(k, n, generator=g, dtype=torch.float64)
    lda, ldb, ldc = k + 3, n + 5, n + 1
    Ad = torch.zeros(m, lda, dtype=torch.float32)
    Ad[:, :k] = A.float()
    Bd = torch.zeros(k, ldb, dtype=torch.float32)
    Bd[:, :n] = B.float()
    Ad, Bd = Ad.cuda(), Bd.cuda()
    C = torch.full((m, ldc), float("nan"), dtype=torch.float32, device="cuda")
    _mm(m, n, k, 1.0, Ad, lda, Bd, ldb, 0.0, C, ldc)
    ref = Ad[:, :k].double().cpu() @ Bd[:, :n].double().cpu()
    got = C[:, :n].double().cpu()
    scale = (Ad[:, :k].double().abs().cpu() @ Bd[:, :n].double().abs().cpu()).max()
    assert torch.isfinite(got).all()
    assert (got - ref).abs().max() <= 2e-6 * scale
    # columns beyond n are untouched
    assert torch.isnan(C[:, n:]).all()
    # alpha and beta: C = 2 A B - 0.5 C
    C2 = C.clone()
    C2[:, n:] = 0
    _mm(m, n, k, 2.0, Ad, lda, Bd, ldb, -0.5, C2, ldc)
    want = 2.0 * ref - 0.5 * got
    assert (C2[:, :n].double().cpu() - want).abs().max() <= 5e-6 * scale


def test_operator_product_beats_plain_tf32_precision():
    """The split products are far more accurate than one TF32 product would
    be (10-bit operands): the error is below 1e-5 of plain TF32's bound."""
    import torch
    g = torch.Generator().manual_seed(5)
    m, k, n = 96, 64, 5 * 256
    A = torch.randn(m, k, generator=g).cuda()
    B = torch.randn(k, n, generator=g).cuda()
    C = torch.empty(m, n, device="cuda")
    _mm(m, n, k, 1.0, A, k, B, n, 0.0, C, n)
    ref = A.double() @ B.double()
    err = (C.double() - ref).abs().max().item()
    scale = (A.double().abs() @ B.double().abs()).max().item()
    assert err <= 1e-6 * scale   # plain TF32 would sit near 2^-11 ~ 5e-4 of scale


def test_operator_product_rejects_bad_shapes():
    import torch
    A = torch.zeros(300, 4, device="cuda")
    B = torch.zeros(4, 10, device="cuda")
    C = torch.zeros(300, 10, device="cuda")
    st = _lib.lib().zb_operator_mm_tf32x3(300, 10, 4, 1.0, ctypes.cast(A.data_ptr(), _FP), 4,
                                          ctypes.cast(B.data_ptr(), _FP), 10, 0.0,
                                          ctypes.cast(C.data_ptr(), _FP), 10, None)
    assert st != 0 and "256" in _lib.lib().zb_last_error().decode()
    st = _lib.lib().zb_operator_mm_tf32x3(4, 10, 4, 1.0, ctypes.cast(A.data_ptr(), _FP), 2,
                                          ctypes.cast(B.data_ptr(), _FP), 10, 0.0,
                                          ctypes.cast(C.data_ptr(), _FP), 10, None)
    assert st == -1  # lda < k
