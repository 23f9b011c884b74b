"""Split-precision product (qd_gemm_split, tcgen05 BF16 slices with FP32
accumulation, FP64 sum) against the FP64 product of the same inputs.

Bars: with 8 slices the result is FP64-accurate (normwise 1e-13 relative to
|A| |B|); with S slices the error is below 2^(-7S) * 8 of the same scale;
integer-valued inputs (|x| <= 127, one slice each) give exact products, which
pins the exactness of the FP32 tensor-core accumulation over whole K chunks."""
import numpy as np
import pytest
import torch

import qd_imsrg_b200 as qd

pytestmark = pytest.mark.gpu


def _ref(A, B, ta, tb):
    a = A.T if ta else A
    b = B.T if tb else B
    return a @ b, a.abs() @ b.abs()


def _mats(m, n, k, ta, tb, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn((k, m) if ta else (m, k), generator=g, dtype=torch.float64, device="cuda")
    B = torch.randn((n, k) if tb else (k, n), generator=g, dtype=torch.float64, device="cuda")
    return A, B


@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (300, 200, 1000), (17, 5, 3), (1264, 16, 1264), (160, 1264, 160)])
@pytest.mark.parametrize("ta,tb", [(False, False), (True, False), (False, True), (True, True)])
def test_fp64_accuracy_at_8_slices(m, n, k, ta, tb):
    A, B = _mats(m, n, k, ta, tb, seed=m * 7 + n + k)
    C = qd.gemm_split(A, B, trans_a=ta, trans_b=tb, slices=8)
    ref, scale = _ref(A, B, ta, tb)
    err = ((C - ref).abs() / scale.clamp_min(1e-300)).max().item()
    assert err < 1e-13, err


@pytest.mark.parametrize("slices", [1, 2, 3, 4, 5, 6, 7, 8])
def test_error_follows_slice_count(slices):
    A, B = _mats(257, 130, 700, False, True, seed=3)
    # rows and columns of very different magnitude: the per-row scaling keeps
    # the relative accuracy of each row
    A *= torch.logspace(-6, 6, A.shape[0], dtype=torch.float64, device="cuda")[:, None]
    B *= torch.logspace(3, -3, B.shape[0], dtype=torch.float64, device="cuda")[:, None]
    C = qd.gemm_split(A, B, trans_b=True, slices=slices)
    ref, scale = _ref(A, B, False, True)
    err = ((C - ref).abs() / scale).max().item()
    assert err < max(8.0 * 2.0 ** (-7 * slices), 5e-14), (slices, err)


@pytest.mark.parametrize("k", [64, 640, 3000])
def test_integer_products_exact(k):
    g = torch.Generator(device="cuda").manual_seed(k)
    A = torch.randint(-127, 128, (192, k), generator=g, device="cuda").double()
    B = torch.randint(-127, 128, (k, 96), generator=g, device="cuda").double()
    A[:, 0] = 127.0  # every row and column reaches the slice range, so one slice is exact
    B[0, :] = -127.0
    C = qd.gemm_split(A, B, slices=1)
    ref = A @ B  # exact: |sums| < 2^53
    assert torch.equal(C, ref)
    # all-extreme values: the largest partial sums a K chunk can hold
    A2 = torch.full((128, k), 127.0, dtype=torch.float64, device="cuda")
    B2 = torch.full((k, 64), 127.0, dtype=torch.float64, device="cuda")
    assert torch.equal(qd.gemm_split(A2, B2, slices=1), A2 @ B2)


def test_alpha_beta_and_accumulate():
    A, B = _mats(200, 70, 90, False, False, seed=11)
    C0 = torch.randn(200, 70, dtype=torch.float64, device="cuda")
    C = C0.clone()
    qd.gemm_split(A, B, C, alpha=-2.5, beta=0.5, slices=8)
    ref = -2.5 * (A @ B) + 0.5 * C0
    assert torch.allclose(C, ref, rtol=1e-13, atol=1e-12)
    Z = qd.gemm_split(A[:, :0].contiguous(), B[:0, :].contiguous(), slices=3)  # K = 0
    assert torch.count_nonzero(Z).item() == 0


def test_bad_arguments():
    with pytest.raises(qd.QDError):
        qd._native.check(qd._native.lib().qd_gemm_split(0, None, b"X", b"N", 4, 4, 4, 1.0, None, 4, None, 4, 0.0,
                                                        None, 4, 4))
    A, B = _mats(8, 8, 8, False, False, seed=1)
    with pytest.raises(qd.QDError):
        qd.gemm_split(A, B, slices=9)
