"""The allocation-free one-body norm, qd_mat_2_norm_noalloc.

It serves callers that must not allocate device memory while they run (for
example a host that reserves its device memory up front and forbids
allocation inside its flow loop): they pass the operator and a device scalar,
and the partial sums live in a fixed static device array.  Checked here,
through the C ABI, against the allocating qd_mat_2_norm on two calls in a
row, at the 1e-12 relative tolerance of the other parity tests."""
import ctypes

import pytest

import qd_imsrg_b200 as qd
from qd_imsrg_b200 import _native

pytestmark = pytest.mark.gpu


def test_noalloc_norm_matches_allocating_entry_point(gpu):
    import torch

    L = qd.Layout(6, 8)
    ops = [qd.FullHam(L, h, qd.random_operator(L, h, seed)) for h, seed in ((-1, 31), (1, 32))]
    L.synchronize()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    lib = _native.lib()
    for op in ops:  # two calls in a row, sharing the static scratch
        ref = qd.mat_2_norm(op)
        rc = lib.qd_mat_2_norm_noalloc(L.h, ctypes.c_void_p(op.device_ptr()), ctypes.c_void_p(out.data_ptr()),
                                       ctypes.c_void_p(stream.cuda_stream))
        _native.check(rc)
        stream.synchronize()
        assert out.item() == pytest.approx(ref, rel=1e-12)
        assert ref > 0.0
