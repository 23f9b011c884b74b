"""The allocation-free norm, qd_mat_2_norm_noalloc.

It serves callers that must not allocate device memory while they run (for
example a host that reserves its device memory up front and forbids
allocation inside its flow loop, or one whose memory belongs to another
allocator, where cudaMalloc can fail or synchronise the device): they pass
the operator and a device scalar, and the partial sums live in a fixed static
device array.  Checked here through the C ABI against the allocating
qd_mat_2_norm on two calls in a row, at the 1e-12 relative tolerance of the
other parity tests; that repeated calls allocate nothing; that with
stream = NULL the call is ordered after asynchronous work on the layout's
stream; and that layouts above the stated maximum are rejected."""
import ctypes

import numpy as np
import pytest

import qd_imsrg_b200 as qd
from qd_imsrg_b200 import _native

MAX_ENTRIES = 4096 * 32768  # QD_NOALLOC_MAX_ENTRIES


def _call(lib, L, op, out, stream):
    return lib.qd_mat_2_norm_noalloc(L.h, ctypes.c_void_p(op.device_ptr()), ctypes.c_void_p(out.data_ptr()),
                                     ctypes.c_void_p(stream))


def test_noalloc_rejects_layouts_above_the_maximum():
    # host-only layout (no device needed): N=20, R=24 holds 221.7 M entries
    L = qd.Layout(20, 24, device=qd.HOST_ONLY)
    assert L.neq - 1 > MAX_ENTRIES
    lib = _native.lib()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.qd_mat_2_norm_noalloc(L.h, dummy, dummy, None)
    assert rc == 1  # QD_ERR_ARG
    assert b"exceed the maximum" in lib.qd_last_error()


@pytest.mark.gpu
def test_noalloc_norm_matches_allocating_entry_point(gpu):
    import torch

    L = qd.Layout(6, 8)
    ops = [qd.FullHam(L, h, qd.random_operator(L, h, seed)) for h, seed in ((-1, 31), (1, 32))]
    L.synchronize()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    lib = _native.lib()
    dev0 = torch.cuda.current_device()
    for op in ops:  # two calls in a row, sharing the static scratch
        ref = qd.mat_2_norm(op)
        v = op.download()
        assert ref == pytest.approx(np.sqrt(np.sum(v[1:] ** 2)), rel=1e-12)  # one- and two-body parts
        _native.check(_call(lib, L, op, out, stream.cuda_stream))
        stream.synchronize()
        assert out.item() == pytest.approx(ref, rel=1e-12)
        assert ref > 0.0
    assert torch.cuda.current_device() == dev0

    # repeated calls allocate nothing: device free memory, torch's reserved
    # bytes and the library's own arena are unchanged
    torch.cuda.synchronize()
    free0, reserved0, ws0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved(), L.workspace_bytes()
    for _ in range(5):
        for op in ops:
            _native.check(_call(lib, L, op, out, stream.cuda_stream))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_reserved() == reserved0
    assert L.workspace_bytes() == ws0


@pytest.mark.gpu
def test_noalloc_null_stream_follows_the_layouts_work(gpu):
    import torch

    L = qd.Layout(6, 8)
    A = qd.FullHam(L, -1, qd.random_operator(L, -1, 41))
    B = qd.FullHam(L, 1, qd.random_operator(L, 1, 42))
    Cop = qd.FullHam(L, 1)
    L.synchronize()
    lib = _native.lib()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for _ in range(2):
        # asynchronous on the layout's stream; stream = NULL orders the norm after it
        _native.check(lib.qd_commutator(A.h, B.h, Cop.h, 0))
        _native.check(_call(lib, L, Cop, out, None))
        L.synchronize()
        got = out.item()
        assert got == pytest.approx(qd.mat_2_norm(Cop), rel=1e-12)
        assert got > 0.0
