"""CPU checks of the C ABI: every function declared in include/qd_imsrg.h is
exported by the in-tree library and bound by the Python front end; the
library refuses to compute without a device instead of falling back."""
import ctypes
import os
import re

import pytest

import qd_imsrg_b200 as qd
from qd_imsrg_b200 import _native
from conftest import HAS_GPU, ROOT

HEADER = os.path.join(ROOT, "include", "qd_imsrg.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(qd_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("qd_commutator_110", "qd_commutator_220", "qd_commutator_111", "qd_commutator_121",
                 "qd_commutator_221", "qd_commutator_122", "qd_commutator_222", "qd_calc_cc",
                 "qd_build_white", "qd_bch_expand", "qd_magnus_expand", "qd_euler_step", "qd_magnus_flow",
                 "qd_add_arrays", "qd_copy_arrays", "qd_set_to_zero", "qd_mat_2_norm", "qd_mbpt2"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_native.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in _native.SIGNATURES, name


def test_version_string():
    assert b"sm_100a" in _native.lib().qd_version()


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_no_silent_cpu_fallback_without_device():
    with pytest.raises(qd.QDError) as e:
        qd.Layout(6, 4)
    assert e.value.code == 7  # QD_ERR_NODEVICE


def test_host_only_layout_refuses_operators():
    L = qd.Layout(2, 3, device=qd.HOST_ONLY)
    with pytest.raises(qd.QDError) as e:
        qd.FullHam(L, 1)
    assert e.value.code == 8  # QD_ERR_STATE


def test_oracle_library_loads():
    import oracle

    assert oracle.get_threads() >= 1
