"""ctypes binding of libqdimsrg.so (the C ABI declared in include/qd_imsrg.h).

The library is loaded from this package directory only.  There is no CPU
fallback: if the library is missing or no CUDA device is present, calls raise
QDError.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqdimsrg.so")

_i64 = C.c_int64
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_ip64 = C.POINTER(C.c_int64)
_lp = C.POINTER(_i64)
_vp = C.c_void_p
_vpp = C.POINTER(C.c_void_p)

QD_OK = 0
QD_PANDYA = 1
QD_BATCH_STREAMS = 4
QD_TBME_QUAD = 1
QD_NSTAGE = 10
STAGES = ["E0", "c111", "c121", "c221", "c122", "calc_cc", "ladder_gemm", "pandya_gemm", "pandya_gather", "glue"]

ERRORS = {
    1: "QD_ERR_ARG", 2: "QD_ERR_LAYOUT", 3: "QD_ERR_CUDA", 4: "QD_ERR_OOM", 5: "QD_ERR_NAN",
    6: "QD_ERR_NOCONV", 7: "QD_ERR_NODEVICE", 8: "QD_ERR_STATE",
}


class QDError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "QD_ERR"), code, msg))
        self.code = code


class FlowStepInfo(C.Structure):
    _fields_ = [("s", C.c_double), ("E0", C.c_double), ("nrm1", C.c_double), ("nrm2", C.c_double),
                ("crit", C.c_double), ("terms", C.c_int), ("accepted", C.c_int), ("converged", C.c_int)]


class FlowResult(C.Structure):
    _fields_ = [("E0", C.c_double), ("s", C.c_double), ("iterations", C.c_int), ("rejected", C.c_int),
                ("commutators", C.c_int), ("rows", C.c_int)]


# name -> (restype, argtypes); every function returns int status
SIGNATURES = {
    "qd_last_error": (C.c_char_p, []),
    "qd_version": (C.c_char_p, []),
    "qd_layout_create": (C.c_int, [C.c_int, C.c_int, _dp, C.c_int, _vpp]),
    "qd_layout_destroy": (C.c_int, [_vp]),
    "qd_layout_info": (C.c_int, [_vp, _ip, _ip, _ip, _lp, _ip]),
    "qd_layout_blocks": (C.c_int, [_vp, _ip]),
    "qd_layout_offsets": (C.c_int, [_vp, _lp]),
    "qd_layout_pairs": (C.c_int, [_vp, C.c_int, C.c_int, _ip, _ip]),
    "qd_layout_set_stream": (C.c_int, [_vp, _vp]),
    "qd_layout_set_split": (C.c_int, [_vp, C.c_int]),
    "qd_layout_set_graphs": (C.c_int, [_vp, C.c_int]),
    "qd_layout_graph_stats": (C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "qd_layout_get_split": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "qd_layout_synchronize": (C.c_int, [_vp]),
    "qd_layout_workspace_bytes": (C.c_int, [_vp, _lp]),
    "qd_layout_profile": (C.c_int, [_vp, C.c_int]),
    "qd_layout_launches": (C.c_int, [_vp, _lp]),
    "qd_layout_profile_read": (C.c_int, [_vp, _dp, _lp, C.c_int]),
    "qd_op_create": (C.c_int, [_vp, C.c_int, _vpp]),
    "qd_op_destroy": (C.c_int, [_vp]),
    "qd_op_upload": (C.c_int, [_vp, _dp, _i64]),
    "qd_op_download": (C.c_int, [_vp, _dp, _i64]),
    "qd_op_upload_device": (C.c_int, [_vp, _vp, _i64]),
    "qd_op_set_herm": (C.c_int, [_vp, C.c_int]),
    "qd_op_get_herm": (C.c_int, [_vp, _ip]),
    "qd_op_device_ptr": (C.c_int, [_vp, C.POINTER(_dp)]),
    "qd_random_operator": (C.c_int, [_vp, C.c_int, C.c_uint64, C.c_double, C.c_int, _dp, _i64]),
    "qd_add_arrays": (C.c_int, [_vp, C.c_double, _vp, C.c_double, _vp]),
    "qd_copy_arrays": (C.c_int, [_vp, _vp]),
    "qd_set_to_zero": (C.c_int, [_vp]),
    "qd_mat_2_norm": (C.c_int, [_vp, _dp]),
    "qd_mat_2_norm_noalloc": (C.c_int, [_vp, _vp, _vp, _vp]),
    "qd_layout_tuning": (C.c_int, [_vp, C.c_char_p, _i64, _ip64]),
    "qd_commutator_110": (C.c_int, [_vp, _vp, _dp]),
    "qd_commutator_220": (C.c_int, [_vp, _vp, _dp]),
    "qd_commutator_111": (C.c_int, [_vp, _vp, _vp]),
    "qd_commutator_121": (C.c_int, [_vp, _vp, _vp]),
    "qd_commutator_221": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "qd_commutator_122": (C.c_int, [_vp, _vp, _vp]),
    "qd_commutator_222": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "qd_commutator": (C.c_int, [_vp, _vp, _vp, C.c_uint]),
    "qd_cc_create": (C.c_int, [_vp, C.c_double, _vpp]),
    "qd_cc_destroy": (C.c_int, [_vp]),
    "qd_cc_set_herm": (C.c_int, [_vp, C.c_double]),
    "qd_calc_cc": (C.c_int, [_vp, _vp]),
    "qd_cc_download": (C.c_int, [_vp, _dp, _i64, _lp]),
    "qd_build_white": (C.c_int, [_vp, _vp]),
    "qd_mbpt2": (C.c_int, [_vp, _dp]),
    "qd_hf_e2": (C.c_int, [_vp, _dp]),
    "qd_bch_expand": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_uint, _ip]),
    "qd_magnus_expand": (C.c_int, [_vp, _vp, _vp]),
    "qd_euler_step": (C.c_int, [_vp, _vp, _dp, C.c_double]),
    "qd_magnus_flow": (C.c_int, [_vp, _vp, C.c_uint, C.c_int, _dp, C.POINTER(FlowResult)]),
    "qd_magnus_flow_batch": (C.c_int, [C.c_int, C.POINTER(_vp), C.POINTER(_vp), C.c_uint, C.c_int,
                                       C.POINTER(FlowResult), C.POINTER(C.c_int)]),
    "qd_flow_create": (C.c_int, [_vp, _vp, C.c_uint, C.POINTER(_vp)]),
    "qd_flow_warm_start": (C.c_int, [_vp, _vp, C.c_double]),
    "qd_flow_step": (C.c_int, [_vp, C.POINTER(FlowStepInfo)]),
    "qd_flow_omega": (C.c_int, [_vp, C.POINTER(_vp)]),
    "qd_flow_state": (C.c_int, [_vp, C.POINTER(FlowResult)]),
    "qd_flow_destroy": (C.c_int, [_vp]),
    "qd_omega_count": (C.c_int, [_vp, _ip64]),
    "qd_omega_gather": (C.c_int, [_vp, _vp, _i64]),
    "qd_omega_scatter": (C.c_int, [_vp, _vp, C.c_float, _vp, _i64]),
    "qd_omega_features": (C.c_int, [_vp, C.c_double, C.c_double, _vp, _i64]),
    "qd_mlp_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(_vp)]),
    "qd_mlp_destroy": (C.c_int, [_vp]),
    "qd_mlp_get_params": (C.c_int, [_vp, C.POINTER(C.c_float), _i64]),
    "qd_mlp_set_params": (C.c_int, [_vp, C.POINTER(C.c_float), _i64]),
    "qd_mlp_forward": (C.c_int, [_vp, _vp, _vp, _i64, _vp]),
    "qd_mlp_grad": (C.c_int, [_vp, _vp, _vp, _i64, _vp, C.POINTER(C.c_float), _vp]),
    "qd_mlp_train_step": (C.c_int, [_vp, _vp, _vp, _i64, C.c_float, C.POINTER(C.c_float), _vp]),
    "qd_dgam": (C.c_int, [_vp, _vp, _vp, _vp]),
    "qd_eom_matvec": (C.c_int, [_vp, _vp, _vp]),
    "qd_eom_dim": (C.c_int, [_vp, C.c_int, C.c_int, _ip64, _ip64]),
    "qd_eom_matvec_target": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp, _i64]),
    "qd_hamiltonian_write": (C.c_int, [_vp, _vp, C.c_char_p]),
    "qd_hamiltonian_read": (C.c_int, [_vp, _vp, C.c_char_p]),
    "qd_export_hamiltonian": (C.c_int, [_vp, C.c_char_p]),
    "qd_import_hamiltonian": (C.c_int, [_vp, C.c_char_p]),
    "qd_gemm_split": (C.c_int, [C.c_int, _vp, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, _vp,
                                C.c_int, _vp, C.c_int, C.c_double, _vp, C.c_int, C.c_int]),
    "qd_tbme_write": (C.c_int, [C.c_int, C.c_char_p, C.c_int, C.c_uint]),
    "qd_hf_hamiltonian": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_char_p, C.c_int, C.c_double, C.c_uint,
                                    _dp, _dp, _i64, _ip]),
    "qd_v_int": (C.c_double, [_ip, _ip, _ip, _ip, C.c_double]),
    "qd_v_int_quad": (C.c_double, [_ip, _ip, _ip, _ip, C.c_double]),
}

_lib = None


def lib():
    """Load libqdimsrg.so from the package directory (raises if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QDError(7, "libqdimsrg.so is not built (run qd_imsrg_b200.build.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != QD_OK:
        raise QDError(rc, lib().qd_last_error().decode(errors="replace"))


def exported_symbols():
    return list(SIGNATURES)
