"""ctypes front end of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker.  The product package
(qd_imsrg_b200) never imports it.

Parity status: unpinned by the reference (no golden vectors or tests exist in
the reference, and no Fortran compiler is available); see oracle.cpp.

Names follow the reference subroutines (commutators.f90, ME_general.f90,
IMSRG_tools.f90, magnus_IMSRG.f90, HFQDmod.f90).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_lib = None

_i64 = C.c_longlong
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(_i64)
_vp = C.c_void_p


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile."""
    src = os.path.join(_HERE, "oracle.cpp")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "-B" if force else "liboracle.so"])
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_SO)
        sig = {
            "orc_set_threads": (None, [C.c_int]),
            "orc_get_threads": (C.c_int, []),
            "orc_layout_new": (_vp, [C.c_int, C.c_int, _dp, _ip]),
            "orc_layout_free": (None, [_vp]),
            "orc_layout_neq": (_i64, [_vp]),
            "orc_layout_nblock": (C.c_int, [_vp]),
            "orc_layout_msp": (C.c_int, [_vp]),
            "orc_layout_ccn": (C.c_int, [_vp]),
            "orc_layout_qn": (None, [_vp, _ip]),
            "orc_layout_blocks": (None, [_vp, _ip, _lp]),
            "orc_layout_pairs": (C.c_int, [_vp, C.c_int, C.c_int, _ip]),
            "orc_layout_i_array": (None, [_vp, _ip]),
            "orc_layout_cc": (None, [_vp, _ip, _ip]),
            "orc_layout_ccmap": (None, [_vp, _ip]),
            "orc_op_new": (_vp, [_vp, C.c_int]),
            "orc_op_free": (None, [_vp]),
            "orc_op_set": (None, [_vp, _dp]),
            "orc_op_get": (None, [_vp, _dp]),
            "orc_op_set_herm": (None, [_vp, C.c_int]),
            "orc_op_get_herm": (C.c_int, [_vp]),
            "orc_cc_new": (_vp, [_vp]),
            "orc_cc_free": (None, [_vp]),
            "orc_cc_set_herm": (None, [_vp, C.c_double]),
            "orc_calc_cc": (None, [_vp, _vp]),
            "orc_cc_get_X": (None, [_vp, _dp]),
            "orc_cc_xsize": (_i64, [_vp]),
            "orc_v_elem": (C.c_double, [C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
            "orc_commutator_110": (C.c_double, [_vp, _vp]),
            "orc_commutator_220": (C.c_double, [_vp, _vp]),
            "orc_commutator_111": (None, [_vp, _vp, _vp]),
            "orc_commutator_121": (None, [_vp, _vp, _vp]),
            "orc_commutator_221": (None, [_vp, _vp, _vp, _vp, _vp]),
            "orc_commutator_122": (None, [_vp, _vp, _vp, C.c_int]),
            "orc_commutator_222": (None, [_vp, _vp, _vp, _vp, _vp, _vp]),
            "orc_commutator": (None, [_vp, _vp, _vp, C.c_int]),
            "orc_build_white": (None, [_vp, _vp]),
            "orc_add_arrays": (None, [_vp, C.c_double, _vp, C.c_double, _vp]),
            "orc_copy_arrays": (None, [_vp, _vp]),
            "orc_set_to_zero": (None, [_vp]),
            "orc_mat_2_norm": (C.c_double, [_vp]),
            "orc_mbpt2": (C.c_double, [_vp]),
            "orc_hf_e2": (C.c_double, [_vp]),
            "orc_bch_expand": (C.c_int, [_vp, _vp, _vp, C.c_int]),
            "orc_magnus_flow": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _dp, _dp]),
            "orc_use_blas": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p]),
            "orc_sampler_new": (_vp, [_vp]),
            "orc_sampler_free": (None, [_vp]),
            "orc_commutator_sample": (None, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
        _attach_blas(L)
    return _lib


BLAS = None  # path of the BLAS library whose dgemm the oracle calls, if any


def _attach_blas(L) -> None:
    """Route the oracle's dgemm to scipy's bundled OpenBLAS when present (the
    reference links BLAS dgemm); otherwise the oracle's own loop dgemm runs."""
    global BLAS
    if os.environ.get("QD_ORACLE_NO_BLAS"):
        return
    try:
        import glob

        import scipy

        libs = glob.glob(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs",
                                      "libscipy_openblas-*.so"))
    except Exception:
        libs = []
    for path in libs:
        if L.orc_use_blas(path.encode(), b"scipy_dgemm_", b"openblas_set_num_threads_local"):
            BLAS = path
            return


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


class Layout:
    """reindex + build_cross_coupled for N holes in emax major shells."""

    def __init__(self, nbody: int, emax: int, eig=None):
        err = C.c_int(0)
        e = None
        if eig is not None:
            self._eig = np.ascontiguousarray(eig, dtype=np.float64)
            e = _dptr(self._eig)
        self.h = lib().orc_layout_new(int(nbody), int(emax), e, C.byref(err))
        if not self.h:
            raise ValueError("oracle layout: holes are not states 1..N (code %d)" % err.value)
        self.n, self.emax = int(nbody), int(emax)
        self.m = int(lib().orc_layout_msp(self.h))
        self.neq = int(lib().orc_layout_neq(self.h))
        self.nblock = int(lib().orc_layout_nblock(self.h))
        self.ccn = int(lib().orc_layout_ccn(self.h))
        dims = np.zeros((self.nblock, 6), np.int32)
        offs = np.zeros((self.nblock, 6), np.int64)
        lib().orc_layout_blocks(self.h, dims.ctypes.data_as(_ip), offs.ctypes.data_as(_lp))
        self.dims, self.offs = dims, offs
        qn = np.zeros((self.m, 3), np.int32)
        lib().orc_layout_qn(self.h, qn.ctypes.data_as(_ip))
        self.qn = qn
        r = np.zeros(self.ccn, np.int32)
        nb = np.zeros(self.ccn, np.int32)
        lib().orc_layout_cc(self.h, r.ctypes.data_as(_ip), nb.ctypes.data_as(_ip))
        self.cc_r, self.cc_nb = r, nb

    def pairs(self, q: int, kind: int) -> np.ndarray:
        """Pair list (1-based states) of block q (1-based); kind 0=hh, 1=ph, 2=pp."""
        d = self.dims[q - 1]
        cnt = [d[0], d[1], d[2]][kind]
        out = np.zeros((max(cnt, 1), 2), np.int32)
        lib().orc_layout_pairs(self.h, q, kind, out.ctypes.data_as(_ip))
        return out[:cnt]

    def i_array(self) -> np.ndarray:
        g = self.m * (self.m - 1) // 2
        out = np.zeros((g, 3), np.int32)
        lib().orc_layout_i_array(self.h, out.ctypes.data_as(_ip))
        return out

    def ccmap(self) -> np.ndarray:
        out = np.zeros((self.m * self.m, 2), np.int32)
        lib().orc_layout_ccmap(self.h, out.ctypes.data_as(_ip))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_layout_free(self.h)
            self.h = None


class Op:
    """type(full_ham) holding its entries in vectorize order."""

    def __init__(self, layout: Layout, herm: int = 1, vec=None):
        self.layout = layout
        self.h = lib().orc_op_new(layout.h, int(herm))
        if vec is not None:
            self.set(vec)

    def set(self, vec) -> None:
        v = np.ascontiguousarray(vec, dtype=np.float64)
        if v.size != self.layout.neq:
            raise ValueError("vector has %d entries, layout needs %d" % (v.size, self.layout.neq))
        lib().orc_op_set(self.h, _dptr(v))

    def get(self) -> np.ndarray:
        v = np.empty(self.layout.neq, np.float64)
        lib().orc_op_get(self.h, _dptr(v))
        return v

    @property
    def herm(self) -> int:
        return int(lib().orc_op_get_herm(self.h))

    @herm.setter
    def herm(self, h: int) -> None:
        lib().orc_op_set_herm(self.h, int(h))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_op_free(self.h)
            self.h = None


class CC:
    """type(cc_mat): cross-coupled X(r,nb) matrices of one operator."""

    def __init__(self, layout: Layout, herm: float = 1.0):
        self.layout = layout
        self.h = lib().orc_cc_new(layout.h)
        lib().orc_cc_set_herm(self.h, float(herm))

    def set_herm(self, h: float) -> None:
        lib().orc_cc_set_herm(self.h, float(h))

    def get_X(self) -> np.ndarray:
        n = int(lib().orc_cc_xsize(self.h))
        out = np.empty(n, np.float64)
        lib().orc_cc_get_X(self.h, _dptr(out))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_cc_free(self.h)
            self.h = None


def v_elem(a, b, c, d, op: Op) -> float:
    return float(lib().orc_v_elem(a, b, c, d, op.h))


def commutator_110(r1: Op, r2: Op) -> float:
    return float(lib().orc_commutator_110(r1.h, r2.h))


def commutator_220(r1: Op, r2: Op) -> float:
    return float(lib().orc_commutator_220(r1.h, r2.h))


def commutator_111(r1, r2, r3):
    lib().orc_commutator_111(r1.h, r2.h, r3.h)


def commutator_121(r1, r2, r3):
    lib().orc_commutator_121(r1.h, r2.h, r3.h)


def commutator_221(r1, r2, r3, w1, w2):
    lib().orc_commutator_221(r1.h, r2.h, r3.h, w1.h, w2.h)


def commutator_122(r1, r2, r3, literal: bool = False):
    lib().orc_commutator_122(r1.h, r2.h, r3.h, int(literal))


def commutator_222(r1, r2, r3, w1, hcc: CC, etacc: CC):
    lib().orc_commutator_222(r1.h, r2.h, r3.h, w1.h, hcc.h, etacc.h)


def calc_cc(op: Op, cc: CC):
    lib().orc_calc_cc(op.h, cc.h)


def commutator(A: Op, B: Op, Cop: Op, pandya: bool = True):
    """Whole [A,B] -> C in the reference's call order (BCH_EXPAND / dGam)."""
    lib().orc_commutator(A.h, B.h, Cop.h, int(pandya))


def build_white(gen: Op, rec: Op):
    lib().orc_build_white(gen.h, rec.h)


def add_arrays(r1, s1, r2, s2, r3):
    lib().orc_add_arrays(r1.h, float(s1), r2.h, float(s2), r3.h)


def copy_arrays(r1, r2):
    lib().orc_copy_arrays(r1.h, r2.h)


def set_to_zero(r1):
    lib().orc_set_to_zero(r1.h)


def mat_2_norm(r) -> float:
    return float(lib().orc_mat_2_norm(r.h))


def mbpt2(r) -> float:
    return float(lib().orc_mbpt2(r.h))


def hf_e2(r) -> float:
    return float(lib().orc_hf_e2(r.h))


def bch_expand(HS: Op, G: Op, H: Op, pandya: bool = False) -> int:
    return int(lib().orc_bch_expand(HS.h, G.h, H.h, 1 if pandya else 0))


class Sampler:
    """Bounded samples of one commutator [A,B] for CPU timing: phase p of
    `stride` does the two-body work of every stride-th block and the
    cross-coupled products of every stride-th cc block (and E0 plus the
    one-body parts, and with pandya calc_cc, on phase 0).  The phases
    together do the work of one whole commutator; without the Pandya channel
    they also give its result (with it, a phase's ph terms see only the
    products formed in that phase)."""

    def __init__(self, A: Op):
        self.h = lib().orc_sampler_new(A.h)

    def run(self, A: Op, B: Op, Cop: Op, stride: int, phase: int, pandya: bool = True) -> None:
        lib().orc_commutator_sample(self.h, A.h, B.h, Cop.h, int(stride), int(phase), int(pandya))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_sampler_free(self.h)
            self.h = None


def magnus_flow(HAM: Op, HS: Op, pandya: bool = False, max_iter: int = 500):
    """s_evolve(build_white); returns (trace[rows,7], s)."""
    trace = np.zeros((max_iter, 7), np.float64)
    s = C.c_double(0.0)
    rows = int(lib().orc_magnus_flow(HAM.h, HS.h, 1 if pandya else 0, int(max_iter), _dptr(trace),
                                     C.byref(s)))
    if rows < 0:
        raise RuntimeError("oracle Magnus flow did not converge within %d iterations" % max_iter)
    return trace[:rows], s.value
