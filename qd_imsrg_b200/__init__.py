"""qd_imsrg_b200 -- B200-native IM-SRG(2) commutator / BCH engine.

Python front end of the C ABI (include/qd_imsrg.h).  Names and argument
meanings follow the reference Fortran subroutines so that host code reads
like the reference:

  reference (nparz/qd_IMSRG)                      here
  type(full_ham)  ME_general.f90:43-62            FullHam (device operator)
  type(cc_mat)    ME_general.f90:19-24            CCMat
  reindex / build_cross_coupled                   Layout
  commutator_110/220/111/121/221/122/222          commutator_110 ... commutator_222
  calc_cc, build_white, add_arrays, copy_arrays,  same names
  set_to_zero, mat_2_norm, MBPT2, HF_E2
  BCH_EXPAND, MAGNUS_EXPAND, euler_step,          bch_expand, magnus_expand,
  s_evolve                                        euler_step, magnus_flow

Operators stay resident in device memory in the reference's (M_L,M_S)-blocked
layout; host arrays are exchanged in the reference's vectorize order.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _native
from ._native import QD_BATCH_STREAMS, QD_PANDYA, QD_TBME_QUAD, FlowResult, FlowStepInfo, QDError, check, lib

__all__ = [
    "Layout", "FullHam", "CCMat", "QDError", "QD_PANDYA", "QD_BATCH_STREAMS",
    "commutator_110", "commutator_220", "commutator_111", "commutator_121", "commutator_221",
    "commutator_122", "commutator_222", "commutator", "calc_cc", "build_white", "add_arrays",
    "copy_arrays", "set_to_zero", "mat_2_norm", "mbpt2", "hf_e2", "bch_expand", "magnus_expand",
    "euler_step", "magnus_flow", "random_operator", "tbme_write", "hf_hamiltonian", "v_int",
    "Flow", "magnus_flow_batch", "dgam", "eom_matvec", "eom_dim", "eom_matvec_target", "gemm_split", "hamiltonian_write", "hamiltonian_read",
    "export_hamiltonian", "import_hamiltonian",
]

_dp = C.POINTER(C.c_double)
HOST_ONLY = -2


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Layout:
    """Basis of N holes in emax major shells, blocked as reindex does.

    eig: optional single-particle energies in states order (default:
    oscillator energies 2n+|ml|+1), used to class pairs as hole/particle.
    device: CUDA device (-1 = current); HOST_ONLY builds only the host tables.
    """

    def __init__(self, nbody: int, emax: int, eig=None, device: int = -1):
        self.h = C.c_void_p()
        e = None
        if eig is not None:
            self._eig = np.ascontiguousarray(eig, dtype=np.float64)
            e = _d(self._eig)
        check(lib().qd_layout_create(int(nbody), int(emax), e, int(device), C.byref(self.h)))
        nb, msp, nblk, ncc = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        neq = C.c_int64()
        check(lib().qd_layout_info(self.h, C.byref(nb), C.byref(msp), C.byref(nblk), C.byref(neq), C.byref(ncc)))
        self.nbody, self.msp, self.nblock, self.neq, self.ncc = nb.value, msp.value, nblk.value, neq.value, ncc.value
        self.emax = int(emax)
        dims = np.zeros((self.nblock, 5), np.int32)
        check(lib().qd_layout_blocks(self.h, dims.ctypes.data_as(C.POINTER(C.c_int))))
        self.dims = dims
        offs = np.zeros((self.nblock, 6), np.int64)
        check(lib().qd_layout_offsets(self.h, offs.ctypes.data_as(C.POINTER(C.c_int64))))
        self.offs = offs

    def pairs(self, q: int, kind: int) -> np.ndarray:
        """1-based (i,j) pairs of block q (0-based); kind 0=hh, 1=ph, 2=pp."""
        cnt = C.c_int()
        check(lib().qd_layout_pairs(self.h, int(q), int(kind), None, C.byref(cnt)))
        out = np.zeros((max(cnt.value, 1), 2), np.int32)
        check(lib().qd_layout_pairs(self.h, int(q), int(kind), out.ctypes.data_as(C.POINTER(C.c_int)),
                                    C.byref(cnt)))
        return out[: cnt.value]

    def synchronize(self) -> None:
        check(lib().qd_layout_synchronize(self.h))

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib().qd_layout_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    @property
    def split(self) -> int:
        """Slices of the split form of the block contractions (0 = plain FP64)."""
        v = C.c_int()
        check(lib().qd_layout_get_split(self.h, C.byref(v)))
        return v.value

    @split.setter
    def split(self, slices: int) -> None:
        check(lib().qd_layout_set_split(self.h, int(slices)))

    def set_graphs(self, enable: bool) -> None:
        """Replay BCH terms as CUDA graphs (default on)."""
        check(lib().qd_layout_set_graphs(self.h, int(enable)))

    def graph_stats(self) -> tuple[int, int]:
        """(graphs captured, replays) of this layout so far."""
        a, b = C.c_int64(), C.c_int64()
        check(lib().qd_layout_graph_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def profile(self, enable: bool = True) -> None:
        """Start (and reset) or stop per-stage CUDA-event timing."""
        check(lib().qd_layout_profile(self.h, int(enable)))

    def profile_read(self) -> dict:
        """{stage: (milliseconds, launches)} accumulated since profile(True)."""
        ms = np.zeros(_native.QD_NSTAGE, np.float64)
        cnt = np.zeros(_native.QD_NSTAGE, np.int64)
        check(lib().qd_layout_profile_read(self.h, _d(ms), cnt.ctypes.data_as(C.POINTER(C.c_int64)),
                                           _native.QD_NSTAGE))
        return {name: (float(ms[i]), int(cnt[i])) for i, name in enumerate(_native.STAGES)}

    def launches(self) -> int:
        """Kernels launched by the library for this layout so far."""
        n = C.c_int64()
        check(lib().qd_layout_launches(self.h, C.byref(n)))
        return n.value

    def tuning(self) -> str:
        """The autotuner's per-bucket timings and choices (text)."""
        need = C.c_int64()
        check(lib().qd_layout_tuning(self.h, None, 0, C.byref(need)))
        buf = C.create_string_buffer(max(1, need.value))
        check(lib().qd_layout_tuning(self.h, buf, need.value, C.byref(need)))
        return buf.value.decode()

    def workspace_bytes(self) -> int:
        b = C.c_int64()
        check(lib().qd_layout_workspace_bytes(self.h, C.byref(b)))
        return b.value

    def close(self) -> None:
        if getattr(self, "h", None) and self.h.value:
            lib().qd_layout_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def random_operator(layout: Layout, herm: int, seed: int, sigma: float = 0.1, conserve: bool = True) -> np.ndarray:
    """Seeded synthetic operator (host vector, vectorize order)."""
    v = np.empty(layout.neq, np.float64)
    check(lib().qd_random_operator(layout.h, int(herm), C.c_uint64(seed), float(sigma), int(conserve), _d(v),
                                   layout.neq))
    return v


class FullHam:
    """A device-resident operator (type(full_ham)); herm = +1 or -1."""

    def __init__(self, layout: Layout, herm: int = 1, vec=None):
        self.layout = layout
        self.h = C.c_void_p()
        check(lib().qd_op_create(layout.h, int(herm), C.byref(self.h)))
        if vec is not None:
            self.upload(vec)

    def upload(self, vec) -> None:
        v = np.ascontiguousarray(vec, dtype=np.float64)
        check(lib().qd_op_upload(self.h, _d(v), v.size))

    def download(self) -> np.ndarray:
        v = np.empty(self.layout.neq, np.float64)
        check(lib().qd_op_download(self.h, _d(v), v.size))
        return v

    @property
    def herm(self) -> int:
        h = C.c_int()
        check(lib().qd_op_get_herm(self.h, C.byref(h)))
        return h.value

    @herm.setter
    def herm(self, h: int) -> None:
        check(lib().qd_op_set_herm(self.h, int(h)))

    def device_ptr(self) -> int:
        p = _dp()
        check(lib().qd_op_device_ptr(self.h, C.byref(p)))
        return C.cast(p, C.c_void_p).value

    @property
    def E0(self) -> float:
        return float(self.download()[0])

    def close(self) -> None:
        if getattr(self, "h", None) and self.h.value:
            if getattr(self, "_owned", True):
                lib().qd_op_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CCMat:
    """Cross-coupled (Pandya) X(r,nb) matrices of one operator (type(cc_mat))."""

    def __init__(self, layout: Layout, herm: float = 1.0):
        self.layout = layout
        self.h = C.c_void_p()
        check(lib().qd_cc_create(layout.h, float(herm), C.byref(self.h)))

    def set_herm(self, h: float) -> None:
        check(lib().qd_cc_set_herm(self.h, float(h)))

    def download(self) -> np.ndarray:
        need = C.c_int64()
        check(lib().qd_cc_download(self.h, None, 0, C.byref(need)))
        out = np.empty(need.value, np.float64)
        check(lib().qd_cc_download(self.h, _d(out), need.value, C.byref(need)))
        return out

    def close(self) -> None:
        if getattr(self, "h", None) and self.h.value:
            lib().qd_cc_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _scalar(fn, *args) -> float:
    out = C.c_double()
    check(fn(*args, C.byref(out)))
    return out.value


def commutator_110(r1: FullHam, r2: FullHam) -> float:
    return _scalar(lib().qd_commutator_110, r1.h, r2.h)


def commutator_220(r1: FullHam, r2: FullHam) -> float:
    return _scalar(lib().qd_commutator_220, r1.h, r2.h)


def commutator_111(r1, r2, r3) -> None:
    check(lib().qd_commutator_111(r1.h, r2.h, r3.h))


def commutator_121(r1, r2, r3) -> None:
    check(lib().qd_commutator_121(r1.h, r2.h, r3.h))


def commutator_221(r1, r2, r3, w1, w2) -> None:
    check(lib().qd_commutator_221(r1.h, r2.h, r3.h, w1.h, w2.h))


def commutator_122(r1, r2, r3) -> None:
    check(lib().qd_commutator_122(r1.h, r2.h, r3.h))


def commutator_222(r1, r2, r3, w1, HCC: CCMat, ETACC: CCMat) -> None:
    check(lib().qd_commutator_222(r1.h, r2.h, r3.h, w1.h if w1 is not None else None, HCC.h, ETACC.h))


def commutator(A: FullHam, B: FullHam, Cop: FullHam, pandya: bool = True) -> None:
    """C = [A,B] in the reference's call order; pandya fills both operators'
    cross-coupled matrices first (as dGam), otherwise the particle-hole
    channel is absent (as run_magnus)."""
    check(lib().qd_commutator(A.h, B.h, Cop.h, QD_PANDYA if pandya else 0))


def dgam(H: FullHam, DER: FullHam, HCC: CCMat | None = None, ETACC: CCMat | None = None) -> None:
    """dGam (gs_IMSRG.f90:223-273): DER = [build_white(H), H] with every term,
    the ODE flow's derivative; fills HCC = calc_cc(H), ETACC = calc_cc(eta)."""
    check(lib().qd_dgam(H.h, DER.h, HCC.h if HCC is not None else None, ETACC.h if ETACC is not None else None))


def eom_matvec(H: FullHam, Q: FullHam, HQ: FullHam) -> None:
    """EOM matrix-vector product (matvec_prod / HQ_comm_1b,2b) for the
    scalar target: HQ's fph and Vpphh = the ph and pphh parts of [H, Q] for
    the excitation amplitudes in Q's fph and Vpphh; other parts zero."""
    check(lib().qd_eom_matvec(H.h, Q.h, HQ.h))


def eom_dim(layout: Layout, ml: int, ms: int) -> tuple[int, int]:
    """(1p1h, 2p2h) entries of the EOM vector for the target (Mltarg, Mstarg)
    = (ml, ms), as unwrap (EOM_IMSRG.f90:815-884) counts them."""
    n1, n2 = C.c_int64(), C.c_int64()
    check(lib().qd_eom_dim(layout.h, int(ml), int(ms), C.byref(n1), C.byref(n2)))
    return n1.value, n2.value


def eom_matvec_target(H: FullHam, ml: int, ms: int, v, w=None):
    """matvec_prod (EOM_IMSRG.f90:551-649) for the target (ml, ms): w = the
    rewrap of HQ_comm_1b/2b of H and the excitation unwrapped from v, both in
    the reference's unwrap order.  v, w: float64 CUDA tensors (torch) of
    n1 + n2 entries on H's device (w is allocated when None); or a numpy v,
    in which case a numpy w is returned (copied through the device)."""
    import torch

    host = isinstance(v, np.ndarray)
    if host:
        v = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).cuda()
    if v.dtype != torch.float64 or not v.is_cuda or not v.is_contiguous() or v.dim() != 1:
        raise ValueError("v must be a contiguous 1-D float64 CUDA tensor")
    if w is None:
        w = torch.empty_like(v)
    # v and w are written on torch's stream, read and written on the layout's
    torch.cuda.current_stream(v.device).synchronize()
    check(lib().qd_eom_matvec_target(H.h, int(ml), int(ms), C.c_void_p(v.data_ptr()), C.c_void_p(w.data_ptr()),
                                     int(v.numel())))
    H.layout.synchronize()
    return w.cpu().numpy() if host else w


def calc_cc(H: FullHam, HCC: CCMat) -> None:
    check(lib().qd_calc_cc(H.h, HCC.h))


def build_white(gen: FullHam, H: FullHam) -> None:
    check(lib().qd_build_white(gen.h, H.h))


def add_arrays(r1, s1, r2, s2, r3) -> None:
    check(lib().qd_add_arrays(r1.h, float(s1), r2.h, float(s2), r3.h))


def copy_arrays(r1, r2) -> None:
    check(lib().qd_copy_arrays(r1.h, r2.h))


def set_to_zero(r1) -> None:
    check(lib().qd_set_to_zero(r1.h))


def mat_2_norm(r) -> float:
    return _scalar(lib().qd_mat_2_norm, r.h)


def mbpt2(r) -> float:
    return _scalar(lib().qd_mbpt2, r.h)


def hf_e2(r) -> float:
    return _scalar(lib().qd_hf_e2, r.h)


def _flags(pandya: bool) -> int:
    return QD_PANDYA if pandya else 0


def bch_expand(HS, G, H, INT1, INT2, AD, w1, w2, HCC: CCMat, OCC: CCMat, pandya: bool = False) -> int:
    """BCH_EXPAND; INT1 is accepted for the reference's argument list and is
    not written (its norm is taken from HS in the update pass)."""
    n = C.c_int()
    check(lib().qd_bch_expand(HS.h, G.h, H.h, INT1.h, INT2.h, AD.h, w1.h, w2.h, HCC.h, OCC.h,
                              _flags(pandya), C.byref(n)))
    return n.value


def magnus_expand(DG, G, ETA) -> None:
    check(lib().qd_magnus_expand(DG.h, G.h, ETA.h))


def euler_step(G, DG, s: float, stp: float) -> float:
    sv = C.c_double(s)
    check(lib().qd_euler_step(G.h, DG.h, C.byref(sv), float(stp)))
    return sv.value


def magnus_flow(HAM: FullHam, HS: FullHam, pandya: bool = False, max_iter: int = 500):
    """s_evolve(build_white): returns (trace[rows,7], FlowResult).  pandya adds
    the particle-hole channel (absent in run_magnus)."""
    trace = np.zeros((max_iter, 7), np.float64)
    res = FlowResult()
    check(lib().qd_magnus_flow(HAM.h, HS.h, _flags(pandya), int(max_iter), _d(trace), C.byref(res)))
    return trace[: res.rows], res


class Flow:
    """s_evolve as a stepping object: Flow(HAM, HS) starts at s = 0;
    warm_start(G, s) seeds Omega = G at flow parameter s; step() runs one
    pass of the loop; omega() is the flow's Omega (owned by the flow)."""

    def __init__(self, HAM: FullHam, HS: FullHam, pandya: bool = False):
        self.layout = HAM.layout
        self.h = C.c_void_p()
        check(lib().qd_flow_create(HAM.h, HS.h, _flags(pandya), C.byref(self.h)))

    def warm_start(self, G: FullHam, s: float) -> None:
        check(lib().qd_flow_warm_start(self.h, G.h, float(s)))

    def step(self) -> FlowStepInfo:
        info = FlowStepInfo()
        check(lib().qd_flow_step(self.h, C.byref(info)))
        return info

    def omega(self) -> FullHam:
        g = C.c_void_p()
        check(lib().qd_flow_omega(self.h, C.byref(g)))
        return _borrowed(self.layout, g)

    def state(self) -> FlowResult:
        r = FlowResult()
        check(lib().qd_flow_state(self.h, C.byref(r)))
        return r

    def run(self, max_iter: int = 500) -> FlowResult:
        """Step until converged; raises QDError after max_iter steps."""
        for _ in range(max_iter + 1):
            if self.step().converged:
                return self.state()
        raise QDError(6, "Flow.run: not converged after %d steps" % max_iter)

    def close(self) -> None:
        if getattr(self, "h", None) and self.h.value:
            lib().qd_flow_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _borrowed(layout: Layout, handle) -> FullHam:
    """A FullHam view of an operator owned by the library (never destroyed
    from Python)."""
    op = FullHam.__new__(FullHam)
    op.layout = layout
    op.h = C.c_void_p(handle.value)
    op._owned = False
    return op


class DeviceView:
    """__cuda_array_interface__ of an operator's device array (float64, neq
    entries, vectorize order): zero-copy access from torch and the like.
    Taking it clears the operator's known-zero parts (writes may follow)."""

    def __init__(self, op: FullHam):
        self.ptr = op.device_ptr()
        self.n = op.layout.neq

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self.n,), "typestr": "<f8", "data": (self.ptr, False), "version": 3, "strides": None}


def magnus_flow_batch(pairs, pandya: bool = False, max_iter: int = 500, raise_on_error: bool = True,
                      streams: bool = False):
    """Run several independent flows: pairs = [(HAM, HS), ...], each pair on
    its own layout.  Default: lockstep, each BCH term's 122 tiles and ladder
    tasks of all instances in one launch per kernel; streams=True: one host
    thread and stream per instance.  Returns ([FlowResult], [status]); with
    raise_on_error, raises QDError for the first failing instance."""
    n = len(pairs)
    hams = (C.c_void_p * n)(*[h.h.value for h, _ in pairs])
    hss = (C.c_void_p * n)(*[s.h.value for _, s in pairs])
    res = (FlowResult * n)()
    st = (C.c_int * n)()
    flags = _flags(pandya) | (QD_BATCH_STREAMS if streams else 0)
    rc = lib().qd_magnus_flow_batch(n, hams, hss, flags, int(max_iter), res, st)
    out = [res[i] for i in range(n)], [int(st[i]) for i in range(n)]
    if raise_on_error:
        check(rc)
    return out


# ---- host-side inputs (the reference's HFQDmod / generate_ME) ----------------
def tbme_write(emax: int, path: str, nthreads: int = 0, quad: bool = False) -> None:
    """Write ME.bin (the reference's Coulomb TBME stream file) for emax shells.
    quad: v_int in __float128 throughout (needed from emax ~ 15 on; without
    it the reference's real(8) sums are kept)."""
    import os

    check(lib().qd_tbme_write(int(emax), path.encode(), int(nthreads or (os.cpu_count() or 1)),
                              QD_TBME_QUAD if quad else 0))


def hf_hamiltonian(nbody: int, emax: int, hw: float, mebin: str | None = None, nthreads: int = 0, mix: float = 1.0,
                   quad: bool = False):
    """Hartree-Fock for N electrons in emax shells at hbar-omega = hw: returns
    (vec, eig, iterations): the normal-ordered HF Hamiltonian in vectorize
    order (vec[0] = E_HF) and the HF single-particle energies (states order),
    ready for Layout(nbody, emax, eig) and FullHam(..., vec).  mix < 1 damps
    the density update (1 = the reference's plain iteration); quad computes
    the TBMEs with v_int in __float128 (see tbme_write)."""
    import os

    L = Layout(nbody, emax, device=HOST_ONLY)
    eig = np.zeros(emax * (emax + 1), np.float64)
    vec = np.zeros(L.neq, np.float64)
    it = C.c_int()
    check(lib().qd_hf_hamiltonian(int(nbody), int(emax), float(hw), mebin.encode() if mebin else None,
                                  int(nthreads or (os.cpu_count() or 1)), float(mix),
                                  QD_TBME_QUAD if quad else 0, _d(eig), _d(vec), L.neq, C.byref(it)))
    return vec, eig, it.value


def v_int(qi, qj, qk, ql, hw: float = 1.0, quad: bool = False) -> float:
    """Coulomb matrix element v_int of the reference, q = (n, ml, ms); quad:
    every sum in __float128 instead of the reference's real(8)."""
    arrs = [(C.c_int * 3)(*[int(x) for x in q]) for q in (qi, qj, qk, ql)]
    fn = lib().qd_v_int_quad if quad else lib().qd_v_int
    return float(fn(*arrs, float(hw)))


def hamiltonian_write(layout: Layout, vec: np.ndarray, path: str) -> None:
    """Write a vectorize-order operator in the reference's export_hamiltonian
    file format (ME_general.f90:207-282)."""
    v = np.ascontiguousarray(vec, np.float64)
    if v.size != layout.neq:
        raise ValueError("hamiltonian_write: %d entries given, layout has %d" % (v.size, layout.neq))
    check(lib().qd_hamiltonian_write(layout.h, v.ctypes.data_as(_dp), os.fsencode(path)))


def hamiltonian_read(layout: Layout, path: str) -> np.ndarray:
    """Read a file of the reference's import_hamiltonian format
    (ME_general.f90:284-361) into a vectorize-order array."""
    v = np.empty(layout.neq, np.float64)
    check(lib().qd_hamiltonian_read(layout.h, v.ctypes.data_as(_dp), os.fsencode(path)))
    return v


def export_hamiltonian(H: "FullHam", path: str) -> None:
    check(lib().qd_export_hamiltonian(H.h, os.fsencode(path)))


def import_hamiltonian(H: "FullHam", path: str) -> None:
    check(lib().qd_import_hamiltonian(H.h, os.fsencode(path)))


def gemm_split(A, B, C=None, alpha: float = 1.0, beta: float = 0.0, trans_a: bool = False, trans_b: bool = False,
               slices: int = 8, device: int = 0, stream=None):
    """C = alpha op(A) op(B) + beta C in the split form (qd_gemm_split) on
    row-major float64 CUDA tensors (torch); op(X) = X.T when trans_x.
    Returns C (allocated when not given)."""
    import torch

    for X in (A, B):
        if X.dtype != torch.float64 or not X.is_cuda or not X.is_contiguous() or X.dim() != 2:
            raise ValueError("gemm_split: A and B must be contiguous 2-D float64 CUDA tensors")
    m, k = (A.shape[1], A.shape[0]) if trans_a else (A.shape[0], A.shape[1])
    k2, n = (B.shape[1], B.shape[0]) if trans_b else (B.shape[0], B.shape[1])
    if k != k2:
        raise ValueError(f"gemm_split: inner dimensions {k} and {k2} differ")
    if C is None:
        C = torch.zeros((m, n), dtype=torch.float64, device=A.device)
        beta = 0.0
    elif C.shape != (m, n) or not C.is_contiguous() or C.dtype != torch.float64:
        raise ValueError("gemm_split: C must be a contiguous float64 tensor of shape (m, n)")
    st = stream if stream is not None else torch.cuda.current_stream(A.device).cuda_stream
    # row-major X is the column-major X^T: C^T = alpha op(B)^T op(A)^T + beta C^T
    tb, ta = (b"T" if trans_b else b"N"), (b"T" if trans_a else b"N")
    check(lib().qd_gemm_split(int(device), st, tb, ta, n, m, k, float(alpha),
                              B.data_ptr(), B.shape[1], A.data_ptr(), A.shape[1], float(beta), C.data_ptr(), n,
                              int(slices)))
    return C
