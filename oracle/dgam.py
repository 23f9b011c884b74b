"""dGam (src/gs_IMSRG.f90:223-273) restated with the oracle's routines, in the
reference's call order, as the checker of qd_dgam.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module."""
from __future__ import annotations

from . import (CC, Op, build_white, calc_cc, commutator_110, commutator_111, commutator_121, commutator_122,
               commutator_220, commutator_221, commutator_222)


def dgam(H: Op, DER: Op, HCC: CC, ETACC: CC) -> None:
    L = H.layout
    ETA, w1, w2 = Op(L, -1), Op(L, 1), Op(L, 1)  # allocate_everything: zero-filled
    calc_cc(H, HCC)
    HCC.set_herm(1.0)
    build_white(ETA, H)
    calc_cc(ETA, ETACC)
    ETACC.set_herm(-1.0)
    e0 = commutator_110(ETA, H) + commutator_220(ETA, H)
    commutator_111(ETA, H, DER)
    commutator_121(ETA, H, DER)
    commutator_221(ETA, H, DER, w1, w2)
    commutator_122(ETA, H, DER)
    commutator_222(ETA, H, DER, w1, HCC, ETACC)
    v = DER.get()
    v[0] = e0  # DER%E0 = ex + ex2
    DER.set(v)
