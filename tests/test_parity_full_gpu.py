"""Parity at the headline size, N=20 electrons in R=20 shells (420
spin-orbitals, 61,947,679 entries per operator), where the largest blocks of
the reference's layout exist: (nh, nph, npp) = (16, 160, 1264), cross-coupled
blocks of up to 2,880 rows, and the largest group-pair tiles of
commutator_122.

1. The FP64 commutator [Omega, H] of the seeded synthetic operators of the
   single-commutator microbenchmark (Philox seeds 2 and 1, entries
   N(0, 0.1^2), (anti)symmetrised), with the particle-hole (Pandya) channel,
   against the oracle at 1e-12 relative per stored part
   (commutators.f90:12-1132, ME_general.f90:923-952).
2. The first BCH commutator of the Magnus flow at hbar-omega = 0.5 on the
   Hartree-Fock Hamiltonian: [Omega, H] with Omega = 0.7 eta(H), eta the
   White generator, ladders only as run_magnus (magnus_IMSRG.f90:207-212,
   298-311), against the oracle at 1e-12.

Each oracle commutator takes about 20 s on 16 host cores."""
import numpy as np
import pytest

import oracle
import qd_imsrg_b200 as qd
from helpers import compare_parts

pytestmark = pytest.mark.gpu

N, R = 20, 20


def test_commutator_n20_r20_matches_oracle(gpu):
    P = qd.Layout(N, R)
    assert P.neq == 61947679
    a = qd.random_operator(P, -1, 2)
    b = qd.random_operator(P, 1, 1)
    A, B, Cq = qd.FullHam(P, -1, a), qd.FullHam(P, 1, b), qd.FullHam(P, 1)
    qd.commutator(A, B, Cq, pandya=True)
    got = Cq.download()
    for o in (A, B, Cq):
        o.close()
    P.close()
    O = oracle.Layout(N, R)
    oA, oB, oC = oracle.Op(O, -1, a), oracle.Op(O, 1, b), oracle.Op(O, 1)
    del a, b
    oracle.commutator(oA, oB, oC, pandya=True)
    ref = oC.get()
    assert got[0] == pytest.approx(ref[0], rel=1e-12, abs=1e-12)
    compare_parts(O, got, ref, rtol=1e-12)


def test_first_bch_commutator_of_the_r20_flow_matches_oracle(gpu):
    vec, eig, _ = qd.hf_hamiltonian(N, R, 0.5, mix=0.5, quad=True)
    stp = float(np.float32(0.7))  # "stp=.7" is a real(4) literal
    P = qd.Layout(N, R, eig=eig)
    H, eta, G, Cq = qd.FullHam(P, 1, vec), qd.FullHam(P, -1), qd.FullHam(P, -1), qd.FullHam(P, 1)
    qd.build_white(eta, H)
    qd.add_arrays(G, 1.0, eta, stp, G)
    qd.commutator(G, H, Cq, pandya=False)
    got = Cq.download()
    for o in (H, eta, G, Cq):
        o.close()
    P.close()
    O = oracle.Layout(N, R, eig)
    oH, oeta, oG, oC = oracle.Op(O, 1, vec), oracle.Op(O, -1), oracle.Op(O, -1), oracle.Op(O, 1)
    oracle.build_white(oeta, oH)
    oracle.add_arrays(oG, 1.0, oeta, stp, oG)
    oracle.commutator(oG, oH, oC, pandya=False)
    ref = oC.get()
    assert got[0] == pytest.approx(ref[0], rel=1e-12)
    compare_parts(O, got, ref, rtol=1e-12)
