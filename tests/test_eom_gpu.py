"""EOM matrix-vector product on the device (qd_eom_matvec) against the
literal restatement of HQ_comm_1b/2b (commutators.f90:1162-1272) over every
(M_L, M_S)-conserving 1p1h and 2p2h entry, 1e-12 relative; and at larger
bases against the oracle's commutator average (the identity the CPU test
pins), with every non-excitation part of HQ zero."""
import numpy as np
import pytest

import oracle
import qd_imsrg_b200 as qd
from helpers import compare_parts
from oracle.eom import HQ
from test_eom_oracle import _restrict

pytestmark = pytest.mark.gpu


def _inputs(n, R, seed):
    P, O = qd.Layout(n, R), oracle.Layout(n, R)
    h = qd.random_operator(P, 1, seed)
    q = _restrict(O, qd.random_operator(P, 1, seed + 1))
    return P, O, h, q


@pytest.mark.parametrize("n,R", [(2, 3), (6, 3)])
def test_matches_literal_hq_comm(n, R):
    P, O, h, q = _inputs(n, R, 90 + n + R)
    out = qd.FullHam(P, 1)
    qd.eom_matvec(qd.FullHam(P, 1, h), qd.FullHam(P, 1, q), out)
    hq = out.download()
    ref = HQ(O, oracle.Op(O, 1, h), h, 1, oracle.Op(O, 1, q), q)
    Hq = oracle.Op(O, 1, hq)
    m, mp = O.m, O.m - O.n
    o_fph = 1 + O.n * O.n + mp * mp
    qn = O.qn
    g, w = [], []
    for a in range(O.n + 1, m + 1):
        for i in range(1, O.n + 1):
            if tuple(qn[a - 1][1:]) == tuple(qn[i - 1][1:]):
                g.append(hq[o_fph + (a - O.n - 1) + (i - 1) * mp])
                w.append(ref.comm_1b(a, i))
    for a in range(O.n + 1, m + 1):
        for b in range(a + 1, m + 1):
            for i in range(1, O.n + 1):
                for j in range(i + 1, O.n + 1):
                    if all(qn[a - 1][k] + qn[b - 1][k] == qn[i - 1][k] + qn[j - 1][k] for k in (1, 2)):
                        g.append(oracle.v_elem(a, b, i, j, Hq))
                        w.append(ref.comm_2b(a, b, i, j))
    g, w = np.array(g), np.array(w)
    assert np.linalg.norm(g - w) <= 1e-12 * np.linalg.norm(w)


@pytest.mark.parametrize("n,R", [(6, 5), (12, 6)])
def test_matches_commutator_average(n, R):
    P, O, h, q = _inputs(n, R, 70 + n + R)
    out = qd.FullHam(P, 1)
    qd.eom_matvec(qd.FullHam(P, 1, h), qd.FullHam(P, 1, q), out)
    H = oracle.Op(O, 1, h)
    parts = []
    for herm in (1, -1):
        C = oracle.Op(O, 1)
        oracle.commutator(H, oracle.Op(O, herm, q), C, pandya=True)
        parts.append(C.get())
    ref = _restrict(O, 0.5 * (parts[0] + parts[1]))
    compare_parts(O, out.download(), ref, 1e-12)
