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


@pytest.mark.parametrize("n,R,ml,ms", [(2, 3, 1, 0), (6, 4, 0, 0), (6, 4, 1, 0), (6, 4, -1, 2), (6, 4, 2, -2),
                                       (6, 5, 3, 0), (12, 5, -2, 0)])
def test_target_matches_literal_matvec_prod(n, R, ml, ms):
    """qd_eom_matvec_target against the literal matvec_prod (unwrap,
    HQ_comm_1b/2b on every target entry, rewrap; EOM_IMSRG.f90:551-649) for
    scalar and non-scalar targets, 1e-12 relative, on a dense one-body H."""
    from oracle.eom import eom_dim, matvec_prod

    P, O = qd.Layout(n, R), oracle.Layout(n, R)
    h = qd.random_operator(P, 1, 300 + n + R, conserve=False)
    n1, n2 = eom_dim(O, ml, ms)
    assert qd.eom_dim(P, ml, ms) == (n1, n2) and n2 > 0
    v = np.random.default_rng(n + R + 7 * ml + ms).standard_normal(n1 + n2)
    H = qd.FullHam(P, 1, h)
    got = qd.eom_matvec_target(H, ml, ms, v)
    got2 = qd.eom_matvec_target(H, ml, ms, v)  # a second call reuses the target's tables
    want = matvec_prod(O, oracle.Op(O, 1, h), h, 1, ml, ms, v)
    assert np.array_equal(got, got2)
    assert np.linalg.norm(got[:n1] - want[:n1]) <= 1e-12 * np.linalg.norm(want[:n1])
    assert np.linalg.norm(got[n1:] - want[n1:]) <= 1e-12 * np.linalg.norm(want[n1:])


@pytest.mark.parametrize("n,R", [(12, 6), (20, 10)])
def test_scalar_target_matches_commutator_path(n, R):
    """At (0, 0) the target kernels equal qd_eom_matvec, which computes the
    same product as the average of two full commutators (particle-hole
    channel on): two independent routes, 1e-12 relative."""
    from helpers import eom_scalar_positions

    P, O = qd.Layout(n, R), oracle.Layout(n, R)
    pos = eom_scalar_positions(O)
    n1, n2 = qd.eom_dim(P, 0, 0)
    assert pos.size == n1 + n2
    h = qd.random_operator(P, 1, 500 + n + R)
    v = np.random.default_rng(n * R).standard_normal(n1 + n2)
    q = np.zeros(P.neq)
    q[pos] = v
    H, out = qd.FullHam(P, 1, h), qd.FullHam(P, 1)
    qd.eom_matvec(H, qd.FullHam(P, 1, q), out)
    want = out.download()[pos]
    got = qd.eom_matvec_target(H, 0, 0, v)
    assert np.linalg.norm(got[:n1] - want[:n1]) <= 1e-12 * np.linalg.norm(want[:n1])
    assert np.linalg.norm(got[n1:] - want[n1:]) <= 1e-12 * np.linalg.norm(want[n1:])


def test_target_rejects_a_wrong_length():
    P = qd.Layout(6, 4)
    n1, n2 = qd.eom_dim(P, 1, 0)
    H = qd.FullHam(P, 1, qd.random_operator(P, 1, 3))
    with pytest.raises(qd.QDError):
        qd.eom_matvec_target(H, 1, 0, np.zeros(n1 + n2 + 1))
