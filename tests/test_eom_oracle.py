"""The EOM matrix-vector product (HQ_comm_1b/2b, commutators.f90:1162-1272)
is the particle-hole and pphh part of [H, Q] for an excitation operator Q;
with Q_exc = (Q+ + Q-)/2, Q+- the same amplitudes as herm +-1 operators,
it is the average of two full commutators (particle-hole channel on).  Checked
here on the CPU with the oracle's commutator against the literal restatement,
over every (M_L, M_S)-conserving ph and pphh entry."""
import numpy as np
import pytest

import oracle
from helpers import numpy_random_op
from oracle.eom import HQ


def _restrict(O, vec):
    """Keep fph and every block's Vpphh; zero the rest."""
    n, m = O.n, O.m
    mp = m - n
    out = np.zeros_like(vec)
    o = 1 + n * n + mp * mp
    out[o:o + mp * n] = vec[o:o + mp * n]
    for q in range(O.nblock):
        nh, npp = int(O.dims[q][0]), int(O.dims[q][2])
        s = int(O.offs[q][2])
        out[s:s + npp * nh] = vec[s:s + npp * nh]
    return out


@pytest.mark.parametrize("n,R", [(2, 3), (6, 3)])
def test_matvec_is_commutator_average(n, R):
    O = oracle.Layout(n, R)
    rng = np.random.default_rng(11 + n + R)
    h = numpy_random_op(O, 1, rng)
    q = _restrict(O, numpy_random_op(O, 1, rng))
    H = oracle.Op(O, 1, h)
    out = []
    for herm in (1, -1):
        Q, C = oracle.Op(O, herm, q), oracle.Op(O, 1)
        oracle.commutator(H, Q, C, pandya=True)
        out.append(C.get())
    hq = 0.5 * (out[0] + out[1])
    ref = HQ(O, H, h, 1, oracle.Op(O, 1, q), q)
    n_, m = O.n, O.m
    mp = m - n_
    o_fph = 1 + n_ * n_ + mp * mp
    qn = O.qn
    got1, want1 = [], []
    for a in range(n_ + 1, m + 1):
        for i in range(1, n_ + 1):
            if qn[a - 1][1] != qn[i - 1][1] or qn[a - 1][2] != qn[i - 1][2]:
                continue
            got1.append(hq[o_fph + (a - n_ - 1) + (i - 1) * mp])
            want1.append(ref.comm_1b(a, i))
    got2, want2 = [], []
    Hq = oracle.Op(O, 1, hq)
    for a in range(n_ + 1, m + 1):
        for b in range(a + 1, m + 1):
            for i in range(1, n_ + 1):
                for j in range(i + 1, n_ + 1):
                    if qn[a - 1][1] + qn[b - 1][1] != qn[i - 1][1] + qn[j - 1][1]:
                        continue
                    if qn[a - 1][2] + qn[b - 1][2] != qn[i - 1][2] + qn[j - 1][2]:
                        continue
                    got2.append(oracle.v_elem(a, b, i, j, Hq))
                    want2.append(ref.comm_2b(a, b, i, j))
    got1, want1, got2, want2 = map(np.array, (got1, want1, got2, want2))
    assert got1.size > 0 and got2.size > 0
    assert np.linalg.norm(got1 - want1) <= 1e-12 * np.linalg.norm(want1)
    assert np.linalg.norm(got2 - want2) <= 1e-12 * np.linalg.norm(want2)


@pytest.mark.parametrize("n,R", [(2, 3), (6, 4)])
def test_dense_ladder_storage_matches_blocked_at_the_scalar_target(n, R):
    """matvec_prod with the reference's dense storage of the ladder operator
    (unwrap, Q_elem over fermionic_tp_index) equals the blocked restatement at
    (Mltarg, Mstarg) = (0, 0): the unwrap order and the signs agree."""
    from helpers import eom_scalar_positions
    from oracle.eom import _targets, eom_dim, matvec_prod

    O = oracle.Layout(n, R)
    rng = np.random.default_rng(5 + n + R)
    h = numpy_random_op(O, 1, rng)
    H = oracle.Op(O, 1, h)
    n1, n2 = eom_dim(O, 0, 0)
    v = rng.standard_normal(n1 + n2)
    w = matvec_prod(O, H, h, 1, 0, 0, v)
    q = np.zeros(O.neq)
    q[eom_scalar_positions(O)] = v
    ref = HQ(O, H, h, 1, oracle.Op(O, 1, q), q)
    one, two = _targets(O, 0, 0)
    want = [ref.comm_1b(ix + n, jx) for ix, jx in one] + [ref.comm_2b(a + n, b + n, i, j) for a, b, i, j in two]
    assert np.array_equal(np.array(want), w)


@pytest.mark.parametrize("n,R", [(6, 5), (12, 6)])
def test_eom_dim_counts_as_unwrap(n, R):
    import qd_imsrg_b200 as qd
    from oracle.eom import eom_dim

    O = oracle.Layout(n, R)
    L = qd.Layout(n, R, device=qd.HOST_ONLY)
    for t in [(0, 0), (1, 0), (-1, 2), (2, -2), (3, 0), (-4, 0), (0, 2)]:
        assert qd.eom_dim(L, *t) == eom_dim(O, *t)
    L.close()
