"""CPU checks of the product's host-side layout (qd_layout_create with
QD_HOST_ONLY) against the oracle's independent restatement of reindex and
build_cross_coupled, and of the seeded synthetic-operator generator."""
import numpy as np
import pytest

import oracle
import qd_imsrg_b200 as qd


@pytest.mark.parametrize("n,R", [(2, 3), (6, 4), (6, 10), (12, 8), (20, 20), (30, 20)])
def test_host_layout_matches_oracle_reindex(n, R):
    P = qd.Layout(n, R, device=qd.HOST_ONLY)
    O = oracle.Layout(n, R)
    assert (P.neq, P.nblock, P.msp) == (O.neq, O.nblock, O.m)
    assert np.array_equal(P.dims[:, :3], O.dims[:, :3])
    assert np.array_equal(P.offs, O.offs)
    for q in range(P.nblock):
        for kind in range(3):
            assert np.array_equal(P.pairs(q, kind), O.pairs(q + 1, kind))


def test_block_quantum_numbers():
    P = qd.Layout(6, 5, device=qd.HOST_ONLY)
    O = oracle.Layout(6, 5)
    assert np.array_equal(P.dims[:, 3:5], O.dims[:, 3:5])


def test_holes_must_be_the_first_states():
    m = 5 * 6
    eig = np.arange(m, 0, -1, dtype=float)  # lowest energies are the LAST states
    with pytest.raises(qd.QDError) as e:
        qd.Layout(6, 5, eig=eig, device=qd.HOST_ONLY)
    assert e.value.code == 2
    with pytest.raises(ValueError):
        oracle.Layout(6, 5, eig)


def test_random_operator_properties():
    L = qd.Layout(6, 6, device=qd.HOST_ONLY)
    for herm in (1, -1):
        v = qd.random_operator(L, herm, seed=7)
        w = qd.random_operator(L, herm, seed=7)
        assert np.array_equal(v, w)
        assert not np.array_equal(v, qd.random_operator(L, herm, seed=8))
        assert v[0] == 0.0
        n, mp = L.nbody, L.msp - L.nbody
        for o, k in ((1, n), (1 + n * n, mp)):
            X = v[o:o + k * k].reshape(k, k, order="F")
            assert np.array_equal(X, herm * X.T)
        for q in range(L.nblock):
            nh, nb, npp = (int(x) for x in L.dims[q, :3])
            for slot, k in ((0, nh), (1, npp), (3, nb)):
                if k:
                    o = int(L.offs[q, slot])
                    X = v[o:o + k * k].reshape(k, k, order="F")
                    assert np.array_equal(X, herm * X.T)
    v = qd.random_operator(L, 1, seed=3, sigma=0.1, conserve=False)
    # the free (not symmetrised) Vpphh, Vppph, Vphhh entries are iid N(0, 0.1^2)
    chunks = []
    for q in range(L.nblock):
        nh, nb, npp = (int(x) for x in L.dims[q, :3])
        for slot, sz in ((2, npp * nh), (4, npp * nb), (5, nb * nh)):
            o = int(L.offs[q, slot])
            chunks.append(v[o:o + sz])
    free = np.concatenate(chunks)
    assert free.size > 1000
    assert abs(free.mean()) < 0.01 and 0.095 < free.std() < 0.105


def test_random_operator_conserves_ml_ms():
    L = qd.Layout(6, 6, device=qd.HOST_ONLY)
    O = oracle.Layout(6, 6)
    g = O.qn[:, 1] * 10 + O.qn[:, 2]
    v = qd.random_operator(L, 1, seed=5, conserve=True)
    n, mp = L.nbody, L.msp - L.nbody
    fph = v[1 + n * n + mp * mp:1 + n * n + mp * mp + mp * n].reshape(mp, n, order="F")
    assert np.all(fph[g[n:, None] != g[None, :n]] == 0.0)
    assert np.any(fph[g[n:, None] == g[None, :n]] != 0.0)
