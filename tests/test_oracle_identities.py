"""CPU checks of the oracle (the C++ restatement in oracle/): layout numbers
of the reference's index builders, algebraic identities of the commutator,
bit-identity of its zero-term skipping, and the reference's quirks."""
import numpy as np
import pytest

import oracle
from helpers import compare_parts, numpy_random_op, part_slices


@pytest.mark.parametrize("n,R,neq,nblock,big", [
    (6, 10, 571598, 111, (3, 24, 168)),
    (20, 20, 61947679, 231, (16, 160, 1264)),
    (6, 16, 14273368, 183, (3, 42, 707)),
    (12, 16, 13660661, 183, (8, 76, 668)),
    (30, 20, 59406670, 231, (29, 222, 1189)),
])
def test_layout_sizes_match_reference_index_builders(n, R, neq, nblock, big):
    # neq = get_num_elements (ME_general.f90:1755-1778); nblock = 12 emax - 9
    L = oracle.Layout(n, R)
    assert L.neq == neq
    assert L.nblock == nblock == 12 * R - 9
    d = L.dims
    assert tuple(int(x) for x in d[np.argmax(d[:, 2]), :3]) == big
    # cross-coupled blocks: 10*MLmax+5 with MLmax = 2(R-1); every ordered pair once
    assert L.ccn == 10 * 2 * (R - 1) + 5
    assert int(L.cc_r.sum()) == L.m * L.m
    assert int(L.cc_nb.sum()) == n * (L.m - n)


def _ops(n, R, seed, conserve=True):
    L = oracle.Layout(n, R)
    rng = np.random.default_rng(seed)
    A = oracle.Op(L, -1, numpy_random_op(L, -1, rng, conserve))
    B = oracle.Op(L, 1, numpy_random_op(L, 1, rng, conserve))
    return L, A, B


@pytest.mark.parametrize("n,R", [(2, 3), (6, 4), (6, 5), (2, 4)])
@pytest.mark.parametrize("pandya", [False, True])
def test_commutator_antisymmetry(n, R, pandya):
    L, A, B = _ops(n, R, 11)
    C1, C2 = oracle.Op(L, 1), oracle.Op(L, 1)
    oracle.commutator(A, B, C1, pandya)
    oracle.commutator(B, A, C2, pandya)
    c1, c2 = C1.get(), C2.get()
    assert np.abs(c1).max() > 1e-3
    assert np.abs(c1 + c2).max() < 1e-14


@pytest.mark.parametrize("n,R", [(2, 3), (6, 5)])
def test_antihermitian_with_hermitian_is_hermitian(n, R):
    L, A, B = _ops(n, R, 12)
    C = oracle.Op(L, 1)
    oracle.commutator(A, B, C, True)
    c = C.get()
    for q in range(L.nblock):
        nh, nb, npp = (int(x) for x in L.dims[q, :3])
        for k, sz in ((0, nh), (1, npp), (3, nb)):
            if sz:
                o = int(L.offs[q, k])
                X = c[o:o + sz * sz].reshape(sz, sz, order="F")
                assert np.abs(X - X.T).max() < 1e-15
    n_, mp = L.n, L.m - L.n
    X = c[1:1 + n_ * n_].reshape(n_, n_, order="F")
    assert np.abs(X - X.T).max() < 1e-15


@pytest.mark.parametrize("n,R,conserve", [(2, 3, True), (6, 4, False), (6, 5, True)])
def test_122_skip_is_bit_identical_to_literal_loop(n, R, conserve):
    L, A, B = _ops(n, R, 13, conserve)
    D1, D2 = oracle.Op(L, 1), oracle.Op(L, 1)
    oracle.commutator_122(A, B, D1, literal=True)
    oracle.commutator_122(A, B, D2, literal=False)
    assert np.array_equal(D1.get(), D2.get())


def test_linearity():
    L, A, B = _ops(6, 4, 14)
    rng = np.random.default_rng(99)
    B2 = oracle.Op(L, 1, numpy_random_op(L, 1, rng))
    Bs = oracle.Op(L, 1)
    oracle.add_arrays(B, 1.0, B2, 1.0, Bs)
    C1, C2, C3 = oracle.Op(L, 1), oracle.Op(L, 1), oracle.Op(L, 1)
    oracle.commutator(A, B, C1, True)
    oracle.commutator(A, B2, C2, True)
    oracle.commutator(A, Bs, C3, True)
    assert np.abs(C1.get() + C2.get() - C3.get()).max() < 1e-13


def test_mat_2_norm_sums_one_and_two_body_parts():
    # ME_general.f90:2112-2138: fph, fpp, fhh, then per block Vhhhh, Vpppp,
    # Vpphh, Vphph, Vphhh, Vppph (E0 excluded)
    L, A, B = _ops(6, 4, 15)
    v = B.get()
    ref = np.sqrt(np.sum(v[1:] ** 2))
    assert oracle.mat_2_norm(B) == pytest.approx(ref, rel=1e-14)
    n, mp = L.n, L.m - L.n
    nb1 = n * n + mp * mp + mp * n
    v[1 + nb1:] *= 7.0   # the two-body parts count
    v[0] = 123.0         # E0 does not
    B.set(v)
    assert oracle.mat_2_norm(B) == pytest.approx(np.sqrt(np.sum(v[1:] ** 2)), rel=1e-14)


def test_bch_with_zero_generator_returns_H():
    L, A, B = _ops(6, 4, 16)
    G = oracle.Op(L, -1)
    HS = oracle.Op(L, 1)
    n = oracle.bch_expand(HS, G, B, pandya=False)
    assert n == 1
    assert np.array_equal(HS.get(), B.get())


def test_magnus_without_cc_drops_particle_hole_channel():
    # run_magnus never fills the cross-coupled X: commutator_222 adds exactly
    # the ladders; with calc_cc on both operators the ph channel appears.
    L, A, B = _ops(6, 4, 17)
    C1, C2 = oracle.Op(L, 1), oracle.Op(L, 1)
    oracle.commutator(A, B, C1, False)
    oracle.commutator(A, B, C2, True)
    d = C2.get() - C1.get()
    n, mp = L.n, L.m - L.n
    nb1 = 1 + n * n + mp * mp + mp * n
    assert np.abs(d[:nb1]).max() == 0.0
    assert np.abs(d[nb1:]).max() > 1e-3


def test_block_sampler_phases_make_the_whole_commutator():
    # the CPU baseline times phases of oracle.Sampler; without the Pandya
    # channel the phases together are exactly one commutator (with it, each
    # phase forms only its own cross-coupled products: the same work, split)
    L = oracle.Layout(6, 5)
    rng = np.random.default_rng(17)
    a, b = numpy_random_op(L, -1, rng), numpy_random_op(L, 1, rng)
    A, B = oracle.Op(L, -1, a), oracle.Op(L, 1, b)
    full = oracle.Op(L, 1)
    oracle.commutator(A, B, full, pandya=False)
    samp = oracle.Op(L, 1)
    S = oracle.Sampler(A)
    for ph in range(3):
        S.run(A, B, samp, 3, ph, pandya=False)
    compare_parts(L, samp.get(), full.get(), rtol=1e-13, atol=1e-15)
