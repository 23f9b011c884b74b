"""GPU parity: every commutator piece, the generator, the algebra and BCH of
the CUDA engine (through the C ABI) against the CPU oracle on the same
seeded inputs.  Tolerance: 1e-12 relative (Frobenius, per stored part),
the plain-form bar; scalars 1e-12 relative."""
import numpy as np
import pytest

import oracle
import qd_imsrg_b200 as qd
from helpers import compare_parts

pytestmark = pytest.mark.gpu

RTOL = 1e-12
SIZES = [(2, 3), (6, 4), (6, 5), (2, 6), (12, 6), (6, 8)]


def setup(n, R, seed, conserve=True):
    P = qd.Layout(n, R)
    O = oracle.Layout(n, R)
    a = qd.random_operator(P, -1, seed, conserve=conserve)
    b = qd.random_operator(P, 1, seed + 1, conserve=conserve)
    c = qd.random_operator(P, 1, seed + 2, conserve=conserve)
    return P, O, a, b, c


def scal(x, y):
    assert x == pytest.approx(y, rel=RTOL, abs=1e-300)


@pytest.mark.parametrize("n,R", SIZES)
@pytest.mark.parametrize("conserve", [True, False])
def test_pieces(gpu, n, R, conserve):
    P, O, a, b, c0 = setup(n, R, 100 + n + R, conserve)
    A, B = qd.FullHam(P, -1, a), qd.FullHam(P, 1, b)
    oA, oB = oracle.Op(O, -1, a), oracle.Op(O, 1, b)
    scal(qd.commutator_110(A, B), oracle.commutator_110(oA, oB))
    scal(qd.commutator_220(A, B), oracle.commutator_220(oA, oB))
    # 111 overwrites the one-body part, 121/221 accumulate, 122 overwrites the
    # two-body part, 222 accumulates: start every piece from the same C0
    for piece in ("111", "121", "221", "122", "222"):
        C, oC = qd.FullHam(P, 1, c0), oracle.Op(O, 1, c0)
        if piece == "111":
            qd.commutator_111(A, B, C); oracle.commutator_111(oA, oB, oC)
        elif piece == "121":
            qd.commutator_121(A, B, C); oracle.commutator_121(oA, oB, oC)
        elif piece == "221":
            w1, w2 = qd.FullHam(P, 1), qd.FullHam(P, 1)
            ow1, ow2 = oracle.Op(O, 1), oracle.Op(O, 1)
            qd.commutator_221(A, B, C, w1, w2); oracle.commutator_221(oA, oB, oC, ow1, ow2)
            compare_parts(O, w1.download(), ow1.get(), RTOL)
            compare_parts(O, w2.download(), ow2.get(), RTOL)
        elif piece == "122":
            qd.commutator_122(A, B, C); oracle.commutator_122(oA, oB, oC)
        else:
            w1 = qd.FullHam(P, 1)
            hcc, ecc = qd.CCMat(P, 1.0), qd.CCMat(P, -1.0)
            qd.commutator_222(A, B, C, w1, hcc, ecc)
            ow1, ohcc, oecc = oracle.Op(O, 1), oracle.CC(O, 1.0), oracle.CC(O, -1.0)
            oracle.commutator_222(oA, oB, oC, ow1, ohcc, oecc)
        compare_parts(O, C.download(), oC.get(), RTOL)


@pytest.mark.parametrize("n,R", SIZES)
def test_pandya_channel(gpu, n, R):
    P, O, a, b, c0 = setup(n, R, 200 + n + R)
    A, B = qd.FullHam(P, -1, a), qd.FullHam(P, 1, b)
    oA, oB = oracle.Op(O, -1, a), oracle.Op(O, 1, b)
    hcc, ecc = qd.CCMat(P, 1.0), qd.CCMat(P, -1.0)
    qd.calc_cc(B, hcc)
    qd.calc_cc(A, ecc)
    ohcc, oecc = oracle.CC(O, 1.0), oracle.CC(O, -1.0)
    oracle.calc_cc(oB, ohcc)
    oracle.calc_cc(oA, oecc)
    assert np.array_equal(hcc.download(), ohcc.get_X())  # gathers: bit-exact
    assert np.array_equal(ecc.download(), oecc.get_X())
    C, oC = qd.FullHam(P, 1, c0), oracle.Op(O, 1, c0)
    qd.commutator_222(A, B, C, None, hcc, ecc)
    oracle.commutator_222(oA, oB, oC, oracle.Op(O, 1), ohcc, oecc)
    compare_parts(O, C.download(), oC.get(), RTOL)


@pytest.mark.parametrize("n,R", SIZES)
@pytest.mark.parametrize("pandya", [False, True])
def test_full_commutator(gpu, n, R, pandya):
    P, O, a, b, _ = setup(n, R, 300 + n + R)
    A, B, C = qd.FullHam(P, -1, a), qd.FullHam(P, 1, b), qd.FullHam(P, 1)
    oA, oB, oC = oracle.Op(O, -1, a), oracle.Op(O, 1, b), oracle.Op(O, 1)
    qd.commutator(A, B, C, pandya)
    oracle.commutator(oA, oB, oC, pandya)
    compare_parts(O, C.download(), oC.get(), RTOL)


@pytest.mark.parametrize("n,R", [(6, 5), (12, 6)])
def test_generator_energies_algebra(gpu, n, R):
    P, O, a, b, c = setup(n, R, 400 + n + R)
    # a Hamiltonian-like operator: dominant diagonal one-body energies so the
    # White denominators are far from zero
    h = b.copy()
    nn, mp = n, P.msp - n
    F = h[1:1 + nn * nn].reshape(nn, nn, order="F"); F[np.diag_indices(nn)] -= 3.0
    h[1:1 + nn * nn] = F.reshape(-1, order="F")
    F = h[1 + nn * nn:1 + nn * nn + mp * mp].reshape(mp, mp, order="F"); F[np.diag_indices(mp)] += 3.0
    h[1 + nn * nn:1 + nn * nn + mp * mp] = F.reshape(-1, order="F")
    H, oH = qd.FullHam(P, 1, h), oracle.Op(O, 1, h)
    E, oE = qd.FullHam(P, -1), oracle.Op(O, -1)
    qd.build_white(E, H)
    oracle.build_white(oE, oH)
    compare_parts(O, E.download(), oE.get(), RTOL)
    scal(qd.mbpt2(H), oracle.mbpt2(oH))
    scal(qd.mat_2_norm(H), oracle.mat_2_norm(oH))
    X, oX = qd.FullHam(P, 1), oracle.Op(O, 1)
    qd.add_arrays(H, 0.7, qd.FullHam(P, 1, c), -1.3, X)
    oracle.add_arrays(oH, 0.7, oracle.Op(O, 1, c), -1.3, oX)
    assert np.array_equal(X.download(), oX.get())
    Y = qd.FullHam(P, 1)
    qd.copy_arrays(X, Y)
    assert np.array_equal(Y.download(), oX.get())
    qd.set_to_zero(Y)
    assert not Y.download().any()


@pytest.mark.parametrize("n,R", [(2, 4), (6, 5)])
@pytest.mark.parametrize("pandya", [False, True])
def test_bch_expand(gpu, n, R, pandya):
    P, O, a, b, _ = setup(n, R, 500 + n + R)
    # a generator-like Omega: only fph and Vpphh non-zero, small enough for
    # the BCH series to truncate after several terms
    g = np.zeros_like(a)
    nn, mp = n, P.msp - n
    o = 1 + nn * nn + mp * mp
    g[o:o + mp * nn] = 0.2 * a[o:o + mp * nn]
    for q in range(P.nblock):
        nh, nb, npp = (int(x) for x in P.dims[q, :3])
        s = int(P.offs[q, 2])
        g[s:s + npp * nh] = 0.2 * a[s:s + npp * nh]
    G, H, HS = qd.FullHam(P, -1, g), qd.FullHam(P, 1, b), qd.FullHam(P, 1)
    ws = [qd.FullHam(P, 1) for _ in range(5)]
    hcc, occ = qd.CCMat(P, 1.0), qd.CCMat(P, -1.0)
    nt = qd.bch_expand(HS, G, H, *ws, hcc, occ, pandya=pandya)
    oG, oH, oHS = oracle.Op(O, -1, g), oracle.Op(O, 1, b), oracle.Op(O, 1)
    ont = oracle.bch_expand(oHS, oG, oH, pandya=pandya)
    assert nt == ont and nt > 2
    compare_parts(O, HS.download(), oHS.get(), RTOL)
