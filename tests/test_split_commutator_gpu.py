"""The split form of the block contractions (qd_layout_set_split) inside the
commutator, the BCH series and the Magnus flow, against the plain FP64
engine on the same inputs (the FP64 engine itself is pinned to the oracle in
test_parity_gpu.py).  Every comparison states its error bar:

* 8 slices: the commutator is FP64-accurate, 1e-12 relative per part (the
  plain form's own bar against the oracle);
* 4 slices: 2^-28-scale truncation, 1e-7 relative per part;
* the N=6, R=10 flow (hbar-omega = 1) with 4 slices: |dE_gs| <= 1e-6 against
  the FP64 flow, the acceptance bar of the split form."""
import numpy as np
import pytest

import oracle
import qd_imsrg_b200 as qd
from helpers import compare_parts

pytestmark = pytest.mark.gpu


def _ops(n, R, seed):
    P = qd.Layout(n, R)
    O = oracle.Layout(n, R)
    a = qd.random_operator(P, -1, seed)
    b = qd.random_operator(P, 1, seed + 1)
    return P, O, a, b


def _commutator(P, a, b, pandya, slices):
    P.split = slices
    A, B, C = qd.FullHam(P, -1, a), qd.FullHam(P, 1, b), qd.FullHam(P, 1)
    qd.commutator(A, B, C, pandya)
    out = C.download()
    for X in (A, B, C):
        X.close()
    return out


@pytest.mark.parametrize("n,R", [(2, 4), (6, 5), (12, 6), (6, 8)])
@pytest.mark.parametrize("pandya", [False, True])
def test_commutator_8_slices_is_fp64(n, R, pandya):
    P, O, a, b = _ops(n, R, 700 + n + R)
    ref = _commutator(P, a, b, pandya, 0)
    got = _commutator(P, a, b, pandya, 8)
    compare_parts(O, got, ref, 1e-12)


@pytest.mark.parametrize("n,R", [(6, 5), (12, 6)])
@pytest.mark.parametrize("pandya", [False, True])
def test_commutator_4_slices(n, R, pandya):
    P, O, a, b = _ops(n, R, 800 + n + R)
    ref = _commutator(P, a, b, pandya, 0)
    got = _commutator(P, a, b, pandya, 4)
    res = compare_parts(O, got, ref, 1e-7)
    # the slices do change the result: the split form is really in use
    assert max(r for r, _ in res.values()) > 1e-14


def test_bch_with_split_matches_fp64():
    n, R = 6, 5
    P, O, a, b = _ops(n, R, 900)
    g = np.zeros_like(a)
    nn, mp = n, P.msp - n
    o = 1 + nn * nn + mp * mp
    g[o:o + mp * nn] = 0.2 * a[o:o + mp * nn]
    for q in range(P.nblock):
        nh, nb, npp = (int(x) for x in P.dims[q, :3])
        s = int(P.offs[q, 2])
        g[s:s + npp * nh] = 0.2 * a[s:s + npp * nh]
    outs = {}
    for slices in (0, 8):
        P.split = slices
        G, H, HS = qd.FullHam(P, -1, g), qd.FullHam(P, 1, b), qd.FullHam(P, 1)
        ws = [qd.FullHam(P, 1) for _ in range(5)]
        hcc, occ = qd.CCMat(P, 1.0), qd.CCMat(P, -1.0)
        nt = qd.bch_expand(HS, G, H, *ws, hcc, occ, pandya=True)
        outs[slices] = (nt, HS.download())
    assert outs[0][0] == outs[8][0]
    compare_parts(O, outs[8][1], outs[0][1], 1e-12)


def test_layout_split_setting():
    P = qd.Layout(2, 3)
    assert P.split == 0
    P.split = 5
    assert P.split == 5
    with pytest.raises(qd.QDError):
        P.split = 9
    P.split = 0


@pytest.fixture(scope="module")
def hf6():
    vec, eig, _ = qd.hf_hamiltonian(6, 10, 1.0)
    return vec, eig


@pytest.mark.parametrize("slices", [4, 8])
def test_config1_flow_split(hf6, slices):
    vec, eig = hf6
    res = {}
    for s in (0, slices):
        P = qd.Layout(6, 10, eig=eig)
        P.split = s
        H, HS = qd.FullHam(P, 1, vec), qd.FullHam(P, 1)
        _, r = qd.magnus_flow(H, HS, pandya=True, max_iter=200)
        res[s] = r.E0
        H.close()
        HS.close()
        P.close()
    assert abs(res[slices] - res[0]) <= 1e-6, (res, slices)
    if slices == 8:
        assert res[slices] == pytest.approx(res[0], rel=1e-10)
