"""The blocked oracle (a restatement of the reference's loops) against an
independent dense statement of the IM-SRG(2) commutator (oracle/dense.py),
and the CUDA path against the same dense statement.

Agreement here pins the commutator sequence (110, 220, 111, 121, 221, 122,
222 with and without the Pandya channel) to the textbook formulas rather
than only to a second reading of the same Fortran."""
import numpy as np
import pytest

import oracle as orc
from helpers import compare_parts, numpy_random_op
from oracle import dense

BASES = [(2, 3), (6, 3), (2, 4), (6, 4), (12, 4)]


def _ops(L, hA, hB, seed):
    rng = np.random.default_rng(seed)
    return numpy_random_op(L, hA, rng), numpy_random_op(L, hB, rng)


def _dense_result(L, a, hA, b, hB, pandya):
    m = L.m
    c0, c1, c2 = dense.commutator(dense.to_dense(L, a, hA), dense.to_dense(L, b, hB), np.arange(m) < L.n,
                                  pandya=pandya)
    return dense.from_dense(L, c0, c1, c2), c2


@pytest.mark.parametrize("n,R", BASES)
def test_dense_round_trip_and_v_elem(n, R):
    L = orc.Layout(n, R)
    a, _ = _ops(L, -1, 1, 3)
    A = orc.Op(L, -1, a)
    E0, f, V = dense.to_dense(L, a, -1)
    assert np.array_equal(dense.from_dense(L, E0, f, V), a)
    rng = np.random.default_rng(4)
    for t in rng.integers(0, L.m, (400, 4)):
        assert orc.v_elem(*(int(x) + 1 for x in t), A) == V[tuple(t)]


@pytest.mark.parametrize("n,R", BASES)
@pytest.mark.parametrize("hA,hB", [(-1, 1), (1, 1), (-1, -1)])
@pytest.mark.parametrize("pandya", [True, False])
def test_oracle_matches_dense(n, R, hA, hB, pandya):
    L = orc.Layout(n, R)
    a, b = _ops(L, hA, hB, 11 + n + R)
    C = orc.Op(L, 1)
    orc.commutator(orc.Op(L, hA, a), orc.Op(L, hB, b), C, pandya=pandya)
    ref, c2 = _dense_result(L, a, hA, b, hB, pandya)
    compare_parts(L, C.get(), ref, rtol=1e-12, atol=1e-15 * np.abs(ref).max())
    # [A,B]^T = -hA hB [A,B]: the dense result has that symmetry and no
    # entries outside the stored block structure
    back = dense.to_dense(L, ref, -hA * hB)[2]
    assert np.abs(c2 - back).max() < 1e-14


def test_particle_hole_channel_is_not_trivial():
    L = orc.Layout(6, 4)
    a, b = _ops(L, -1, 1, 21)
    on, _ = _dense_result(L, a, -1, b, 1, True)
    off, _ = _dense_result(L, a, -1, b, 1, False)
    assert np.linalg.norm(on - off) > 0.1 * np.linalg.norm(on[1 + L.m * L.m:])


@pytest.mark.parametrize("n,R", [(2, 4), (6, 4), (12, 4)])
def test_mbpt2_matches_dense(n, R):
    L = orc.Layout(n, R)
    rng = np.random.default_rng(8)
    from helpers import synth_hamiltonian

    h = synth_hamiltonian(L, rng, gap=2.0, vs=0.1, fs=0.0)
    _, f, V = dense.to_dense(L, h, 1)
    got = orc.mbpt2(orc.Op(L, 1, h))
    assert got == pytest.approx(dense.mbpt2(f, V, n), rel=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("n,R", [(2, 4), (6, 4), (12, 4)])
@pytest.mark.parametrize("pandya", [True, False])
def test_gpu_matches_dense(n, R, pandya):
    import qd_imsrg_b200 as qd

    L = orc.Layout(n, R)
    a, b = _ops(L, -1, 1, 31 + n)
    P = qd.Layout(n, R, device=0)
    A, B, C = qd.FullHam(P, -1, a), qd.FullHam(P, 1, b), qd.FullHam(P, 1)
    qd.commutator(A, B, C, pandya=pandya)
    ref, _ = _dense_result(L, a, -1, b, 1, pandya)
    compare_parts(L, C.download(), ref, rtol=1e-12)
    for o in (A, B, C):
        o.close()
    P.close()
