"""GPU parity of the whole Magnus flow (s_evolve with build_white,
magnus_IMSRG.f90:194-248): per-step trace (s, E0, ||eta||, crit, BCH terms,
rejections) and the converged Hamiltonian, CUDA engine vs oracle, on
synthetic Hamiltonians, with and without the particle-hole channel."""
import numpy as np
import pytest

import oracle
import qd_imsrg_b200 as qd
from helpers import compare_parts, synth_hamiltonian

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,R,gap,vs,fs,pandya,rejects", [
    (2, 4, 2.0, 0.05, 0.05, False, 0),
    (6, 4, 2.0, 0.05, 0.05, True, 0),
    (6, 5, 2.0, 0.05, 0.05, False, 0),
    (6, 4, 0.2, 0.4, 0.01, False, 1),   # one step rejected on eta-norm growth
])
def test_magnus_flow_matches_oracle(gpu, n, R, gap, vs, fs, pandya, rejects):
    O = oracle.Layout(n, R)
    h = synth_hamiltonian(O, np.random.default_rng(9 if rejects else 5), gap, vs, fs)
    oH, oHS = oracle.Op(O, 1, h), oracle.Op(O, 1)
    otr, os_ = oracle.magnus_flow(oH, oHS, pandya=pandya, max_iter=300)
    P = qd.Layout(n, R)
    H, HS = qd.FullHam(P, 1, h), qd.FullHam(P, 1)
    tr, res = qd.magnus_flow(H, HS, pandya=pandya, max_iter=300)
    assert tr.shape == otr.shape
    assert int((tr[:, 6] < 0).sum()) == rejects == res.rejected
    assert np.array_equal(tr[:, 6], otr[:, 6])           # BCH terms per step (sign: rejected)
    assert np.array_equal(tr[:, 0], otr[:, 0])           # iteration counter
    assert np.allclose(tr[:, 1], otr[:, 1], rtol=0, atol=1e-15)  # s
    assert np.allclose(tr[:, 2:6], otr[:, 2:6], rtol=1e-10, atol=1e-14)  # E0, nrm1, nrm2, crit
    assert res.E0 == pytest.approx(oHS.get()[0], rel=1e-10, abs=1e-13)
    compare_parts(O, HS.download(), oHS.get(), rtol=1e-10)
