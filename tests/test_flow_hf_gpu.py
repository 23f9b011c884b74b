"""The reference's own CPU-runnable case on the GPU: N=6 electrons, R=10
shells, hbar-omega = 1, Hartree-Fock basis (host), Magnus flow with the White
generator on the device, against the oracle's flow on the same Hamiltonian,
with the reference's default semantics (mat_2_norm over one- and two-body
parts for the BCH truncation and the step rejection), without and with the
particle-hole channel."""
import numpy as np
import pytest

import oracle
import qd_imsrg_b200 as qd
from helpers import compare_parts

pytestmark = pytest.mark.gpu

N, R, HW = 6, 10, 1.0


@pytest.fixture(scope="module")
def hf_input():
    vec, eig, _ = qd.hf_hamiltonian(N, R, HW)
    return vec, eig


@pytest.mark.parametrize("pandya", [False, True])
def test_config1_flow_matches_oracle(gpu, hf_input, pandya):
    vec, eig = hf_input
    O = oracle.Layout(N, R, eig)
    oH, oHS = oracle.Op(O, 1, vec), oracle.Op(O, 1)
    otr, _ = oracle.magnus_flow(oH, oHS, pandya=pandya, max_iter=200)
    P = qd.Layout(N, R, eig=eig)
    H, HS = qd.FullHam(P, 1, vec), qd.FullHam(P, 1)
    tr, res = qd.magnus_flow(H, HS, pandya=pandya, max_iter=200)
    assert tr.shape == otr.shape
    assert np.array_equal(tr[:, 6], otr[:, 6])           # BCH terms per step, rejections
    assert res.E0 == pytest.approx(oHS.get()[0], rel=1e-10)
    assert np.allclose(tr[:, 2], otr[:, 2], rtol=1e-10)  # E0 per step
    assert np.allclose(tr[:, 3:6], otr[:, 3:6], rtol=1e-9)  # nrm1, nrm2, crit
    compare_parts(O, HS.download(), oHS.get(), rtol=1e-9)
    # the flow lowers the HF energy by roughly the second-order correction
    assert vec[0] - 0.6 < res.E0 < vec[0] - 0.2
