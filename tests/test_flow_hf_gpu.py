"""The reference's own CPU-runnable case on the GPU: N=6 electrons, R=10
shells, hbar-omega = 1, Hartree-Fock basis (host), Magnus flow with the White
generator on the device, against the oracle's flow on the same Hamiltonian.

The reference's mat_2_norm sums one-body parts only; on an HF Hamiltonian
(vanishing ph Fock block) the initial eta norm is ~1e-16 and run_magnus
rejects every step.  The literal mode reproduces that stall (compared row by
row over a few steps); QD_FULL_NORM takes the norms over one- and two-body
parts and converges, without and with the particle-hole channel."""
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
def test_config1_flow_full_norm(gpu, hf_input, pandya):
    vec, eig = hf_input
    O = oracle.Layout(N, R, eig)
    oH, oHS = oracle.Op(O, 1, vec), oracle.Op(O, 1)
    otr, _ = oracle.magnus_flow(oH, oHS, pandya=pandya, full_norm=True, max_iter=200)
    P = qd.Layout(N, R, eig=eig)
    H, HS = qd.FullHam(P, 1, vec), qd.FullHam(P, 1)
    tr, res = qd.magnus_flow(H, HS, pandya=pandya, full_norm=True, max_iter=200)
    assert tr.shape == otr.shape
    assert np.array_equal(tr[:, 6], otr[:, 6])
    assert res.E0 == pytest.approx(oHS.get()[0], rel=1e-10)
    assert np.allclose(tr[:, 2], otr[:, 2], rtol=1e-10)
    compare_parts(O, HS.download(), oHS.get(), rtol=1e-9)
    # the flow lowers the HF energy by roughly the second-order correction
    assert vec[0] - 0.6 < res.E0 < vec[0] - 0.2


def test_config1_literal_mode_stalls_like_the_reference(gpu, hf_input):
    vec, eig = hf_input
    O = oracle.Layout(N, R, eig)
    oH, oHS = oracle.Op(O, 1, vec), oracle.Op(O, 1)
    import ctypes

    otr = np.zeros((6, 7))
    s = ctypes.c_double()
    rows = oracle.lib().orc_magnus_flow(oH.h, oHS.h, 0, 6, otr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        ctypes.byref(s))
    assert rows == -1 and np.all(otr[:, 6] < 0)  # every step rejected
    P = qd.Layout(N, R, eig=eig)
    H, HS = qd.FullHam(P, 1, vec), qd.FullHam(P, 1)
    with pytest.raises(qd.QDError) as e:
        qd.magnus_flow(H, HS, max_iter=6)
    assert e.value.code == 6  # QD_ERR_NOCONV
