"""dGam (src/gs_IMSRG.f90:223-273) on the device against the oracle's
restatement in the reference's call order (1e-12 relative per part, the
plain form's bar), and the ODE form of the flow driven by a host integrator
through qd_dgam, as the reference's adams_ode drives dGam: the device-driven
and oracle-driven integrations agree, and the energy flows to the Magnus
flow's ground state."""
import numpy as np
import pytest

import oracle
import qd_imsrg_b200 as qd
from helpers import compare_parts
from oracle import dgam as odgam

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,R", [(2, 4), (6, 5), (12, 6)])
def test_dgam_matches_oracle(n, R):
    P, O = qd.Layout(n, R), oracle.Layout(n, R)
    h = qd.random_operator(P, 1, 40 + n + R)
    H, DER = qd.FullHam(P, 1, h), qd.FullHam(P, 1)
    HCC, ETACC = qd.CCMat(P, 1.0), qd.CCMat(P, -1.0)
    qd.dgam(H, DER, HCC, ETACC)
    oH, oD = oracle.Op(O, 1, h), oracle.Op(O, 1)
    oHCC, oECC = oracle.CC(O, 1.0), oracle.CC(O, -1.0)
    odgam.dgam(oH, oD, oHCC, oECC)
    compare_parts(O, DER.download(), oD.get(), 1e-12)
    assert np.allclose(HCC.download(), oHCC.get_X(), rtol=1e-12, atol=1e-14)
    assert np.allclose(ETACC.download(), oECC.get_X(), rtol=1e-12, atol=1e-14)


def test_ode_flow_through_dgam():
    from scipy.integrate import solve_ivp

    n, R, hw = 6, 4, 1.0
    vec, eig, _ = qd.hf_hamiltonian(n, R, hw)
    P, O = qd.Layout(n, R, eig=eig), oracle.Layout(n, R, eig)
    H, DER = qd.FullHam(P, 1), qd.FullHam(P, 1)
    oH, oD = oracle.Op(O, 1), oracle.Op(O, 1)
    occ = (oracle.CC(O, 1.0), oracle.CC(O, -1.0))

    def f_dev(s, y):  # repackage -> dGam -> vectorize, as the reference's solver callback
        H.upload(y)
        qd.dgam(H, DER)
        return DER.download()

    def f_orc(s, y):
        oH.set(y)
        odgam.dgam(oH, oD, *occ)
        return oD.get()

    s_end = 4.0
    kw = dict(method="DOP853", rtol=1e-8, atol=1e-10, dense_output=False)
    dev = solve_ivp(f_dev, (0.0, s_end), vec, **kw)
    orc = solve_ivp(f_orc, (0.0, s_end), vec, **kw)
    assert dev.success and orc.success
    assert dev.y[0, -1] == pytest.approx(orc.y[0, -1], rel=1e-10)
    # the ODE form flows to the same ground state as the Magnus form
    HS = qd.FullHam(P, 1)
    H.upload(vec)
    _, res = qd.magnus_flow(H, HS, pandya=True, max_iter=300)
    assert abs(dev.y[0, -1] - res.E0) < 1e-3 * abs(res.E0), (dev.y[0, -1], res.E0)
    assert dev.y[0, -1] < vec[0]  # correlation lowers the HF energy
