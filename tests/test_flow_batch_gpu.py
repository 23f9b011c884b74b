"""Batched flows (qd_magnus_flow_batch): independent instances of different
sizes, run in lockstep with each BCH term's 122 tiles and ladder tasks of all
instances in one launch per kernel (default), or one host thread and stream
each, must give exactly what each gives alone; repeated flows on one layout
reuse its workspaces; the stepping object (qd_flow_*) reproduces
qd_magnus_flow."""
import numpy as np
import pytest

import qd_imsrg_b200 as qd
from helpers import synth_hamiltonian

pytestmark = pytest.mark.gpu

CASES = [(2, 4, 2.0, 0.05, 0.05), (6, 5, 2.0, 0.05, 0.05), (6, 6, 1.5, 0.08, 0.03), (12, 6, 2.0, 0.05, 0.05)]


def _instance(n, R, gap, vs, fs, seed):
    import oracle

    O = oracle.Layout(n, R)
    h = synth_hamiltonian(O, np.random.default_rng(seed), gap, vs, fs)
    P = qd.Layout(n, R)
    return P, qd.FullHam(P, 1, h), qd.FullHam(P, 1)


@pytest.mark.parametrize("pandya", [False, True])
def test_batch_equals_separate(gpu, pandya):
    inst = [_instance(*c, seed=11 + i) for i, c in enumerate(CASES)]
    alone = []
    for P, H, HS in inst:
        _, res = qd.magnus_flow(H, HS, pandya=pandya, max_iter=300)
        alone.append((res.E0, res.iterations, res.commutators, HS.download()))
    for streams in (False, True):
        results, status = qd.magnus_flow_batch([(H, HS) for _, H, HS in inst], pandya=pandya, max_iter=300,
                                               streams=streams)
        assert status == [0] * len(inst)
        for (P, H, HS), r, (e0, it, nc, v) in zip(inst, results, alone):
            assert r.E0 == e0 and r.iterations == it and r.commutators == nc
            assert np.array_equal(HS.download(), v)


def test_repeated_flow_reuses_workspaces(gpu):
    P, H, HS = _instance(6, 5, 2.0, 0.05, 0.05, seed=3)
    _, r1 = qd.magnus_flow(H, HS, max_iter=300)
    v1 = HS.download()
    _, r2 = qd.magnus_flow(H, HS, max_iter=300)
    assert r1.E0 == r2.E0 and r1.commutators == r2.commutators and np.array_equal(HS.download(), v1)


def test_stepping_flow_matches_magnus_flow(gpu):
    P, H, HS = _instance(6, 5, 2.0, 0.05, 0.05, seed=4)
    _, ref = qd.magnus_flow(H, HS, max_iter=300)
    vref = HS.download()
    HS2 = qd.FullHam(P, 1)
    f = qd.Flow(H, HS2)
    res = f.run(300)
    assert res.E0 == ref.E0 and res.iterations == ref.iterations and np.array_equal(HS2.download(), vref)
    f.close()


def test_warm_start_from_converged_omega_is_converged(gpu):
    # seeding the flow with its own converged Omega must reproduce the
    # converged Hamiltonian (one BCH evaluation, no further steps)
    P, H, HS = _instance(6, 5, 2.0, 0.05, 0.05, seed=5)
    f = qd.Flow(H, HS)
    res = f.run(300)
    G = qd.FullHam(P, -1)
    qd.copy_arrays(f.omega(), G)
    v = HS.download()
    f.close()
    HS2 = qd.FullHam(P, 1)
    f2 = qd.Flow(H, HS2)
    f2.warm_start(G, res.s)
    info = f2.step()
    assert info.converged and not info.accepted
    assert f2.state().E0 == pytest.approx(res.E0, abs=1e-12)
    assert np.allclose(HS2.download(), v, rtol=0, atol=1e-12)
    f2.close()


def test_batch_rejects_shared_layout(gpu):
    P, H, HS = _instance(2, 4, 2.0, 0.05, 0.05, seed=1)
    HS2 = qd.FullHam(P, 1)
    with pytest.raises(qd.QDError):
        qd.magnus_flow_batch([(H, HS), (H, HS2)])
