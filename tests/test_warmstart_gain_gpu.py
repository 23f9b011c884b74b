"""What the learned warm start gains.  The per-entry network is trained on
the plain flow's own Omega(s) trajectories (12 draws of hbar-omega ~
U[0.3, 1.0] at N=12, R=10, by the library's forward/backward/Adam kernels);
on 6 held-out draws the plain Magnus flow then runs once from Omega = 0 and
once from the network's Omega at half the training flows' median final s,
each to the reference's criterion |MBPT2| <= 1e-9.  The flow judges the
prediction and restarts from Omega = 0 if it rejects it
(magnus_IMSRG.f90:220-228); the abandoned work is counted.

Bars: every warm-started E_gs within 1e-6 hbar-omega of the plain flow's, at
least half the predictions accepted, and at least 15% fewer commutators in
total over the held-out draws (measured: about 25%)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, R = 12, 10


def test_warm_start_saves_commutators_on_held_out_draws(gpu):
    import torch

    from qd_imsrg_b200 import warmstart as ws

    rng = np.random.default_rng(3)
    Xs, Ts, sfin = [], [], []
    for _ in range(12):
        inst = ws.Instance(N, R, float(rng.uniform(0.3, 1.0)))
        idx, sv, om, res = ws.trajectory(inst, 2048, rng)
        X, T = ws.samples(inst, idx, sv, om)
        Xs.append(X)
        Ts.append(T)
        sfin.append(res.s)
        inst.close()
    mlp = ws.MLP(0, seed=7)
    hist = ws.train(mlp, torch.cat(Xs), torch.cat(Ts), steps=1500, batch=8192, lr=1e-3, seed=1, log_every=500)
    assert hist[-1][1] < hist[0][1]
    s_target = 0.5 * float(np.median(sfin))
    erng = np.random.default_rng(99)
    cold_c = warm_c = accepted = 0
    rows = []
    for _ in range(6):
        hw = float(erng.uniform(0.3, 1.0))
        inst = ws.Instance(N, R, hw)
        cold = ws.cold_flow(inst)
        warm = ws.warm_flow(mlp, inst, s_target)
        inst.close()
        assert abs(warm["E"] - cold["E"]) <= 1e-6
        cold_c += cold["commutators"]
        warm_c += warm["commutators"]
        accepted += int(warm["accepted"])
        rows.append((hw, cold["commutators"], warm["commutators"], warm["accepted"]))
    mlp.close()
    print("held-out (hw, cold, warm, accepted):", rows, "gain %.3f" % (1.0 - warm_c / cold_c))
    assert accepted >= 3
    assert warm_c <= 0.85 * cold_c
