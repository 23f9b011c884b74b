"""The warm-start network's CUDA kernels against the numpy statement
(oracle/mlp.py, rounding to bfloat16 where the kernels do): forward values
and gradients; training lowers the loss; the Omega feature, gather and
scatter kernels against host-side statements on a small basis."""
import numpy as np
import pytest

from oracle import mlp as om

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def test_forward_and_gradient_match_oracle(gpu):
    torch = _torch()
    from qd_imsrg_b200.warmstart import MLP

    m = MLP(0, seed=3)
    p = m.params().astype(np.float64)
    rng = np.random.default_rng(1)
    n = 256
    X = rng.normal(0, 1, (n, om.NI)).astype(np.float32)
    T = rng.normal(0, 1, n).astype(np.float32)
    dX, dT = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    y = torch.empty(n, dtype=torch.float32, device="cuda")
    m.forward(dX, y)
    yref, _ = om.forward(p, X)
    assert np.allclose(y.cpu().numpy(), yref, rtol=2e-3, atol=2e-3 * np.abs(yref).max())
    g = torch.empty(om.NPARAM, dtype=torch.float32, device="cuda")
    loss = m.grad(dX, dT, g)
    gref, lref = om.grad(p, X, T)
    assert loss == pytest.approx(lref, rel=2e-3)
    gg = g.cpu().numpy()
    for lo, hi in [(om.O_W1, om.O_B1), (om.O_B1, om.O_W2), (om.O_W2, om.O_B2), (om.O_B2, om.O_W3),
                   (om.O_W3, om.O_B3), (om.O_B3, om.NPARAM)]:
        err = np.linalg.norm(gg[lo:hi] - gref[lo:hi]) / max(np.linalg.norm(gref[lo:hi]), 1e-30)
        assert err < 5e-3, (lo, hi, err)
    m.close()


def test_training_lowers_the_loss(gpu):
    torch = _torch()
    from qd_imsrg_b200.warmstart import MLP, train

    rng = np.random.default_rng(2)
    X = rng.uniform(-1, 1, (65536, om.NI)).astype(np.float32)
    T = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2]).astype(np.float32)
    dX, dT = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    m = MLP(0, seed=4)
    hist = train(m, dX, dT, steps=400, batch=4096, lr=2e-3, log_every=399)
    assert hist[-1][1] < 0.1 * hist[0][1], hist
    m.close()


def test_omega_kernels_match_host_statements(gpu):
    torch = _torch()
    import oracle
    import qd_imsrg_b200 as qd
    from helpers import numpy_random_op
    from qd_imsrg_b200 import warmstart as ws

    n, R, hw = 6, 5, 0.7
    O = oracle.Layout(n, R)
    v = numpy_random_op(O, -1, np.random.default_rng(5))
    P = qd.Layout(n, R)
    P.set_stream(torch.cuda.current_stream().cuda_stream)
    G = qd.FullHam(P, -1, v)
    N = ws.omega_count(P)
    m, mp = O.m, O.m - O.n
    # host statement of the entry list: fph, then every block's Vpphh
    idx = [1 + n * n + mp * mp + e for e in range(mp * n)]
    for q in range(O.nblock):
        nh, npp = int(O.dims[q, 0]), int(O.dims[q, 2])
        idx += list(range(int(O.offs[q, 2]), int(O.offs[q, 2]) + nh * npp))
    assert N == len(idx)
    buf = torch.empty(N, dtype=torch.float64, device="cuda")
    ws.omega_gather(G, buf)
    assert np.array_equal(buf.cpu().numpy(), v[idx])
    # scatter back: zero elsewhere, the entries (through float32) in place
    G2 = qd.FullHam(P, -1)
    ws.omega_scatter(G2, buf.float(), 1.0)
    w = G2.download()
    ref = np.zeros_like(v)
    ref[idx] = v[idx].astype(np.float32)
    assert np.array_equal(w, ref)
    # with a per-entry factor (the warm start's eta0 scaling)
    fac = torch.linspace(-2.0, 2.0, N, dtype=torch.float64, device="cuda")
    ws.omega_scatter(G2, buf.float(), 0.5, fac)
    w = G2.download()
    ref = np.zeros_like(v)
    ref[idx] = 0.5 * v[idx].astype(np.float32).astype(np.float64) * fac.cpu().numpy()
    assert np.allclose(w, ref, rtol=1e-15, atol=0)
    # features of a Hamiltonian-like operator at s = 3.5
    from helpers import synth_hamiltonian

    h = synth_hamiltonian(O, np.random.default_rng(6))
    H = qd.FullHam(P, 1, h)
    X = torch.empty((N, 16), dtype=torch.float32, device="cuda")
    ws.omega_features(H, hw, 3.5, X)
    X = X.cpu().numpy()
    fhh = h[1:1 + n * n].reshape(n, n, order="F")
    fpp = h[1 + n * n:1 + n * n + mp * mp].reshape(mp, mp, order="F")
    eps = np.concatenate([np.diag(fhh), np.diag(fpp)])
    rows = []
    for e in range(mp * n):
        a, i = n + e % mp, e // mp
        rows.append([eps[a], 0, eps[i], 0, 0, 0, 1, 0, h[idx[e]], 0, 0, 1])
    nml = O.nblock // 3
    k = mp * n
    for q in range(O.nblock):
        pp, hh = O.pairs(q + 1, 2) - 1, O.pairs(q + 1, 0) - 1
        ML, MS = q % nml - (nml - 1) // 2, 2 * (q // nml) - 2
        for c in range(len(hh)):
            for r in range(len(pp)):
                rows.append([eps[pp[r, 0]], eps[pp[r, 1]], eps[hh[c, 0]], eps[hh[c, 1]], 0, 0, 1, 1, h[idx[k]],
                             ML, MS, 0])
                k += 1
    rows = np.array(rows, np.float64)
    ref = np.zeros((N, 16))
    ref[:, 0:4] = rows[:, 0:4] / (10 * hw)
    ref[:, 4:8] = rows[:, 4:8]
    ref[:, 8] = rows[:, 8] / np.sqrt(hw) * 10
    ref[:, 9], ref[:, 10] = hw, n / 20
    ref[:, 11], ref[:, 12] = rows[:, 9] / 10, rows[:, 10] / 2
    ref[:, 13], ref[:, 14], ref[:, 15] = 0.35, R / 20, rows[:, 11]
    assert np.allclose(X, ref, rtol=1e-6, atol=1e-6)
    for o in (G, G2, H):
        o.close()
    P.close()
