"""The numpy statement of the warm-start network (oracle/mlp.py): its
backward pass against central finite differences in float64."""
import numpy as np

from oracle import mlp as om


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.2, om.NPARAM)
    X = rng.normal(0, 1, (8, om.NI))
    T = rng.normal(0, 1, 8)
    g, _ = om.grad(p, X, T, emulate=False)
    picks = np.concatenate([rng.integers(lo, hi, 6) for lo, hi in
                            [(om.O_W1, om.O_B1), (om.O_B1, om.O_W2), (om.O_W2, om.O_B2), (om.O_B2, om.O_W3),
                             (om.O_W3, om.O_B3), (om.O_B3, om.NPARAM)]])
    h = 1e-6
    for k in picks:
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (om.grad(pp, X, T, emulate=False)[1] - om.grad(pm, X, T, emulate=False)[1]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3], np.float32)
    r = om.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7 and r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2 ** -8
