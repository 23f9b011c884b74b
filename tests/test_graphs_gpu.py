"""BCH terms replayed as CUDA graphs give results identical to eager
launches: the N=6, R=10 flow (both channel settings) traced step by step with
graphs on and off, and graphs were really captured and replayed."""
import numpy as np
import pytest

import qd_imsrg_b200 as qd

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hf6():
    vec, eig, _ = qd.hf_hamiltonian(6, 10, 1.0)
    return vec, eig


@pytest.mark.parametrize("pandya", [False, True])
def test_flow_graphs_identical(hf6, pandya):
    vec, eig = hf6
    out = {}
    for graphs in (False, True):
        P = qd.Layout(6, 10, eig=eig)
        P.set_graphs(graphs)
        H, HS = qd.FullHam(P, 1, vec), qd.FullHam(P, 1)
        trs = []
        for _ in range(2):  # the second flow replays the first flow's graphs
            tr, res = qd.magnus_flow(H, HS, pandya=pandya, max_iter=200)
            trs.append((tr, res.E0, HS.download()))
        out[graphs] = (trs, P.graph_stats())
        for o in (H, HS):
            o.close()
        P.close()
    (eager, st0), (graph, st1) = out[False], out[True]
    assert st0 == (0, 0)
    assert st1[0] > 0 and st1[1] > st1[0]
    for (t0, e0, h0), (t1, e1, h1) in zip(eager, graph):
        assert np.array_equal(t0, t1)
        assert e0 == e1
        assert np.array_equal(h0, h1)
