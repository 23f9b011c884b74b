"""The autotuner of commutator_122: the first commutator on a layout times
every launch bucket of four bucketings with 64-, 128- and 256-thread CTAs
and keeps the fastest; qd_layout_tuning reports the timings.  The choice never changes a result:
the commutator before tuning (the tuned launch) and after it are
bit-identical."""
import numpy as np
import pytest

import qd_imsrg_b200 as qd

pytestmark = pytest.mark.gpu


def test_tuning_report_and_identical_results(gpu):
    P = qd.Layout(12, 8)
    A = qd.FullHam(P, -1, qd.random_operator(P, -1, 5))
    B = qd.FullHam(P, 1, qd.random_operator(P, 1, 6))
    C = qd.FullHam(P, 1)
    qd.commutator(A, B, C, pandya=True)
    first = C.download()
    rep = P.tuning()
    assert "commutator_122" in rep and "->" in rep
    for line in rep.splitlines():
        if line.startswith("commutator_122"):
            assert "bucketing" in line and "kept" in line
        else:
            assert line.rstrip().endswith(("-> 64", "-> 128", "-> 256"))
    qd.commutator(A, B, C, pandya=True)
    assert np.array_equal(C.download(), first)
