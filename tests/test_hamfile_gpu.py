"""export_hamiltonian / import_hamiltonian of a device operator: the file is
the host writer's, and an operator read back is bit-identical."""
import numpy as np
import pytest

import qd_imsrg_b200 as qd

pytestmark = pytest.mark.gpu


def test_device_round_trip(tmp_path):
    P = qd.Layout(6, 5)
    v = qd.random_operator(P, 1, 77)
    H = qd.FullHam(P, 1, v)
    path = tmp_path / "H.bin"
    qd.export_hamiltonian(H, str(path))
    ref = tmp_path / "ref.bin"
    qd.hamiltonian_write(P, v, str(ref))
    assert path.read_bytes() == ref.read_bytes()
    G = qd.FullHam(P, 1)
    qd.import_hamiltonian(G, str(path))
    assert np.array_equal(G.download(), v)
