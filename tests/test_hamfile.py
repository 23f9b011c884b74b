"""On-disk Hamiltonian format (export/import_hamiltonian,
src/ME_general.f90:207-361): the library's files are byte-identical to the
oracle's literal restatement of the Fortran write loops, read back exactly,
and malformed files are rejected.  Host-only layouts: no GPU needed."""
import numpy as np
import pytest

import qd_imsrg_b200 as qd
from oracle import hamfile


@pytest.mark.parametrize("n,R", [(2, 3), (6, 4), (6, 5), (12, 6)])
def test_bytes_match_the_fortran_loops(tmp_path, n, R):
    P = qd.Layout(n, R, device=qd.HOST_ONLY)
    v = qd.random_operator(P, 1, 31 + n + R)
    v[0] = 1.25  # E0 written first
    ours, ref = tmp_path / "ours.bin", tmp_path / "ref.bin"
    qd.hamiltonian_write(P, v, str(ours))
    hamfile.export_hamiltonian(v, P.nbody, P.msp, P.dims, P.offs, str(ref))
    assert ours.read_bytes() == ref.read_bytes()
    assert ours.stat().st_size == 16 * P.neq
    back = qd.hamiltonian_read(P, str(ref))
    assert np.array_equal(back, v)
    assert np.array_equal(hamfile.import_hamiltonian(P.nbody, P.msp, P.dims, P.offs, P.neq, str(ours)), v)


def test_first_records(tmp_path):
    # E0, then fhh(1,1), fhh(1,2): row by row, although vectorize is column-major
    P = qd.Layout(2, 3, device=qd.HOST_ONLY)
    v = np.arange(P.neq, dtype=np.float64)
    path = tmp_path / "h.bin"
    qd.hamiltonian_write(P, v, str(path))
    raw = path.read_bytes()
    rec = [np.frombuffer(raw[16 * k + 4:16 * k + 12], np.float64)[0] for k in range(4)]
    assert rec == [0.0, 1.0, 3.0, 2.0]  # E0, fhh(1,1), fhh(1,2) = v[1+0+1*2], fhh(2,1)
    assert np.frombuffer(raw[:4], np.int32)[0] == 8 and np.frombuffer(raw[12:16], np.int32)[0] == 8


def test_rejects_malformed_files(tmp_path):
    P = qd.Layout(2, 3, device=qd.HOST_ONLY)
    v = qd.random_operator(P, 1, 5)
    path = tmp_path / "h.bin"
    qd.hamiltonian_write(P, v, str(path))
    raw = bytearray(path.read_bytes())
    (tmp_path / "short.bin").write_bytes(bytes(raw[:-16]))
    with pytest.raises(qd.QDError):
        qd.hamiltonian_read(P, str(tmp_path / "short.bin"))
    raw[16 * 3] = 4  # a record marker that is not 8
    (tmp_path / "bad.bin").write_bytes(bytes(raw))
    with pytest.raises(qd.QDError):
        qd.hamiltonian_read(P, str(tmp_path / "bad.bin"))
    with pytest.raises(qd.QDError):
        qd.hamiltonian_read(P, str(tmp_path / "missing.bin"))
    # a file of another layout has the wrong size
    P2 = qd.Layout(6, 4, device=qd.HOST_ONLY)
    with pytest.raises(qd.QDError):
        qd.hamiltonian_read(P2, str(path))
