"""Restatement of the reference's export_hamiltonian / import_hamiltonian
(src/ME_general.f90:207-361) in plain Python, as the checker of the library's
file format.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module.

The Fortran code opens the file `form='unformatted'` (sequential access) and
executes one `write(20) value` per entry, so each entry is a record: a 4-byte
length marker (8), the 8-byte value, the marker again (the gfortran/ifort
default record layout).  The loops below follow the Fortran loops literally
(i outer, j inner), with the part order of the reference: E0, fhh, fph, fpp,
then per block Vhhhh, Vpppp, Vpphh, Vphph, Vphhh, Vppph.  Operators are held
in vectorize order (ME_general.f90:1871-1989): column-major parts, fhh, fpp,
fph, then per block Vhhhh, Vpppp, Vpphh, Vphph, Vppph, Vphhh.
"""
from __future__ import annotations

import struct


def _parts(n, m, dims, offs):
    """Yield vectorize indices in export_hamiltonian's loop order.
    dims[q] = (nhh, nph, npp, ...), offs[q] = vectorize offsets of
    (Vhhhh, Vpppp, Vpphh, Vphph, Vppph, Vphhh)."""
    mp = m - n
    o_fhh = 1
    o_fpp = o_fhh + n * n
    o_fph = o_fpp + mp * mp
    yield 0                                  # write(20) H%E0
    for i in range(n):                       # ME_general.f90:220-224
        for j in range(n):
            yield o_fhh + i + j * n
    for i in range(mp):                      # :226-230
        for j in range(n):
            yield o_fph + i + j * mp
    for i in range(mp):                      # :232-236
        for j in range(mp):
            yield o_fpp + i + j * mp
    for q in range(len(dims)):               # :238-278
        nh, nb, npp = int(dims[q][0]), int(dims[q][1]), int(dims[q][2])
        hhhh, pppp, pphh, phph, ppph, phhh = (int(x) for x in offs[q][:6])
        for i in range(nh):
            for j in range(nh):
                yield hhhh + i + j * nh
        for i in range(npp):
            for j in range(npp):
                yield pppp + i + j * npp
        for i in range(npp):
            for j in range(nh):
                yield pphh + i + j * npp
        for i in range(nb):
            for j in range(nb):
                yield phph + i + j * nb
        for i in range(nb):
            for j in range(nh):
                yield phhh + i + j * nb
        for i in range(npp):
            for j in range(nb):
                yield ppph + i + j * npp


def export_hamiltonian(vec, n, m, dims, offs, path):
    with open(path, "wb") as fh:
        for idx in _parts(n, m, dims, offs):
            fh.write(struct.pack("<idi", 8, float(vec[idx]), 8))


def import_hamiltonian(n, m, dims, offs, neq, path):
    import numpy as np

    out = np.zeros(neq)
    with open(path, "rb") as fh:
        data = fh.read()
    pos = 0
    for idx in _parts(n, m, dims, offs):
        a, v, b = struct.unpack_from("<idi", data, pos)
        assert a == 8 and b == 8, "record markers"
        out[idx] = v
        pos += 16
    assert pos == len(data), "trailing bytes"
    return out
